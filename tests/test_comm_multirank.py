"""The multi-process halo/collective backend (gpu-wm-next_b200/comm.py): the reference's
MPI halo exchange, face exchange, interface sync (src/comm/halo_exchange.cpp:399-561)
and allreduce_sum_in_place (src/comm/collectives.cpp:11-45) between processes over
torch.distributed, run here as gloo ranks on 127.0.0.1 (no GPU; between GPUs the same
code runs over NCCL).

Each rank builds its halo-padded storage from one seeded global field
(gwm_b200_global_to_ranks), runs the operator, and the parent compares every rank's
array with the oracle's restatement of the same operator on all ranks at once: the
exchange bit for bit against gwo_halo; the interface sync against the MPI rule (average
with the neighbour's copy wherever a neighbour exists, periodic wrap included)."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ORIENTS = {"cell": 0, "x": 1, "y": 2, "z": 3}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _global(shape, seed):
    return np.random.default_rng(seed).uniform(-1.0, 2.0, shape).astype(np.float32)


def _rank_main(rank, world, port, case, q):
    import datetime
    import importlib

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        gwm = importlib.import_module("gpu-wm-next_b200")
        comm = importlib.import_module("gpu-wm-next_b200.comm")
        nx, ny, nz, h, rx, ry, px, py = case["layout"]
        hc = comm.HaloComm(nx, ny, nz, h, rx, ry, px, py)
        out = {}
        for name, o in ORIENTS.items():
            shp = (nz + (o == 3), ny + (o == 2), nx + (o == 1))
            glob = _global(shp, case["seed"] + o)
            ranks = [np.zeros(comm_shape(hc.rows[r], nz, h, o), np.float32) for r in range(world)]
            gwm.global_to_ranks(glob, ranks, nx, ny, nz, h, rx, ry, px, py, o)
            t = torch.from_numpy(ranks[rank].copy())
            assert tuple(t.shape) == hc.shape(o)
            out[("exchange", name)] = hc.exchange(t.clone(), o).numpy()
            if o in (1, 2):
                out[("sync", name)] = hc.synchronize_owned_face_interfaces(t.clone(), o).numpy()
        sums = torch.arange(8, dtype=torch.int64) * (rank + 1) + (1 << 40) * rank
        hc.allreduce_sum(sums)
        vals = torch.full((3,), 0.25 * (rank + 1), dtype=torch.float64)
        hc.allreduce_sum(vals)
        out["sums"], out["vals"] = sums.numpy(), vals.numpy()
        q.put((rank, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def comm_shape(row, nz, h, o):
    nxl, nyl = int(row[4] - row[3]), int(row[6] - row[5])
    return (nz + (o == 3), nyl + (o == 2) + 2 * h, nxl + (o == 1) + 2 * h)


CASES = {
    "2x1_periodic": dict(layout=(13, 7, 3, 1, 2, 1, True, True), seed=11),
    "2x1_open_halo2": dict(layout=(12, 9, 2, 2, 2, 1, False, True), seed=12),
    "1x2_open": dict(layout=(8, 11, 2, 1, 1, 2, True, False), seed=13),
    "2x2_periodic": dict(layout=(10, 9, 2, 1, 2, 2, True, True), seed=14),
    "2x2_open_halo2": dict(layout=(11, 10, 3, 2, 2, 2, False, False), seed=15),
    "4x1_mixed": dict(layout=(17, 5, 2, 1, 4, 1, True, False), seed=16),
}


@pytest.mark.parametrize("name", list(CASES))
def test_distributed_halo_operators_match_the_reference(gwm, orc, name):
    import torch.multiprocessing as mp
    comm = __import__("importlib").import_module("gpu-wm-next_b200.comm")
    case = CASES[name]
    nx, ny, nz, h, rx, ry, px, py = case["layout"]
    world = rx * ry
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, out = q.get(timeout=180)
        results[r] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rows = gwm.layout(nx, ny, nz, h, rx, ry, px, py)
    for oname, o in ORIENTS.items():
        shp = (nz + (o == 3), ny + (o == 2), nx + (o == 1))
        glob = _global(shp, case["seed"] + o)
        ranks = [np.zeros(comm_shape(rows[r], nz, h, o), np.float32) for r in range(world)]
        gwm.global_to_ranks(glob, ranks, nx, ny, nz, h, rx, ry, px, py, o)
        want = orc.halo([a.astype(np.float64) for a in ranks], nx, ny, nz, h, rx, ry, px, py, oname, "exchange")
        for r in range(world):
            np.testing.assert_array_equal(results[r][("exchange", oname)], want[r].astype(np.float32),
                                          err_msg=f"{name} exchange {oname} rank {r}")
        if o in (1, 2):
            want = comm.mpi_interface_sync_reference(ranks, rows, h, o)
            for r in range(world):
                np.testing.assert_array_equal(results[r][("sync", oname)], want[r],
                                              err_msg=f"{name} sync {oname} rank {r}")
    total = sum(np.arange(8, dtype=np.int64) * (r + 1) + (1 << 40) * r for r in range(world))
    for r in range(world):
        np.testing.assert_array_equal(results[r]["sums"], total)
        np.testing.assert_array_equal(results[r]["vals"], np.full(3, sum(0.25 * (k + 1) for k in range(world))))


def test_layout_mismatch_is_refused(gwm):
    # a process group whose size is not ranks_x * ranks_y is rejected before any message
    import datetime

    import torch.distributed as dist
    comm = __import__("importlib").import_module("gpu-wm-next_b200.comm")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=datetime.timedelta(seconds=30))
    try:
        with pytest.raises(ValueError, match="process group of 1 ranks"):
            comm.HaloComm(8, 8, 2, 1, 2, 1, True, True)
        hc = comm.HaloComm(8, 6, 2, 1, 1, 1, True, False)   # one rank, periodic in x: its own neighbour
        import torch
        f = torch.from_numpy(np.arange(2 * 8 * 10, dtype=np.float32).reshape(2, 8, 10))
        g = hc.exchange(f.clone(), 0)
        assert torch.equal(g[:, 1:7, 0], f[:, 1:7, 8]) and torch.equal(g[:, 1:7, 9], f[:, 1:7, 1])
        assert torch.count_nonzero(g[:, 0, :]) == 0 and torch.count_nonzero(g[:, 7, :]) == 0  # open in y
    finally:
        dist.destroy_process_group()


# ---- the reference's own MPI unit tests (tests/unit/test_mpi_scalar_halo_exchange.cpp,
# test_mpi_face_halo_exchange.cpp, test_mpi_face_interface_sync.cpp,
# test_mpi_halo_mismatch_rejects.cpp): a 2 x 2 periodic layout of 8 x 8 x 2, every owned
# storage value 1000 k + 100 gj + gi of its global index, the MPI operators against the
# virtual-rank operators on the same fields
KAT = (8, 8, 2, 1, 2, 2, True, True)


def _kat_field(row, nz, h, o):
    nxl, nyl = int(row[4] - row[3]), int(row[6] - row[5])
    a = np.zeros((nz + (o == 3), nyl + (o == 2) + 2 * h, nxl + (o == 1) + 2 * h), np.float32)
    k, j, i = np.meshgrid(np.arange(a.shape[0]), np.arange(nyl + (o == 2)), np.arange(nxl + (o == 1)),
                          indexing="ij")
    a[:, h:h + nyl + (o == 2), h:h + nxl + (o == 1)] = 1000 * k + 100 * (row[5] + j) + (row[3] + i)
    return a


def _rank_kat(rank, world, port, q):
    import datetime
    import importlib

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        comm = importlib.import_module("gpu-wm-next_b200.comm")
        nx, ny, nz, h, rx, ry, px, py = KAT
        hc = comm.HaloComm(nx, ny, nz, h, rx, ry, px, py)
        out = {}
        for o in (0, 1, 2, 3):
            t = torch.from_numpy(_kat_field(hc.rows[rank], nz, h, o))
            out[("exchange", o)] = hc.exchange(t.clone(), o).numpy()
            if o in (1, 2):
                out[("sync", o)] = hc.synchronize_owned_face_interfaces(t.clone(), o).numpy()
        # test_mpi_halo_mismatch_rejects: a layout whose rank count is not the group's
        try:
            comm.HaloComm(nx, ny, nz, h, 1, 1, px, py)
            out["mismatch"] = False
        except ValueError:
            out["mismatch"] = True
        q.put((rank, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reference_mpi_unit_tests(gwm, orc):
    import torch.multiprocessing as mp
    comm = __import__("importlib").import_module("gpu-wm-next_b200.comm")
    nx, ny, nz, h, rx, ry, px, py = KAT
    world = rx * ry
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_kat, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rows = gwm.layout(nx, ny, nz, h, rx, ry, px, py)
    names = {0: "cell", 1: "x", 2: "y", 3: "z"}
    for o in (0, 1, 2, 3):
        fields = [_kat_field(r, nz, h, o) for r in rows]
        virt = orc.halo([f.astype(np.float64) for f in fields], nx, ny, nz, h, rx, ry, px, py, names[o], "exchange")
        for r in range(world):  # test_mpi_scalar_halo_exchange / test_mpi_face_halo_exchange
            np.testing.assert_array_equal(res[r][("exchange", o)], virt[r].astype(np.float32))
        if o in (1, 2):
            # test_mpi_face_interface_sync expects the virtual-rank result.  The two agree on
            # every interface between distinct subdomains; on the periodic wrap interface the
            # MPI code (halo_exchange.cpp:463-561) averages the two copies, 1000 k + 100 gj + nx
            # and 1000 k + 100 gj + 0 here, where the virtual-rank sync leaves them, so the
            # backend follows the MPI code there
            virt = orc.halo([f.astype(np.float64) for f in fields], nx, ny, nz, h, rx, ry, px, py, names[o], "sync")
            mpi = comm.mpi_interface_sync_reference(fields, rows, h, o)
            for r in range(world):
                got = res[r][("sync", o)]
                np.testing.assert_array_equal(got, mpi[r])
                row = rows[r]
                nxl, nyl = int(row[4] - row[3]), int(row[6] - row[5])
                interior = np.ones(got.shape, bool)  # drop the wrap interfaces
                if o == 1:
                    if row[3] == 0:
                        interior[:, :, h] = False
                    if row[4] == nx:
                        interior[:, :, h + nxl] = False
                else:
                    if row[5] == 0:
                        interior[:, h, :] = False
                    if row[6] == ny:
                        interior[:, h + nyl, :] = False
                np.testing.assert_array_equal(got[interior], virt[r].astype(np.float32)[interior])
    assert all(res[r]["mismatch"] for r in range(world))
