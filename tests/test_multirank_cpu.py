"""The N>1 path of bench.py on CPU: two gloo ranks (127.0.0.1), no GPU.

Each rank advances an independent replica (no data-path collective), so the only
cross-rank steps are the timing reduction (max over ranks) and the whole-job
throughput; the reference arm runs on rank 0 alone.  These tests run those host
pieces under a real two-process torch.distributed group.
"""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank            # rank 1 is the slow one
        ms_max = bench.max_over_ranks(local_ms, torch, dist, "cpu")
        value = bench.job_throughput(1000, 4, world, ms_max)
        # the reference arm: rank 0 alone works, the other ranks return at once
        class A:
            steps, warmup = 1, 0
        if rank != 0:
            bench.run_reference(A(), rank, world)
        dist.barrier()
        q.put((rank, ms_max, value))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_reduction():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0, f"rank exited with {p.exitcode}"
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms_max, value in got:
        assert ms_max == pytest.approx(15.0), rank           # max over ranks, on every rank
        assert value == pytest.approx(1000 * 4 * 2 / 15e-3)  # whole job: both replicas


def test_single_rank_helpers_without_group():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, torch, None, "cpu") == 7.5
    assert bench.job_throughput(10, 3, 1, 2.0) == pytest.approx(10 * 3 / 2e-3)


def test_bench_reads_the_committed_traffic_summaries():
    # the roofline object's `traffic` comes from the committed ncu summaries of the
    # substep kernels (per-cell DRAM bytes scaled to the bench grid); a summary that
    # lost its machine-readable line would silently turn it into null
    sys.path.insert(0, ROOT)
    import bench

    class G:
        nx, ny, nz = 1024, 1024, 64

    for tile in bench.TRAFFIC_PROFILES:
        t = bench.read_traffic(G, tile)
        assert t is not None, bench.TRAFFIC_PROFILES[tile]
        per_cell = t / (G.nx * G.ny * G.nz)
        assert 30.0 < per_cell < 60.0, (tile, per_cell)


def test_reference_arm_loads_no_product_code():
    # the reference arm times the oracle alone: neither the product package nor its
    # CUDA library may be imported or mapped by that process
    import subprocess
    code = ("import sys, json; sys.path.insert(0, %r); import bench\n"
            "bench.CPU_SAMPLE = 16\n"
            "class A:\n    steps, warmup = 1, 1\n"
            "bench.run_reference(A(), 0, 1)\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(json.dumps({'pkg': any('gpu-wm-next_b200' in m for m in sys.modules),\n"
            "                  'so': 'libgwm_b200' in maps, 'torch': 'torch' in sys.modules}))\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, check=True)
    import json
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    ref, flags = lines[0], lines[-1]
    assert ref["impl"] == "reference" and ref["value"] > 0 and ref["sampled_grid"]["nx"] == 16
    assert ref["config"]["nx"] == 1024 and ref["cpu_baseline"]["kind"] == "port"
    assert flags == {"pkg": False, "so": False, "torch": False}, flags


def test_clock_sampler_decodes_nvml_reasons(monkeypatch):
    # The clock record reads NVML only; a fake NVML module stands in for the device.
    import types
    import time

    sys.path.insert(0, ROOT)
    import bench
    seq = iter([(1965, 0x0), (1965, 0x4), (1800, 0x4 | 0x8)] + [(1965, 0x1)] * 10000)
    fake = types.SimpleNamespace(
        NVML_CLOCK_SM=1, nvmlInit=lambda: None,
        nvmlDeviceGetHandleByIndex=lambda i: ("dev", i),
        nvmlDeviceGetHandleByPciBusId=lambda b: ("dev", b),
        nvmlDeviceGetMaxClockInfo=lambda h, k: 1965)
    cur = {}

    def clock(h, k):
        cur["s"] = next(seq)
        return cur["s"][0]

    fake.nvmlDeviceGetClockInfo = clock
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: cur["s"][1]
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    c = bench.ClockSampler(0, period_s=0.001)
    c.start()
    c.wait_first(2.0)
    time.sleep(0.05)
    c.stop()
    s = c.summary()
    assert c.source == "nvml" and s["samples"] >= 4
    assert s["sm_max_mhz"] == 1965 and s["sm_mhz"] == 1965
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    # samples before mark() do not describe the timed region
    c2 = bench.ClockSampler(0)
    c2.samples = [(1200.0, 1965.0, {"hw_slowdown"}), (1965.0, 1965.0, set())]
    c2._start = 1
    assert c2.summary()["reasons"] == [] and c2.summary()["sm_mhz"] == 1965.0
