"""Multi-process halo exchange and level collectives: the reference's MPI path
(HaloExchange::exchange_scalar / exchange_face / synchronize_owned_face_interfaces with
an MpiCartesianContext, src/comm/halo_exchange.cpp:399-561; allreduce_sum_in_place,
src/comm/collectives.cpp:11-45) for one rank per process over torch.distributed: NCCL
between GPUs (NVLink / NVSwitch), gloo between host processes.

A rank's field is the reference's per-rank halo-padded storage as a torch tensor,
(nz[+1], ny_local[+1] + 2 halo, nx_local[+1] + 2 halo) with storage index (i, j, k) at
[k, j + halo, i + halo], the layout gwm_b200_global_to_ranks writes.  The layout and the
neighbour ranks are VirtualRankLayout::build and the cartesian topology
(gwm_b200_layout): a neighbour beyond an open side is -1 and its halo reads zero, as
MPI_PROC_NULL leaves it.

Messages carry no tags here, so every phase uses one channel: each rank sends at most
one message to a neighbour and receives at most one, and the pairing is unique even
where the west and east neighbour are the same rank (two ranks along a periodic axis).
A rank that is its own neighbour (one rank along a periodic axis) copies locally.
"""
from __future__ import annotations


import numpy as np

CELL, FACE_X, FACE_Y, FACE_Z = 0, 1, 2, 3


class HaloComm:
    """The MPI halo operators of one rank over a torch.distributed process group whose
    size is ranks_x * ranks_y (rank r of the group owns subdomain r of the layout)."""

    def __init__(self, nx: int, ny: int, nz: int, halo: int, ranks_x: int, ranks_y: int, periodic_x: bool,
                 periodic_y: bool, group=None):
        import importlib

        import torch.distributed as dist
        gwm = importlib.import_module(__package__ or "gpu-wm-next_b200")
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        world = dist.get_world_size(group)
        if world != ranks_x * ranks_y:
            raise ValueError(f"process group of {world} ranks for a {ranks_x} x {ranks_y} layout")
        if halo < 1:
            raise ValueError("halo must be at least 1")
        rows = gwm.layout(nx, ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y)
        row = rows[self.rank]
        self.nx_local, self.ny_local = int(row[4] - row[3]), int(row[6] - row[5])
        self.i_begin, self.j_begin = int(row[3]), int(row[5])
        self.west, self.east, self.south, self.north = (int(v) for v in row[7:11])
        self.nz, self.halo = nz, halo
        self.rows = rows

    # -- shapes -------------------------------------------------------------------------
    def shape(self, orientation: int):
        """The rank's storage shape for a field of this orientation."""
        h = self.halo
        return (self.nz + (orientation == FACE_Z), self.ny_local + (orientation == FACE_Y) + 2 * h,
                self.nx_local + (orientation == FACE_X) + 2 * h)

    def _global_rank(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    # -- point to point -----------------------------------------------------------------
    def _phase(self, send, dest: int, recv_like, source: int):
        """One channel: send to dest (-1: none) and receive from source (-1: zeros)."""
        import torch
        out = torch.zeros_like(recv_like)
        if dest == self.rank and source == self.rank:
            out.copy_(send)
            return out
        ops = []
        if dest >= 0:
            ops.append(self.dist.P2POp(self.dist.isend, send.contiguous(), self._global_rank(dest), self.group))
        if source >= 0:
            ops.append(self.dist.P2POp(self.dist.irecv, out, self._global_rank(source), self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        return out

    # -- HaloExchange::exchange_scalar / exchange_face (halo_exchange.cpp:399-461) ----------
    def exchange(self, f, orientation: int = CELL):
        """Fill the halo of f (in place) from the neighbours' owned values: x first, then
        y over the full padded width, so the corners come from the diagonal neighbour."""
        if tuple(f.shape) != self.shape(orientation):
            raise ValueError(f"field shape {tuple(f.shape)} is not {self.shape(orientation)}")
        h = self.halo
        onx = self.nx_local + (orientation == FACE_X)
        ony = self.ny_local + (orientation == FACE_Y)
        rows = slice(h, h + ony)
        # pack_face_x_faces_impl / pack_scalar_x_faces: X faces skip the shared face 0
        wi = 1 + h if orientation == FACE_X else h
        ei = self.nx_local if orientation == FACE_X else onx
        west_send = f[:, rows, wi:wi + h]
        east_send = f[:, rows, ei:ei + h]
        east_recv = self._phase(west_send, self.west, east_send, self.east)
        west_recv = self._phase(east_send, self.east, west_send, self.west)
        f[:, rows, 0:h] = west_recv
        f[:, rows, onx + h:onx + 2 * h] = east_recv
        # pack_face_y_faces_impl / pack_scalar_y_faces: whole padded rows
        sj = 1 + h if orientation == FACE_Y else h
        nj = self.ny_local if orientation == FACE_Y else ony
        south_send = f[:, sj:sj + h, :]
        north_send = f[:, nj:nj + h, :]
        north_recv = self._phase(south_send, self.south, north_send, self.north)
        south_recv = self._phase(north_send, self.north, south_send, self.south)
        f[:, 0:h, :] = south_recv
        f[:, ony + h:ony + 2 * h, :] = north_recv
        return f

    # -- HaloExchange::synchronize_owned_face_interfaces (halo_exchange.cpp:463-561) -------
    def synchronize_owned_face_interfaces(self, f, orientation: int):
        """Average each shared face with the neighbour's copy where the neighbour exists
        (0.5f (own + theirs), in FP32); Z faces have no lateral interface."""
        import torch
        if orientation == FACE_Z:
            return f
        if orientation not in (FACE_X, FACE_Y):
            raise ValueError("interface sync is defined for X and Y faces")
        if tuple(f.shape) != self.shape(orientation):
            raise ValueError(f"field shape {tuple(f.shape)} is not {self.shape(orientation)}")
        h = self.halo
        half = torch.tensor(0.5, dtype=f.dtype, device=f.device)
        if orientation == FACE_X:
            rows = slice(h, h + self.ny_local)
            lo, hi = f[:, rows, h], f[:, rows, h + self.nx_local]
            a, b = self.west, self.east
        else:
            cols = slice(h, h + self.nx_local)
            lo, hi = f[:, h, cols], f[:, h + self.ny_local, cols]
            a, b = self.south, self.north
        lo_send, hi_send = lo.clone(), hi.clone()
        # channel "high face -> the high neighbour's low face", then the reverse
        lo_recv = self._phase(hi_send, b, lo_send, a)
        hi_recv = self._phase(lo_send, a, hi_send, b)
        if a >= 0:
            lo.copy_(half * (lo_send + lo_recv))
        if b >= 0:
            hi.copy_(half * (hi_send + hi_recv))
        return f

    # -- allreduce_sum_in_place (collectives.cpp:11-45) ---------------------------------
    def allreduce_sum(self, values):
        """Sum over the ranks in place: float64 values, or 64-bit integers (the unsigned
        fixed-point level sums add the same in two's complement)."""
        import torch
        t = values
        if t.dtype == torch.uint64:
            t = values.view(torch.int64)
        if t.dtype not in (torch.float64, torch.int64):
            raise TypeError("allreduce_sum takes float64 or 64-bit integer values")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return values


def mpi_interface_sync_reference(rank_arrays, rows, halo: int, orientation: int):
    """The MPI interface sync applied to all ranks' arrays at once (numpy, for checking a
    distributed run): each shared face averaged with the neighbour's copy where the
    neighbour exists, periodic wrap included (halo_exchange.cpp:463-561)."""
    out = [np.array(a, dtype=np.float32, copy=True) for a in rank_arrays]
    h = halo
    for r, row in enumerate(rows):
        nxl, nyl = int(row[4] - row[3]), int(row[6] - row[5])
        west, east, south, north = (int(v) for v in row[7:11])
        src = rank_arrays[r]
        if orientation == FACE_X:
            if west >= 0:
                wn = int(rows[west][4] - rows[west][3])
                out[r][:, h:h + nyl, h] = np.float32(0.5) * (src[:, h:h + nyl, h] + rank_arrays[west][:, h:h + nyl, h + wn])
            if east >= 0:
                out[r][:, h:h + nyl, h + nxl] = np.float32(0.5) * (src[:, h:h + nyl, h + nxl] +
                                                                   rank_arrays[east][:, h:h + nyl, h])
        elif orientation == FACE_Y:
            if south >= 0:
                sn = int(rows[south][6] - rows[south][5])
                out[r][:, h, h:h + nxl] = np.float32(0.5) * (src[:, h, h:h + nxl] + rank_arrays[south][:, h + sn, h:h + nxl])
            if north >= 0:
                out[r][:, h + nyl, h:h + nxl] = np.float32(0.5) * (src[:, h + nyl, h:h + nxl] +
                                                                   rank_arrays[north][:, h, h:h + nxl])
    return out

