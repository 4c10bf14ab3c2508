"""Slab decomposition across ranks: one elastic grid cut along x into one slab per rank (one
GPU each), stepped in lockstep with a halo exchange after every step, as the reference's MPI tree
exchanges its halo strips (mpi/src/cpp/namespaces.hpp:611-635).

`partition` chooses the cuts; `SlabRun` owns one rank's slab and moves its halo rows to and from
the neighbouring ranks with torch.distributed point-to-point calls (NCCL between GPUs): each edge
is packed by the library into one contiguous device buffer (tw_slab_pack), sent, and the
neighbour's buffer unpacked into the halo rows (tw_slab_unpack). Exchanges alternate between the
even and the odd edges so that every send meets its receive without a deadlock. The energies of
the slabs add up to the whole grid's (`reduce_energy`), and so do their traces.
"""
from __future__ import annotations

import numpy as np

MIN_ROWS = 16     # rows per slab, and from an inner cut to a free surface (tw_create_slab)


def partition(Mx: int, n: int) -> list:
    """Balanced cuts 0 = c_0 < c_1 < ... < c_n = Mx of the x rows into n slabs of MIN_ROWS rows or
    more. Raises ValueError when the grid is too small for n slabs."""
    if n < 1 or Mx < n * MIN_ROWS:
        raise ValueError(f"{Mx} rows cannot hold {n} slabs of {MIN_ROWS} rows")
    return [round(k * Mx / n) for k in range(n + 1)]


def schedule(rank: int, world: int) -> list:
    """The point-to-point steps of one exchange for `rank`, in order: (phase, peer, my side). In
    phase 0 the edges between ranks 2i and 2i+1 exchange, in phase 1 those between 2i+1 and 2i+2;
    on each edge the upper rank sends first and the lower receives first."""
    steps = []
    for phase in (0, 1):
        if rank % 2 == phase and rank + 1 < world:
            steps.append((phase, rank + 1, 1))    # the edge below me
        if (rank - 1) % 2 == phase and rank - 1 >= 0:
            steps.append((phase, rank - 1, 0))    # the edge above me
    return steps


class SlabRun:
    """One rank's slab of an Mx x My elastic grid. `tw` is the library's Python front end; `dist`
    the initialised torch.distributed module; the remaining keywords go to Solver.slab. `slab`
    replaces the library handle by any object with the same pack / unpack / halo_bytes / sync /
    step methods (with device=None its buffers live on the host: a test of the exchange on CPU)."""

    def __init__(self, tw, dist, Mx: int, My: int, num_dx: int, den_dx: int, dt: float, slab=None, **kw):
        import torch
        self.torch, self.dist = torch, dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.cuts = partition(Mx, self.world)
        r0, r1 = self.cuts[self.rank], self.cuts[self.rank + 1]
        self.device = kw.get("device", 0) if slab is None else kw.get("device")
        self.s = slab if slab is not None else tw.Solver.slab(Mx, My, num_dx, den_dx, dt, r0, r1, **kw)
        where = "cpu" if self.device is None else f"cuda:{self.device}"
        self.buf = {}
        for side in (0, 1):
            if (side == 0 and self.rank > 0) or (side == 1 and self.rank + 1 < self.world):
                n = self.s.halo_bytes(side)
                self.buf[side] = (torch.empty(n, dtype=torch.uint8, device=where),
                                  torch.empty(n, dtype=torch.uint8, device=where))

    def exchange(self):
        """Swap halo rows with both neighbours (the handle's queued steps are finished first)."""
        torch = self.torch
        self.s.sync()
        for _, peer, side in schedule(self.rank, self.world):
            send, recv = self.buf[side]
            self.s.pack(side, send.data_ptr())
            if self.device is not None:
                torch.cuda.synchronize(self.device)   # (the pack runs on the handle's stream)
            else:
                self.s.sync()
            if side == 1:   # upper end of the edge: send, then receive
                self.dist.send(send, peer)
                self.dist.recv(recv, peer)
            else:
                self.dist.recv(recv, peer)
                self.dist.send(send, peer)
            if self.device is not None:
                torch.cuda.synchronize(self.device)   # (the transfer may run on the library's own stream)
            self.s.unpack(side, recv.data_ptr())
        self.s.sync()

    def run(self, n: int):
        for _ in range(n):
            self.s.step(1)
            self.exchange()

    def reduce_energy(self) -> list:
        """E_k, E_p0, E_p1 of the whole grid: the slabs' records summed over ranks."""
        torch = self.torch
        out = []
        for e in self.s.read_energy():
            t = torch.tensor(np.asarray(e), dtype=torch.float64, device=f"cuda:{self.device}")
            self.dist.all_reduce(t)
            out.append(t.cpu().numpy())
        return out

    def close(self):
        self.s.close()
