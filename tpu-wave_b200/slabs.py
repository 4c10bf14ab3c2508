"""Slab decomposition across ranks: one elastic grid cut along x into one slab per rank (one
GPU each), stepped in lockstep with a halo exchange after every step, as the reference's MPI tree
exchanges its halo strips (mpi/src/cpp/namespaces.hpp:611-635).

`partition` chooses the cuts; `SlabRun` owns one rank's slab and moves its halo rows to and from
the neighbouring ranks with torch.distributed point-to-point calls (NCCL between GPUs). The rows
travel where they lie: every field array's owned rows next to a cut are sent straight from the
slab's state, and the neighbour receives straight into its halo rows (tw_slab_halo gives both
spans, which are contiguous per array), so no pack or unpack kernel runs. All transfers of a rank
(both edges, every array) go out as one batch of non-blocking sends and receives, which cannot
deadlock whatever the order in which ranks reach it. On GPUs the host never waits: the transfers
are ordered after the step by a CUDA event on the handle's stream, and the next step after the
transfers by an event the handle's stream waits on. The energies of the slabs add up to the whole
grid's (`reduce_energy`), and so do their traces.
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


def edges(rank: int, world: int) -> list:
    """The cuts `rank` shares: (side, peer), side 0 the edge above it (shared with rank - 1), 1 the
    edge below (shared with rank + 1)."""
    out = []
    if rank > 0:
        out.append((0, rank - 1))
    if rank + 1 < world:
        out.append((1, rank + 1))
    return out


def tag(f: int, downward: bool) -> int:
    """Message tag of array slot f crossing a cut: downward (from the upper slab's bottom rows into
    the lower slab's top halo) or upward."""
    return 2 * f + (0 if downward else 1)


class _DeviceSpan:
    """A span of device memory as a CUDA array (zero-copy view for torch.as_tensor)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


class SlabRun:
    """One rank's slab of an Mx x My elastic grid. `tw` is the library's Python front end; `dist`
    the initialised torch.distributed module; the remaining keywords go to Solver.slab. `slab`
    replaces the library handle by any object with the same halo_spans / sync / step methods (with
    device=None its spans are writable numpy arrays on the host: a test of the exchange on CPU)."""

    def __init__(self, tw, dist, Mx: int, My: int, num_dx: int, den_dx: int, dt: float, slab=None, **kw):
        import torch
        self.torch, self.dist = torch, dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.cuts = partition(Mx, self.world)
        r0, r1 = self.cuts[self.rank], self.cuts[self.rank + 1]
        self.device = kw.get("device", 0) if slab is None else kw.get("device")
        self.s = slab if slab is not None else tw.Solver.slab(Mx, My, num_dx, den_dx, dt, r0, r1, **kw)
        if self.device is not None:
            self.stream = torch.cuda.ExternalStream(self.s.stream(), device=f"cuda:{self.device}")

    def _views(self, side: int, recv: int) -> list:
        """(slot, tensor) of every array's span at one edge: the owned rows the neighbour needs
        (recv 0) or the halo rows to fill (recv 1), of the current buffers."""
        torch = self.torch
        out = []
        for f, span in self.s.halo_spans(side, recv):
            if self.device is None:
                out.append((f, torch.from_numpy(span)))   # host stand-in: a writable numpy view
            else:
                ptr, n = span
                out.append((f, torch.as_tensor(_DeviceSpan(ptr, n), device=f"cuda:{self.device}")))
        return out

    def exchange(self):
        """Swap halo rows with both neighbours, straight between the slabs' state arrays."""
        torch, dist = self.torch, self.dist
        ops = []
        for side, peer in edges(self.rank, self.world):
            # my bottom rows go down (to the next rank's top halo); my top rows go up
            for f, t in self._views(side, 0):
                ops.append(dist.P2POp(dist.isend, t, peer, tag=tag(f, downward=side == 1)))
            for f, t in self._views(side, 1):
                ops.append(dist.P2POp(dist.irecv, t, peer, tag=tag(f, downward=side == 0)))
        if not ops:
            return
        if self.device is None:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            return
        cur = torch.cuda.current_stream(self.device)
        done = torch.cuda.Event()
        done.record(self.stream)        # the step has written the rows the sends read
        cur.wait_event(done)
        for r in dist.batch_isend_irecv(ops):
            r.wait()                    # (NCCL: the current stream waits for the transfers)
        landed = torch.cuda.Event()
        landed.record(cur)
        self.stream.wait_event(landed)  # the next step reads the halos after they landed

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
