"""Host logic of the rank-parallel slab decomposition (no GPU): the cuts, the deadlock-free
exchange schedule, and three `gloo` ranks swapping halo rows through the same code path with a
host stand-in for the library's slab handle (pack / unpack of four rows per edge)."""
import importlib.util
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 4


def load_slabs():
    spec = importlib.util.spec_from_file_location("twave_slabs", os.path.join(ROOT, "tpu-wave_b200", "slabs.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["twave_slabs"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_partition():
    sl = load_slabs()
    assert sl.partition(72, 3) == [0, 24, 48, 72]
    c = sl.partition(1000, 7)
    assert c[0] == 0 and c[-1] == 1000 and min(b - a for a, b in zip(c[:-1], c[1:])) >= sl.MIN_ROWS
    with pytest.raises(ValueError):
        sl.partition(40, 3)


def test_schedule_pairs_every_edge_once_per_phase():
    sl = load_slabs()
    for world in (1, 2, 3, 4, 7):
        seen = {}
        for r in range(world):
            for phase, peer, side in sl.schedule(r, world):
                seen.setdefault((phase, min(r, peer), max(r, peer)), []).append((r, side))
        assert len(seen) == world - 1
        for (phase, a, b), ends in seen.items():
            assert b == a + 1 and phase == a % 2 and sorted(ends) == [(a, 1), (b, 0)]


class FakeSlab:
    """Host stand-in: local rows [off, off + n) of a global (Mx, W) array of float64."""

    def __init__(self, glob, r0, r1):
        Mx = glob.shape[0]
        self.off = r0 - H if r0 > 0 else 0
        end = r1 + H if r1 < Mx else Mx
        self.own0, self.own1 = r0 - self.off, r1 - self.off
        self.a = np.full((end - self.off, glob.shape[1]), np.nan)
        self.a[self.own0:self.own1] = glob[r0:r1]   # halos unknown until exchanged

    def halo_bytes(self, side):
        return H * self.a.shape[1] * 8

    def rows(self, side, recv):
        if side == 0:
            return slice(self.own0 - H, self.own0) if recv else slice(self.own0, self.own0 + H)
        return slice(self.own1, self.own1 + H) if recv else slice(self.own1 - H, self.own1)

    def pack(self, side, ptr):
        import ctypes
        blk = np.ascontiguousarray(self.a[self.rows(side, 0)])
        ctypes.memmove(ptr, blk.ctypes.data, blk.nbytes)

    def unpack(self, side, ptr):
        import ctypes
        blk = np.empty_like(self.a[self.rows(side, 1)])
        ctypes.memmove(blk.ctypes.data, ptr, blk.nbytes)
        self.a[self.rows(side, 1)] = blk

    def sync(self):
        pass


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sl = load_slabs()
    Mx, W = 72, 5
    glob = np.arange(Mx * W, dtype=np.float64).reshape(Mx, W)
    cuts = sl.partition(Mx, world)
    fake = FakeSlab(glob, cuts[rank], cuts[rank + 1])
    run = sl.SlabRun(None, dist, Mx, W, 1, Mx, 1e-3, slab=fake, device=None)
    run.exchange()
    dist.destroy_process_group()
    q.put((rank, fake.off, fake.a))


@pytest.mark.timeout(120)
def test_three_gloo_ranks_fill_their_halos():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_rank_main, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    glob = np.arange(72 * 5, dtype=np.float64).reshape(72, 5)
    for rank, off, a in (q.get() for _ in range(3)):
        assert np.array_equal(a, glob[off:off + a.shape[0]]), rank   # owned rows and both halos
