"""Host logic of the rank-parallel slab decomposition (no GPU): the cuts, the edges and message
tags, and three `gloo` ranks swapping halo rows through the same code path (one batch of
non-blocking sends and receives straight between the arrays' rows) with a host stand-in for the
library's slab handle. Not run on several GPUs: NCCL needs one GPU per rank."""
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


def test_edges_and_tags_pair_every_send_with_one_receive():
    sl = load_slabs()
    for world in (1, 2, 3, 4, 7):
        sends, recvs = [], []
        for r in range(world):
            for side, peer in sl.edges(r, world):
                assert peer == (r - 1 if side == 0 else r + 1)
                for f in (0, 3, 7):
                    sends.append((r, peer, sl.tag(f, downward=side == 1)))
                    recvs.append((peer, r, sl.tag(f, downward=side == 0)))
        assert sorted(sends) == sorted(recvs) and len(set(sends)) == len(sends)


class FakeSlab:
    """Host stand-in: local rows [off, off + n) of global (Mx, W) arrays of float64, one per slot
    (two slots of different widths, so that a send paired with the wrong receive shows)."""

    WIDTHS = {0: 5, 3: 7}

    def __init__(self, globs, r0, r1):
        Mx = globs[0].shape[0]
        self.off = r0 - H if r0 > 0 else 0
        end = r1 + H if r1 < Mx else Mx
        self.own0, self.own1 = r0 - self.off, r1 - self.off
        self.a = {}
        for f, g in globs.items():
            a = np.full((end - self.off, g.shape[1]), np.nan)
            a[self.own0:self.own1] = g[r0:r1]   # halos unknown until exchanged
            self.a[f] = a

    def rows(self, side, recv):
        if side == 0:
            return slice(self.own0 - H, self.own0) if recv else slice(self.own0, self.own0 + H)
        return slice(self.own1, self.own1 + H) if recv else slice(self.own1 - H, self.own1)

    def halo_spans(self, side, recv):
        return [(f, a[self.rows(side, recv)].reshape(-1).view(np.uint8)) for f, a in self.a.items()]

    def sync(self):
        pass


def _globs(Mx):
    return {f: np.arange(Mx * w, dtype=np.float64).reshape(Mx, w) * (f + 1) for f, w in FakeSlab.WIDTHS.items()}


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sl = load_slabs()
    Mx = 72
    cuts = sl.partition(Mx, world)
    fake = FakeSlab(_globs(Mx), cuts[rank], cuts[rank + 1])
    run = sl.SlabRun(None, dist, Mx, 5, 1, Mx, 1e-3, slab=fake, device=None)
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
    globs = _globs(72)
    for rank, off, arrs in (q.get() for _ in range(3)):
        for f, a in arrs.items():
            assert np.array_equal(a, globs[f][off:off + a.shape[0]]), (rank, f)   # owned rows and both halos
