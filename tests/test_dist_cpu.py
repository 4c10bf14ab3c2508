"""Multi-rank host logic of bench.py on CPU: two `gloo` ranks agree on the max-over-ranks time
and each rank gets its own shot (the source moves with the rank)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    d = bench.Dist()
    d.init("gloo")
    d.barrier()
    got = d.reduce_max(float(10 + 7 * rank))
    src = bench.build_model(rank)[4]
    d.finish()
    q.put((rank, got, src))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_max_and_split_shots():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    assert [r[1] for r in res] == [17.0, 17.0]
    assert res[0][2] != res[1][2]
