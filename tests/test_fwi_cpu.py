"""The FWI outer loop's host logic on CPU (no GPU): shots dealt to two `gloo` ranks, gradients
and misfits summed by all-reduce, identical models on every rank, the misfit decreasing; with a
linear stand-in for the per-shot solve (J_s = 1/2 |A_s m - d_s|^2)."""
import importlib.util
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_fwi():
    spec = importlib.util.spec_from_file_location("twave_fwi", os.path.join(ROOT, "tpu-wave_b200", "fwi.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["twave_fwi"] = mod   # (dataclasses look their module up here)
    spec.loader.exec_module(mod)
    return mod


def problem(n_shots=5, shape=(6, 7), seed=3):
    rng = np.random.default_rng(seed)
    n = shape[0] * shape[1]
    A = [rng.standard_normal((12, n)) / np.sqrt(n) for _ in range(n_shots)]
    truth = 2.0 + 0.1 * rng.standard_normal(shape)
    d = [a @ truth.reshape(-1) for a in A]
    return A, d, truth


def make_shot_fn(A, d):
    def shot_fn(model, shot, want_gradient):
        k = shot.src_ix
        r = A[k] @ model["vp"].reshape(-1) - d[k]
        g = {"vp": (A[k].T @ r).reshape(model["vp"].shape)} if want_gradient else {}
        return 0.5 * float(r @ r), g
    return shot_fn


def shots(fwi, n):
    return [fwi.Shot(0, k, 0, [], np.zeros(1)) for k in range(n)]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fwi = load_fwi()
    A, d, truth = problem()
    f = fwi.FWI(shots(fwi, len(A)), make_shot_fn(A, d), params=("vp",), rank=rank, world=world,
                allreduce=fwi.torch_allreduce())
    model = {"vp": np.full(truth.shape, 2.0)}
    J, g = f.gradient(model)
    Js = []
    for _ in range(4):
        model, J0, J1 = f.iterate(model, step=0.05)
        Js.append((J0, J1))
    dist.destroy_process_group()
    q.put((rank, J, g["vp"], model["vp"], Js))


@pytest.mark.timeout(120)
def test_two_ranks_sum_gradients_and_agree_on_the_model():
    fwi = load_fwi()
    A, d, truth = problem()
    single = fwi.FWI(shots(fwi, len(A)), make_shot_fn(A, d), params=("vp",))
    J_ref, g_ref = single.gradient({"vp": np.full(truth.shape, 2.0)})
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    res = sorted((q.get() for _ in range(2)), key=lambda x: x[0])
    for rank, J, g, m, Js in res:
        assert abs(J - J_ref) <= 1e-12 * J_ref
        assert np.allclose(g, g_ref["vp"], rtol=1e-12, atol=1e-14)
        assert all(j1 < j0 for j0, j1 in Js)
    assert np.array_equal(res[0][3], res[1][3])


def test_line_search_keeps_the_model_when_no_step_helps():
    fwi = load_fwi()
    A, d, truth = problem()
    f = fwi.FWI(shots(fwi, len(A)), make_shot_fn(A, d), params=("vp",))
    m, J0, J1 = f.iterate({"vp": truth.copy()}, step=0.5)   # already the minimiser
    assert J1 <= J0 and np.allclose(m["vp"], truth, atol=1e-6)
