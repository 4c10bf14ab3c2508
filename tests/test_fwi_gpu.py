"""The FWI outer loop on the GPU: three shots on a small elastic grid, observed data from a
medium with a vp anomaly, the misfit falling at every iteration from the background model; and
the reference's data misfit (tw_data_misfit) equal to twice the adjoint's J."""
import importlib.util
import os
import sys

import numpy as np
import pytest

from cases import load_twave

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_fwi():
    spec = importlib.util.spec_from_file_location("twave_fwi", os.path.join(ROOT, "tpu-wave_b200", "fwi.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["twave_fwi"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_fwi_iterations_reduce_the_misfit():
    tw, fwi = load_twave(), load_fwi()
    M, den, nt = 48, 48, 160
    dt = 0.4 * (1 / den) / (np.sqrt(2) * 3.3)
    P = (M + 2, M + 2)
    rho, vp = np.full(P, 2.0), np.full(P, 3.0)
    X, Y = np.meshgrid(np.arange(P[0]), np.arange(P[1]), indexing="ij")
    true_vp = vp * (1 + 0.08 * np.exp(-((X - 26) ** 2 + (Y - 24) ** 2) / 30.0))
    vs = vp / np.sqrt(3)
    rcv = [(tw.NM, np.full(M // 2, 3), np.arange(0, M, 2))]
    run = fwi.elastic_shot_fn(tw, M, M, 1, den, dt, nt, central_f=6.0, time_delay=0.15, precision="f64", ckpt_every=40)
    shots = []
    for iy in (8, 24, 40):
        sh = fwi.Shot(tw.MM, 6, iy, rcv, np.zeros((M // 2, 2, nt)))
        s = tw.Solver(M, M, 1, den, dt, precision="f64", central_f=6.0, time_delay=0.15, max_steps=nt, energy=False)
        s.set_material_model(rho, true_vp, vs)
        s.set_source(tw.MM, 6, iy)
        s.add_receivers(*rcv[0])
        s.run(nt)
        sh.obs = s.read_receivers()
        s.close()
        shots.append(sh)
    model = {"rho": rho, "vp": vp.copy(), "vs": vs}
    f = fwi.FWI(shots, run, params=("vp",), bounds={"vp": (1.0, 6.0)})
    Js = []
    for _ in range(3):
        model, J0, J1 = f.iterate(model, step=0.03)
        Js.append((J0, J1))
    assert all(j1 < j0 for j0, j1 in Js), Js
    assert Js[-1][1] < 0.9 * Js[0][0], Js   # (measured: 19 % lower after three iterations)
    # the reference's data misfit is twice the adjoint's J
    s = tw.Solver(M, M, 1, den, dt, precision="f64", central_f=6.0, time_delay=0.15, max_steps=nt, energy=False)
    s.set_material_model(rho, vp, vs)
    s.set_source(tw.MM, 6, 24)
    s.add_receivers(*rcv[0])
    out = s.adjoint_gradient(nt, shots[1].obs, ckpt_every=40, model=False)
    tot, per = s.data_misfit(shots[1].obs)
    assert abs(tot - 2 * out["misfit"]) <= 1e-12 * tot and abs(per.sum() - tot) <= 1e-12 * tot
    s.close()
