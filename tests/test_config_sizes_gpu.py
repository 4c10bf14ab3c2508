"""Parity and the energy check at the benchmark configurations' own sizes.

* C2, elastic 2048 x 2048 FP32 (the benchmark's workload: 8-layer seeded medium, explosive
  Ricker source, 16 receivers): the first 30 steps against the reference's own FP32 solver built
  from its sources (oracle/_ref), every field and trace bit for bit; a random state of the whole
  grid stepped 3 times against the C restatement, so that every interior warp, strip, row segment
  and the periodic seam carry data; 4000 steps with the energy every step, whose 100-step block
  maxima must not grow after the source has stopped.
* C1, acoustic 512 x 512 FP32, 1000 steps: the periodic mode against the reference's single-core
  solver (fields, 16 traces, energies), the free-surface mode against the reference's elastic
  solver with vs = 0 (p = sxx = syy; fields and traces).

Reference code paths: cuda/src/cpp/forward_simulation.cpp:21-182 (elastic loop),
singlecore/src/main_cpp/cpu_acoustic.cpp:231-345 (single-core acoustic loop).
"""
import numpy as np
import pytest

import bench
from cases import load_twave, product_acoustic_periodic, product_elastic
from conftest import has_ref_binaries
from oracle import oracle as orc
from oracle import refrun

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not has_ref_binaries(), reason="oracle/_ref binaries not built")
E_RTOL = 1e-12


def energy_close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= E_RTOL * max(np.abs(b).max(), 1e-300)


@needs_ref
def test_c2_elastic_2048_first_steps_match_reference():
    case = bench.reference_case(30)
    want = refrun.run_elastic(case, "f32")
    got = product_elastic(case, "f32")
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    assert np.abs(got["traces"]).max() > 0 or np.abs(got["fields"]["MM0"]).max() > 0
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


def test_c2_elastic_2048_random_state_matches_restatement():
    """Every point of the 2048^2 grid carries data (random fields and the benchmark's medium),
    so the interior warps, their strips and segment edges, the boundary CTAs and the periodic
    seam all meet non-zero values; 3 steps, bit for bit with the C restatement."""
    case = bench.reference_case(3)
    Mx, My = case.Mx, case.My
    rng = np.random.default_rng(2048)
    shapes = [(Mx + 1, My + 1), (Mx, My + 1), (Mx + 1, My), (Mx, My), (Mx, My)]
    f0 = [(rng.standard_normal(s) * 1e-2).astype(np.float32).astype(np.float64) for s in shapes]
    want = orc.elastic_run(case, "f32", fields0=f0)
    got = product_elastic(case, "f32", fields0=f0)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


def test_c2_elastic_2048_energy_does_not_grow():
    """4000 FP32 steps of the benchmark workload with the discrete energy E = E_k + (E_p0 + E_p1)/2
    every step (grid_energy.cpp:180-216). After the source has stopped (t > delay + 3/f0), the
    maximum over each 100-step block may not exceed the previous block's by more than 1e-6
    relative (the reference's energy oscillates at O(dt) within a block, so blocks are compared
    by their maxima)."""
    tw = load_twave()
    rho, vp, vs, dt, (sx, sy) = bench.build_model(0)
    rx, ry = bench.receivers()
    nt = 4000
    s = tw.Solver(bench.MX, bench.MY, 1, bench.DEN_DX, dt, physics=tw.ELASTIC, precision="f32", cpst="00",
                  central_f=bench.F0, time_delay=bench.DELAY, max_steps=nt, energy=True)
    try:
        s.set_material_model(rho, vp, vs)
        s.set_source(tw.MM, sx, sy)
        s.add_receivers(tw.NM, rx, ry)
        s.run(nt)
        ek, ep0, ep1 = s.read_energy()
    finally:
        s.close()
    E = ek + 0.5 * (ep0 + ep1)
    assert np.isfinite(E).all() and E.max() > 0
    first = int(np.ceil((bench.DELAY + 3.0 / bench.F0) / dt)) + 1
    blocks = E[first:first + 100 * ((nt - first) // 100)].reshape(-1, 100).max(axis=1)
    assert len(blocks) >= 10   # the source stops near step 2390 of 4000
    ratios = blocks[1:] / blocks[:-1]
    assert ratios.max() <= 1 + 1e-6, ratios.max()


def _c1_geometry():
    n = 512
    dx = 1.0 / n
    dt = 0.5 * dx / np.sqrt(2.0)
    rcv_ix, rcv_iy = np.full(16, 128), 16 + 32 * np.arange(16)
    return n, dx, dt, rcv_ix, rcv_iy


@needs_ref
def test_c1_acoustic_512_periodic_matches_reference():
    n, dx, dt, rcv_ix, rcv_iy = _c1_geometry()
    case = refrun.AcousticCase(Nx=n, Ny=n, dx=dx, dt=dt, coef_vx=np.ones((n + 1, n)), coef_vy=np.ones((n, n + 1)),
                               coef_p=np.ones((n, n)), src=(n // 2, n // 2),
                               rcvs=[(2, int(a), int(b)) for a, b in zip(rcv_ix, rcv_iy)], Nt=1000, cpst="0",
                               central_f=10.0, time_delay=0.25)
    case.rho_vx, case.rho_vy = np.ones((n + 1, n)), np.ones((n, n + 1))
    want = refrun.run_acoustic(case, "f32")
    got = product_acoustic_periodic(case, "f32")
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    assert np.abs(want.traces).max() > 0
    assert energy_close(got["E_k"], want.energy[0] + want.energy[1])
    assert energy_close(got["E_p1"], want.energy[2])


@needs_ref
def test_c1_acoustic_512_free_surface_matches_reference_elastic_vs0():
    n, dx, dt, rcv_ix, rcv_iy = _c1_geometry()
    P = (n + 2, n + 2)
    case = refrun.ElasticCase(Mx=n, My=n, num_dx=1, den_dx=n, dt=dt, rho=np.ones(P).reshape(-1),
                              vp=np.ones(P).reshape(-1), vs=np.zeros(P).reshape(-1),
                              src=("M", "M", 2 * (n // 2) + 1, 2 * n, 2 * (n // 2) + 1, 2 * n),
                              rcvs=[("M", "M", 2 * int(a) + 1, 2 * n, 2 * int(b) + 1, 2 * n)
                                    for a, b in zip(rcv_ix, rcv_iy)],
                              Nt=1000, cpst="00", central_f=10.0, time_delay=0.25)
    want = refrun.run_elastic(case, "f32")
    assert np.array_equal(want.fields["MM0"], want.fields["MM1"])
    got = product_elastic(case, "f32", acoustic=True, energy=False)
    for k in ("MN", "NM", "MM0"):
        assert np.array_equal(got["fields"][k], want.fields[k]), k
    assert np.array_equal(got["traces"][:, 0], want.traces[:, 0])
    assert np.abs(want.traces).max() > 0
