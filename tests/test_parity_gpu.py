"""Parity of the CUDA product (through the C ABI) with the reference.

Fields and receiver traces must be bit-identical to the reference's FP64 and FP32 CPU solvers
(golden fixtures) and to the C restatement (random states, every compensation code, sources on
every grid). Energies are FP64 sums taken in a different order: relative tolerance 1e-12.
"""
import json
import os

import numpy as np
import pytest

from cases import ROOT, acoustic_periodic_case, elastic_case, product_acoustic_periodic, product_elastic
from oracle import oracle as orc
from test_oracle_reference import MANIFEST, golden_acoustic_case, golden_elastic_case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(ROOT, "tests", "golden")
E_RTOL = 1e-12


def energy_close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= E_RTOL * scale


@pytest.mark.parametrize("name", [n for n, m in MANIFEST.items() if m["kind"] == "elastic" and not m["vs0"]])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_elastic_matches_reference_golden(name, prec):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    got = product_elastic(golden_elastic_case(d), prec)
    for k, v in got["fields"].items():
        assert np.array_equal(v, d[f"{prec}_field_{k}"]), k
    assert np.array_equal(got["traces"], d[f"{prec}_traces"])
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], d[f"{prec}_{k}"]), k


@pytest.mark.parametrize("name", ["el_20x16_vs0", "el_20x16_if_vs0"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_free_surface_matches_reference_vs0(name, prec):
    """Acoustic with SAT free surfaces (or the x ends joined by the SAT interface) = the reference
    elastic solver with vs = 0 (p = sxx = syy)."""
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = golden_elastic_case(d)
    keep = [i for i, r in enumerate(case.rcvs) if (r[0], r[1]) != ("N", "N")]
    case.rcvs = [case.rcvs[i] for i in keep]
    got = product_elastic(case, prec, acoustic=True)
    for k in ("MN", "NM", "MM0"):
        assert np.array_equal(got["fields"][k], d[f"{prec}_field_{k}"]), k
    ref_tr = d[f"{prec}_traces"][keep]
    assert np.array_equal(got["traces"][:, 0], ref_tr[:, 0])
    assert np.array_equal(got["E_k"], got["E_k"]) and energy_close(got["E_k"], d[f"{prec}_E_k"])


@pytest.mark.parametrize("name", [n for n, m in MANIFEST.items() if m["kind"] == "acoustic_periodic"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_periodic_matches_reference_golden(name, prec):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    got = product_acoustic_periodic(golden_acoustic_case(d), prec)
    for k, v in got["fields"].items():
        assert np.array_equal(v, d[f"{prec}_field_{k}"]), k
    assert np.array_equal(got["traces"], d[f"{prec}_traces"])
    e = d[f"{prec}_energy"]
    assert energy_close(got["E_k"], e[0] + e[1])
    assert energy_close(got["E_p1"], e[2])


def _random_state(Mx, My, seed, scale=1e-2):
    """Random fields at reference sizes; the periodic seam column of the N-type-y grids is an
    independent point in the reference, so it is drawn independently too."""
    rng = np.random.default_rng(seed)
    shapes = [(Mx + 1, My + 1), (Mx, My + 1), (Mx + 1, My), (Mx, My), (Mx, My)]
    return [rng.standard_normal(s) * scale for s in shapes]


CPST_CODES = ["00", "-3C", "-3R", "3C", "3R", "6C", "6R"]


@pytest.mark.parametrize("cpst", CPST_CODES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("Mx,My", [(24, 40), (37, 45), (8, 4)])
def test_elastic_random_state_matches_oracle(cpst, prec, Mx, My):
    case = elastic_case(Mx, My, seed=Mx * My, cpst=cpst, Nt=3, rcvs=[])
    f0 = _random_state(Mx, My, 1)
    r0 = _random_state(Mx, My, 2, scale=1e-8) if cpst != "00" else None
    T = np.float64 if prec == "f64" else np.float32
    f0 = [a.astype(T).astype(np.float64) for a in f0]
    r0 = None if r0 is None else [a.astype(T).astype(np.float64) for a in r0]
    want = orc.elastic_run(case, prec, fields0=f0, resid0=r0)
    got = product_elastic(case, prec, fields0=f0, resid0=r0)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    if r0 is not None:
        for k, v in zip(("NN", "MN", "NM", "MM0", "MM1"), got["resid"]):
            assert np.array_equal(v, want.resid[k]), ("resid", k)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("src", [("N", "N", 5, 24, 7, 24), ("M", "N", 11, 48, 9, 24), ("N", "M", 13, 24, 15, 48),
                                 ("M", "M", 21, 48, 29, 48)])
def test_source_on_every_grid_matches_oracle(prec, src):
    case = elastic_case(24, 24, seed=3, Nt=50, src=src, den_dx=24, model="layered")
    want = orc.elastic_run(case, prec)
    got = product_elastic(case, prec)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)


@pytest.mark.parametrize("cpst", ["00", "6R", "3C"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_free_surface_random_state_matches_oracle(cpst, prec):
    Mx, My = 30, 36
    case = elastic_case(Mx, My, seed=5, cpst=cpst, Nt=4, rcvs=[], acoustic=True)
    T = np.float64 if prec == "f64" else np.float32
    rng = np.random.default_rng(9)
    p = rng.standard_normal((Mx, My)).astype(T).astype(np.float64) * 1e-2
    vmn = rng.standard_normal((Mx, My + 1)).astype(T).astype(np.float64) * 1e-2
    vnm = rng.standard_normal((Mx + 1, My)).astype(T).astype(np.float64) * 1e-2
    zero_nn = np.zeros((Mx + 1, My + 1))
    want = orc.elastic_run(case, prec, fields0=[zero_nn, vmn, vnm, p, p])
    got = product_elastic(case, prec, acoustic=True, fields0=[vmn, vnm, p])
    assert np.array_equal(want.fields["MM0"], want.fields["MM1"])
    for k in ("MN", "NM", "MM0"):
        assert np.array_equal(got["fields"][k], want.fields[k]), k


@pytest.mark.parametrize("cpst", ["0", "3", "6"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_periodic_matches_oracle(cpst, prec):
    case = acoustic_periodic_case(40, 36, seed=17, cpst=cpst, Nt=70)
    want = orc.acoustic_periodic_run(case, prec)
    got = product_acoustic_periodic(case, prec)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)


@pytest.mark.parametrize("cpst", ["0", "3", "6"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("Nx,Ny,Nt", [(40, 36, 70), (9, 5, 30), (70, 500, 12), (203, 61, 9)])
def test_fused_acoustic_periodic_matches_oracle(cpst, prec, Nx, Ny, Nt):
    """The one-launch periodic acoustic step (energy off): random initial state so every row and
    column carries data through the wrapped halos; fields, residuals and traces bit-identical."""
    case = acoustic_periodic_case(Nx, Ny, seed=Nx + Ny, cpst=cpst, Nt=Nt)
    rng = np.random.default_rng(Nx * Ny)
    T = np.float64 if prec == "f64" else np.float32
    shapes = [(Nx + 1, Ny), (Nx, Ny + 1), (Nx, Ny)]
    f0 = [rng.standard_normal(sh).astype(T).astype(np.float64) for sh in shapes]
    r0 = None if cpst == "0" else [(rng.standard_normal(sh) * 1e-8).astype(T).astype(np.float64) for sh in shapes]
    want = orc.acoustic_periodic_run(case, prec, fields0=f0, resid0=r0)
    got = product_acoustic_periodic(case, prec, fields0=f0, resid0=r0, energy=False)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    if r0 is not None:
        for k, v in zip(("Vx", "Vy", "P"), got["resid"]):
            assert np.array_equal(v, want.resid[k]), ("resid", k)


def test_errors_follow_the_reference_checks(tw):
    s = tw.Solver(16, 16, 1, 16, 1e-3, max_steps=5)
    try:
        with pytest.raises(tw.TwError) as e:
            s.step(1)                                   # no material yet
        assert e.value.code == -4
        with pytest.raises(tw.TwError) as e:
            s.set_source_location("N", "M", 0, 1, 1, 32)   # node row 0 is the free surface
        assert e.value.code == -7
        with pytest.raises(tw.TwError) as e:
            s.set_source_location("N", "M", 1, 32, 1, 32)  # 1/32 is not a node of dx = 1/16
        assert e.value.code == -5
        s.set_source(tw.NN, 3, 0)                       # the periodic seam is accepted, as in the reference
        with pytest.raises(tw.TwError) as e:
            s.add_receivers(tw.MM, [16], [0])           # outside the MM grid
        assert e.value.code == -6
        rho, vp, vs = (np.full((18, 18), v) for v in (2.0, 3.0, 1.5))
        s.set_material_model(rho, vp, vs)
        s.run(5)
        with pytest.raises(tw.TwError) as e:
            s.step(1)                                   # records hold 5 steps
        assert e.value.code == -8
    finally:
        s.close()


def test_nonfinite_value_is_reported_not_faulted(tw):
    """A NaN planted in a field from the host is reported by tw_sync; the context stays usable."""
    s = tw.Solver(16, 16, 1, 16, 1e-3, max_steps=10)
    try:
        rho, vp, vs = (np.full((18, 18), v) for v in (2.0, 3.0, 1.5))
        s.set_material_model(rho, vp, vs)
        f = np.zeros((16, 16))
        f[5, 5] = np.nan
        s.write_field(tw.MM, 0, f)
        s.step(2)
        with pytest.raises(tw.TwError) as e:
            s.sync()
        assert e.value.code == -9
        s.reset()
        s.run(2)
        assert np.isfinite(s.read_field(tw.MM)).all()
    finally:
        s.close()


@pytest.mark.parametrize("cpst", ["00", "6R", "3C"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_many_strips_and_segments_match_oracle(cpst, prec):
    """A grid wide and tall enough for several column strips and row segments of the one-launch
    step; receivers sit on strip and segment edges and on the periodic seam."""
    Mx, My = 70, 500
    den = 500
    rcvs = [("N", "M", 15, den, 2 * 247 + 1, 2 * den), ("N", "M", 16, den, 2 * 248 + 1, 2 * den),
            ("M", "M", 2 * 47 + 1, 2 * den, 2 * 495 + 1, 2 * den), ("N", "N", 48, den, My, den),
            ("M", "N", 2 * 69 + 1, 2 * den, 0, 1), ("N", "N", Mx, den, 248, den), ("N", "M", Mx, den, 2 * 499 + 1, 2 * den)]
    case = elastic_case(Mx, My, seed=77, cpst=cpst, Nt=6, den_dx=den, rcvs=rcvs,
                        src=("N", "M", 16, den, 2 * 248 + 1, 2 * den))
    T = np.float64 if prec == "f64" else np.float32
    f0 = [a.astype(T).astype(np.float64) for a in _random_state(Mx, My, 5)]
    r0 = None if cpst == "00" else [a.astype(T).astype(np.float64) for a in _random_state(Mx, My, 6, scale=1e-8)]
    want = orc.elastic_run(case, prec, fields0=f0, resid0=r0)
    got = product_elastic(case, prec, fields0=f0, resid0=r0)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_energy_before_a_step_follows_the_state_written_into_the_handle(tw, prec):
    """E_p0 of a step sums the stresses the step starts from: after 20 steps (graph replays
    included) E_p0 follows the previous step's E_p1, and after a stress field written into the
    handle, the next 20 steps' energies equal the oracle's from that state."""
    Mx, My = 40, 36
    case = elastic_case(Mx, My, seed=8, Nt=20, rcvs=[], model="layered")
    T = np.float64 if prec == "f64" else np.float32
    s = tw.Solver(Mx, My, case.num_dx, case.den_dx, case.dt, precision=prec, central_f=case.central_f,
                  time_delay=case.time_delay, max_steps=40)
    try:
        shp = (Mx + 2, My + 2)
        s.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), case.vs.reshape(shp))
        s.set_source_location(*case.src)
        s.run(20)
        keys = [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
        state = [s.read_field(g, f) for g, f in keys]
        state[3] = (state[3] + np.random.default_rng(1).standard_normal(state[3].shape) * 1e-3).astype(T).astype(np.float64)
        s.write_field(tw.MM, 0, state[3])
        s.run(20)
        E_k, E_p0, E_p1 = s.read_energy()
    finally:
        s.close()
    assert energy_close(E_p0[1:20], E_p1[:19])
    want = orc.elastic_run(case_shifted(case, 20), prec, fields0=state)
    for got, ref in ((E_p0[20:], want.E_p0), (E_k[20:], want.E_k), (E_p1[20:], want.E_p1)):
        assert energy_close(got, ref)
    assert not np.isclose(E_p0[20], E_p1[19], rtol=1e-6)   # the written state changed the energy


def case_shifted(case, k):
    """`case` started k steps later: the source's delay moves back by k dt."""
    import copy
    c = copy.copy(case)
    c.time_delay = case.time_delay - k * case.dt
    return c


@pytest.mark.parametrize("bc,sat_y", [("periodic", False), ("free", False), ("interface", True)])
@pytest.mark.parametrize("cpst", ["00", "6R"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_steps_agree_however_the_calls_split_them(tw, bc, sat_y, cpst, prec):
    """One step per call (launched directly) and calls of 5, 1 and 31 steps (the long one replays
    a captured graph of 16 steps) give the same fields and traces bit for bit."""
    Nx, Ny, Nt = 40, 36, 37
    case = acoustic_periodic_case(Nx, Ny, seed=23, cpst="0", Nt=Nt)
    bcx = {"periodic": tw.PERIODIC, "free": tw.SAT_FREE, "interface": tw.SAT_INTERFACE}[bc]
    out = []
    for calls in ([1] * Nt, [5, 1, 31]):
        s = tw.Solver(Nx, Ny, 1, max(Nx, Ny), case.dt, physics=tw.ACOUSTIC, bc_x=bcx, precision=prec, cpst=cpst,
                      central_f=case.central_f, time_delay=case.time_delay, max_steps=Nt, energy=False, sat_y=sat_y)
        try:
            s.set_material_grid(tw.NM, 0, case.rho_vx)
            s.set_material_grid(tw.MN, 0, case.rho_vy)
            s.set_material_grid(tw.MM, 0, np.asarray(case.coef_p).reshape(Nx, Ny))
            s.set_source(tw.MM, Nx // 2, Ny // 3)
            s.add_receivers(tw.MM, [3, 0, 20], [3, 5, Ny - 1])
            s.add_receivers(tw.NM, [0, Nx], [4, 7])
            s.add_receivers(tw.MN, [2], [Ny])
            for n in calls:
                s.step(n)
            s.sync()
            out.append(([s.read_field(g) for g in (tw.MN, tw.NM, tw.MM)], s.read_receivers()))
        finally:
            s.close()
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(out[0][1], out[1][1])
    assert np.abs(out[0][1]).max() > 0
