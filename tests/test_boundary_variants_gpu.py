"""Parity of the boundary variants on the GPU (the two-launch kernels, through the C ABI):

* the x ends joined by the SBP-SAT interface penalty (the reference's secure_bdry branch for a
  boundary type other than 'F', grid_drvt.tpp:575-693): bit-identical to the reference's own
  solver (golden fixtures `*_if_*`, in test_parity_gpu.py) and to the restatement here;
* free surfaces on all four sides (no reference run): bit-identical to the restatement, whose
  y operators the transposition test of test_boundary_variants_cpu.py holds to the x ones; from
  16 columns on they run on the fused step with the points next to the y ends recomputed, below
  on the two-launch kernels, and the sizes here cover both (and strips of several warps).

Energies are FP64 sums taken in a different order: relative tolerance 1e-12.
"""
import numpy as np
import pytest

from cases import elastic_case, load_twave, product_elastic
from oracle import oracle as orc
from test_parity_gpu import CPST_CODES, _random_state, energy_close

pytestmark = pytest.mark.gpu

MODES = [("I", False), ("F", True), ("I", True)]


@pytest.mark.parametrize("bc,sat_y", MODES)
@pytest.mark.parametrize("cpst", CPST_CODES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("Mx,My", [(24, 40), (37, 9), (8, 8), (30, 117)])
def test_elastic_variant_random_state_matches_oracle(bc, sat_y, cpst, prec, Mx, My):
    case = elastic_case(Mx, My, seed=Mx * My + 1, cpst=cpst, Nt=3, rcvs=[])
    case.bc_x, case.sat_y = bc, sat_y
    T = np.float64 if prec == "f64" else np.float32
    f0 = [a.astype(T).astype(np.float64) for a in _random_state(Mx, My, 3)]
    r0 = None if cpst == "00" else [a.astype(T).astype(np.float64) for a in _random_state(Mx, My, 4, scale=1e-8)]
    want = orc.elastic_run(case, prec, fields0=f0, resid0=r0)
    got = product_elastic(case, prec, fields0=f0, resid0=r0)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    if r0 is not None:
        for k, v in zip(("NN", "MN", "NM", "MM0", "MM1"), got["resid"]):
            assert np.array_equal(v, want.resid[k]), ("resid", k)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


@pytest.mark.parametrize("bc,sat_y", MODES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_elastic_variant_long_run_matches_oracle(bc, sat_y, prec):
    """A source and receivers on every grid, 400 steps: the waves cross all four sides."""
    rcvs = [("N", "M", 0, 1, 2 * 3 + 1, 2 * 32), ("M", "N", 2 * 5 + 1, 2 * 32, 0, 1), ("N", "N", 1, 1, 1, 2),
            ("M", "M", 2 * 30 + 1, 2 * 32, 2 * 20 + 1, 2 * 32), ("M", "N", 1, 64, 24, 32)]
    case = elastic_case(32, 24, seed=41, Nt=400, rcvs=rcvs, den_dx=32, model="layered")
    case.bc_x, case.sat_y = bc, sat_y
    want = orc.elastic_run(case, prec)
    got = product_elastic(case, prec)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


@pytest.mark.parametrize("bc,sat_y", MODES)
@pytest.mark.parametrize("cpst", ["00", "6R", "3C"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_variant_matches_elastic_vs0_oracle(bc, sat_y, cpst, prec):
    """The acoustic SAT kernels are the elastic scheme with mu = 0 under every boundary variant."""
    Mx, My = 30, 20
    case = elastic_case(Mx, My, seed=6, cpst=cpst, Nt=5, rcvs=[], acoustic=True)
    case.bc_x, case.sat_y = bc, sat_y
    T = np.float64 if prec == "f64" else np.float32
    rng = np.random.default_rng(10)
    p = rng.standard_normal((Mx, My)).astype(T).astype(np.float64) * 1e-2
    vmn = rng.standard_normal((Mx, My + 1)).astype(T).astype(np.float64) * 1e-2
    vnm = rng.standard_normal((Mx + 1, My)).astype(T).astype(np.float64) * 1e-2
    want = orc.elastic_run(case, prec, fields0=[np.zeros((Mx + 1, My + 1)), vmn, vnm, p, p])
    got = product_elastic(case, prec, acoustic=True, fields0=[vmn, vnm, p])
    assert np.array_equal(want.fields["MM0"], want.fields["MM1"])
    for k in ("MN", "NM", "MM0"):
        assert np.array_equal(got["fields"][k], want.fields[k]), k


def test_variant_rules():
    """A source on an end column of an N-type-y grid is on a weak boundary once y is free; the
    variants take FP64/FP32 storage."""
    tw = load_twave()
    s = tw.Solver(16, 16, 1, 16, 1e-3, sat_y=True, max_steps=4)
    try:
        for grid, ix, iy in ((tw.NN, 3, 0), (tw.MN, 3, 16)):
            with pytest.raises(tw.TwError) as e:
                s.set_source(grid, ix, iy)
            assert e.value.name == "TW_ERR_WEAK_BOUNDARY"
        s.set_source(tw.NM, 3, 0)   # M type along y: an ordinary point
    finally:
        s.close()
    for kw in ({"precision": "bf16"}, {"precision": "f32", "coef_fp16": True}):
        with pytest.raises(tw.TwError) as e:
            tw.Solver(16, 16, 1, 16, 1e-3, sat_y=True, max_steps=4, **kw)
        assert e.value.name == "TW_ERR_UNSUPPORTED"
