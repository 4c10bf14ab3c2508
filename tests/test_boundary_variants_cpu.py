"""Boundary variants beyond the reference's runs, on the oracle (CPU):

* the two x ends joined by the SBP-SAT interface penalty: the branch of the reference's
  secure_bdry for a boundary type other than 'F' (grid_drvt.tpp:575-693). The reference's inputs
  never select it, but its own solver runs it when the harness sets the type, so the restatement
  is pinned bit for bit (golden fixtures `*_if_*` and, where built, live runs);
* free surfaces on all four sides (closures and penalties along y as along x): no reference run,
  so parity is unpinned; the checks are the discrete energy after the source has stopped and the
  x <-> y transposition symmetry of the scheme.
"""
import numpy as np
import pytest

from cases import elastic_case
from conftest import has_ref_binaries
from oracle import oracle as orc
from oracle import refrun


def energy_after_source(case, r):
    E = r.E_k + 0.5 * (r.E_p0 + r.E_p1)
    return E[int((case.time_delay + 3.0 / case.central_f) / case.dt) + 1:]


@pytest.mark.skipif(not has_ref_binaries(), reason="reference binaries (oracle/_ref) not built")
@pytest.mark.parametrize("Mx,My,cpst,seed,ac", [(26, 14, "00", 31, False), (13, 11, "6R", 32, False),
                                                 (30, 9, "3C", 33, False), (16, 16, "00", 34, True)])
def test_interface_oracle_matches_live_reference(Mx, My, cpst, seed, ac):
    case = elastic_case(Mx, My, seed=seed, cpst=cpst, Nt=90, model="layered", acoustic=ac)
    case.bc_x = "I"
    for prec in ("f64", "f32"):
        ref = refrun.run_elastic(case, prec)
        got = orc.elastic_run(case, prec)
        for k, v in ref.fields.items():
            assert np.array_equal(got.fields[k], v), (prec, k)
        assert np.array_equal(got.traces, ref.traces)
        for k in ("E_k", "E_p0", "E_p1"):
            assert np.array_equal(getattr(got, k), getattr(ref, k), equal_nan=True), k


def test_interface_changes_the_x_ends_only_through_the_penalty():
    """Before the wave reaches an x end the interface run equals the free-surface run; after it,
    the interface couples the two ends (the NN grid, unpenalised under free surfaces, differs)."""
    case = elastic_case(48, 24, seed=35, Nt=4, model="layered", rcvs=[])   # reach: 4 rows a step
    free = orc.elastic_run(case, "f64")
    case.bc_x = "I"
    inter = orc.elastic_run(case, "f64")
    for k in free.fields:
        assert np.array_equal(free.fields[k], inter.fields[k]), k
    case.Nt = 400
    inter = orc.elastic_run(case, "f64")
    case.bc_x = "F"
    free = orc.elastic_run(case, "f64")
    assert not np.array_equal(free.fields["NN"][0], inter.fields["NN"][0])


@pytest.mark.parametrize("Mx,My,seed,model,bc", [(48, 40, 3, "layered", "F"), (40, 56, 5, "random", "F"),
                                                 (33, 41, 9, "random", "I"), (64, 32, 7, "layered", "I")])
def test_all_sides_energy_is_bounded(Mx, My, seed, model, bc):
    """Free surfaces on all four sides: after the source stops, the discrete energy (kinetic plus
    the mean of the potential energies around it) stays within 1 % over 3000 steps and no
    100-step block exceeds the previous block's maximum by more than 0.2 %."""
    case = elastic_case(Mx, My, seed=seed, Nt=3000, model=model, rcvs=[])
    case.bc_x, case.sat_y = bc, True
    r = orc.elastic_run(case, "f64")
    E = energy_after_source(case, r)
    assert np.all(np.isfinite(E)) and E[0] > 0
    assert E.min() / E.max() > 0.99
    blocks = [E[i:i + 100].max() for i in range(0, len(E) - 99, 100)]
    assert max(b / a for a, b in zip(blocks, blocks[1:])) < 1.002


def transpose_case(case):
    """The same problem with data x and y exchanged (Mx == My)."""
    n = case.Mx + 2
    t = elastic_case(case.Mx, case.My, Nt=case.Nt, rcvs=[])
    for k in ("rho", "vp", "vs"):
        setattr(t, k, np.ascontiguousarray(getattr(case, k).reshape(n, n).T).reshape(-1))
    s = case.src
    t.src = (s[1], s[0], s[4], s[5], s[2], s[3])
    t.dt, t.time_delay, t.central_f, t.cpst = case.dt, case.time_delay, case.central_f, case.cpst
    t.sat_y = case.sat_y
    return t


@pytest.mark.parametrize("prec,tol", [("f64", 1e-11), ("f32", 2e-4)])
def test_all_sides_is_symmetric_under_transposition(prec, tol):
    """With free surfaces on all four sides the scheme treats x and y alike: the run of the
    transposed medium and source is the transposed run (NN -> NN^T, MN <-> NM^T, sxx <-> syy^T),
    up to the rounding of the terms' order. This holds the y closures and penalties against the
    x ones, which the reference pins."""
    case = elastic_case(28, 28, seed=36, Nt=300, model="random", rcvs=[],
                        src=("M", "M", 2 * 9 + 1, 2 * 28, 2 * 15 + 1, 2 * 28))
    case.sat_y = True
    a = orc.elastic_run(case, prec)
    b = orc.elastic_run(transpose_case(case), prec)
    pairs = (("NN", "NN"), ("MN", "NM"), ("NM", "MN"), ("MM0", "MM1"), ("MM1", "MM0"))
    scale = max(np.abs(v).max() for v in a.fields.values())
    for ka, kb in pairs:
        assert np.abs(a.fields[ka] - b.fields[kb].T).max() <= tol * scale, (ka, kb)
    # the waves have reached all four sides
    assert np.abs(a.fields["NM"][0]).max() > 1e-3 * scale and np.abs(a.fields["MN"][:, 0]).max() > 1e-3 * scale
