"""Pin the oracle: the plain-C restatement (oracle/twave_oracle.c) must reproduce the reference's
own solvers bit for bit, against the committed golden fixtures (generated from the reference by
tests/golden/make_golden.py) and, where the reference binaries are present, against fresh runs."""
import json
import os

import numpy as np
import pytest

from cases import ROOT, acoustic_periodic_case, elastic_case
from conftest import has_ref_binaries
from oracle import oracle as orc
from oracle import refrun

GOLDEN = os.path.join(ROOT, "tests", "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))


def golden_elastic_case(d):
    return refrun.ElasticCase(Mx=int(d["Mx"]), My=int(d["My"]), num_dx=int(d["num_dx"]), den_dx=int(d["den_dx"]),
                              dt=float(d["dt"]), rho=d["rho"], vp=d["vp"], vs=d["vs"],
                              src=tuple(json.loads(str(d["src"]))), rcvs=[tuple(r) for r in json.loads(str(d["rcvs"]))],
                              Nt=int(d["Nt"]), cpst=str(d["cpst"]), central_f=float(d["central_f"]),
                              time_delay=float(d["time_delay"]), bc_x=str(d["bc_x"]) if "bc_x" in d else "F")


def golden_acoustic_case(d):
    c = refrun.AcousticCase(Nx=int(d["Nx"]), Ny=int(d["Ny"]), dx=float(d["dx"]), dt=float(d["dt"]),
                            coef_vx=1.0 / d["rho_vx"], coef_vy=1.0 / d["rho_vy"], coef_p=d["coef_p"],
                            src=tuple(int(v) for v in d["src"]), rcvs=[tuple(int(v) for v in r) for r in d["rcvs"]],
                            Nt=int(d["Nt"]), cpst=str(d["cpst"]), central_f=float(d["central_f"]),
                            time_delay=float(d["time_delay"]))
    c.rho_vx, c.rho_vy = d["rho_vx"], d["rho_vy"]
    return c


@pytest.mark.parametrize("name", [n for n, m in MANIFEST.items() if m["kind"] == "elastic"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_oracle_matches_golden_elastic(name, prec):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    r = orc.elastic_run(golden_elastic_case(d), prec)
    for k, v in r.fields.items():
        assert np.array_equal(v, d[f"{prec}_field_{k}"]), k
        if not (MANIFEST[name]["vs0"] and k == "NN"):   # shear stress stays zero when vs = 0
            assert np.abs(v).max() > 0, "fixture must exercise the field"
    for k, v in r.coefs.items():
        assert np.array_equal(v, d[f"{prec}_coef_{k}"]), k
    for k, v in r.weights.items():
        assert np.array_equal(v, d[f"{prec}_weight_{k}"], equal_nan=True), k
    assert np.array_equal(r.traces, d[f"{prec}_traces"])
    for k in ("E_k", "E_p0", "E_p1"):
        assert np.array_equal(getattr(r, k), d[f"{prec}_{k}"], equal_nan=True), k


@pytest.mark.parametrize("name", [n for n, m in MANIFEST.items() if m["kind"] == "acoustic_periodic"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_oracle_matches_golden_acoustic(name, prec):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    r = orc.acoustic_periodic_run(golden_acoustic_case(d), prec)
    for k, v in r.fields.items():
        assert np.array_equal(v, d[f"{prec}_field_{k}"]), k
    assert np.array_equal(r.traces, d[f"{prec}_traces"])
    assert np.array_equal(r.energy, d[f"{prec}_energy"])


def test_vs0_gives_identical_normal_stresses():
    """The acoustic limit of the elastic reference: sxx == syy bit for bit when vs = 0."""
    for name in ("el_20x16_vs0", "el_20x16_if_vs0"):
        d = np.load(os.path.join(GOLDEN, name + ".npz"))
        for prec in ("f64", "f32"):
            assert np.array_equal(d[f"{prec}_field_MM0"], d[f"{prec}_field_MM1"])
            assert not np.any(d[f"{prec}_field_NN"])


@pytest.mark.skipif(not has_ref_binaries(), reason="reference binaries (oracle/_ref) not built")
@pytest.mark.parametrize("Mx,My,cpst,seed", [(13, 11, "6R", 11), (26, 9, "3R", 12), (9, 33, "-3C", 13), (30, 22, "00", 14)])
def test_oracle_matches_live_reference(Mx, My, cpst, seed):
    case = elastic_case(Mx, My, seed=seed, cpst=cpst, Nt=45, model="layered")
    for prec in ("f64", "f32"):
        ref = refrun.run_elastic(case, prec)
        got = orc.elastic_run(case, prec)
        for k in ref.fields:
            assert np.array_equal(ref.fields[k], got.fields[k]), (prec, k)
        assert np.array_equal(ref.traces, got.traces)
        assert np.array_equal(ref.E_k, got.E_k) and np.array_equal(ref.E_p1, got.E_p1)


@pytest.mark.skipif(not has_ref_binaries(), reason="reference binaries (oracle/_ref) not built")
def test_reference_warm_up_pass_leaves_outputs_unchanged():
    """The benchmark's reference arm times the pass after an untimed one: that pass starts
    from rest again and must give the outputs of a single pass, bit for bit."""
    import dataclasses
    case = elastic_case(17, 12, seed=15, cpst="00", Nt=30, model="layered")
    one = refrun.run_elastic(case, "f32", perf=True)
    two = refrun.run_elastic(dataclasses.replace(case, warm_passes=1), "f32", perf=True)
    for k in one.fields:
        assert np.array_equal(one.fields[k], two.fields[k]), k
    assert np.array_equal(one.traces, two.traces)
    for a, b in ((one.E_k, two.E_k), (one.E_p0, two.E_p0), (one.E_p1, two.E_p1)):
        assert np.array_equal(a, b)


@pytest.mark.skipif(not has_ref_binaries(), reason="reference binaries (oracle/_ref) not built")
def test_oracle_matches_live_reference_acoustic():
    case = acoustic_periodic_case(14, 22, seed=21, cpst="6", Nt=40)
    for prec in ("f64", "f32"):
        ref = refrun.run_acoustic(case, prec)
        got = orc.acoustic_periodic_run(case, prec)
        for k in ref.fields:
            assert np.array_equal(ref.fields[k], got.fields[k]), (prec, k)
        assert np.array_equal(ref.energy, got.energy)


def test_location_mapping_edges():
    """forward.cpp:31-51: N-type locations are multiples of dx, M-type ones are half-cell offsets."""
    assert orc.location_to_index("N", 3, 50, 1, 50) == 3
    assert orc.location_to_index("M", 7, 100, 1, 50) == 3
    assert orc.location_to_index("N", 0, 1, 1, 50) == 0
    with pytest.raises(ValueError):
        orc.location_to_index("N", 7, 100, 1, 50)
    with pytest.raises(ValueError):
        orc.location_to_index("M", 3, 50, 1, 50)
