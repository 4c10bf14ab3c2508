"""Mixed precision on the GPU: BF16 / FP16 field storage with FP32 arithmetic.

Two codes: "00" stores each new value rounded to 16 bits; "split" stores the pair hi + lo (lo =
the rounded remainder) and every read takes their FP32 sum, a compensated (Kahan-style) storage
of about 16 (BF16) or 22 (FP16) significant bits. Fields and traces must equal the oracle's
mixed-precision restatement bit for bit (energies: FP64 sums, relative 1e-12), and the split
code must stay close to an FP64 run of the same scheme: within 1e-4 (relative L2) with FP16
storage, 1e-3 with BF16.
"""
import ctypes

import numpy as np
import pytest

from cases import elastic_case, load_twave, product_elastic
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
E_RTOL = 1e-12
KEYS = ("NN", "MN", "NM", "MM0", "MM1")


def round16(a, prec):
    import torch
    t = torch.tensor(np.asarray(a, np.float32))
    return t.to(torch.bfloat16 if prec == "bf16" else torch.float16).to(torch.float32).double().numpy()


def _state(Mx, My, seed, prec, cpst, scale=1e-2):
    rng = np.random.default_rng(seed)
    shapes = [(Mx + 1, My + 1), (Mx, My + 1), (Mx + 1, My), (Mx, My), (Mx, My)]
    f = [(rng.standard_normal(s) * scale).astype(np.float32).astype(np.float64) for s in shapes]
    # plain 16-bit storage holds 16-bit values; the split pair is formed from the FP32 value
    return [round16(a, prec) for a in f] if cpst == "00" else f


def energy_close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= E_RTOL * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("cpst", ["00", "split"])
@pytest.mark.parametrize("prec", ["bf16", "fp16"])
@pytest.mark.parametrize("Mx,My,Nt", [(24, 40, 3), (37, 45, 3), (8, 4, 3), (70, 500, 6)])
def test_mixed_matches_oracle(cpst, prec, Mx, My, Nt):
    den = max(Mx, My)
    rcvs = [("N", "M", 2, den, 2 * (My - 1) + 1, 2 * den), ("M", "M", 2 * (Mx // 2) + 1, 2 * den, 2 * (My // 2) + 1, 2 * den),
            ("N", "N", Mx, den, My, den), ("M", "N", 2 * (Mx - 1) + 1, 2 * den, 0, 1)]
    case = elastic_case(Mx, My, seed=Mx + My, cpst=cpst, Nt=Nt, rcvs=rcvs)
    f0 = _state(Mx, My, 3, prec, cpst)
    want = orc.elastic_run(case, prec, fields0=f0)
    got = product_elastic(case, prec, fields0=f0)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    if cpst == "split":
        for k, v in zip(KEYS, got["resid"]):
            assert np.array_equal(v, want.resid[k]), ("lo", k)
    assert np.array_equal(got["traces"], want.traces)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


def test_split_storage_error_against_fp64():
    """A source-driven run from rest on a layered medium (160 x 160, 1200 steps): relative L2
    error of all fields together and of the traces against FP64. FP16 split storage meets 1e-4
    (measured on a B200: 1.3e-5); BF16 split storage does not (4.8e-4: 16 significant bits) and is
    held to 1e-3; plain 16-bit storage drifts far more (BF16 0.36, FP16 0.05) and is only checked
    for sanity. FP16 coefficients quantise the medium itself (measured 8.0e-4 here, with FP32 or
    FP16-split fields alike) and are held to 2e-3."""
    Mx = My = 160
    den = 500
    rcvs = [("N", "M", 8, den, 2 * k + 1, 2 * den) for k in range(4, My, 16)]
    base = dict(Nt=1200, model="layered", den_dx=den, rcvs=rcvs, time_delay=0.06)
    ref = product_elastic(elastic_case(Mx, My, seed=9, **base), "f64", energy=False)
    errs = {}
    for prec in ("bf16", "fp16"):
        for cpst in ("00", "split"):
            got = product_elastic(elastic_case(Mx, My, seed=9, cpst=cpst, **base), prec, energy=False)
            num = sum(np.sum((got["fields"][k] - ref["fields"][k]) ** 2) for k in KEYS)
            den_ = sum(np.sum(ref["fields"][k] ** 2) for k in KEYS)
            tr = np.linalg.norm(got["traces"] - ref["traces"]) / np.linalg.norm(ref["traces"])
            errs[(prec, cpst)] = (np.sqrt(num / den_), tr)
    print({k: f"{v[0]:.2e}/{v[1]:.2e}" for k, v in errs.items()})
    for prec, cpst in (("f32", "00"), ("fp16", "split")):   # FP16 coefficients
        got = product_elastic(elastic_case(Mx, My, seed=9, cpst=cpst, **base), prec, energy=False, coef_fp16=True)
        num = sum(np.sum((got["fields"][k] - ref["fields"][k]) ** 2) for k in KEYS)
        den_ = sum(np.sum(ref["fields"][k] ** 2) for k in KEYS)
        tr = np.linalg.norm(got["traces"] - ref["traces"]) / np.linalg.norm(ref["traces"])
        errs[(prec + "+c16", cpst)] = (np.sqrt(num / den_), tr)
    print({k: f"{v[0]:.2e}/{v[1]:.2e}" for k, v in errs.items()})
    for key in (("f32+c16", "00"), ("fp16+c16", "split")):
        assert errs[key][0] <= 2e-3 and errs[key][1] <= 2e-3, errs
    bound = {"fp16": 1e-4, "bf16": 1e-3}
    for prec in ("bf16", "fp16"):
        assert errs[(prec, "split")][0] <= bound[prec] and errs[(prec, "split")][1] <= bound[prec], errs
        assert errs[(prec, "00")][0] < 1.0, errs
    assert errs[("fp16", "split")][0] < errs[("bf16", "split")][0]


def fp16_material(case):
    """Stepping coefficients and energy weights as FP16 coefficient storage keeps them: each FP64
    quantity rounded to FP32, then to FP16; the weights follow from the stored values."""
    mu, rho_mn, rho_nm, lam, m2 = orc.material(case)
    h = lambda x: np.asarray(x, np.float64).astype(np.float32).astype(np.float16).astype(np.float32)
    coefs = {"NN_mu": h(mu), "MN_irho": h(1.0 / rho_mn), "NM_irho": h(1.0 / rho_nm), "MM_lambda": h(lam), "MM_2mu": h(m2)}
    Mx, My = case.Mx, case.My
    w = [np.zeros((Mx + 1, My + 1)), np.zeros((Mx, My + 1)), np.zeros((Mx + 1, My)), np.zeros((Mx, My)), np.zeros((Mx, My))]
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    stored = [h(mu), h(rho_mn), h(rho_nm), h(lam), h(m2)]
    orc.lib().two_energy_weights_f32(ctypes.c_int(Mx), ctypes.c_int(My), ctypes.c_double(case.num_dx / case.den_dx),
                                     *[p(a) for a in stored], *[p(a) for a in w])
    return coefs, dict(zip(("NN", "MN", "NM", "MM_P1", "MM_P2"), w))


@pytest.mark.parametrize("prec,cpst", [("f32", "00"), ("fp16", "split"), ("bf16", "00")])
@pytest.mark.parametrize("Mx,My,Nt", [(24, 40, 3), (70, 500, 6)])
def test_fp16_coefficients_match_oracle(prec, cpst, Mx, My, Nt):
    den = max(Mx, My)
    rcvs = [("N", "M", 2, den, 2 * (My - 1) + 1, 2 * den), ("M", "M", 2 * (Mx // 2) + 1, 2 * den, 2 * (My // 2) + 1, 2 * den)]
    case = elastic_case(Mx, My, seed=Mx * 3 + My, cpst=cpst, Nt=Nt, rcvs=rcvs)
    f0 = _state(Mx, My, 5, prec if prec != "f32" else "fp16", cpst) if prec != "f32" else \
        [a.astype(np.float32).astype(np.float64) for a in _state(Mx, My, 5, "fp16", "split")]
    coefs, weights = fp16_material(case)
    want = orc.elastic_run(case, prec, fields0=f0, coefs=coefs, weights=weights)
    got = product_elastic(case, prec, fields0=f0, coef_fp16=True)
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    for k in ("E_k", "E_p0", "E_p1"):
        assert energy_close(got[k], getattr(want, k)), k


def test_fp16_coefficients_reject_a_medium_outside_their_range():
    tw = load_twave()
    case = elastic_case(24, 20, seed=2, Nt=3)
    s = tw.Solver(24, 20, 1, 24, case.dt, coef_fp16=True, max_steps=3)
    shp = (26, 22)
    with pytest.raises(tw.TwError) as e:   # lambda ~ rho vp^2 ~ 2e6: above the FP16 range
        s.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp) * 1000, case.vs.reshape(shp) * 1000)
    assert e.value.code == -10
    s.close()


@pytest.mark.parametrize("energy", [False, True])
@pytest.mark.parametrize("Mx,My", [(40, 300), (57, 421)])
def test_fixed_point_coefficients_match_oracle(Mx, My, energy):
    """Coefficients stored as 16-bit codes on a per-array affine map (coef_fp16 = 2): every decoded
    value lies within half a step of the FP32 coefficient, and the run equals the restatement given
    the decoded coefficients bit for bit (fields, traces; energies to 1e-12)."""
    tw = load_twave()
    den = max(Mx, My)
    rcvs = [("N", "M", 9, den, 2 * 100 + 1, 2 * den), ("M", "M", 2 * (Mx // 2) + 1, 2 * den, 2 * 177 + 1, 2 * den),
            ("N", "N", Mx // 3, den, My, den), ("M", "N", 2 * 11 + 1, 2 * den, 0, 1)]
    case = elastic_case(Mx, My, seed=Mx * My, Nt=5, rcvs=rcvs, den_dx=den)
    shp = (Mx + 2, My + 2)
    keys = [(tw.NN, 0, "NN_mu"), (tw.MN, 0, "MN_irho"), (tw.NM, 0, "NM_irho"), (tw.MM, 0, "MM_lambda"), (tw.MM, 1, "MM_2mu")]

    def handle(q16):
        s = tw.Solver(Mx, My, 1, den, case.dt, precision="f32", cpst="00", central_f=case.central_f,
                      time_delay=case.time_delay, max_steps=case.Nt, energy=energy, coef_q16=q16)
        s.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), case.vs.reshape(shp))
        s.set_source_location(*case.src)
        for r in case.rcvs:
            s.add_receiver_location(*r)
        return s
    plain = handle(False)
    full = {name: plain.read_coefficients(g, i) for g, i, name in keys}
    plain.close()
    s = handle(True)
    try:
        dec = {name: s.read_coefficients(g, i) for g, i, name in keys}
        for name in dec:
            lo, hi = full[name].min(), full[name].max()
            step = np.float32((hi - lo) / 65535.0)
            assert np.abs(dec[name] - full[name]).max() <= 0.5 * step * (1 + 1e-3) + 4 * np.spacing(np.float32(hi)), name
        f0 = [(a * 0.1).astype(np.float32).astype(np.float64) for a in _state(Mx, My, 7, "f32", "split")]
        for (g, f), a in zip([(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)], f0):
            s.write_field(g, f, a)
        s.run(case.Nt)
        got = [s.read_field(g, f) for g, f in [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]]
        traces = s.read_receivers()
        E = s.read_energy() if energy else None
    finally:
        s.close()
    want = orc.elastic_run(case, "f32", fields0=f0, coefs=dec)
    for k, v in zip(KEYS, got):
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(traces, want.traces)
    if energy:
        for k, v in zip(("E_k", "E_p0", "E_p1"), E):
            assert energy_close(v, getattr(want, k)), k
