"""The oracle's mixed-precision restatement (CPU): every stored value is a 16-bit number (plain
code) or a pair hi + lo of 16-bit numbers with |lo| at most half a unit in the last place of hi
(split code), and the result stays close to the FP32 run."""
import numpy as np
import pytest

from cases import elastic_case
from oracle import oracle as orc

KEYS = ("NN", "MN", "NM", "MM0", "MM1")


def round16(a, prec):
    torch = pytest.importorskip("torch")
    t = torch.tensor(np.asarray(a, np.float32))
    return t.to(torch.bfloat16 if prec == "bf16" else torch.float16).to(torch.float32).double().numpy()


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
@pytest.mark.parametrize("cpst", ["00", "split"])
def test_stored_values_are_16_bit(prec, cpst):
    case = elastic_case(24, 20, seed=4, cpst=cpst, Nt=30, rcvs=[])
    r = orc.elastic_run(case, prec)
    f32 = orc.elastic_run(elastic_case(24, 20, seed=4, Nt=30, rcvs=[]), "f32")
    for k in KEYS:
        v = r.fields[k]
        if cpst == "00":
            assert np.array_equal(v, round16(v, prec)), k
        else:
            lo = r.resid[k]
            hi = (v.astype(np.float32) - lo.astype(np.float32)).astype(np.float64)
            assert np.array_equal(hi, round16(hi, prec)), k
            assert np.array_equal(lo, round16(lo, prec)), k
            # hi is v rounded (|lo| <= ulp(hi)/2); where v lies half-way, rounding may pick the neighbour
            rv = round16(v, prec)
            off = rv != hi
            assert np.array_equal(np.abs(rv - hi)[off], 2 * np.abs(lo)[off]), k
        scale = np.abs(f32.fields[k]).max()
        tol = {"bf16": 3e-2, "fp16": 5e-3}[prec] if cpst == "00" else {"bf16": 1e-4, "fp16": 1e-5}[prec]
        assert np.abs(v - f32.fields[k]).max() <= tol * scale, k
