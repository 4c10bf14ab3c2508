"""The TMA-staged fused elastic step (FP32, plain update): grids around its strip geometry.

Strips of 120 core columns start at column 56; the columns before them and from the end of the
last strip to the seam column My are stepped by warp strips. The widths below put the last
strip's end at, just below and just above the seam, with one strip or several; rows give one or
many segments. Every field carries random data, receivers sit on both sides of every strip edge,
on the seam and on segment edges, and the source sits in a strip. Fields, traces and energies are
compared with the C restatement (bit for bit; energies 1e-12) and with the per-warp kernel
(TW_TMA=0), which must agree bit for bit too. The warp strips run both ways: as the first work
items of the strips' launch and in the side launch (TW_TMA_WITEMS).
"""
import os

import numpy as np
import pytest

from cases import elastic_case, product_elastic
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _rcv(tx, ty, ix, iy, den):
    loc = lambda t, i: (i, den) if t == "N" else (2 * i + 1, 2 * den)
    (nx, dx_), (ny, dy_) = loc(tx, ix), loc(ty, iy)
    return (tx, ty, nx, dx_, ny, dy_)


def _case(Mx, My, seed):
    den = max(Mx, My)
    n_t = (My - 180) // 120 + 1 if My >= 180 else 0
    y_end = 56 + 120 * n_t
    cols = sorted({0, 1, 3, 54, 55, 56, 57, 59, 175, 176, 177, y_end - 2, y_end - 1, y_end, y_end + 1, My - 1})
    cols = [c for c in cols if 0 <= c < My]
    rows = sorted({8, 9, Mx // 3, Mx // 2, Mx - 9, Mx - 8})
    rcvs = []
    for k, c in enumerate(cols):
        r = rows[k % len(rows)]
        rcvs += [_rcv("N", "M", r, c, den), _rcv("M", "N", r, c, den), _rcv("M", "M", r, c, den)]
    rcvs += [_rcv("N", "N", Mx // 2, My, den), _rcv("M", "N", Mx // 2, My, den)]
    src = _rcv("M", "M", Mx // 2, min(100, My - 10), den)
    case = elastic_case(Mx, My, seed=seed, Nt=4, rcvs=rcvs, src=src, den_dx=den)
    return case


def _random_state(Mx, My, seed):
    rng = np.random.default_rng(seed)
    shapes = [(Mx + 1, My + 1), (Mx, My + 1), (Mx + 1, My), (Mx, My), (Mx, My)]
    return [(rng.standard_normal(s) * 1e-2).astype(np.float32).astype(np.float64) for s in shapes]


@pytest.mark.parametrize("witems", ["1", "0"])
@pytest.mark.parametrize("energy", [False, True])
@pytest.mark.parametrize("Mx,My", [(24, 180), (40, 299), (33, 300), (57, 301), (100, 420), (26, 1000), (300, 181)])
def test_tma_step_matches_restatement_and_warp_kernel(Mx, My, energy, witems, monkeypatch):
    case = _case(Mx, My, seed=Mx + 7 * My)
    f0 = _random_state(Mx, My, Mx * My)
    monkeypatch.setenv("TW_TMA_WITEMS", witems)   # the warp strips in the strips' launch, or the side launch
    want = orc.elastic_run(case, "f32", fields0=f0)
    os.environ["TW_TMA"] = "1"
    try:
        got = product_elastic(case, "f32", fields0=f0, energy=energy)
    finally:
        del os.environ["TW_TMA"]
    for k, v in got["fields"].items():
        assert np.array_equal(v, want.fields[k]), k
    assert np.array_equal(got["traces"], want.traces)
    if energy:
        for k in ("E_k", "E_p0", "E_p1"):
            ref = getattr(want, k)
            assert np.abs(got[k] - ref).max() <= 1e-12 * np.abs(ref).max(), k
    os.environ["TW_TMA"] = "0"
    try:
        warp = product_elastic(case, "f32", fields0=f0, energy=energy)
    finally:
        del os.environ["TW_TMA"]
    for k, v in got["fields"].items():
        assert np.array_equal(v, warp["fields"][k]), k
    assert np.array_equal(got["traces"], warp["traces"])
