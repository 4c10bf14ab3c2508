"""Host-side checks that need no GPU: the C-ABI library loads, exports every entry point that
include/twave.h declares, validates arguments before touching the device, and maps rational
locations to grid indices exactly as the reference does."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc


def test_library_exports_every_declared_symbol(tw):
    names = tw.declared_symbols()
    assert len(names) >= 20
    L = tw.lib()
    for n in names:
        assert hasattr(L, n), n
    nm = subprocess.run(["nm", "-D", "--defined-only", tw.library_path()], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in nm.splitlines() if " T " in line}
    assert set(names) <= exported
    # the product never carries the oracle
    assert not any(s.startswith("two_") for s in exported)


def test_library_does_not_link_the_oracle(tw):
    out = subprocess.run(["ldd", tw.library_path()], capture_output=True, text=True).stdout
    assert "oracle" not in out


def test_strerror(tw):
    L = tw.lib()
    assert L.tw_strerror(0) == b"ok"
    assert b"weak boundary" in L.tw_strerror(-7)
    assert L.tw_strerror(12345) == b"unknown status"


def test_location_to_index_matches_reference_rule(tw):
    rng = np.random.default_rng(0)
    for _ in range(2000):
        t = "NM"[rng.integers(2)]
        num_dx, den_dx = int(rng.integers(1, 4)), int(rng.integers(1, 600))
        den = int(rng.integers(1, 2000))
        num = int(rng.integers(-50, 4000))
        try:
            want = orc.location_to_index(t, num, den, num_dx, den_dx)
        except ValueError:
            want = None
        try:
            got = tw.location_to_index(t, num, den, num_dx, den_dx)
        except tw.TwError as e:
            assert e.code == -5
            got = None
        assert got == want, (t, num, den, num_dx, den_dx)


def _desc(tw, **kw):
    base = dict(physics=0, bc_x=0, precision=1, cpst=0, Mx=64, My=64, num_dx=1, den_dx=64, dt=1e-3,
                central_f=5.0, time_delay=0.1, source_scaling=1.0, max_steps=10, energy=1, device=0)
    base.update(kw)
    return tw.GridDesc(**base)


@pytest.mark.parametrize("kw,code", [
    (dict(Mx=7), -1), (dict(My=3), -1), (dict(dt=0.0), -1), (dict(num_dx=0), -1), (dict(max_steps=0), -1),
    (dict(physics=5), -1), (dict(cpst=9), -1), (dict(source_scaling=0.0), -1),
    (dict(physics=0, bc_x=1), -10),                 # elastic needs the SAT x boundaries
    (dict(physics=1, bc_x=1, cpst=5), -10),         # the single-core tree has no 'C' compensation
    (dict(precision=4), -1),
    (dict(precision=2, cpst=4), -10),               # 16-bit storage: plain or split only
    (dict(precision=1, cpst=7), -10),               # the split pair needs 16-bit storage
    (dict(physics=1, precision=3), -10),            # 16-bit storage is elastic only
    (dict(coef_fp16=3), -1),
    (dict(coef_fp16=2), -10),                       # 16-bit coefficient codes need a TMA strip (My >= 180)
    (dict(coef_fp16=2, precision=0, My=256), -10),  # ... and FP32 fields
    (dict(coef_fp16=1, precision=0), -10),          # FP16 coefficients need FP32 arithmetic
    (dict(coef_fp16=1, cpst=6), -10),               # ... and the plain update
    (dict(coef_fp16=1, physics=1, bc_x=1), -10),    # ... and the elastic stepper
    (dict(bc_x=3), -1), (dict(sat_y=2), -1),
    (dict(sat_y=1, My=7), -1),                      # free y ends need 8 columns
    (dict(sat_y=1, physics=1, bc_x=1), -10),        # free y ends with periodic x
    (dict(bc_x=2, precision=2), -10),               # the variants: FP64 / FP32 storage
    (dict(sat_y=1, coef_fp16=1), -10),
])
def test_create_rejects_bad_descriptors_before_touching_the_device(tw, kw, code):
    h = C.c_void_p()
    assert tw.lib().tw_create(C.byref(h), C.byref(_desc(tw, **kw))) == code
    assert not h.value


def test_null_handles_are_rejected(tw):
    L = tw.lib()
    assert L.tw_step(None, 1) == -1
    assert L.tw_sync(None) == -1
    assert L.tw_reset(None) == -1
    L.tw_destroy(None)
