"""Batched stepping of many acoustic shots (tw_batch_*) through the C ABI.

A batch advances shots of different sizes with one launch per half-step for all of them. Every
shot must come out bit-identical to the same handle stepped alone (which the parity tests pin
to the reference), for every launch shape the autotuner may pick, and small shots must also
equal the oracle's single-core restatement.
"""
import ctypes

import numpy as np
import pytest

from cases import acoustic_periodic_case, load_twave
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
CP = {"0": "00", "3": "3R", "6": "6R"}


def make_shot(tw, case, precision, energy=False, bc_x=None, sat_y=False):
    s = tw.Solver(case.Nx, case.Ny, 1, max(case.Nx, case.Ny), case.dt, physics=tw.ACOUSTIC,
                  bc_x=tw.PERIODIC if bc_x is None else bc_x, precision=precision, cpst=CP[case.cpst],
                  central_f=case.central_f, time_delay=case.time_delay, max_steps=max(case.Nt, 1) + 64,
                  energy=energy, sat_y=sat_y)
    s.set_material_grid(tw.NM, 0, case.rho_vx)
    s.set_material_grid(tw.MN, 0, case.rho_vy)
    s.set_material_grid(tw.MM, 0, np.asarray(case.coef_p).reshape(case.Nx, case.Ny))
    s.set_source(tw.MM, *case.src)
    grid = {0: tw.NM, 1: tw.MN, 2: tw.MM}
    for m, ix, iy in case.rcvs:
        s.add_receivers(grid[m], [ix], [iy])
    return s


def state(tw, s):
    return [s.read_field(g) for g in (tw.NM, tw.MN, tw.MM)], s.read_receivers()


SIZES = [(40, 36), (64, 64), (17, 90), (128, 40), (9, 5)]


@pytest.mark.parametrize("cpst", ["0", "3", "6"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_equals_each_shot_alone_and_the_oracle(cpst, prec):
    tw = load_twave()
    cases = [acoustic_periodic_case(nx, ny, seed=100 + k, cpst=cpst, Nt=37) for k, (nx, ny) in enumerate(SIZES)]
    alone = []
    for c in cases:
        s = make_shot(tw, c, prec)
        s.run(c.Nt)
        alone.append(state(tw, s))
        s.close()
    shots = [make_shot(tw, c, prec) for c in cases]
    b = tw.Batch(shots)
    b.run(cases[0].Nt)
    for k, (s, c) in enumerate(zip(shots, cases)):
        f, t = state(tw, s)
        for a, w in zip(f, alone[k][0]):
            assert np.array_equal(a, w), k
        assert np.array_equal(t, alone[k][1]), k
        want = orc.acoustic_periodic_run(c, prec)
        assert np.array_equal(f[2], want.fields["P"]), k
        assert np.array_equal(t[:, 0, :], want.traces), k
    b.close()
    for s in shots:
        s.close()


@pytest.mark.parametrize("shape", [(32, 8, 1, 0), (64, 4, 2, 0), (128, 2, 4, 3), (256, 1, 1, 1), (32, 1, 3, 7)])
def test_every_launch_shape_gives_the_same_result(shape):
    """Free-surface shots use the tiled per-point kernels, whose launch shape is free."""
    tw = load_twave()
    cases = [acoustic_periodic_case(nx, ny, seed=7 + k, cpst="6", Nt=20) for k, (nx, ny) in enumerate(SIZES)]
    ref_shots = [make_shot(tw, c, "f32", bc_x=tw.SAT_FREE) for c in cases]
    for s in ref_shots:
        s.run(20)
    ref = [state(tw, s) for s in ref_shots]
    b0 = None
    shots = [make_shot(tw, c, "f32", bc_x=tw.SAT_FREE) for c in cases]
    b = tw.Batch(shots)
    b.set_shape(*shape)
    assert b.shape() == shape[:3] + ((shape[3] or b.shape()[3]),)
    b.step(16)     # one graph replay
    b.step(4)      # eager remainder
    b.sync()
    for s, r in zip(shots, ref):
        f, t = state(tw, s)
        for a, w in zip(f, r[0]):
            assert np.array_equal(a, w)
        assert np.array_equal(t, r[1])
    for h in [b] + shots + ref_shots:
        h.close()


def test_batch_of_boundary_variants_equals_each_shot_alone():
    """Shots with the x ends joined by the SAT interface and with free y ends batch with the
    free-surface shots: each carries its variant in its own arguments."""
    tw = load_twave()
    modes = [(tw.SAT_INTERFACE, False), (tw.SAT_FREE, True), (tw.SAT_INTERFACE, True), (tw.SAT_FREE, False)]
    cases = [acoustic_periodic_case(nx, ny, seed=27 + k, cpst="3", Nt=60) for k, (nx, ny) in enumerate(SIZES[:4])]
    ref_shots = [make_shot(tw, c, "f64", bc_x=m[0], sat_y=m[1]) for c, m in zip(cases, modes)]
    for s in ref_shots:
        s.run(60)
    ref = [state(tw, s) for s in ref_shots]
    shots = [make_shot(tw, c, "f64", bc_x=m[0], sat_y=m[1]) for c, m in zip(cases, modes)]
    b = tw.Batch(shots)
    b.run(60)
    for s, r in zip(shots, ref):
        f, t = state(tw, s)
        for a, w in zip(f, r[0]):
            assert np.array_equal(a, w)
        assert np.array_equal(t, r[1])
    for h in [b] + shots + ref_shots:
        h.close()


@pytest.mark.parametrize("per_sm", [1, 3, 15, 40])
def test_fused_batch_segmentation_gives_the_same_result(per_sm):
    """Periodic shots step with the fused kernel; its segmentation target changes nothing."""
    tw = load_twave()
    cases = [acoustic_periodic_case(nx, ny, seed=17 + k, cpst="3", Nt=21) for k, (nx, ny) in enumerate(SIZES)]
    ref = []
    for c in cases:
        s = make_shot(tw, c, "f32")
        s.run(21)
        ref.append(state(tw, s))
        s.close()
    shots = [make_shot(tw, c, "f32") for c in cases]
    b = tw.Batch(shots)
    b.set_shape(0, 0, 0, per_sm)
    assert b.shape()[2] == per_sm
    b.step(16)
    b.step(5)
    b.sync()
    for s, r in zip(shots, ref):
        f, t = state(tw, s)
        for a, w in zip(f, r[0]):
            assert np.array_equal(a, w)
        assert np.array_equal(t, r[1])
    for h in [b] + shots:
        h.close()


def test_tune_picks_a_shape_and_resets_the_shots():
    tw = load_twave()
    cases = [acoustic_periodic_case(nx, ny, seed=3 + k, cpst="0", Nt=24) for k, (nx, ny) in enumerate(SIZES)]
    shots = [make_shot(tw, c, "f32") for c in cases]
    b = tw.Batch(shots)
    ms = b.tune(4)
    assert ms > 0
    for s in shots:
        assert s.info().steps_done == 0
        assert all(not np.any(f) for f in state(tw, s)[0])
    b.run(24)
    for s, c in zip(shots, cases):
        want = orc.acoustic_periodic_run(c, "f32")
        assert np.array_equal(s.read_field(tw.MM), want.fields["P"])
    for h in [b] + shots:
        h.close()


def test_shots_stay_usable_alone_after_batched_steps():
    tw = load_twave()
    c = acoustic_periodic_case(40, 36, seed=5, cpst="3", Nt=30)
    s1 = make_shot(tw, c, "f32")
    s1.run(30)
    want = state(tw, s1)
    s2 = make_shot(tw, c, "f32")
    b = tw.Batch([s2])
    b.step(18)
    s2.step(12)    # ordered after the batch on the shot's own stream
    s2.sync()
    got = state(tw, s2)
    for a, w in zip(got[0], want[0]):
        assert np.array_equal(a, w)
    assert np.array_equal(got[1], want[1])
    for h in (b, s1, s2):
        h.close()


def test_batch_rejections():
    tw = load_twave()
    c = acoustic_periodic_case(16, 16, seed=1, cpst="0", Nt=4)
    a = make_shot(tw, c, "f32")
    e = make_shot(tw, c, "f32", energy=True)
    d = make_shot(tw, c, "f64")
    el = tw.Solver(16, 16, 1, 16, 1e-3, precision="f32")
    L = tw.lib()
    for group, code in [([a, a], -1), ([a, e], -10), ([a, d], -10), ([el], -10)]:
        h = ctypes.c_void_p()
        arr = (ctypes.c_void_p * len(group))(*[g.h for g in group])
        assert L.tw_batch_create(ctypes.byref(h), arr, len(group)) == code
        assert not h.value
    b = tw.Batch([a])
    assert L.tw_batch_set_shape(b.h, 48, 3, 1, 0) == -1      # 144 threads: not whole warps
    assert L.tw_batch_set_shape(b.h, 64, 8, 1, 0) == -1      # 512 threads: above the kernel's bound
    assert L.tw_batch_step(b.h, 10**6) == -8
    for h in (b, a, e, d, el):
        h.close()
