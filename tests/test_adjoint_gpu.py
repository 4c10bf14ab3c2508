"""Adjoint gradients (tw_adjoint_gradient) through the C ABI.

The reference has no adjoint, so nothing pins these to it; they are pinned by the two identities
that define a correct discrete adjoint:
  * dot-product test: for the linear map L from the initial fields to the receiver traces (no
    source), <L x, y> = <x, L^T y>, where L^T y is the gradient with respect to the initial state
    for residual y; FP64, relative 1e-12;
  * central finite differences of the misfit along random directions of the node model (rho, vp,
    vs): FP64, relative error at most 1e-3 with h = 1e-3 (the bound asked of the method) and at
    most 2e-5 with h = 1e-4 (second-order convergence of the differences to the adjoint value).
Checkpoint spacing must not change the gradient, and the handle must end as after tw_step(nt).
"""
import numpy as np
import pytest

from cases import elastic_case, load_twave

pytestmark = pytest.mark.gpu
KEYS = ("NN", "MN", "NM", "MM0", "MM1")


def rcvs_for(Mx, My, den):
    return [("N", "M", 2, den, 2 * 3 + 1, 2 * den), ("M", "M", 2 * 5 + 1, 2 * den, 2 * (My // 2) + 1, 2 * den),
            ("N", "N", Mx // 2, den, My, den), ("M", "N", 2 * (Mx - 1) + 1, 2 * den, 0, 1),
            ("N", "M", 0, 1, 2 * (My - 1) + 1, 2 * den), ("N", "M", 4, den, 2 * 9 + 1, 2 * den)]


def solver(tw, case, precision="f64", source=True, rho=None, vp=None, vs=None):
    s = tw.Solver(case.Mx, case.My, case.num_dx, case.den_dx, case.dt, precision=precision, cpst=case.cpst,
                  central_f=case.central_f, time_delay=case.time_delay, max_steps=case.Nt, energy=False)
    shp = (case.Mx + 2, case.My + 2)
    s.set_material_model((case.rho if rho is None else rho).reshape(shp), (case.vp if vp is None else vp).reshape(shp),
                         (case.vs if vs is None else vs).reshape(shp))
    if source:
        s.set_source_location(*case.src)
    for r in case.rcvs:
        s.add_receiver_location(*r)
    return s


def single_field_mask(tw, case):
    """1 where a trace entry exists (field 1 only on the MM grid)."""
    m = np.ones((len(case.rcvs), 2, 1))
    for q, r in enumerate(case.rcvs):
        if (r[0], r[1]) != ("M", "M"):
            m[q, 1] = 0
    return m


def random_state(case, seed):
    rng = np.random.default_rng(seed)
    Mx, My = case.Mx, case.My
    return [rng.standard_normal(s) for s in [(Mx + 1, My + 1), (Mx, My + 1), (Mx + 1, My), (Mx, My), (Mx, My)]]


@pytest.mark.parametrize("nt,K", [(1, 1), (30, 7), (30, 50)])
def test_dot_product_identity_of_the_state_map(nt, K):
    tw = load_twave()
    Mx, My, den = 24, 20, 24
    case = elastic_case(Mx, My, seed=3, Nt=nt, den_dx=den, rcvs=rcvs_for(Mx, My, den))
    x = random_state(case, 1)
    slots = [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
    s = solver(tw, case, source=False)
    for (g, f), a in zip(slots, x):
        s.write_field(g, f, a)
    s.run(nt)
    d = s.read_receivers()
    s.close()
    y = np.random.default_rng(2).standard_normal(d.shape) * single_field_mask(tw, case)
    s = solver(tw, case, source=False)
    for (g, f), a in zip(slots, x):
        s.write_field(g, f, a)
    out = s.adjoint_gradient(nt, d - y, ckpt_every=K, model=False, state=True)
    s.close()
    lhs = float(np.sum(d * y))
    rhs = float(sum(np.sum(a * out["state"][k]) for a, k in zip(x, KEYS)))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.sqrt(np.sum(d * d) * np.sum(y * y)))
    assert abs(out["misfit"] - 0.5 * np.sum(y * y)) <= 1e-12 * np.sum(y * y)


def _misfit_case():
    Mx, My, den = 32, 32, 32
    rcvs = [("N", "M", 3, den, 2 * k + 1, 2 * den) for k in range(1, My, 3)]
    case = elastic_case(Mx, My, seed=11, Nt=90, den_dx=den, rcvs=rcvs, model="layered",
                        src=("M", "M", 2 * 20 + 1, 2 * den, 2 * 13 + 1, 2 * den), time_delay=0.1, central_f=8.0)
    return case


def test_gradient_matches_central_differences():
    tw = load_twave()
    case = _misfit_case()
    nt = case.Nt
    shp = (case.Mx + 2, case.My + 2)
    rho, vp, vs = (np.asarray(a, np.float64).reshape(shp) for a in (case.rho, case.vp, case.vs))
    # observed traces from a perturbed medium (a Gaussian anomaly in vp and vs)
    X, Y = np.meshgrid(np.arange(shp[0]), np.arange(shp[1]), indexing="ij")
    bump = 1.0 + 0.05 * np.exp(-((X - 14) ** 2 + (Y - 18) ** 2) / 18.0)
    s = solver(tw, case, vp=vp * bump, vs=vs * bump)
    s.run(nt)
    obs = s.read_receivers()
    s.close()

    def J(r, p, q):
        h = solver(tw, case, rho=r, vp=p, vs=q)
        h.run(nt)
        t = h.read_receivers()
        h.close()
        return 0.5 * float(np.sum((t - obs) ** 2))

    s = solver(tw, case)
    g = s.adjoint_gradient(nt, obs, ckpt_every=25)
    s.close()
    assert abs(g["misfit"] - J(rho, vp, vs)) <= 1e-12 * g["misfit"]
    rng = np.random.default_rng(5)
    for k in range(8):
        d = [rng.standard_normal(shp) * a for a in (rho, vp, vs)]   # relative perturbation directions
        ana = sum(float(np.sum(gg * dd)) for gg, dd in zip((g["rho"], g["vp"], g["vs"]), d))
        err = {}
        for eps in (1e-3, 1e-4):
            fd = (J(rho + eps * d[0], vp + eps * d[1], vs + eps * d[2]) -
                  J(rho - eps * d[0], vp - eps * d[1], vs - eps * d[2])) / (2 * eps)
            err[eps] = abs(fd - ana) / abs(ana)
        # the bound asked of the method at h = 1e-3, and the second-order convergence of central
        # differences towards the adjoint value (the gap is their truncation error, not the adjoint's)
        assert err[1e-3] <= 1e-3 and err[1e-4] <= 2e-5, (k, err)


def test_checkpoint_spacing_does_not_change_the_gradient_and_the_handle_ends_at_nt():
    tw = load_twave()
    case = _misfit_case()
    nt = case.Nt
    ref = solver(tw, case, precision="f32")
    ref.run(nt)
    fields = [ref.read_field(g, f) for g, f in ((tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1))]
    traces = ref.read_receivers()
    ref.close()
    obs = traces * 0.9
    outs = []
    for K in (1, 13, nt):
        s = solver(tw, case, precision="f32")
        outs.append(s.adjoint_gradient(nt, obs, ckpt_every=K))
        assert s.info().steps_done == nt
        assert np.array_equal(s.read_receivers(), traces)
        for (gr, f), a in zip(((tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)), fields):
            assert np.array_equal(s.read_field(gr, f), a)
        s.close()
    for o in outs[1:]:
        for k, v in o["grid"].items():   # one thread per point, same order: identical
            assert np.array_equal(v, outs[0]["grid"][k]), k
        for k in ("rho", "vp", "vs"):    # the node scatter adds with atomics: equal to rounding
            assert np.abs(o[k] - outs[0][k]).max() <= 1e-12 * np.abs(outs[0][k]).max(), k


def test_adjoint_rejections():
    tw = load_twave()
    case = elastic_case(16, 16, seed=1, Nt=10, den_dx=16, rcvs=[("N", "M", 2, 16, 7, 32)])
    obs = np.zeros((1, 2, 10))
    s = solver(tw, case)
    s.step(1)
    with pytest.raises(tw.TwError) as e:
        s.adjoint_gradient(5, obs[:, :, :5])
    assert e.value.code == -4
    s.close()
    c6 = elastic_case(16, 16, seed=1, Nt=10, den_dx=16, cpst="6R", rcvs=[("N", "M", 2, 16, 7, 32)])
    s = solver(tw, c6)
    with pytest.raises(tw.TwError) as e:
        s.adjoint_gradient(10, obs)
    assert e.value.code == -10
    s.close()
