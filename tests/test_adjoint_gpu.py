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


class StateMap:
    """The linear map from the initial fields to the traces (no source) and its transpose by the
    adjoint, for the autograd wrapper Traces (adjoint_torch.py)."""

    def __init__(self, tw, case, nt, K=0, slots=0):
        self.tw, self.case, self.nt, self.K, self.slots = tw, case, nt, K, slots
        self.keys = [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
        self.misfit = None

    def _handle(self, x):
        s = solver(self.tw, self.case, source=False)
        for (g, f), a in zip(self.keys, x):
            s.write_field(g, f, a)
        return s

    def forward(self, x):
        s = self._handle(x)
        s.run(self.nt)
        d = s.read_receivers()
        s.close()
        return d

    def transpose(self, x, obs):
        s = self._handle(x)
        out = s.adjoint_gradient(self.nt, obs, ckpt_every=max(self.K, 1), model=False, state=True, slots=self.slots)
        s.close()
        self.misfit = out["misfit"]
        return [out["state"][k] for k in KEYS]


@pytest.mark.parametrize("nt,K,slots", [(1, 1, 0), (30, 7, 0), (30, 50, 0), (30, 0, 1), (30, 0, 4)])
def test_dot_product_identity_of_the_state_map(nt, K, slots):
    """<L x, y> = <x, L^T y> with L^T y from autograd's vector-Jacobian product of the traces."""
    import torch
    from adjoint_torch import Traces
    tw = load_twave()
    Mx, My, den = 24, 20, 24
    case = elastic_case(Mx, My, seed=3, Nt=nt, den_dx=den, rcvs=rcvs_for(Mx, My, den))
    x = [torch.from_numpy(a).requires_grad_(True) for a in random_state(case, 1)]
    runner = StateMap(tw, case, nt, K=K, slots=slots)
    d = Traces.apply(*x, runner)
    y = torch.from_numpy(np.random.default_rng(2).standard_normal(tuple(d.shape)) * single_field_mask(tw, case))
    g = torch.autograd.grad(d, x, grad_outputs=y)
    lhs = float(torch.sum(d * y))
    rhs = float(sum(torch.sum(a * b) for a, b in zip(x, g)))
    dd, yy = float(torch.sum(d * d)), float(torch.sum(y * y))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.sqrt(dd * yy))
    assert abs(runner.misfit - 0.5 * yy) <= 1e-12 * yy


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

    import torch
    from adjoint_torch import Misfit

    def runner(r, p, q):
        h = solver(tw, case, rho=r, vp=p, vs=q)
        out = h.adjoint_gradient(nt, obs, ckpt_every=25)
        h.close()
        return out["misfit"], out

    m = [torch.from_numpy(a.copy()).requires_grad_(True) for a in (rho, vp, vs)]
    Jt = Misfit.apply(*m, runner)
    grads = torch.autograd.grad(Jt, m)
    assert abs(float(Jt) - J(rho, vp, vs)) <= 1e-12 * float(Jt)
    rng = np.random.default_rng(5)
    for k in range(8):
        d = [rng.standard_normal(shp) * a for a in (rho, vp, vs)]   # relative perturbation directions
        ana = sum(float(torch.sum(gg * torch.from_numpy(dd))) for gg, dd in zip(grads, d))
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


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_revolve_schedule_gives_the_same_gradient(prec):
    """Binomial checkpointing in 1, 2, 3, 7 and nt state slots against checkpoints every 13 steps:
    the same forward states reach every adjoint step, so the per-grid gradients are bit-identical
    and the node gradients (FP64 atomics) equal to 1e-12; the handle ends as after tw_step(nt)."""
    tw = load_twave()
    case = _misfit_case()
    nt = case.Nt
    ref = solver(tw, case, precision=prec)
    ref.run(nt)
    traces = ref.read_receivers()
    fields = [ref.read_field(g, f) for g, f in ((tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1))]
    ref.close()
    obs = traces * 0.9
    s = solver(tw, case, precision=prec)
    want = s.adjoint_gradient(nt, obs, ckpt_every=13)
    s.close()
    for slots in (1, 2, 3, 7, nt):
        s = solver(tw, case, precision=prec)
        got = s.adjoint_gradient(nt, obs, slots=slots)
        assert s.info().steps_done == nt
        assert np.array_equal(s.read_receivers(), traces)
        for (gr, f), a in zip(((tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)), fields):
            assert np.array_equal(s.read_field(gr, f), a)
        s.close()
        assert got["misfit"] == want["misfit"]
        for k, v in got["grid"].items():
            assert np.array_equal(v, want["grid"][k]), (slots, k)
        for k in ("rho", "vp", "vs"):
            assert np.abs(got[k] - want[k]).max() <= 1e-12 * np.abs(want[k]).max(), (slots, k)


@pytest.mark.parametrize("slots", [0, 3])
def test_recomputed_steps_leave_the_energy_records_alone(slots):
    """With the energy on, the gradient call's records equal a plain run's: steps recomputed from
    checkpoints add nothing to them."""
    tw = load_twave()
    case = _misfit_case()
    nt = case.Nt
    shp = (case.Mx + 2, case.My + 2)

    def make():
        h = tw.Solver(case.Mx, case.My, case.num_dx, case.den_dx, case.dt, precision="f64", central_f=case.central_f,
                      time_delay=case.time_delay, max_steps=nt, energy=True)
        h.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), case.vs.reshape(shp))
        h.set_source_location(*case.src)
        for r in case.rcvs:
            h.add_receiver_location(*r)
        return h
    h = make()
    h.run(nt)
    want = h.read_energy()
    obs = h.read_receivers() * 0.9
    h.close()
    h = make()
    h.adjoint_gradient(nt, obs, ckpt_every=11, slots=slots)
    got = h.read_energy()
    h.close()
    for a, b in zip(got, want):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_gradient_at_the_c5_size_matches_central_differences():
    """The C5 configuration's grid and length in FP64 (1024 x 1024, 2000 steps, one of its shots on
    row 16, 256 receivers on NM row 4, the layered medium with observed data from the 5 % anomaly):
    central differences of the misfit along 3 random relative directions at h = 1e-3 and 5e-4, and
    their Richardson extrapolation (4 D(h/2) - D(h)) / 3, which removes the h^2 truncation term,
    against the adjoint value from autograd (Misfit wrapper)."""
    import torch
    import bench
    from adjoint_torch import Misfit
    tw = load_twave()
    n, nt = bench.ADJ_N, 2000
    rho, vp, vs, bump = bench.adjoint_media()
    dt = bench.CFL * (1.0 / bench.DEN_DX) / (np.sqrt(2.0) * (vp * bump).max())
    rx, ry = np.full(256, 4), 4 * np.arange(256)

    def run(r, p, q, adjoint_obs=None):
        h = tw.Solver(n, n, 1, bench.DEN_DX, dt, precision="f64", central_f=bench.F0, time_delay=bench.DELAY,
                      max_steps=nt, energy=False)
        h.set_material_model(r, p, q)
        h.set_source(tw.MM, 16, 512)
        h.add_receivers(tw.NM, rx, ry)
        if adjoint_obs is not None:
            out = h.adjoint_gradient(nt, adjoint_obs, ckpt_every=50)
            h.close()
            return out
        h.run(nt)
        t = h.read_receivers()
        h.close()
        return t

    obs = run(rho, vp * bump, vs * bump)

    def J(r, p, q):
        return 0.5 * float(np.sum((run(r, p, q) - obs) ** 2))

    def runner(r, p, q):
        out = run(r, p, q, adjoint_obs=obs)
        return out["misfit"], out

    m = [torch.from_numpy(a.copy()).requires_grad_(True) for a in (rho, vp, vs)]
    grads = torch.autograd.grad(Misfit.apply(*m, runner), m)
    rng = np.random.default_rng(bench.ADJ_SEED + 1)
    for k in range(3):
        d = [rng.standard_normal(rho.shape) * a for a in (rho, vp, vs)]
        ana = sum(float(torch.sum(g * torch.from_numpy(dd))) for g, dd in zip(grads, d))

        def D(h):
            return (J(rho + h * d[0], vp + h * d[1], vs + h * d[2]) - J(rho - h * d[0], vp - h * d[1], vs - h * d[2])) / (2 * h)
        d1, d2 = D(1e-3), D(5e-4)
        rich = (4 * d2 - d1) / 3
        e1, e2, er = (abs(v - ana) / abs(ana) for v in (d1, d2, rich))
        print(f"direction {k}: rel err h=1e-3 {e1:.3e}, h=5e-4 {e2:.3e}, Richardson {er:.3e}")
        assert e2 <= e1 * 0.35 + 1e-9          # second-order convergence of the differences
        assert er <= 1e-4, (k, e1, e2, er)      # the extrapolated difference agrees with the adjoint


@pytest.mark.parametrize("slots", [0, 4])
def test_fp32_gradient_on_a_tma_handle_equals_the_per_warp_kernels(slots, monkeypatch):
    """An FP32 handle wide enough for the TMA-staged step (My >= 180) steps its own buffers with
    it, while the adjoint's recomputation (and every revolve sweep) steps between other buffers
    with the per-warp kernel in its own layout. Both kernels give bit-identical states, so the
    gradient, misfit, traces and final fields must equal those of the same handle made with the
    TMA step switched off (TW_TMA=0), bit for bit, for checkpoints every 7 steps and for 4 slots."""
    tw = load_twave()
    Mx, My, den = 40, 300, 300
    case = elastic_case(Mx, My, seed=31, Nt=30, rcvs=rcvs_for(Mx, My, den), den_dx=den, src=("M", "M", 2 * 20 + 1, 2 * den, 2 * 150 + 1, 2 * den))
    ref = solver(tw, case, precision="f32")
    assert ref.info().step_kind == 2      # the TMA-staged step
    ref.run(case.Nt)
    obs = ref.read_receivers() * 0.9
    ref.close()
    out = {}
    for tma in ("1", "0"):
        monkeypatch.setenv("TW_TMA", tma)
        s = solver(tw, case, precision="f32")
        assert s.info().step_kind == (2 if tma == "1" else 1)
        g = s.adjoint_gradient(case.Nt, obs, ckpt_every=7, slots=slots)
        g["traces"] = s.read_receivers()
        g["fields"] = [s.read_field(gr, f) for gr, f in ((tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1))]
        s.close()
        out[tma] = g
    a, b = out["1"], out["0"]
    assert a["misfit"] == b["misfit"] and a["misfit"] > 0
    assert np.array_equal(a["traces"], b["traces"])
    for x, y in zip(a["fields"], b["fields"]):
        assert np.array_equal(x, y)
    for k in a["grid"]:
        assert np.array_equal(a["grid"][k], b["grid"][k]), k
    for k in ("rho", "vp", "vs"):
        assert np.array_equal(a[k], b[k]) or np.abs(a[k] - b[k]).max() <= 1e-12 * np.abs(b[k]).max(), k
