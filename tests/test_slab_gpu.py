"""Slab decomposition of one elastic grid (tw_create_slab / tw_slab_exchange / tw_slab_run), on
one GPU: the grid cut into slabs along x, every slab stepped and the halos exchanged after each
step (by copies, by packed buffers, by copies between the per-array spans the rank-parallel
driver hands to NCCL, or by the step kernel's own stores into the neighbours' halo rows), must give the whole grid's fields on every owned row and its traces bit for bit, and its
energies to 1e-12 (sums in another order). Covers the free-surface zones of the first and last
slab, open inner edges, compensation arrays in the halo, sources and receivers in any slab."""
import numpy as np
import pytest

from cases import elastic_case, load_twave
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
SLOTS = None


def packed_exchange(up, lo):
    """The same halo swap through flat device buffers (tw_slab_pack / tw_slab_unpack), as a
    multi-GPU driver moves them with NCCL."""
    import torch
    n = up.halo_bytes(1)
    assert n == lo.halo_bytes(0)
    a = torch.empty(n, dtype=torch.uint8, device="cuda:0")
    b = torch.empty(n, dtype=torch.uint8, device="cuda:0")
    up.sync()
    lo.sync()
    up.pack(1, a.data_ptr())
    lo.pack(0, b.data_ptr())
    up.sync()
    lo.sync()
    lo.unpack(0, a.data_ptr())
    up.unpack(1, b.data_ptr())
    up.sync()
    lo.sync()


def spans_exchange(up, lo):
    """The halo swap the rank-parallel driver makes with NCCL (tpu-wave_b200/slabs.py): every
    array's rows straight from the owned span into the neighbour's halo span, here by device
    copies between the same zero-copy views."""
    import importlib.util
    import os
    import torch
    spec = importlib.util.spec_from_file_location(
        "twave_slabs", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tpu-wave_b200", "slabs.py"))
    sl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sl)
    up.sync()
    lo.sync()
    for src_h, src_side, dst_h, dst_side in ((up, 1, lo, 0), (lo, 0, up, 1)):
        src, dst = dict(src_h.halo_spans(src_side, 0)), dict(dst_h.halo_spans(dst_side, 1))
        assert src.keys() == dst.keys() and len(src) in (5, 10)
        for f in src:
            assert src[f][1] == dst[f][1]
            a = torch.as_tensor(sl._DeviceSpan(*src[f]), device="cuda:0")
            b = torch.as_tensor(sl._DeviceSpan(*dst[f]), device="cuda:0")
            b.copy_(a)
    torch.cuda.synchronize()


def run(tw, case, prec, cuts, f0, r0, Nt, slab=True, mode="copy"):
    shp = (case.Mx + 2, case.My + 2)
    kw = dict(precision=prec, cpst=case.cpst, central_f=case.central_f, time_delay=case.time_delay, max_steps=Nt)
    slots = [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
    if slab:
        hs = [tw.Solver.slab(case.Mx, case.My, 1, case.den_dx, case.dt, a, b, **kw) for a, b in zip(cuts[:-1], cuts[1:])]
    else:
        hs = [tw.Solver(case.Mx, case.My, 1, case.den_dx, case.dt, **kw)]
    for h in hs:
        h.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), case.vs.reshape(shp))
        h.set_source_location(*case.src)
        for r in case.rcvs:
            h.add_receiver_location(*r)
        off = h.row_off if slab else 0
        for (g, f), a in zip(slots, f0):
            h.write_field(g, f, a[off:off + h.shape(g)[0]])
        if r0 is not None:
            for (g, f), a in zip(slots, r0):
                h.write_resid(g, f, a[off:off + h.shape(g)[0]])
    if mode == "fused":   # in two calls: the buffers alternate across calls too
        tw.Solver.slab_run(hs, 3)
        tw.Solver.slab_run(hs, Nt - 3)
    for _ in range(Nt if mode != "fused" else 0):
        for h in hs:
            h.step(1)
        for up, lo in zip(hs[:-1], hs[1:]):
            if mode == "packed":
                packed_exchange(up, lo)
            elif mode == "spans":
                spans_exchange(up, lo)
            else:
                up.exchange(lo)
    if mode != "fused":   # after a linked run each handle alone is ordered after its neighbours' stores
        for h in hs:
            h.sync()
    fields = [np.zeros_like(a) for a in f0]
    for h in hs:
        off = h.row_off if slab else 0
        own = h.own if slab else (0, case.Mx)
        for k, (g, f) in enumerate(slots):
            loc = h.read_field(g, f)
            hi = own[1] + (1 if (g in (tw.NN, tw.NM) and own[1] == case.Mx) else 0)
            fields[k][own[0]:hi] = loc[own[0] - off:hi - off]
    traces = sum(h.read_receivers() for h in hs)
    energy = [sum(h.read_energy()[i] for h in hs) for i in range(3)]
    for h in hs:
        h.close()
    return fields, traces, energy


@pytest.mark.parametrize("mode", ["copy", "packed", "spans", "fused"])
@pytest.mark.parametrize("prec,cpst", [("f32", "00"), ("f64", "6R"), ("f32", "3C")])
@pytest.mark.parametrize("cuts", [(0, 24, 48, 72), (0, 40, 72), (0, 16, 56, 72)])
def test_slabs_equal_the_whole_grid(prec, cpst, cuts, mode):
    tw = load_twave()
    Mx, My, den, Nt = 72, 60, 72, 9
    rcvs = [("N", "M", 2, den, 7, 2 * den), ("M", "M", 2 * 23 + 1, 2 * den, 2 * 9 + 1, 2 * den),
            ("N", "N", 24, den, 31, den), ("M", "N", 2 * 40 + 1, 2 * den, 0, 1), ("N", "M", Mx, den, 2 * 59 + 1, 2 * den),
            ("N", "N", 56, den, My, den)]
    case = elastic_case(Mx, My, seed=5, cpst=cpst, Nt=Nt, den_dx=den, rcvs=rcvs,
                        src=("M", "M", 2 * 47 + 1, 2 * den, 2 * 20 + 1, 2 * den))
    rng = np.random.default_rng(4)
    T = np.float64 if prec == "f64" else np.float32
    shapes = [(Mx + 1, My + 1), (Mx, My + 1), (Mx + 1, My), (Mx, My), (Mx, My)]
    f0 = [(rng.standard_normal(s) * 1e-2).astype(T).astype(np.float64) for s in shapes]
    r0 = None if cpst == "00" else [(rng.standard_normal(s) * 1e-9).astype(T).astype(np.float64) for s in shapes]
    want = run(tw, case, prec, None, f0, r0, Nt, slab=False)
    got = run(tw, case, prec, cuts, f0, r0, Nt, mode=mode)
    for k in range(5):
        assert np.array_equal(got[0][k], want[0][k]), k
    assert np.array_equal(got[1], want[1])
    for a, b in zip(got[2], want[2]):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    # and the assembled slabs against the C restatement (pinned to the reference's solver)
    ref = orc.elastic_run(case, prec, fields0=f0, resid0=r0)
    for k, key in enumerate(("NN", "MN", "NM", "MM0", "MM1")):
        assert np.array_equal(got[0][k], ref.fields[key]), key
    assert np.array_equal(got[1], ref.traces)
    for a, key in zip(got[2], ("E_k", "E_p0", "E_p1")):
        b = getattr(ref, key)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), key


def test_slab_arguments():
    tw = load_twave()
    with pytest.raises(tw.TwError):
        tw.Solver.slab(72, 60, 1, 72, 1e-3, 0, 10)      # fewer than 16 rows
    with pytest.raises(tw.TwError):
        tw.Solver.slab(72, 60, 1, 72, 1e-3, 8, 40)      # an inner cut 8 rows from the free surface
    a = tw.Solver.slab(72, 60, 1, 72, 1e-3, 0, 40)
    b = tw.Solver.slab(72, 60, 1, 72, 1e-3, 48, 72)
    with pytest.raises(tw.TwError):
        a.exchange(b)                                     # not adjacent
    with pytest.raises(tw.TwError):
        tw.Solver.slab_run([a, b], 1)                     # not the whole grid, not consecutive
    shp = (74, 62)
    rho, vp, vs = np.full(shp, 2.0), np.full(shp, 3.0), np.full(shp, 1.7)
    c = tw.Solver.slab(72, 60, 1, 72, 1e-3, 40, 72, max_steps=4)
    c.set_material_model(rho, vp, vs)
    with pytest.raises(tw.TwError):
        tw.Solver.slab_run([a, c], 1)                     # a has no material yet
    a.close()
    b.close()
    c.close()
