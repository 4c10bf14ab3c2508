"""Writers of the reference's output files (tw_io_write_records) on a real run: file names,
formats and values against the records read through the C ABI."""
import os

import numpy as np
import pytest

from cases import elastic_case, load_twave
from conftest import has_ref_binaries
from oracle import refrun

pytestmark = pytest.mark.gpu


def test_signal_energy_and_snapshot_files(tmp_path):
    tw = load_twave()
    den = 24
    case = elastic_case(24, 20, seed=8, Nt=12, den_dx=den,
                        rcvs=[("N", "M", 3, den, 2 * 5 + 1, 2 * den), ("M", "M", 2 * 7 + 1, 2 * den, 2 * 9 + 1, 2 * den)])
    s = tw.Solver(case.Mx, case.My, 1, den, case.dt, central_f=case.central_f, time_delay=case.time_delay,
                  max_steps=case.Nt, energy=True)
    shp = (case.Mx + 2, case.My + 2)
    s.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), case.vs.reshape(shp))
    s.set_source(tw.MM, 12, 6)
    for r in case.rcvs:
        s.add_receiver_location(*r)
    s.run(case.Nt)
    s.write_records(str(tmp_path), src_index=4, rcv_index=[10, 11], snapshots=True)
    tr = s.read_receivers()
    Ek, Ep0, Ep1 = s.read_energy()
    names = sorted(os.listdir(tmp_path))
    sig0 = "Signal_src_4_MM_6_12_rcv_10_MN_5_3.txt"      # NM receiver: data-y type first
    sig1 = "Signal_src_4_MM_6_12_rcv_11_MM_9_7.txt"
    assert sig0 in names and sig1 in names
    a = np.loadtxt(tmp_path / sig0)
    assert a.shape == (case.Nt, 2) and np.array_equal(a[:, 0], np.arange(case.Nt))
    assert np.allclose(a[:, 1], tr[0, 0], rtol=1e-14, atol=0)
    b = np.loadtxt(tmp_path / sig1)
    assert b.shape == (case.Nt, 3)
    assert np.allclose(b[:, 1:], tr[1].T, rtol=1e-14, atol=0)
    e = np.loadtxt(tmp_path / "Energy_src_4_MM_6_12.txt")
    assert np.allclose(e, Ek + (Ep0 + Ep1) / 2, rtol=1e-14, atol=0)
    for gname, g, f in (("NN_Sxy_0", tw.NN, 0), ("NM_Vx_0", tw.MN, 0), ("MN_Vy_0", tw.NM, 0), ("MM_SMM_0", tw.MM, 0),
                        ("MM_SMM_1", tw.MM, 1)):
        v = np.loadtxt(tmp_path / f"Snapshot_{gname}.txt")
        assert np.allclose(v, s.read_field(g, f).reshape(-1), rtol=1e-14, atol=0), gname
    s.close()


def _product_run(tw, case, prec):
    s = tw.Solver(case.Mx, case.My, case.num_dx, case.den_dx, case.dt, precision=prec, central_f=case.central_f,
                  time_delay=case.time_delay, max_steps=case.Nt, energy=True)
    shp = (case.Mx + 2, case.My + 2)
    s.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), case.vs.reshape(shp))
    s.set_source_location(*case.src)
    for r in case.rcvs:
        s.add_receiver_location(*r)
    s.run(case.Nt)
    return s


@pytest.mark.skipif(not has_ref_binaries(), reason="oracle/_ref binaries not built")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_writers_match_the_reference_writers(tmp_path, prec):
    """The Signal and Energy files of tw_io_write_records against the files the reference's own
    output_solution_record / output_energy (forward.cpp:215-325) write for the same run: the same
    file names; Signal files byte for byte (the traces are bit-identical); Energy values to 1e-12
    relative (FP64 sums taken in another order)."""
    tw = load_twave()
    case = elastic_case(30, 26, seed=12, Nt=40, model="layered")
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    refrun.run_elastic(case, prec, out_folder=str(ref_dir))
    s = _product_run(tw, case, prec)
    try:
        s.write_records(str(our_dir), src_index=0)
    finally:
        s.close()
    ref_names, our_names = sorted(os.listdir(ref_dir)), sorted(os.listdir(our_dir))
    assert ref_names == our_names
    for name in ref_names:
        a, b = (ref_dir / name).read_bytes(), (our_dir / name).read_bytes()
        if name.startswith("Signal"):
            assert a == b, name
        else:
            x, y = np.loadtxt(ref_dir / name), np.loadtxt(our_dir / name)
            assert x.shape == y.shape and np.abs(x - y).max() <= 1e-12 * np.abs(x).max(), name


@pytest.mark.skipif(not has_ref_binaries(), reason="oracle/_ref binaries not built")
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_data_misfit_matches_the_reference(prec):
    """tw_data_misfit against the reference's calculate_data_misfit (forward.cpp:414-445) on the
    same run and the same observed traces: per receiver bit for bit (the same traces, summed in
    the same order), the total to 1e-14 relative (the reference adds receivers grid by grid)."""
    tw = load_twave()
    case = elastic_case(30, 26, seed=13, Nt=40, model="layered")
    probe = refrun.run_elastic(case, prec)
    obs = probe.traces + np.random.default_rng(5).standard_normal(probe.traces.shape) * 1e-3
    ref = refrun.run_elastic(case, prec, obs=obs)
    s = _product_run(tw, case, prec)
    try:
        total, per = s.data_misfit(obs)
    finally:
        s.close()
    assert np.array_equal(np.asarray(per), ref.misfit_rcv)
    assert abs(total - ref.misfit_total) <= 1e-14 * abs(ref.misfit_total)
