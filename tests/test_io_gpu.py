"""Writers of the reference's output files (tw_io_write_records) on a real run: file names,
formats and values against the records read through the C ABI."""
import os

import numpy as np
import pytest

from cases import elastic_case, load_twave

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
