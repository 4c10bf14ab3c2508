"""Readers of the reference's input files (no GPU): InputFile.txt entries, SrcRcv.txt points and
raw model files, on fixtures written here in the reference's formats and, where the reference
tree is present, on its own example files."""
import os

import numpy as np
import pytest

from cases import load_twave
from oracle.refrun import REFERENCE_DIR

REF_DATA = os.path.join(REFERENCE_DIR, "cuda", "data", "homogeneous")


@pytest.fixture(scope="module")
def tw():
    return load_twave()


def test_input_file_entries(tw, tmp_path):
    p = tmp_path / "InputFile.txt"
    p.write_text("model_300_200                   // X then Y: model cells\n\n"
                 "dxM_1_100    // model spacing (numerator_denominator)\n"
                 "dxS_1_200\n"
                 "grids_600_400\n"
                 "bdry_ffpp\n"
                 "Nt_1500\n"
                 "MAXdt_2.5e-04\n"
                 "CFL_0.4\n"
                 "frequency_7.5\n"
                 "delay_0.125\n"
                 "device_3\n"
                 "something_else_99\n")
    r = tw.io_read_input(str(p))
    assert (r.Mx_prmt, r.My_prmt, r.Mx, r.My) == (200, 300, 400, 600)   # 'X' is data y
    assert (r.num_dxM, r.den_dxM, r.num_dx, r.den_dx) == (1, 100, 1, 200)
    assert bytes(r.bdry) == b"FFPP"
    assert r.Nt == 1500 and r.device == 3
    assert r.dt_max == 2.5e-4 and r.cfl == 0.4 and r.dt == 2.5e-4 * 0.4
    assert r.central_f == 7.5 and r.time_delay == 0.125


def test_input_file_defaults_and_errors(tw, tmp_path):
    p = tmp_path / "InputFile.txt"
    p.write_text("grids_8_9\n#bdry_PPFF\n")
    r = tw.io_read_input(str(p))
    assert (r.Mx, r.My) == (9, 8) and r.cfl == 0.625 and r.central_f == 5.0 and r.time_delay == 0.25
    assert bytes(r.bdry) == b""   # absent: zeros
    with pytest.raises(tw.TwError) as e:
        tw.io_read_input(str(tmp_path / "missing.txt"))
    assert e.value.code == -13
    (tmp_path / "bad.txt").write_text("Nt_many\n")
    with pytest.raises(tw.TwError):
        tw.io_read_input(str(tmp_path / "bad.txt"))


def test_srcrcv_points(tw, tmp_path):
    p = tmp_path / "SrcRcv.txt"
    p.write_text("# comment_line\n"
                 "Src_7_MN_401_250_20_250\n"
                 "Rcv_7_0_MN_801_250_20_250\n"
                 "rcv_7_1_NM_3_2_5_4\n"
                 "Src_2_NN_1_1_0_1\n")
    pts = tw.io_read_srcrcv(str(p))
    assert len(pts) == 4
    s = pts[0]
    assert (s.src_index, s.rcv_index, s.type_x, s.type_y) == (7, -1, b"N", b"M")
    assert (s.num_x, s.den_x, s.num_y, s.den_y) == (20, 250, 401, 250)
    r = pts[2]
    assert (r.src_index, r.rcv_index, r.type_x, r.type_y, r.num_x, r.den_x, r.num_y, r.den_y) == (7, 1, b"M", b"N", 5, 4, 3, 2)
    (tmp_path / "orphan.txt").write_text("Rcv_1_0_MN_1_2_1_2\nSrc_1_MN_1_2_1_2\n")
    with pytest.raises(tw.TwError) as e:
        tw.io_read_srcrcv(str(tmp_path / "orphan.txt"))
    assert e.value.code == -13


def test_model_file_padding(tw, tmp_path):
    Mx, My = 5, 7
    raw = np.arange((Mx + 1) * (My + 1), dtype=np.float64).reshape(Mx + 1, My + 1) * 0.5 + 1.0
    (tmp_path / "vp.bin").write_bytes(raw.tobytes())
    m = tw.io_read_model(str(tmp_path / "vp.bin"), Mx, My)
    assert m.shape == (Mx + 2, My + 2)
    assert np.array_equal(m[:Mx + 1, :My + 1], raw) and not m[Mx + 1].any() and not m[:, My + 1].any()
    with pytest.raises(tw.TwError) as e:
        tw.io_read_model(str(tmp_path / "vp.bin"), Mx + 1, My)
    assert e.value.code == -13


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference example files not present")
def test_reference_example_files(tw):
    r = tw.io_read_input(os.path.join(REF_DATA, "InputFile.txt"))
    assert (r.Mx_prmt, r.My_prmt, r.Mx, r.My) == (600, 600, 600, 600)
    assert (r.num_dxM, r.den_dxM, r.num_dx, r.den_dx) == (1, 125, 1, 125)
    assert r.Nt == 60000 and r.cfl == 0.625 and r.central_f == 5.0 and r.time_delay == 0.25
    pts = tw.io_read_srcrcv(os.path.join(REF_DATA, "SrcRcv.txt"))
    assert [(p.src_index, p.rcv_index) for p in pts] == [(1, -1), (1, 1)]
    assert (pts[0].type_x, pts[0].type_y, pts[0].num_y, pts[0].den_y, pts[0].num_x, pts[0].den_x) == (b"N", b"M", 401, 250, 20, 250)


def test_reference_gpu_program_inputs(tw, tmp_path):
    """The InputFile.txt and SrcRcv.txt that oracle/ref_gpu_timing.py writes for the reference's
    own GPU program read back, through the readers of the reference's formats, as the 2048^2
    workload meant: grid and spacing, dt = MAXdt x CFL 1, the Ricker parameters, the source on the
    centre MM point and 16 receivers on MM points."""
    from oracle import ref_gpu_timing as rg
    dt = 0.00012871690627155345
    rg.write_inputs(str(tmp_path), 2048, 500, dt, 15.0, 0.1)
    r = tw.io_read_input(str(tmp_path / "InputFile.txt"))
    assert (r.Mx, r.My, r.Mx_prmt, r.My_prmt) == (2048, 2048, 2048, 2048)
    assert (r.num_dx, r.den_dx, r.num_dxM, r.den_dxM) == (1, 500, 1, 500)
    assert r.dt == dt and r.central_f == 15.0 and r.time_delay == 0.1
    pts = tw.io_read_srcrcv(str(tmp_path / "SrcRcv.txt"))
    assert len(pts) == 17
    src, rcvs = pts[0], pts[1:]
    assert (src.rcv_index, src.type_x, src.type_y) == (-1, b"M", b"M")
    assert tw.location_to_index("M", src.num_x, src.den_x, 1, 500) == 1024
    assert tw.location_to_index("M", src.num_y, src.den_y, 1, 500) == 1024
    for k, q in enumerate(rcvs):
        c = (64 + 128 * k) % 2048
        assert (q.src_index, q.rcv_index, q.type_x, q.type_y) == (1, k + 1, b"M", b"M")
        assert tw.location_to_index("M", q.num_x, q.den_x, 1, 500) == c
        assert tw.location_to_index("M", q.num_y, q.den_y, 1, 500) == c
