"""Drive the reference's own CPU solvers (built into oracle/_ref by oracle/Makefile).

ORACLE / TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module; tests, the
golden-vector generator and bench.py's CPU-baseline and reference legs do.

Two executables are wrapped:
  * twref_elastic_{f64,f32}: the reference's elastic SBP-SAT host solver
    (cuda/src/cpp/forward_simulation.cpp:21-182 and everything it calls), free surface on the
    data-x ends and periodic in data-y.
  * twref_acoustic_{f64,f32}: the reference's single-core acoustic solver
    (singlecore/src/cpp/namespaces.hpp:566-668), periodic on all sides.
Each call runs one simulation in a fresh process (the single-core reference keeps its fields
in process-wide globals).
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")
# where the reference's sources are (only the oracle build and the tests of its example files
# read them); TW_REFERENCE_DIR overrides the default location
REFERENCE_DIR = os.environ.get("TW_REFERENCE_DIR", "/root/reference")

CPST_CODES = {"00": (0, "0"), "-3C": (-3, "C"), "-3R": (-3, "R"), "3C": (3, "C"),
              "3R": (3, "R"), "6C": (6, "C"), "6R": (6, "R")}


def ref_binary(name: str) -> str:
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: build it with `make -C oracle ref`")
    return path


@dataclass
class ElasticCase:
    """One elastic run in the reference's terms (all locations in data order x=slow, y=fast).

    rho/vp/vs: padded model arrays of shape (Mx_prmt + 2, My_prmt + 2) (the reference pads the
    (Mx_prmt + 1) x (My_prmt + 1) node model with one extra row and column, inverse.cpp:79-90).
    src = (type_x, type_y, num_x, den_x, num_y, den_y) physical location as rationals;
    rcvs = list of the same 6-tuples.
    """
    Mx: int
    My: int
    num_dx: int
    den_dx: int
    dt: float
    rho: np.ndarray
    vp: np.ndarray
    vs: np.ndarray
    src: tuple
    rcvs: list = field(default_factory=list)
    Nt: int = 10
    cpst: str = "00"
    central_f: float = 5.0
    time_delay: float = 0.25
    Mx_prmt: int | None = None
    My_prmt: int | None = None
    num_dxM: int | None = None
    den_dxM: int | None = None
    bc_x: str = "F"      # "F" free surfaces; "I" x ends joined by the SAT interface penalty
    sat_y: bool = False  # free surfaces on the y ends too (restatement only: no reference run)
    warm_passes: int = 0  # untimed runs of the same Nt steps before the timed one (outputs unchanged)


@dataclass
class ElasticResult:
    loop_seconds: float
    E_k: np.ndarray
    E_p0: np.ndarray
    E_p1: np.ndarray
    traces: np.ndarray         # [n_rcv, 2, Nt] (second field zero on single-field grids)
    fields: dict               # NN, MN, NM, MM0, MM1 at reference sizes
    coefs: dict                # NN_mu, MN_irho, NM_irho, MM_lambda, MM_2mu
    weights: dict              # NN, MN, NM, MM_P1, MM_P2 (energy weights incl. norms)
    misfit_total: float | None = None      # calculate_data_misfit against `obs` (when given)
    misfit_rcv: np.ndarray | None = None   # per receiver, input order


def _elastic_sizes(Mx, My):
    return {"NN": (Mx + 1, My + 1), "MN": (Mx, My + 1), "NM": (Mx + 1, My), "MM0": (Mx, My), "MM1": (Mx, My)}


def run_elastic(case: ElasticCase, precision: str = "f64", perf: bool = False, obs: np.ndarray | None = None,
                out_folder: str | None = None) -> ElasticResult:
    """Run the reference's elastic solver on `case`. obs ([n_rcv][2][Nt] observed traces): also
    return the reference's calculate_data_misfit against them. out_folder: let the reference's
    own writers (output_solution_record, output_energy) put their text files there."""
    Mxp = case.Mx if case.Mx_prmt is None else case.Mx_prmt
    Myp = case.My if case.My_prmt is None else case.My_prmt
    ndM = case.num_dx if case.num_dxM is None else case.num_dxM
    ddM = case.den_dx if case.den_dxM is None else case.den_dxM
    P = (Mxp + 2) * (Myp + 2)
    for a in (case.rho, case.vp, case.vs):
        assert a.size == P, (a.shape, P)
    if case.sat_y:
        raise ValueError("the reference has no run with free surfaces on the y ends")
    cn, cs = CPST_CODES[case.cpst]
    ih = np.zeros(32, np.int64)
    ih[20] = 0 if case.bc_x == "F" else ord(case.bc_x)
    ih[21] = case.warm_passes
    ih[22] = 1 if obs is not None else 0
    ih[:20] = [0x5457454C, case.Mx, case.My, Mxp, Myp, case.num_dx, case.den_dx, ndM, ddM,
               case.Nt, cn, ord(cs), ord(case.src[0]), ord(case.src[1]), *case.src[2:6],
               len(case.rcvs), 1]
    dh = np.zeros(8, np.float64)
    dh[:3] = [case.dt, case.central_f, case.time_delay]
    rcv = np.array([[ord(r[0]), ord(r[1]), *r[2:6]] for r in case.rcvs], np.int64).reshape(-1, 6)
    name = f"twref_elastic_{precision}" + ("_perf" if perf else "")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(ih.tobytes()); f.write(dh.tobytes())
            for a in (case.rho, case.vp, case.vs):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(rcv.tobytes())
            if obs is not None:
                f.write(np.ascontiguousarray(obs, np.float64).reshape(len(case.rcvs), 2, case.Nt).tobytes())
        cmd = [ref_binary(name), fin, fout] + ([out_folder] if out_folder else [])
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        out = np.fromfile(fout, np.float64)
    Nt, n = case.Nt, len(case.rcvs)
    pos = 0

    def take(count, shape=None):
        nonlocal pos
        a = out[pos:pos + count]
        pos += count
        return a.reshape(shape) if shape is not None else a

    loop = float(take(1)[0])
    E_k, E_p0, E_p1 = take(Nt), take(Nt), take(Nt)
    traces = take(n * 2 * Nt, (n, 2, Nt))
    sizes = _elastic_sizes(case.Mx, case.My)
    fields = {k: take(s[0] * s[1], s) for k, s in sizes.items()}
    coefs = {}
    for key, g in (("NN_mu", "NN"), ("MN_irho", "MN"), ("NM_irho", "NM"), ("MM_lambda", "MM0"), ("MM_2mu", "MM1")):
        s = sizes[g]
        coefs[key] = take(s[0] * s[1], s)
    weights = {}
    for key, g in (("NN", "NN"), ("MN", "MN"), ("NM", "NM"), ("MM_P1", "MM0"), ("MM_P2", "MM1")):
        s = sizes[g]
        weights[key] = take(s[0] * s[1], s)
    mt, mr = None, None
    if obs is not None:
        mt = float(take(1)[0])
        mr = take(n).copy()
    assert pos == out.size, (pos, out.size)
    return ElasticResult(loop, E_k, E_p0, E_p1, traces, fields, coefs, weights, mt, mr)


@dataclass
class AcousticCase:
    """One periodic acoustic run in the single-core reference's terms.

    Grids (unpadded, x slow): Vx is N in x and M in y, (Nx+1, Ny); Vy is (Nx, Ny+1); P is (Nx, Ny).
    coef_vx / coef_vy = 1/rho on the velocity grids, coef_p = kappa = rho vp^2 on P.
    rcvs: list of (mesh, ix, iy) with mesh 0=Vx, 1=Vy, 2=P.
    """
    Nx: int
    Ny: int
    dx: float
    dt: float
    coef_vx: np.ndarray
    coef_vy: np.ndarray
    coef_p: np.ndarray
    src: tuple                  # (ix, iy) on P
    rcvs: list = field(default_factory=list)
    Nt: int = 10
    cpst: str = "0"
    central_f: float = 5.0
    time_delay: float = 0.25


@dataclass
class AcousticResult:
    loop_seconds: float
    energy: np.ndarray          # [3, Nt] per-mesh weighted sums (Vx, Vy, P)
    traces: np.ndarray          # [n_rcv, Nt]
    fields: dict                # Vx, Vy, P


def run_acoustic(case: AcousticCase, precision: str = "f64", perf: bool = False) -> AcousticResult:
    ih = np.zeros(16, np.int64)
    ih[:9] = [0x54574143, case.Nx, case.Ny, case.Nt, ord(case.cpst), case.src[0], case.src[1], len(case.rcvs), 1]
    dh = np.zeros(8, np.float64)
    dh[:4] = [case.dx, case.dt, case.central_f, case.time_delay]
    rcv = np.array(case.rcvs, np.int64).reshape(-1, 3)
    name = f"twref_acoustic_{precision}" + ("_perf" if perf else "")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(ih.tobytes()); f.write(dh.tobytes())
            for a in (case.coef_vx, case.coef_vy, case.coef_p):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(rcv.tobytes())
        subprocess.run([ref_binary(name), fin, fout], check=True, stdout=subprocess.DEVNULL)
        out = np.fromfile(fout, np.float64)
    Nt, n, Nx, Ny = case.Nt, len(case.rcvs), case.Nx, case.Ny
    loop = float(out[0])
    pos = 1
    energy = out[pos:pos + 3 * Nt].reshape(3, Nt); pos += 3 * Nt
    traces = out[pos:pos + n * Nt].reshape(n, Nt); pos += n * Nt
    fields = {}
    for key, s in (("Vx", (Nx + 1, Ny)), ("Vy", (Nx, Ny + 1)), ("P", (Nx, Ny))):
        fields[key] = out[pos:pos + s[0] * s[1]].reshape(s); pos += s[0] * s[1]
    assert pos == out.size
    return AcousticResult(loop, energy, traces, fields)
