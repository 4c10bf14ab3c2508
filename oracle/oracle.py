"""ctypes front end of the plain-C oracle (oracle/twave_oracle.c).

ORACLE / TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg as the checker. The product never imports it.

`elastic_run` takes the same `refrun.ElasticCase` as the reference driver and returns the same
`refrun.ElasticResult`, so a test can hold the restatement against the reference bit for bit.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

try:
    from . import refrun  # type: ignore
except ImportError:  # loaded by path
    import refrun  # type: ignore

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libtwave_oracle.so")
CPST_INDEX = {"00": 0, "-3C": 1, "-3R": 2, "3C": 3, "3R": 4, "6C": 5, "6R": 6, "split": 7}
STORE16 = {"bf16": 2, "fp16": 3}   # mixed precision: 16-bit storage, FP32 arithmetic
GRID_INDEX = {("N", "N"): 0, ("M", "N"): 1, ("N", "M"): 2, ("M", "M"): 3}

_lib = None


class _ElasticCfg(C.Structure):
    _fields_ = [("Mx", C.c_int), ("My", C.c_int), ("dx", C.c_double), ("dt", C.c_double),
                ("central_f", C.c_double), ("time_delay", C.c_double), ("cpst", C.c_int), ("Nt", C.c_int),
                ("src_grid", C.c_int), ("src_ix", C.c_long), ("src_iy", C.c_long), ("n_rcv", C.c_int),
                ("rcv_grid", C.POINTER(C.c_int)), ("rcv_ix", C.POINTER(C.c_long)), ("rcv_iy", C.POINTER(C.c_long)),
                ("bc_x", C.c_int), ("sat_y", C.c_int)]


class _AcousticCfg(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("dx", C.c_double), ("dt", C.c_double),
                ("central_f", C.c_double), ("time_delay", C.c_double), ("cpst", C.c_int), ("Nt", C.c_int),
                ("src_ix", C.c_long), ("src_iy", C.c_long), ("n_rcv", C.c_int),
                ("rcv_mesh", C.POINTER(C.c_int)), ("rcv_ix", C.POINTER(C.c_long)), ("rcv_iy", C.POINTER(C.c_long))]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: build it with `make -C oracle oracle`")
        _lib = C.CDLL(LIB_PATH)
        _lib.two_ricker.restype = C.c_double
        _lib.two_ricker.argtypes = [C.c_double, C.c_double]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def location_to_index(gtype: str, num: int, den: int, num_dx: int, den_dx: int) -> int:
    """Rational physical location -> grid index (forward.cpp:31-51); ValueError if not on the grid."""
    if gtype == "N":
        n, d = num * den_dx, den * num_dx
    else:
        n, d = 2 * num * den_dx - den * num_dx, 2 * den * num_dx
    if d == 0 or n % d != 0:
        raise ValueError("location is not a grid point")
    return n // d


def ricker(t: float, f0: float) -> float:
    return lib().two_ricker(t, f0)


def material(case: refrun.ElasticCase):
    """FP64 coefficients before rounding: NN mu, MN rho, NM rho, MM lambda, MM 2mu."""
    Mx, My = case.Mx, case.My
    Mxp = Mx if case.Mx_prmt is None else case.Mx_prmt
    Myp = My if case.My_prmt is None else case.My_prmt
    ndM = case.num_dx if case.num_dxM is None else case.num_dxM
    ddM = case.den_dx if case.den_dxM is None else case.den_dxM
    out = [np.zeros((Mx + 1, My + 1)), np.zeros((Mx, My + 1)), np.zeros((Mx + 1, My)), np.zeros((Mx, My)), np.zeros((Mx, My))]
    rho, vp, vs = (np.ascontiguousarray(a, np.float64) for a in (case.rho, case.vp, case.vs))
    rc = lib().two_material_map(Mx, My, case.num_dx, case.den_dx, Mxp, Myp, ndM, ddM, _p(rho), _p(vp), _p(vs),
                                *[_p(o) for o in out])
    if rc != 0:
        raise ValueError("material interpolation stepped out of the model")
    return out


BC_X = {"F": 0, "I": 2}


def elastic_coefficients(case: refrun.ElasticCase, precision: str):
    """Stored coefficients (T) and energy weights (FP64), as the reference prepares them."""
    T = np.float64 if precision == "f64" else np.float32
    mu, rho_mn, rho_nm, lam, m2 = material(case)
    stored = {"NN_mu": mu.astype(T), "MN_rho": rho_mn.astype(T), "NM_rho": rho_nm.astype(T),
              "MM_lambda": lam.astype(T), "MM_2mu": m2.astype(T),
              "MN_irho": (1.0 / rho_mn).astype(T), "NM_irho": (1.0 / rho_nm).astype(T)}
    Mx, My = case.Mx, case.My
    w = [np.zeros((Mx + 1, My + 1)), np.zeros((Mx, My + 1)), np.zeros((Mx + 1, My)), np.zeros((Mx, My)), np.zeros((Mx, My))]
    fn = lib().two_energy_weights_ext_f64 if precision == "f64" else lib().two_energy_weights_ext_f32
    dx = case.num_dx / case.den_dx
    fn(C.c_int(Mx), C.c_int(My), C.c_double(dx), C.c_int(int(case.sat_y)), _p(stored["NN_mu"]), _p(stored["MN_rho"]), _p(stored["NM_rho"]),
       _p(stored["MM_lambda"]), _p(stored["MM_2mu"]), *[_p(a) for a in w])
    weights = dict(zip(("NN", "MN", "NM", "MM_P1", "MM_P2"), w))
    return stored, weights


def elastic_run(case: refrun.ElasticCase, precision: str = "f64", fields0=None, resid0=None,
                coefs=None, weights=None) -> refrun.ElasticResult:
    """Run the restated elastic stepper. fields0/resid0: optional initial state (5 arrays,
    reference sizes). coefs/weights: optional overrides of the stored coefficients
    (keys NN_mu, MN_irho, NM_irho, MM_lambda, MM_2mu) and energy weights. precision "bf16" /
    "fp16" runs the mixed-precision restatement (FP32 arithmetic and coefficients, 16-bit field
    storage; case.cpst "00" or "split")."""
    T = np.float64 if precision == "f64" else np.float32
    stored, w = elastic_coefficients(case, "f64" if precision == "f64" else "f32")
    if coefs is not None:
        stored.update({k: np.ascontiguousarray(v, T) for k, v in coefs.items()})
    if weights is not None:
        w.update({k: np.ascontiguousarray(v, np.float64) for k, v in weights.items()})
    Mx, My, Nt = case.Mx, case.My, case.Nt
    sizes = refrun._elastic_sizes(Mx, My)
    keys = ("NN", "MN", "NM", "MM0", "MM1")
    fields = [np.zeros(sizes[k], T) if fields0 is None else np.array(fields0[i], T) for i, k in enumerate(keys)]
    resid = [np.zeros(sizes[k], T) if resid0 is None else np.array(resid0[i], T) for i, k in enumerate(keys)]
    nd, dd = case.num_dx, case.den_dx
    s = case.src
    if s is None:
        src_grid, sx, sy = -1, 0, 0
    else:
        src_grid = GRID_INDEX[(s[0], s[1])]
        sx = location_to_index(s[0], s[2], s[3], nd, dd)
        sy = location_to_index(s[1], s[4], s[5], nd, dd)
    n = len(case.rcvs)
    rg = np.array([GRID_INDEX[(r[0], r[1])] for r in case.rcvs] or [0], np.int32)
    rx = np.array([location_to_index(r[0], r[2], r[3], nd, dd) for r in case.rcvs] or [0], np.int64)
    ry = np.array([location_to_index(r[1], r[4], r[5], nd, dd) for r in case.rcvs] or [0], np.int64)
    cfg = _ElasticCfg(Mx, My, nd / dd, case.dt, case.central_f, case.time_delay, CPST_INDEX[case.cpst], Nt,
                      src_grid, sx, sy, n, rg.ctypes.data_as(C.POINTER(C.c_int)),
                      rx.ctypes.data_as(C.POINTER(C.c_long)), ry.ctypes.data_as(C.POINTER(C.c_long)),
                      BC_X[case.bc_x], int(case.sat_y))
    traces = np.zeros((n, 2, Nt))
    E_k, E_p0, E_p1 = np.zeros(Nt), np.zeros(Nt), np.zeros(Nt)
    FA = C.c_void_p * 5
    if precision in STORE16:
        fn = lambda cfgp, *rest: lib().two_elastic_run_mixed(cfgp, STORE16[precision], *rest)
    else:
        fn = lib().two_elastic_run_f64 if precision == "f64" else lib().two_elastic_run_f32
    rc = fn(C.byref(cfg), _p(stored["NN_mu"]), _p(stored["MN_irho"]), _p(stored["NM_irho"]),
            _p(stored["MM_lambda"]), _p(stored["MM_2mu"]), _p(w["NN"]), _p(w["MN"]), _p(w["NM"]),
            _p(w["MM_P1"]), _p(w["MM_P2"]), FA(*[f.ctypes.data for f in fields]),
            FA(*[r.ctypes.data for r in resid]), _p(traces), _p(E_k), _p(E_p0), _p(E_p1))
    if rc != 0:
        raise ValueError(f"oracle elastic run failed: {rc}")
    coef_out = {"NN_mu": stored["NN_mu"], "MN_irho": stored["MN_irho"], "NM_irho": stored["NM_irho"],
                "MM_lambda": stored["MM_lambda"], "MM_2mu": stored["MM_2mu"]}
    res = refrun.ElasticResult(0.0, E_k, E_p0, E_p1, traces, dict(zip(keys, fields)), coef_out, w)
    res.resid = dict(zip(keys, resid))
    return res


def acoustic_periodic_run(case: refrun.AcousticCase, precision: str = "f64", fields0=None, resid0=None):
    T = np.float64 if precision == "f64" else np.float32
    Nx, Ny, Nt = case.Nx, case.Ny, case.Nt
    shapes = ((Nx + 1, Ny), (Nx, Ny + 1), (Nx, Ny))
    coefs = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(s), T)
             for a, s in zip((case.coef_vx, case.coef_vy, case.coef_p), shapes)]
    fields = [np.zeros(s, T) if fields0 is None else np.array(fields0[i], T) for i, s in enumerate(shapes)]
    resid = [np.zeros(s, T) if resid0 is None else np.array(resid0[i], T) for i, s in enumerate(shapes)]
    n = len(case.rcvs)
    rm = np.array([r[0] for r in case.rcvs] or [0], np.int32)
    rx = np.array([r[1] for r in case.rcvs] or [0], np.int64)
    ry = np.array([r[2] for r in case.rcvs] or [0], np.int64)
    src = case.src if case.src is not None else (-1, 0)
    cfg = _AcousticCfg(Nx, Ny, case.dx, case.dt, case.central_f, case.time_delay, int(case.cpst), Nt,
                       src[0], src[1], n, rm.ctypes.data_as(C.POINTER(C.c_int)),
                       rx.ctypes.data_as(C.POINTER(C.c_long)), ry.ctypes.data_as(C.POINTER(C.c_long)))
    traces = np.zeros((n, Nt))
    energy = np.zeros((3, Nt))
    FA = C.c_void_p * 3
    fn = lib().two_acoustic_periodic_run_f64 if precision == "f64" else lib().two_acoustic_periodic_run_f32
    rc = fn(C.byref(cfg), *[_p(c) for c in coefs], FA(*[f.ctypes.data for f in fields]),
            FA(*[r.ctypes.data for r in resid]), _p(traces), _p(energy))
    if rc != 0:
        raise ValueError(f"oracle acoustic run failed: {rc}")
    res = refrun.AcousticResult(0.0, energy, traces, dict(zip(("Vx", "Vy", "P"), fields)))
    res.resid = dict(zip(("Vx", "Vy", "P"), resid))
    return res
