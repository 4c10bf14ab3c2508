"""Python front end of libtwave.so, the B200 SBP-SAT stepper (C ABI in include/twave.h).

The package loads the in-tree library built by tpu-wave_b200/build.py and raises if it is
missing: there is no CPU or pure-PyTorch path. `Solver` mirrors the reference's object protocol
(Class_Grid / Class_Forward_Specs in cuda/src/cpp): create the grids, set the material, place the
source and receivers, step, read fields, traces and energies.

The directory name is not a Python identifier; load it by path, e.g.

    spec = importlib.util.spec_from_file_location("twave", "tpu-wave_b200/__init__.py")
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libtwave.so")
HEADER = os.path.join(HERE, "..", "include", "twave.h")

ELASTIC, ACOUSTIC = 0, 1
SAT_FREE, PERIODIC, SAT_INTERFACE = 0, 1, 2
FP64, FP32, BF16, FP16 = 0, 1, 2, 3
CPST = {"00": 0, "-3C": 1, "-3R": 2, "3C": 3, "3R": 4, "6C": 5, "6R": 6, "split": 7}
NN, MN, NM, MM = 0, 1, 2, 3
GRID = {("N", "N"): NN, ("M", "N"): MN, ("N", "M"): NM, ("M", "M"): MM}
PRECISION = {"f64": FP64, "f32": FP32, "bf16": BF16, "fp16": FP16}

ERRORS = {0: "TW_OK", -1: "TW_ERR_INVALID", -2: "TW_ERR_CUDA", -3: "TW_ERR_NOMEM", -4: "TW_ERR_STATE",
          -5: "TW_ERR_LOCATION", -6: "TW_ERR_OUTSIDE", -7: "TW_ERR_WEAK_BOUNDARY", -8: "TW_ERR_RECORD_FULL",
          -9: "TW_ERR_NONFINITE", -10: "TW_ERR_UNSUPPORTED", -11: "TW_ERR_MODEL_BOUNDS", -12: "TW_ERR_TOO_LARGE", -13: "TW_ERR_IO", -14: "TW_ERR_TIMEOUT"}


class TwError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        self.name = ERRORS.get(code, str(code))
        super().__init__(f"{what}: {self.name}")


class GridDesc(C.Structure):
    _fields_ = [("physics", C.c_int), ("bc_x", C.c_int), ("precision", C.c_int), ("cpst", C.c_int),
                ("Mx", C.c_long), ("My", C.c_long), ("num_dx", C.c_int), ("den_dx", C.c_int),
                ("dt", C.c_double), ("central_f", C.c_double), ("time_delay", C.c_double),
                ("source_scaling", C.c_double), ("max_steps", C.c_int), ("energy", C.c_int), ("device", C.c_int),
                ("coef_fp16", C.c_int), ("sat_y", C.c_int)]


class Info(C.Structure):
    _fields_ = [("rows", C.c_long * 4), ("cols", C.c_long * 4), ("pitch", C.c_long), ("steps_done", C.c_int),
                ("n_rcv", C.c_int), ("bytes_per_update", C.c_double), ("device_bytes", C.c_double),
                ("row_off", C.c_long), ("own_rows", C.c_long * 2), ("Mx_glob", C.c_long),
                ("step_kind", C.c_int), ("launches_per_step", C.c_int)]


_lib = None


def library_path() -> str:
    return LIB_PATH


class IoInput(C.Structure):
    _fields_ = [("Mx_prmt", C.c_long), ("My_prmt", C.c_long), ("Mx", C.c_long), ("My", C.c_long),
                ("num_dxM", C.c_int), ("den_dxM", C.c_int), ("num_dx", C.c_int), ("den_dx", C.c_int),
                ("bdry", C.c_char * 4), ("Nt", C.c_long), ("dt_max", C.c_double), ("cfl", C.c_double),
                ("dt", C.c_double), ("central_f", C.c_double), ("time_delay", C.c_double), ("device", C.c_int)]


class IoPoint(C.Structure):
    _fields_ = [("src_index", C.c_long), ("rcv_index", C.c_long), ("type_x", C.c_char), ("type_y", C.c_char),
                ("num_x", C.c_long), ("den_x", C.c_long), ("num_y", C.c_long), ("den_y", C.c_long)]


def lib() -> C.CDLL:
    """Load libtwave.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python tpu-wave_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        vp, dp, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_long)
        L.tw_create.argtypes = [C.POINTER(vp), C.POINTER(GridDesc)]
        L.tw_destroy.argtypes = [vp]
        L.tw_destroy.restype = None
        L.tw_release_cached_memory.argtypes = [C.c_int]
        L.tw_set_material_model.argtypes = [vp, dp, dp, dp, C.c_long, C.c_long, C.c_int, C.c_int]
        L.tw_set_material_grid.argtypes = [vp, C.c_int, C.c_int, dp, C.c_long]
        L.tw_set_source_location.argtypes = [vp, C.c_char, C.c_char, C.c_long, C.c_long, C.c_long, C.c_long]
        L.tw_set_source.argtypes = [vp, C.c_int, C.c_long, C.c_long]
        L.tw_clear_source.argtypes = [vp]
        L.tw_add_receiver_location.argtypes = [vp, C.c_char, C.c_char, C.c_long, C.c_long, C.c_long, C.c_long]
        L.tw_add_receivers.argtypes = [vp, C.c_int, lp, lp, C.c_int]
        L.tw_reset.argtypes = [vp]
        L.tw_step.argtypes = [vp, C.c_int]
        L.tw_sync.argtypes = [vp]
        for name in ("tw_read_field", "tw_write_field", "tw_read_resid", "tw_write_resid"):
            getattr(L, name).argtypes = [vp, C.c_int, C.c_int, dp, C.c_long]
        L.tw_read_receivers.argtypes = [vp, dp]
        L.tw_read_coefficients.argtypes = [vp, C.c_int, C.c_int, dp, C.c_long]
        L.tw_read_energy.argtypes = [vp, dp, dp, dp]
        L.tw_get_info.argtypes = [vp, C.POINTER(Info)]
        L.tw_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.tw_profile.argtypes = [vp, C.c_int, dp]
        L.tw_material_map_noalloc.argtypes = [vp, vp, vp, C.c_long, C.c_long, C.c_int, C.c_int, C.c_long, C.c_long,
                                              C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
        L.tw_location_to_index.argtypes = [C.c_char, C.c_long, C.c_long, C.c_int, C.c_int, lp]
        L.tw_adjoint_gradient.argtypes = [vp, C.c_int, dp, C.c_int, dp, C.POINTER(dp), dp, dp, dp, C.POINTER(dp)]
        L.tw_adjoint_gradient_revolve.argtypes = [vp, C.c_int, dp, C.c_int, dp, C.POINTER(dp), dp, dp, dp, C.POINTER(dp)]
        L.tw_revolve_plan.argtypes = [C.c_int, C.c_int, lp, C.POINTER(C.c_int)]
        L.tw_io_read_input.argtypes = [C.c_char_p, C.POINTER(IoInput)]
        L.tw_io_read_srcrcv.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.tw_io_read_model.argtypes = [C.c_char_p, C.c_long, C.c_long, dp]
        L.tw_io_write_records.argtypes = [vp, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.tw_data_misfit.argtypes = [vp, dp, dp, dp]
        L.tw_create_slab.argtypes = [C.POINTER(vp), C.POINTER(GridDesc), C.c_long, C.c_long]
        L.tw_slab_exchange.argtypes = [vp, vp]
        L.tw_slab_run.argtypes = [C.POINTER(vp), C.c_int, C.c_int]
        L.tw_slab_pack.argtypes = [vp, C.c_int, vp, lp]
        L.tw_slab_unpack.argtypes = [vp, C.c_int, vp]
        L.tw_slab_halo.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(vp), lp, lp, lp]
        L.tw_batch_create.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int]
        L.tw_batch_destroy.argtypes = [vp]
        L.tw_batch_destroy.restype = None
        L.tw_batch_set_shape.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.tw_batch_get_shape.argtypes = [vp, C.POINTER(C.c_int)]
        L.tw_batch_tune.argtypes = [vp, C.c_int, dp]
        L.tw_batch_step.argtypes = [vp, C.c_int]
        L.tw_batch_sync.argtypes = [vp]
        L.tw_strerror.restype = C.c_char_p
        L.tw_strerror.argtypes = [C.c_int]
        L.tw_last_cuda_error.restype = C.c_char_p
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    """Names of the entry points include/twave.h declares (TW_API lines)."""
    import re
    with open(HEADER) as f:
        text = f.read()
    return re.findall(r"^TW_API[^(]*?\b(tw_\w+)\(", text, flags=re.M)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ok(code: int, what: str):
    if code != 0:
        if code == -2:
            what = f"{what} ({lib().tw_last_cuda_error().decode()})"
        raise TwError(code, what)


def io_read_input(path: str) -> IoInput:
    """The reference's InputFile.txt (tw_io_read_input)."""
    out = IoInput()
    _ok(lib().tw_io_read_input(path.encode(), C.byref(out)), "tw_io_read_input")
    return out


def io_read_srcrcv(path: str) -> list:
    """The Src and Rcv lines of the reference's SrcRcv.txt, in file order (tw_io_read_srcrcv)."""
    n = C.c_int()
    _ok(lib().tw_io_read_srcrcv(path.encode(), None, 0, C.byref(n)), "tw_io_read_srcrcv")
    arr = (IoPoint * max(n.value, 1))()
    _ok(lib().tw_io_read_srcrcv(path.encode(), arr, n.value, C.byref(n)), "tw_io_read_srcrcv")
    return [arr[i] for i in range(n.value)]


def io_read_model(path: str, Mx_prmt: int, My_prmt: int) -> np.ndarray:
    """A model file in the padded (Mx_prmt+2) x (My_prmt+2) layout (tw_io_read_model)."""
    out = np.zeros((Mx_prmt + 2, My_prmt + 2))
    _ok(lib().tw_io_read_model(path.encode(), Mx_prmt, My_prmt, _dp(out)), "tw_io_read_model")
    return out


def release_cached_memory(device: int = 0):
    """Give the device memory that destroyed handles left in the per-device pool back to the driver."""
    _ok(lib().tw_release_cached_memory(device), "tw_release_cached_memory")


def revolve_plan(nt: int, slots: int):
    """(forward steps, actions) of the binomial checkpointing schedule (tw_revolve_plan; host only)."""
    f, n = C.c_long(), C.c_int()
    _ok(lib().tw_revolve_plan(nt, slots, C.byref(f), C.byref(n)), "tw_revolve_plan")
    return f.value, n.value


def location_to_index(gtype: str, num: int, den: int, num_dx: int, den_dx: int) -> int:
    """Rational location -> grid index through the library (forward.cpp:31-51)."""
    out = C.c_long()
    _ok(lib().tw_location_to_index(gtype.encode(), num, den, num_dx, den_dx, C.byref(out)), "tw_location_to_index")
    return out.value


class Solver:
    """One simulation: the reference's four grids + forward specs, on one GPU stream."""

    def __init__(self, Mx: int, My: int, num_dx: int, den_dx: int, dt: float, *, physics: int = ELASTIC,
                 bc_x: int = SAT_FREE, precision: str = "f32", cpst: str = "00", central_f: float = 5.0,
                 time_delay: float = 0.25, source_scaling: float = 1.0, max_steps: int = 1000,
                 energy: bool = True, device: int = 0, coef_fp16: bool = False, sat_y: bool = False,
                 coef_q16: bool = False):
        """coef_fp16: stepping coefficients stored in FP16; coef_q16: stored as 16-bit fixed-point
        codes on a per-array affine map (tw_grid_desc.coef_fp16 = 1 / 2)."""
        self.desc = GridDesc(physics, bc_x, PRECISION[precision], CPST[cpst], Mx, My, num_dx, den_dx, dt,
                             central_f, time_delay, source_scaling, max_steps, 1 if energy else 0, device,
                             2 if coef_q16 else (1 if coef_fp16 else 0), 1 if sat_y else 0)
        self.h = C.c_void_p()
        _ok(lib().tw_create(C.byref(self.h), C.byref(self.desc)), "tw_create")
        self.Mx, self.My, self.physics, self.bc_x = Mx, My, physics, bc_x
        self.n_rcv = 0

    @classmethod
    def slab(cls, Mx: int, My: int, num_dx: int, den_dx: int, dt: float, row0: int, row1: int, **kw):
        """The handle of global rows [row0, row1) of an Mx x My elastic grid (tw_create_slab)."""
        self = cls.__new__(cls)
        energy = kw.pop("energy", True)
        self.desc = GridDesc(ELASTIC, SAT_FREE, PRECISION[kw.pop("precision", "f32")], CPST[kw.pop("cpst", "00")], Mx, My,
                             num_dx, den_dx, dt, kw.pop("central_f", 5.0), kw.pop("time_delay", 0.25),
                             kw.pop("source_scaling", 1.0), kw.pop("max_steps", 1000), 1 if energy else 0,
                             kw.pop("device", 0), 1 if kw.pop("coef_fp16", False) else 0, 0)
        if kw:
            raise TypeError(f"unexpected arguments {sorted(kw)}")
        self.h = C.c_void_p()
        _ok(lib().tw_create_slab(C.byref(self.h), C.byref(self.desc), row0, row1), "tw_create_slab")
        inf = self.info()
        self.Mx, self.My, self.physics, self.bc_x = int(inf.rows[3]), My, ELASTIC, SAT_FREE   # local cells
        self.n_rcv = 0
        self.Mx_glob = Mx
        self.row_off, self.own = int(inf.row_off), (int(inf.own_rows[0]), int(inf.own_rows[1]))
        return self

    def halo_spans(self, side: int, recv: int) -> list:
        """(slot, (device pointer, bytes)) of every state array's rows at one edge (tw_slab_halo):
        the owned rows the neighbour on `side` (0 top, 1 bottom) needs (recv 0) or this slab's halo
        rows there (recv 1), of the current buffers, each one contiguous span (the rows with the
        pitch padding between them)."""
        out = []
        for f in range(10):
            ptr, rows, rb, pb = C.c_void_p(), C.c_long(), C.c_long(), C.c_long()
            rc = lib().tw_slab_halo(self.h, side, recv, f, C.byref(ptr), C.byref(rows), C.byref(rb), C.byref(pb))
            if rc != 0:
                if f < 5:
                    _ok(rc, "tw_slab_halo")
                continue   # no compensation array in this slot
            out.append((f, (ptr.value, (rows.value - 1) * pb.value + rb.value)))
        return out

    def halo_bytes(self, side: int) -> int:
        n = C.c_long()
        _ok(lib().tw_slab_pack(self.h, side, None, C.byref(n)), "tw_slab_pack")
        return n.value

    def pack(self, side: int, dst_ptr: int):
        """The owned rows the neighbour on `side` (0 top, 1 bottom) needs, into device memory."""
        n = C.c_long()
        _ok(lib().tw_slab_pack(self.h, side, C.c_void_p(dst_ptr), C.byref(n)), "tw_slab_pack")

    def unpack(self, side: int, src_ptr: int):
        """A buffer packed by the neighbour on `side` into this slab's halo rows there."""
        _ok(lib().tw_slab_unpack(self.h, side, C.c_void_p(src_ptr)), "tw_slab_unpack")

    def exchange(self, lower: "Solver"):
        """Refresh the halo rows shared with the slab just below (tw_slab_exchange)."""
        _ok(lib().tw_slab_exchange(self.h, lower.h), "tw_slab_exchange")

    @staticmethod
    def slab_run(slabs, steps: int):
        """Step all slabs of a grid (top to bottom) `steps` steps with the halo exchange fused into
        the step kernel (tw_slab_run); returns after queuing."""
        arr = (C.c_void_p * len(slabs))(*[s.h.value for s in slabs])
        _ok(lib().tw_slab_run(arr, len(slabs), steps), "tw_slab_run")

    def close(self):
        if self.h:
            lib().tw_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- sizes
    def shape(self, grid: int):
        Mx, My = self.Mx, self.My
        return {NN: (Mx + 1, My + 1), MN: (Mx, My + 1), NM: (Mx + 1, My), MM: (Mx, My)}[grid]

    # ---- material
    def set_material_model(self, rho, vp, vs=None, Mx_prmt=None, My_prmt=None, num_dxM=None, den_dxM=None):
        Mxp = getattr(self, "Mx_glob", self.Mx) if Mx_prmt is None else Mx_prmt   # a slab: the whole grid's
        Myp = self.My if My_prmt is None else My_prmt
        nd = self.desc.num_dx if num_dxM is None else num_dxM
        dd = self.desc.den_dx if den_dxM is None else den_dxM
        P = (Mxp + 2) * (Myp + 2)
        arrs = [np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1)) for a in (rho, vp)]
        arrs.append(np.zeros(P) if vs is None else np.ascontiguousarray(np.asarray(vs, np.float64).reshape(-1)))
        for a in arrs:
            if a.size != P:
                raise ValueError(f"model arrays must hold (Mx_prmt+2)*(My_prmt+2) = {P} values")
        _ok(lib().tw_set_material_model(self.h, *[_dp(a) for a in arrs], Mxp, Myp, nd, dd), "tw_set_material_model")
        self.model_shape = (Mxp + 2, Myp + 2)

    def set_material_grid(self, grid: int, idx: int, coef):
        a = np.ascontiguousarray(np.asarray(coef, np.float64))
        r, c = self.shape(grid)
        if a.shape != (r, c):
            raise ValueError(f"expected shape {(r, c)}, got {a.shape}")
        _ok(lib().tw_set_material_grid(self.h, grid, idx, _dp(a), c), "tw_set_material_grid")

    # ---- source / receivers
    def set_source(self, grid: int, ix: int, iy: int):
        _ok(lib().tw_set_source(self.h, grid, ix, iy), "tw_set_source")

    def set_source_location(self, tx, ty, nx, dxn, ny, dyn):
        _ok(lib().tw_set_source_location(self.h, tx.encode(), ty.encode(), nx, dxn, ny, dyn), "tw_set_source_location")

    def clear_source(self):
        _ok(lib().tw_clear_source(self.h), "tw_clear_source")

    def add_receivers(self, grid: int, ix, iy):
        ix = np.ascontiguousarray(np.atleast_1d(ix), np.int64)
        iy = np.ascontiguousarray(np.atleast_1d(iy), np.int64)
        lp = C.POINTER(C.c_long)
        _ok(lib().tw_add_receivers(self.h, grid, ix.ctypes.data_as(lp), iy.ctypes.data_as(lp), int(ix.size)),
            "tw_add_receivers")
        self.n_rcv += int(ix.size)

    def add_receiver_location(self, tx, ty, nx, dxn, ny, dyn):
        _ok(lib().tw_add_receiver_location(self.h, tx.encode(), ty.encode(), nx, dxn, ny, dyn), "tw_add_receiver_location")
        self.n_rcv += 1

    # ---- stepping
    def reset(self):
        _ok(lib().tw_reset(self.h), "tw_reset")

    def step(self, n: int):
        _ok(lib().tw_step(self.h, n), "tw_step")

    def sync(self):
        _ok(lib().tw_sync(self.h), "tw_sync")

    def run(self, n: int):
        self.step(n)
        self.sync()

    # ---- readback
    def read_field(self, grid: int, field: int = 0) -> np.ndarray:
        r, c = self.shape(grid)
        out = np.empty((r, c))
        _ok(lib().tw_read_field(self.h, grid, field, _dp(out), c), "tw_read_field")
        return out

    def write_field(self, grid: int, field: int, values):
        a = np.ascontiguousarray(np.asarray(values, np.float64))
        r, c = self.shape(grid)
        if a.shape != (r, c):
            raise ValueError(f"expected shape {(r, c)}")
        _ok(lib().tw_write_field(self.h, grid, field, _dp(a), c), "tw_write_field")

    def read_coefficients(self, grid: int, idx: int = 0) -> np.ndarray:
        """The stepping coefficient the handle steps with (tw_read_coefficients): NN mu, MN / NM
        1/rho, MM lambda (idx 0) and 2mu (idx 1), at reference sizes."""
        out = np.zeros(self.shape(grid))
        _ok(lib().tw_read_coefficients(self.h, grid, idx, _dp(out), out.shape[1]), "tw_read_coefficients")
        return out

    def read_resid(self, grid: int, field: int = 0) -> np.ndarray:
        r, c = self.shape(grid)
        out = np.empty((r, c))
        _ok(lib().tw_read_resid(self.h, grid, field, _dp(out), c), "tw_read_resid")
        return out

    def write_resid(self, grid: int, field: int, values):
        a = np.ascontiguousarray(np.asarray(values, np.float64))
        r, c = self.shape(grid)
        _ok(lib().tw_write_resid(self.h, grid, field, _dp(a), c), "tw_write_resid")

    def info(self) -> Info:
        inf = Info()
        _ok(lib().tw_get_info(self.h, C.byref(inf)), "tw_get_info")
        return inf

    def read_receivers(self) -> np.ndarray:
        n = self.info().steps_done
        out = np.zeros((self.n_rcv, 2, n))
        if self.n_rcv and n:
            _ok(lib().tw_read_receivers(self.h, _dp(out)), "tw_read_receivers")
        return out

    def read_energy(self):
        n = self.info().steps_done
        E_k, E_p0, E_p1 = np.zeros(n), np.zeros(n), np.zeros(n)
        if n:
            _ok(lib().tw_read_energy(self.h, _dp(E_k), _dp(E_p0), _dp(E_p1)), "tw_read_energy")
        return E_k, E_p0, E_p1

    def profile(self, n: int) -> np.ndarray:
        """Mean ms per launch of [velocity, stress, energy, gather] over n eagerly launched steps."""
        ms = np.zeros(4)
        _ok(lib().tw_profile(self.h, n, _dp(ms)), "tw_profile")
        return ms

    def adjoint_gradient(self, nt: int, obs, ckpt_every: int = 50, model: bool = True, state: bool = False,
                         slots: int = 0):
        """Misfit and gradients (tw_adjoint_gradient; with slots > 0 tw_adjoint_gradient_revolve,
        binomial checkpointing in that many states). obs: [n_rcv, 2, nt]. Returns a dict with
        "misfit", "grid" (NN mu, MN rho, NM rho, MM lambda, MM 2mu), and "rho", "vp", "vs" (padded
        node model, when model=True) and "state" (initial fields, when state=True)."""
        o = np.ascontiguousarray(np.asarray(obs, np.float64).reshape(self.n_rcv, 2, nt)) if self.n_rcv else np.zeros(1)
        shapes = [self.shape(g) for g in (NN, MN, NM, MM, MM)]
        grid = [np.zeros(sh) for sh in shapes]
        garr = (C.POINTER(C.c_double) * 5)(*[_dp(g) for g in grid])
        out = {"grid": dict(zip(("NN_mu", "MN_rho", "NM_rho", "MM_lambda", "MM_2mu"), grid))}
        mdl = [None, None, None]
        if model:
            mdl = [np.zeros(self.model_shape) for _ in range(3)]
        st = [np.zeros(sh) for sh in shapes] if state else None
        sarr = (C.POINTER(C.c_double) * 5)(*[_dp(g) for g in st]) if state else None
        J = C.c_double()
        fn, arg = (lib().tw_adjoint_gradient_revolve, slots) if slots > 0 else (lib().tw_adjoint_gradient, ckpt_every)
        _ok(fn(self.h, nt, _dp(o), arg, C.byref(J), garr, *[(_dp(m) if m is not None else None) for m in mdl], sarr),
            "tw_adjoint_gradient")
        out["misfit"] = J.value
        if model:
            out["rho"], out["vp"], out["vs"] = mdl
        if state:
            out["state"] = dict(zip(("NN", "MN", "NM", "MM0", "MM1"), st))
        return out

    def data_misfit(self, obs):
        """(total, per receiver) sum of squared trace residuals (tw_data_misfit)."""
        n = self.info().steps_done
        o = np.ascontiguousarray(np.asarray(obs, np.float64).reshape(self.n_rcv, 2, n))
        tot, per = C.c_double(), np.zeros(max(self.n_rcv, 1))
        _ok(lib().tw_data_misfit(self.h, _dp(o), C.byref(tot), _dp(per)), "tw_data_misfit")
        return tot.value, per[:self.n_rcv]

    def write_records(self, folder: str, src_index: int = 0, rcv_index=None, snapshots: bool = False):
        """The reference's Signal / Energy / Snapshot text files (tw_io_write_records)."""
        ri = None
        if rcv_index is not None:
            ri = (C.c_int * len(rcv_index))(*rcv_index)
        _ok(lib().tw_io_write_records(self.h, folder.encode(), src_index, ri, int(snapshots)), "tw_io_write_records")

    def stream(self) -> int:
        p = C.c_void_p()
        _ok(lib().tw_get_stream(self.h, C.byref(p)), "tw_get_stream")
        return p.value or 0


class Batch:
    """Many acoustic Solver handles stepped together (one launch per half-step for all shots).
    The shots keep their own set-up and readback; see tw_batch_create."""

    def __init__(self, shots):
        self.shots = list(shots)
        arr = (C.c_void_p * len(self.shots))(*[s.h for s in self.shots])
        self.h = C.c_void_p()
        _ok(lib().tw_batch_create(C.byref(self.h), arr, len(self.shots)), "tw_batch_create")

    def close(self):
        if self.h:
            lib().tw_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, tx: int, ty: int, rows_per_thread: int = 1, ctas: int = 0):
        _ok(lib().tw_batch_set_shape(self.h, tx, ty, rows_per_thread, ctas), "tw_batch_set_shape")

    def shape(self):
        out = (C.c_int * 4)()
        _ok(lib().tw_batch_get_shape(self.h, out), "tw_batch_get_shape")
        return tuple(out)

    def tune(self, steps: int = 8) -> float:
        """Pick the fastest launch shape; resets every shot afterwards."""
        ms = C.c_double()
        _ok(lib().tw_batch_tune(self.h, steps, C.byref(ms)), "tw_batch_tune")
        return ms.value

    def step(self, n: int):
        _ok(lib().tw_batch_step(self.h, n), "tw_batch_step")

    def sync(self):
        _ok(lib().tw_batch_sync(self.h), "tw_batch_sync")

    def run(self, n: int):
        self.step(n)
        self.sync()
