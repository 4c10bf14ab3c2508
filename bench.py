#!/usr/bin/env python
"""Benchmark of the B200 SBP-SAT stepper on the elastic 2048^2 FP32 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one shot per GPU, weak scaling): 2D elastic, 2048 x 2048 cells, dx = 1/500, FP32,
seeded layered medium of 8 horizontal layers (per layer vp ~ U(1.5, 4.5), rho ~ U(1.8, 2.7);
vs = vp/sqrt(3) * U(0.9, 1.1) per node), CFL 0.4 (dt = 0.4 dx / (sqrt(2) vp_max)), explosive
Ricker source f0 = 15 on the normal-stress grid near the centre, 16 receivers on the NM grid.
A "step" is one leapfrog time step of the whole grid; one grid-point update (Gpt) is one cell
advanced one step with all five fields.

Printed JSON (rank 0): `value` = device-timed Gpt-updates/s over all ranks (inputs resident in
HBM); `e2e` = the same metric through the public C ABI with host buffers (model upload,
stepping, trace and energy readback inside the timed region); `roofline` = the dominant kernel's
algorithmic bytes per launch over its CUDA-event duration against the measured HBM copy
bandwidth; `cpu_baseline` = the reference's own CPU solver (oracle/_ref) on a bounded sample.
`--impl reference` times only the reference's CPU solver on the host cores.

`--workload mixed` measures the mixed-precision configuration instead: elastic 8192 x 8192,
seeded Gaussian-random-field medium, 2000 steps, every storage variant (FP64, FP32, BF16 and
FP16, plain and split) device-timed, with the relative L2 / Linf field error and the trace error
of each against the FP64 run of the same scheme.

`--workload batch` measures batching: 64 acoustic shots (periodic, FP32) of sizes drawn from
{256, 512, 1024, 2048}^2, each with its own seeded 8-layer medium and source, stepped together by
one batched launch per half-step (launch shape from the autotuner) against the same 64 handles
solved one after another; the traces of the two must agree bit for bit.

`--workload acoustic512` measures the plain-method acoustic configuration: 512 x 512 on [0,1]^2,
c = 1, rho = 1, FP32, CFL 0.5, Ricker f0 = 10 at the centre, 1000 steps, 16 receivers, in the
periodic and the free-surface mode (both two launches per step at this size), with
the reference's single-core solver on a sample of the same run for the CPU baseline and a
bit-for-bit trace comparison.

`--workload adjoint` measures the adjoint gradient: elastic 1024 x 1024 FP32, 2000 steps, 8
shots along row 16, 256 receivers on NM row 4; observed traces from the layered medium with a 5 %
Gaussian anomaly, gradient of the misfit with respect to rho, vp, vs of the layered medium,
checkpoints every 50 steps; checked against central differences (h = 1e-3) along 8 random
directions and by the dot-product identity of the state map (FP64).

`--workload variants` times the boundary variants on the elastic 2048 x 2048 FP32 workload: the x
ends joined by the SAT interface, free surfaces on all four sides, and both, beside the
reference's configuration.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpt-updates/s & %HBM roofline; plain FP32 vs mixed/batched at L2 err≤1e-4"
UNIT = "Gpt-updates/s"
MX = MY = 2048
DEN_DX = 500
CFL = 0.4
F0 = 15.0
DELAY = 0.1
SEED = 20261203 + 2
N_RCV = 16
L2_BYTES = 126 * 2**20


def workload_desc():
    return {"workload": "elastic 2048x2048 FP32, 8-layer seeded medium, CFL 0.4, Ricker f0=15 explosive, 16 receivers",
            "grid": [MX, MY], "dx": f"1/{DEN_DX}", "precision": "fp32", "compensation": "00",
            "energy": "off in value (on in e2e_energy)", "steps_per_shot_in_config": 4000,
            "l2": "inputs larger than L2 (fields + coefficients = 168 MB vs 126 MB L2), no flush"}


def build_model(rank: int = 0, n: int = MX):
    """Padded (n+2)x(n+2) node model in the reference layout (inverse.cpp:79-90, padding 0) of the
    8-layer medium on an n x n grid (n = 2048: the benchmark's workload)."""
    rng = np.random.default_rng(SEED)
    nl = 8
    vp_l, rho_l = rng.uniform(1.5, 4.5, nl), rng.uniform(1.8, 2.7, nl)
    P = (n + 2, n + 2)
    vp = np.zeros(P); rho = np.zeros(P)
    layer = np.minimum(np.arange(n + 1) * nl // (n + 1), nl - 1)
    vp[:n + 1, :n + 1] = vp_l[layer][:, None]
    rho[:n + 1, :n + 1] = rho_l[layer][:, None]
    vs = vp / np.sqrt(3.0) * rng.uniform(0.9, 1.1, P)
    vs[n + 1, :] = 0.0
    vs[:, n + 1] = 0.0
    dx = 1.0 / DEN_DX
    dt = CFL * dx / (np.sqrt(2.0) * vp.max())
    # one shot per rank: the source moves along y with the rank
    src_iy = (n // 2 + 16 * rank) % n
    return rho, vp, vs, dt, (n // 2, src_iy)


def receivers():
    return np.full(N_RCV, 8), 64 + 128 * np.arange(N_RCV)


def load_twave():
    import importlib.util
    spec = importlib.util.spec_from_file_location("twave", os.path.join(ROOT, "tpu-wave_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["twave"] = mod
    spec.loader.exec_module(mod)
    return mod


# ---------------------------------------------------------------- distributed plumbing
class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend: str):
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.pg.get_backend() == "nccl":
                import torch
                self.pg.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def reduce_max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = torch.device("cuda", self.local) if self.pg.get_backend() == "nccl" else torch.device("cpu")
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def finish(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks during the timed region
class ClockSampler:
    """SM clocks and clock-event reasons of one GPU, polled through NVML about every millisecond
    by a separate process (reading only; nothing is set), each sample stamped with the system-wide
    monotonic clock; `window(t0, t1)` summarises the samples between two time.monotonic() stamps
    of this process, so that a timed region of a few milliseconds still carries samples (a thread
    of this process would wait on the interpreter lock while the timed calls run). nvidia-smi at
    its fastest period (100 ms) is the fallback when NVML cannot be loaded."""
    CHILD = r"""
import sys, time, pynvml as nv
nv.nvmlInit()
try:
    h = nv.nvmlDeviceGetHandleByPciBusId(sys.argv[1])
except Exception:
    h = nv.nvmlDeviceGetHandleByIndex(int(sys.argv[2]))
names = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"), ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
         ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"), ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
         ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown")]
masks = [(n, getattr(nv, c)) for n, c in names if hasattr(nv, c)]
smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
while True:
    t = time.monotonic()
    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
    print(t, sm, smax, ",".join(n for n, m in masks if r & m) or "-", flush=True)
    time.sleep(0.001)
"""

    def __init__(self, device: int):
        self.device = device
        self.samples = []      # (monotonic time, sm MHz, max sm MHz, [reason names])
        self.proc = None
        self.out = None
        self.source = None

    def start(self):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            bus = ""
        self.out = tempfile.TemporaryFile(mode="w+")
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", self.CHILD, bus, str(self.device)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
            self.source = "nvml in a separate process, ~1 ms period"
            t0 = time.monotonic()   # the timed region must not begin before sampling does
            while time.monotonic() - t0 < 10.0 and self.proc.poll() is None:
                self.out.seek(0, io.SEEK_END)
                if self.out.tell() > 0:
                    break
                time.sleep(0.01)
            if self.proc.poll() is not None:
                raise OSError("nvml sampler exited")
        except OSError:
            self.proc = None
            self._start_smi()

    def _start_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.source = "nvidia-smi, 100 ms period"
        self.out = tempfile.TemporaryFile(mode="w+")
        try:
            self.smi = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                         "--format=csv,noheader,nounits", "-lms", "100"],
                                        stdout=self.out, stderr=subprocess.DEVNULL)
            self.t_smi = time.monotonic()
        except OSError:
            self.smi = None

    def _refresh(self):
        """Parse the complete lines the sampling process has written since the last call."""
        if not self.proc:
            return
        self.out.seek(getattr(self, "_pos", 0))
        text = self.out.read()
        cut = text.rfind("\n") + 1
        self._pos = getattr(self, "_pos", 0) + len(text[:cut].encode())
        for line in text[:cut].splitlines():
            f = line.split()
            if len(f) != 4:
                continue
            try:
                self.samples.append((float(f[0]), float(f[1]), float(f[2]), [] if f[3] == "-" else f[3].split(",")))
            except ValueError:
                pass

    def stop(self):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self._refresh()
            self.proc = None
        elif getattr(self, "smi", None):
            self.smi.terminate()
            self.smi.wait()
            self.out.seek(0)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) >= 6]
            for k, row in enumerate(rows):   # approximate times: one row per 100 ms from the start
                try:
                    self.samples.append((self.t_smi + 0.1 * k, float(row[0]), float(row[1]),
                                         [n for n, v in zip(names, row[2:6]) if v.strip().lower() == "active"]))
                except ValueError:
                    pass

    def window(self, t0: float, t1: float, min_samples: int = 5) -> dict:
        """Median SM clock, max clock and every reason seen between t0 and t1 (host times). A
        region too short for `min_samples` samples is widened symmetrically, 10 ms at a time up
        to 200 ms on each side (the GPU is busy with the warm-up before it and the per-kernel
        timing after it), and the margin is reported."""
        time.sleep(0.005)   # the samples just after the region
        self._refresh()
        margin = 0.0
        inside = [x for x in self.samples if t0 <= x[0] <= t1]
        while len(inside) < min_samples and margin < 0.2:
            margin += 0.01
            inside = [x for x in self.samples if t0 - margin <= x[0] <= t1 + margin]
        out = {"source": self.source, "samples": len(inside), "window_widened_ms_each_side": round(margin * 1e3)}
        if not inside:
            out.update({"sm_mhz": None, "sm_max_mhz": None, "reasons": []})
            return out
        out.update({"sm_mhz": statistics.median(x[1] for x in inside), "sm_max_mhz": max(x[2] for x in inside),
                    "sm_mhz_min": min(x[1] for x in inside),
                    "reasons": sorted({r for x in inside for r in x[3]})})
        return out


# ---------------------------------------------------------------- CPU baseline (reference solver)
def reference_case(steps: int, rank: int = 0):
    """The 2048^2 workload as a case of the reference's own solver (oracle/refrun.py)."""
    from oracle import refrun
    rho, vp, vs, dt, (sx, sy) = build_model(rank)
    rx, ry = receivers()
    return refrun.ElasticCase(Mx=MX, My=MY, num_dx=1, den_dx=DEN_DX, dt=dt, rho=rho.reshape(-1), vp=vp.reshape(-1),
                              vs=vs.reshape(-1), src=("M", "M", 2 * sx + 1, 2 * DEN_DX, 2 * sy + 1, 2 * DEN_DX),
                              rcvs=[("N", "M", int(a), DEN_DX, 2 * int(b) + 1, 2 * DEN_DX) for a, b in zip(rx, ry)],
                              Nt=steps, cpst="00", central_f=F0, time_delay=DELAY)


def reference_parity(tw, steps: int, dev: int = 0):
    """The first `steps` steps of the workload on the GPU (energy on) against the reference's own
    FP32 solver built from its sources (oracle/_ref, parity build): every field, the 16 traces and
    the three energy records. This is the checker, not a measured leg."""
    from oracle import refrun
    case = reference_case(steps)
    try:
        want = refrun.run_elastic(case, "f32")
    except (FileNotFoundError, OSError) as e:
        return {"steps": steps, "status": f"unavailable: {e}"}
    rho, vp, vs = (a.reshape(MX + 2, MY + 2) for a in (case.rho, case.vp, case.vs))
    s = tw.Solver(MX, MY, 1, DEN_DX, case.dt, physics=tw.ELASTIC, precision="f32", cpst="00", central_f=F0,
                  time_delay=DELAY, max_steps=steps, energy=True, device=dev)
    s.set_material_model(rho, vp, vs)
    s.set_source_location(*case.src)
    for r in case.rcvs:
        s.add_receiver_location(*r)
    s.run(steps)
    keys = {"NN": (tw.NN, 0), "MN": (tw.MN, 0), "NM": (tw.NM, 0), "MM0": (tw.MM, 0), "MM1": (tw.MM, 1)}
    fields_same = all(np.array_equal(s.read_field(*keys[k]), want.fields[k]) for k in keys)
    traces_same = bool(np.array_equal(s.read_receivers(), want.traces))
    ek, ep0, ep1 = s.read_energy()
    s.close()
    erel = max(float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
               for a, b in ((ek, want.E_k), (ep0, want.E_p0), (ep1, want.E_p1)))
    ok = fields_same and traces_same and erel <= 1e-12
    return {"steps": steps, "status": "bit-identical" if ok else "MISMATCH", "fields_bit_identical": fields_same,
            "traces_bit_identical": traces_same, "energy_max_rel_diff": erel,
            "against": "the reference's elastic FP32 host solver built from its sources (oracle/_ref/twref_elastic_f32)"}


def reference_sample(steps: int, procs: int = 1, rank: int = 0, warm: int = 0):
    """Run the reference's own elastic FP32 CPU solver (oracle/_ref, built from its sources) on
    `steps` time steps of the same workload in `procs` concurrent processes, each first making
    `warm` untimed passes of the same steps; returns (Gpt-updates/s aggregated over the
    processes, loop seconds of the timed pass per process, kind)."""
    from oracle import refrun
    case = reference_case(steps, rank)
    rho, vp, vs = (a.reshape(MX + 2, MY + 2) for a in (case.rho, case.vp, case.vs))
    dt = case.dt
    binary = os.path.join(refrun.REF_DIR, "twref_elastic_f32_perf")
    if not os.path.exists(binary):
        return None
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        ih = np.zeros(32, np.int64)
        cn, cs = refrun.CPST_CODES["00"]
        ih[:20] = [0x5457454C, MX, MY, MX, MY, 1, DEN_DX, 1, DEN_DX, steps, cn, ord(cs), ord("M"), ord("M"),
                   *case.src[2:6], len(case.rcvs), 1]
        ih[21] = warm
        dh = np.zeros(8); dh[:3] = [dt, F0, DELAY]
        with open(fin, "wb") as f:
            f.write(ih.tobytes()); f.write(dh.tobytes())
            for a in (rho, vp, vs):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(np.array([[ord("N"), ord("M"), *r[2:6]] for r in case.rcvs], np.int64).tobytes())
        ps = [subprocess.Popen([binary, fin, os.path.join(td, f"out{k}.bin")], stdout=subprocess.DEVNULL)
              for k in range(procs)]
        for p in ps:
            if p.wait() != 0:
                return None
        loops = [float(np.fromfile(os.path.join(td, f"out{k}.bin"), np.float64, count=1)[0]) for k in range(procs)]
    gpts = procs * MX * MY * steps / max(loops) / 1e9
    return gpts, loops, "reference"


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args, dist: Dist):
    if dist.rank != 0:
        return
    procs = max(1, min(cpu_threads(), 32))
    steps = max(1, min(args.steps, 20))
    warm = 1 if args.warmup > 0 else 0   # one untimed pass of the same steps first
    res = reference_sample(steps, procs, warm=warm)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU solver binary oracle/_ref missing"}))
        return
    gpts, loops, kind = res
    sample = (f"{procs} concurrent single-threaded processes of the reference elastic FP32 host solver, each "
              f"{steps} time steps of the 2048x2048 workload (energy every step, as the reference asserts), "
              f"timed after {warm * steps} untimed warm-up steps")
    line = {"metric": METRIC, "value": gpts, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm * steps, "ms_per_step": max(loops) / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_desc(),
            "cpu_baseline": {"value": gpts, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample},
            "e2e": {"value": gpts, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        line["gpu_executable"] = reference_gpu_executable()
    print(json.dumps(line), flush=True)


def reference_gpu_executable():
    """The reference's own GPU program (nvcc_device_FDM_2D.cu, unmodified, built for sm_100a) on
    the 2048^2 grid at the workload's dt, energy on as it requires: ms per step from runs of 200
    and 2200 steps (the fastest of two each, after a warm-up run; context beside the CPU arm, not
    its value)."""
    import shutil
    if shutil.which("nvidia-smi") is None:
        return {"unavailable": "no GPU visible"}
    try:
        from oracle import ref_gpu_timing
        dt = float(build_model(0, MX)[3])
        rec = ref_gpu_timing.time_reference_gpu(MX, DEN_DX, dt, F0, DELAY, (200, 2200))
    except Exception as e:  # a failed run is reported, not fatal to the CPU arm
        return {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    return rec if rec is not None else {"unavailable": "oracle/_ref/twref_elastic_gpu_f32 not built"}


# ---------------------------------------------------------------- our arm
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "of measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "of fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if one exists."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        e = t.get(kernel)
        return None if e is None else float(e["bytes_per_launch_full_size"])
    except (OSError, ValueError, KeyError):
        return None


def run_ours(args, dist: Dist):
    import torch
    tw = load_twave()
    dev = dist.local
    torch.cuda.set_device(dev)
    dist.init("nccl")
    rho, vp, vs, dt, (sx, sy) = build_model(dist.rank)
    rx, ry = receivers()
    K, W = args.steps, args.warmup
    P = min(max(K // 8, 20), 400)   # eagerly launched steps for the per-kernel timing
    s = tw.Solver(MX, MY, 1, DEN_DX, dt, physics=tw.ELASTIC, precision="f32", cpst="00", central_f=F0,
                  time_delay=DELAY, max_steps=W + K + P, energy=False, device=dev)
    s.set_material_model(rho, vp, vs)
    s.set_source(tw.MM, sx, sy)
    s.add_receivers(tw.NM, rx, ry)
    stream = torch.cuda.ExternalStream(s.stream(), device=dev)
    clocks = ClockSampler(dev)
    clocks.start()
    s.run(W)   # warm-up; its first call also captures the 16-step graph the timed call replays
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    th0 = time.monotonic()
    e0.record(stream)
    s.step(K)
    e1.record(stream)
    e1.synchronize()
    s.sync()
    torch.cuda.synchronize()
    th1 = time.monotonic()
    dist.barrier()
    clk = clocks.window(th0, th1)
    ms = e0.elapsed_time(e1)
    ms_max = dist.reduce_max(ms)
    updates = MX * MY * K * dist.world
    value = updates / (ms_max / 1e3) / 1e9

    # per-kernel durations (CUDA events around each launch on the solver's stream)
    info = s.info()
    prof = s.profile(P)
    if info.step_kind == 2:
        # TMA-staged step: one launch (boundary, warp-strip and TMA items of the persistent
        # strips' grid) or two side by side (the strips and the boundary / seam CTAs), timed
        # together; compulsory bytes = 5 fields read and written once + 5 coefficients read once
        # = 60 B per cell in FP32
        launches_per_step = int(info.launches_per_step)
        name = "k_elastic_tma (one launch a step)" if launches_per_step == 1 else "k_elastic_tma + k_elastic_side (one step)"
        alg, ms_k = MX * MY * 60, float(prof[0])
    elif prof[1] == 0.0:
        # fused path: the whole step is one launch
        name, alg, ms_k = "k_elastic_fused", MX * MY * 60, float(prof[0])
        launches_per_step = 1
    else:
        names = ["k_elastic_velocity", "k_elastic_stress"]
        algs = [MX * MY * (3 * 4 + 2 * 4 + 2 * 2 * 4), MX * MY * (2 * 4 + 3 * 4 + 3 * 2 * 4)]
        k = int(np.argmax(prof[:2]))
        name, alg, ms_k = names[k], algs[k], float(prof[k])
        launches_per_step = 3
    ms_bracketed = ms_k
    if launches_per_step == 1:
        # one launch a step: its average duration inside the timed region is the step time there
        # (graph replay; the gaps between launches count against it). tw_profile's figure, each
        # launch bracketed by its own events outside a graph, is reported beside it
        ms_k = ms_max / K
    achieved = alg / (ms_k / 1e3) / 1e9
    peak, peak_note = measured_peaks()
    tkey = name if info.step_kind != 2 else ("tma_step1@2048" if launches_per_step == 1 else "tma_step@2048")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": ncu_traffic(tkey), "kernel": name, "peak_source": peak_note,
                "algorithmic_bytes_per_launch": alg, "ms_per_launch": ms_k,
                "ms_per_launch_source": ("CUDA events over the timed region / steps (one launch a step)"
                                         if launches_per_step == 1 else "tw_profile: events around each step's launches"),
                "ms_per_launch_bracketed": ms_bracketed,
                "ms_per_launch_all": [float(x) for x in prof], "step_bytes_algorithmic_per_update": 60,
                "frac_of_step_time": alg / (ms_max / K / 1e3) / 1e9 / peak}
    s.close()

    e2e = run_e2e(args, dist, tw, torch, clocks, (rho, vp, vs, dt, (sx, sy)))
    target = None
    if not args.no_target and dist.world == 1:
        target = run_target_8192(args, tw, torch, clocks, dev)
    cpu, parity = None, None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        res = reference_sample(args.cpu_steps, 1)
        if res is not None:
            cpu = {"value": res[0], "unit": UNIT, "cores": 1, "kind": res[2],
                   "sample": f"{args.cpu_steps} time steps of this 2048x2048 workload, one process of the reference "
                             f"elastic FP32 host solver built from its sources (energy every step, as it asserts)"}
        parity = reference_parity(tw, min(K, 30), dev)
    clocks.stop()
    if dist.rank == 0:
        cfg = workload_desc()
        cfg["graph"] = "the 16-step CUDA graph is captured by the first (warm-up) call, outside the timed region"
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": K, "warmup": W,
                "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": cfg, "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": K * launches_per_step, "clocks": clk,
                "parity": parity, "target_8192": target}
        print(json.dumps(line), flush=True)
    dist.finish()


def run_e2e(args, dist: Dist, tw, torch, clocks, model):
    """The metric end to end through the C ABI with host buffers: handle creation, model upload
    from pinned host memory and FP64 interpolation on the GPU, K steps with the energy every step
    (as the reference computes it) and 16 receivers, trace and energy readback. One untimed pass
    first (the steady state of a caller that simulates shot after shot: kernels loaded, the
    handle pool holding memory), then the timed pass, then an untimed pass synchronised after
    each phase for the breakdown."""
    rho, vp, vs, dt, (sx, sy) = model
    rx, ry = receivers()
    K = args.steps
    dev = dist.local

    t0 = time.monotonic()
    pins = []
    for a in (rho, vp, vs):   # the caller's model in pinned host memory (staged once, reported)
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        pins.append(t)
    staging_s = time.monotonic() - t0
    host = [p.numpy() for p in pins]

    def one_pass(breakdown: bool):
        marks = []

        def mark(name):
            if breakdown:
                torch.cuda.synchronize(dev)
                marks.append((name, time.monotonic()))
        t0 = time.monotonic()
        s2 = tw.Solver(MX, MY, 1, DEN_DX, dt, physics=tw.ELASTIC, precision="f32", cpst="00", central_f=F0,
                       time_delay=DELAY, max_steps=K, energy=True, device=dev)
        mark("create")
        s2.set_material_model(*host)
        mark("material: model upload, interpolation, coefficients and energy weights")
        s2.set_source(tw.MM, sx, sy)
        s2.add_receivers(tw.NM, rx, ry)
        mark("source table and receivers")
        s2.step(K)
        if breakdown:
            marks.append(("steps enqueued (graph capture and launches, host side)", time.monotonic()))
        mark("steps run (energy every step)")
        traces = s2.read_receivers()
        energy = s2.read_energy()
        t1 = time.monotonic()
        mark("trace and energy readback")
        s2.close()
        phases = {}
        prev = t0
        for name, t in marks:
            phases[name] = (t - prev) * 1e3
            prev = t
        return t1 - t0, traces, energy, phases

    one_pass(False)
    torch.cuda.synchronize()
    dist.barrier()
    th0 = time.monotonic()
    secs, traces, energy, _ = one_pass(False)
    th1 = time.monotonic()
    clk = clocks.window(th0, th1)
    _, _, _, phases = one_pass(True)
    del pins, host
    e2e_s = dist.reduce_max(secs)
    h2d = 3 * rho.size * 8
    d2h = traces.nbytes + sum(e.nbytes for e in energy)
    return {"value": MX * MY * K * dist.world / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
            "d2h_bytes_per_step": d2h / K, "seconds": e2e_s,
            "includes": "handle creation, model upload from pinned host memory + FP64 interpolation on the "
                        "GPU, K steps with energy every step and 16 receivers, trace and energy readback",
            "warmup": "one untimed pass of the same calls first", "clocks": clk,
            "breakdown_ms": phases, "pinned_staging_ms_not_timed": staging_s * 1e3}


def run_target_8192(args, tw, torch, clocks, dev: int):
    """The plain FP32 stepper on an 8192 x 8192 grid of the same 8-layer medium (energy off):
    device-timed, with the dominant kernel's roofline fraction."""
    n, T, W = 8192, 48, 3
    rho, vp, vs, dt, (sx, sy) = build_model(0, n)
    s = tw.Solver(n, n, 1, DEN_DX, dt, physics=tw.ELASTIC, precision="f32", cpst="00", central_f=F0,
                  time_delay=DELAY, max_steps=W + T + 8, energy=False, device=dev)
    s.set_material_model(rho, vp, vs)
    del rho, vp, vs
    s.set_source(tw.MM, sx, sy)
    s.add_receivers(tw.NM, np.full(16, 8), 256 + 512 * np.arange(16))
    stream = torch.cuda.ExternalStream(s.stream(), device=dev)
    s.run(W)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    th0 = time.monotonic()
    e0.record(stream)
    s.step(T)
    e1.record(stream)
    e1.synchronize()
    s.sync()
    th1 = time.monotonic()
    ms = e0.elapsed_time(e1)
    tma = s.info().step_kind == 2
    one = int(s.info().launches_per_step) == 1
    prof = s.profile(8)
    s.close()
    peak, peak_note = measured_peaks()
    alg = n * n * 60
    ms_k = float(prof[0])
    kname = ("k_elastic_tma (one launch a step)" if one else "k_elastic_tma + k_elastic_side (one step)") if tma else "k_elastic_fused"
    return {"workload": f"elastic {n}x{n} FP32, the same 8-layer medium, energy off, 16 receivers",
            "steps": T, "warmup": W, "ms_per_step": ms / T, "gpts": n * n * T / (ms / 1e3) / 1e9,
            "roofline": {"kernel": kname, "algorithmic_bytes_per_launch": alg, "ms_per_launch": ms_k,
                         "achieved": alg / (ms_k / 1e3) / 1e9, "peak": peak, "peak_source": peak_note,
                         "frac": alg / (ms_k / 1e3) / 1e9 / peak,
                         "frac_of_step_time": alg / (ms / T / 1e3) / 1e9 / peak,
                         "traffic": ncu_traffic(("tma_step1@8192" if one else "tma_step@8192") if tma else "k_elastic_fused@8192")},
            "clocks": clocks.window(th0, th1), "l2": "inputs far larger than L2 (4 GB a step), no flush"}


# ---------------------------------------------------------------- mixed-precision workload
MIX_N = 8192
MIX_CORR = 32.0        # correlation length of the medium, cells
MIX_SEED = 20261203 + 3


def grf_model(n: int, seed: int):
    """Padded (n+2)^2 node model: vp a Gaussian random field (white noise filtered by a Gaussian
    whose autocorrelation exp(-r^2 / (2 L^2)) has L = MIX_CORR cells), normalised to mean 3.0
    and standard deviation 0.3; vs = vp / sqrt(3); rho = 2.0."""
    import torch
    m = n + 2
    w = torch.from_numpy(np.random.default_rng(seed).standard_normal((m, m))).cuda()
    k = torch.fft.fftfreq(m, device="cuda", dtype=torch.float64)
    sigma = MIX_CORR / np.sqrt(2.0)   # kernel width: g * g has variance 2 sigma^2 = L^2
    g = torch.exp(-2 * np.pi ** 2 * sigma ** 2 * (k[:, None] ** 2 + k[None, :] ** 2))
    f = torch.fft.ifft2(torch.fft.fft2(w) * g).real
    f = (f - f.mean()) / f.std()
    vp = (3.0 + 0.3 * f).cpu().numpy()
    del w, g, f
    torch.cuda.empty_cache()
    return np.full_like(vp, 2.0), vp, vp / np.sqrt(3.0)


def run_mixed(args):
    import torch
    tw = load_twave()
    torch.cuda.set_device(0)
    n, K = MIX_N, args.steps
    rho, vp, vs = grf_model(n, MIX_SEED)
    dx = 1.0 / DEN_DX
    dt = CFL * dx / (np.sqrt(2.0) * vp.max())
    # 64 receivers on the NM grid along a row 160 cells from the source, within reach in 2000 steps
    rx, ry = np.full(64, n // 2 - 160), n // 2 - 320 + 10 * np.arange(64)
    # (storage, compensation, coefficient storage, algorithmic bytes per update); coefficients:
    # "full" = the compute type, "c16" = FP16, "q16" = 16-bit fixed-point codes on a per-array map
    variants = [("f64", "00", "full", 120), ("f32", "00", "full", 60), ("f32", "00", "q16", 50),
                ("f32", "00", "c16", 50), ("bf16", "00", "full", 40), ("bf16", "split", "full", 60),
                ("fp16", "00", "full", 40), ("fp16", "split", "full", 60), ("fp16", "split", "c16", 50)]
    if args.variant:   # e.g. "f32-00" or "f32-00-q16": run only these (errors need "f64-00" first)
        names = args.variant.split(",")
        variants = [v for v in variants if f"{v[0]}-{v[1]}" + ("" if v[2] == "full" else "-" + v[2]) in names]
        if not variants:
            raise SystemExit(f"--variant {args.variant}: no such variant")
    peak, peak_note = measured_peaks()
    keys = [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
    ref = None
    out = []
    for prec, cpst, cstore, bpu in variants:
        s = tw.Solver(n, n, 1, DEN_DX, dt, physics=tw.ELASTIC, precision=prec, cpst=cpst, central_f=F0,
                      time_delay=DELAY, max_steps=args.warmup + K, energy=False, coef_fp16=cstore == "c16",
                      coef_q16=cstore == "q16")
        s.set_material_model(rho, vp, vs)
        s.set_source(tw.MM, n // 2, n // 2)
        s.add_receivers(tw.NM, rx, ry)
        stream = torch.cuda.ExternalStream(s.stream())
        # warm-up on a copy of the run: reset afterwards so every variant steps K from rest
        s.run(args.warmup)
        s.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(K)
        e1.record(stream)
        e1.synchronize()
        s.sync()
        ms = e0.elapsed_time(e1)
        fields = [s.read_field(g, f) for g, f in keys]
        traces = s.read_receivers()
        kind = s.info().step_kind
        s.close()
        gpts = n * n * K / (ms / 1e3) / 1e9
        row = {"precision": prec, "compensation": cpst,
               "coefficients": {"full": "compute type", "c16": "fp16", "q16": "16-bit fixed point"}[cstore],
               "step": {2: "TMA-staged (two launches)", 1: "one-launch per-warp kernel"}.get(kind, "other"),
               "gpts": gpts, "ms_per_step": ms / K,
               "bytes_per_update": bpu, "hbm_frac": gpts * bpu / peak}
        if prec != "f64" and ref is None:
            row.update({"l2_err": None, "linf_err": None, "trace_err": None})
        elif ref is None:
            ref = (fields, traces)
            row.update({"l2_err": 0.0, "linf_err": 0.0, "trace_err": 0.0})
        else:
            num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(fields, ref[0]))
            den = sum(float(np.sum(b ** 2)) for b in ref[0])
            linf = max(float(np.abs(a - b).max()) for a, b in zip(fields, ref[0]))
            scale = max(float(np.abs(b).max()) for b in ref[0])
            row.update({"l2_err": (num / den) ** 0.5, "linf_err": linf / scale,
                        "trace_err": float(np.linalg.norm(traces - ref[1]) / np.linalg.norm(ref[1]))})
        del fields, traces
        out.append(row)
    best = max((r for r in out if (r["precision"] in ("bf16", "fp16") or r["coefficients"] != "compute type")
                and r["l2_err"] is not None and r["l2_err"] <= 1e-4), key=lambda r: r["gpts"], default=None)
    f32 = next((r for r in out if r["precision"] == "f32" and r["coefficients"] == "compute type"), None)
    line = {"metric": METRIC, "value": best["gpts"] if best else None, "unit": UNIT, "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "higher_is_better": True,
            "dtype": f"{best['precision']} fields, {best['coefficients']} coefficients, f32 arithmetic" if best else None,
            "data": "synthetic",
            "config": {"workload": f"mixed precision: elastic {n}x{n}, Gaussian-random-field medium (vp mean 3.0, "
                                   f"std 0.3, correlation length {MIX_CORR:g} cells, vs = vp/sqrt(3), rho = 2.0), "
                                   f"CFL 0.4, Ricker f0=15 at the centre, 64 receivers on an NM row 160 cells from it",
                       "errors": "relative L2 over all five fields, Linf / max |FP64|, trace L2, vs the FP64 run",
                       "l2": f"inputs far larger than L2, no flush", "peak": f"{peak} GB/s {peak_note}"},
            "variants": out,
            "best_mixed_over_plain_fp32": (best["gpts"] / f32["gpts"]) if best and f32 else None}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batched acoustic workload
BATCH_SEED = 20261203 + 4


def batch_shots(tw, n_shots: int, steps: int):
    rng = np.random.default_rng(BATCH_SEED)
    shots, cells = [], 0
    for k in range(n_shots):
        side = int(rng.choice([256, 512, 1024, 2048]))
        nl = 8
        c_l, rho_l = rng.uniform(1.0, 3.0, nl), rng.uniform(1.0, 2.5, nl)
        dx = 1.0 / side
        dt = 0.5 * dx / (np.sqrt(2.0) * c_l.max())
        sx, sy = (int(v) for v in rng.integers(8, side - 8, 2))
        s = tw.Solver(side, side, 1, side, dt, physics=tw.ACOUSTIC, bc_x=tw.PERIODIC, precision="f32", cpst="00",
                      central_f=10.0, time_delay=0.1, max_steps=steps + 128, energy=False)
        lay = np.minimum(np.arange(side + 1) * nl // side, nl - 1)
        lay[side] = lay[0]   # the periodic seam row repeats row 0
        rho_x = rho_l[lay][:, None] * np.ones((1, side))            # Vx: (side+1) x side
        rho_y = rho_l[lay[:side]][:, None] * np.ones((1, side + 1))  # Vy: side x (side+1)
        kap = (rho_l * c_l ** 2)[lay[:side]][:, None] * np.ones((1, side))
        s.set_material_grid(tw.NM, 0, rho_x)
        s.set_material_grid(tw.MN, 0, rho_y)
        s.set_material_grid(tw.MM, 0, kap)
        s.set_source(tw.MM, sx, sy)
        s.add_receivers(tw.MM, np.full(16, (sx + 10) % side), (sy + np.arange(16) * (side // 16)) % side)
        shots.append(s)
        cells += side * side
    return shots, cells


def run_batch(args):
    import torch
    tw = load_twave()
    torch.cuda.set_device(0)
    K = args.steps
    shots, cells = batch_shots(tw, 64, K)
    # 64 sequential plain solves (each handle stepped alone, graphs of 16 steps); the warm-up is
    # long enough to capture every handle's graph before the timed region
    warm = max(args.warmup, 32)
    for s in shots:
        s.run(warm)
        s.reset()
    torch.cuda.synchronize()
    t0 = time.monotonic()
    for s in shots:
        s.run(K)
    t_seq = time.monotonic() - t0
    seq_traces = [s.read_receivers() for s in shots]
    for s in shots:
        s.reset()
    b = tw.Batch(shots)
    tuned_ms = b.tune(8)
    shape = b.shape()
    b.run(warm)
    for s in shots:
        s.reset()
    clocks = ClockSampler(0)
    clocks.start()
    torch.cuda.synchronize()
    t0 = time.monotonic()
    b.run(K)
    t1 = time.monotonic()
    t_bat = t1 - t0
    clocks.stop()
    clk = clocks.window(t0, t1)
    same = all(np.array_equal(s.read_receivers(), t) for s, t in zip(shots, seq_traces))
    b.close()
    for s in shots:
        s.close()
    peak, peak_note = measured_peaks()
    v_bat, v_seq = cells * K / t_bat / 1e9, cells * K / t_seq / 1e9
    line = {"metric": METRIC, "value": v_bat, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": args.warmup,
            "ms_per_step": t_bat / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batching: 64 acoustic periodic shots, sides drawn from {256,512,1024,2048} (seeded), "
                                   "8-layer media c ~ U(1,3), rho ~ U(1,2.5), Ricker f0=10, CFL 0.5, 16 receivers each",
                       "cells_per_step": cells, "timing": "host clock around the whole run, synchronised (both arms)"},
            "sequential": {"value": v_seq, "unit": UNIT, "seconds": t_seq},
            "batched": {"seconds": t_bat, "shape": shape, "tuned_ms_per_step": tuned_ms,
                        "speedup_vs_sequential": t_seq / t_bat, "traces_identical_to_sequential": same,
                        "hbm_frac_at_36B": v_bat * 36 / peak, "peak": f"{peak} GB/s {peak_note}"},
            "clocks": clk}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- plain acoustic 512^2
def run_acoustic512(args):
    import torch
    from oracle import refrun
    tw = load_twave()
    torch.cuda.set_device(0)
    n, K = 512, args.steps
    dx = 1.0 / n
    dt = 0.5 * dx / np.sqrt(2.0)
    rcv_ix, rcv_iy = np.full(16, 128), 16 + 32 * np.arange(16)
    out = {}
    for mode, bc, sat_y in (("periodic", tw.PERIODIC, False), ("free_surface", tw.SAT_FREE, False),
                            ("all_sides", tw.SAT_FREE, True)):
        s = tw.Solver(n, n, 1, n, dt, physics=tw.ACOUSTIC, bc_x=bc, precision="f32", cpst="00", central_f=10.0,
                      time_delay=0.25, max_steps=K + 64, energy=False, sat_y=sat_y)
        s.set_material_grid(tw.NM, 0, np.ones((n + 1, n)))
        s.set_material_grid(tw.MN, 0, np.ones((n, n + 1)))
        s.set_material_grid(tw.MM, 0, np.ones((n, n)))
        s.set_source(tw.MM, n // 2, n // 2)
        s.add_receivers(tw.MM, rcv_ix, rcv_iy)
        s.run(32)
        s.reset()
        stream = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(K)
        e1.record(stream)
        s.sync()
        ms = e0.elapsed_time(e1)
        out[mode] = {"gpts": n * n * K / (ms / 1e3) / 1e9, "ms_per_step": ms / K,
                     "hbm_frac_at_36B": n * n * K / (ms / 1e3) * 36 / 1e9 / measured_peaks()[0],
                     "traces": s.read_receivers()[:, 0, :]}
        s.close()
        if mode == "all_sides":
            # no reference run exists for free y ends: the discrete energy after the source stops
            # (t > delay + 3 / f0) is the check, over 2000 steps (FP64, energy every step)
            ne = 2000
            s = tw.Solver(n, n, 1, n, dt, physics=tw.ACOUSTIC, bc_x=bc, precision="f64", cpst="00",
                          central_f=10.0, time_delay=0.25, max_steps=ne, energy=True, sat_y=True)
            s.set_material_grid(tw.NM, 0, np.ones((n + 1, n)))
            s.set_material_grid(tw.MN, 0, np.ones((n, n + 1)))
            s.set_material_grid(tw.MM, 0, np.ones((n, n)))
            s.set_source(tw.MM, n // 2, n // 2)
            s.run(ne)
            ek, ep0, ep1 = s.read_energy()
            s.close()
            E = (ek + 0.5 * (ep0 + ep1))[int((0.25 + 3 / 10.0) / dt) + 1:]
            out[mode]["energy_min_over_max_after_source"] = float(E.min() / E.max())
            out[mode]["energy_steps"] = ne
    # the reference's single-core solver (periodic) on the first steps of the same run
    cs = min(K, args.cpu_steps * 10)
    case = refrun.AcousticCase(Nx=n, Ny=n, dx=dx, dt=dt, coef_vx=np.ones((n + 1, n)), coef_vy=np.ones((n, n + 1)),
                               coef_p=np.ones((n, n)), src=(n // 2, n // 2),
                               rcvs=[(2, int(a), int(b)) for a, b in zip(rcv_ix, rcv_iy)], Nt=cs, cpst="0",
                               central_f=10.0, time_delay=0.25)
    ref = refrun.run_acoustic(case, "f32", perf=True)   # timing build (the reference's -O3 flags)
    cpu = {"value": n * n * cs / ref.loop_seconds / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
           "sample": f"the first {cs} steps of this run, periodic mode, the reference's single-core acoustic FP32 solver"}
    case.Nt = 100                                         # parity build: traces bit for bit
    par = refrun.run_acoustic(case, "f32", perf=False)
    same = bool(np.array_equal(par.traces, out["periodic"]["traces"][:, :100]))
    for v in out.values():
        v.pop("traces")
    line = {"metric": METRIC, "value": out["periodic"]["gpts"], "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": 32,
            "ms_per_step": out["periodic"]["ms_per_step"], "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "plain acoustic 512x512 on [0,1]^2, c=1, rho=1, FP32, CFL 0.5, Ricker f0=10 at the "
                                   "centre, 16 receivers on P row 128; value: periodic mode (at this size the handle runs the "
                                   "two-launch step, faster than the fused one below 2^20 points)",
                       "l2": "grid far smaller than L2 (fields and coefficients 6 MB)"},
            "modes": out, "cpu_baseline": cpu, "traces_identical_to_reference_on_sample": same}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- adjoint workload
ADJ_N = 1024
ADJ_SEED = 20261203 + 5


def adjoint_media():
    rng = np.random.default_rng(ADJ_SEED)
    nl, n = 8, ADJ_N
    vp_l, rho_l = rng.uniform(1.5, 4.5, nl), rng.uniform(1.8, 2.7, nl)
    P = (n + 2, n + 2)
    layer = np.minimum(np.arange(n + 2) * nl // (n + 1), nl - 1)
    vp = np.repeat(vp_l[layer][:, None], n + 2, axis=1)
    rho = np.repeat(rho_l[layer][:, None], n + 2, axis=1)
    vs = vp / np.sqrt(3.0) * rng.uniform(0.9, 1.1, P)
    X, Y = np.meshgrid(np.arange(n + 2), np.arange(n + 2), indexing="ij")
    bump = 1.0 + 0.05 * np.exp(-((X - 150.0) ** 2 + (Y - n / 2) ** 2) / (2 * 40.0 ** 2))
    return rho, vp, vs, bump


def run_adjoint(args):
    import torch
    tw = load_twave()
    torch.cuda.set_device(0)
    n, K = ADJ_N, args.steps
    rho, vp, vs, bump = adjoint_media()
    dt = CFL * (1.0 / DEN_DX) / (np.sqrt(2.0) * (vp * bump).max())
    shots = [(16, 64 + 128 * k) for k in range(8)]
    rx, ry = np.full(256, 4), 4 * np.arange(256)

    def make(prec, r, p, q, src, energy=False):
        s = tw.Solver(n, n, 1, DEN_DX, dt, precision=prec, cpst="00", central_f=F0, time_delay=DELAY,
                      max_steps=K, energy=energy)
        s.set_material_model(r, p, q)
        if src is not None:
            s.set_source(tw.MM, *src)
        s.add_receivers(tw.NM, rx, ry)
        return s

    def traces(prec, r, p, q, src):
        s = make(prec, r, p, q, src)
        s.run(K)
        t = s.read_receivers()
        s.close()
        return t

    obs = [traces("f32", rho, vp * bump, vs * bump, src) for src in shots]
    # forward alone (device time), then the gradient call (host clock, synchronised), per shot
    s = make("f32", rho, vp, vs, shots[0])
    stream = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step(K)
    e1.record(stream)
    s.sync()
    fwd_ms = e0.elapsed_time(e1)
    s.close()
    g = {"rho": 0., "vp": 0., "vs": 0.}
    J0 = 0.
    t_grad = 0.
    for src, o in zip(shots, obs):
        s = make("f32", rho, vp, vs, src)
        torch.cuda.synchronize()
        t0 = time.monotonic()
        out = s.adjoint_gradient(K, o, ckpt_every=50)
        t_grad += time.monotonic() - t0
        s.close()
        J0 += out["misfit"]
        for k in g:
            g[k] = g[k] + out[k]

    # binomial checkpointing in a fixed number of state slots (tw_adjoint_gradient_revolve): the
    # first shot's gradient with 8 and 24 slots against the checkpoints every 50 steps above
    revolve = []
    for n_slots in (8, 24):
        s = make("f32", rho, vp, vs, shots[0])
        torch.cuda.synchronize()
        t0 = time.monotonic()
        out = s.adjoint_gradient(K, obs[0], slots=n_slots)
        dt_s = time.monotonic() - t0
        s.close()
        fwd_steps, _ = tw.revolve_plan(K, n_slots)
        revolve.append({"slots": n_slots, "seconds": dt_s, "forward_steps": fwd_steps,
                        "state_bytes": n_slots * 5 * (n + 1) * (n + 1) * 4})
    # the same gradient in FP64, and central differences of the FP64 misfit along 8 random
    # directions (unit normal perturbations of every node value of rho, vp, vs; h = 1e-3 and 1e-4)
    obs64 = [traces("f64", rho, vp * bump, vs * bump, src) for src in shots]
    g64 = {"rho": 0., "vp": 0., "vs": 0.}
    for src, o in zip(shots, obs64):
        s = make("f64", rho, vp, vs, src)
        out = s.adjoint_gradient(K, o, ckpt_every=50)
        s.close()
        for k in g64:
            g64[k] = g64[k] + out[k]

    def misfit64(r, p, q):
        return sum(0.5 * float(np.sum((traces("f64", r, p, q, src) - o) ** 2)) for src, o in zip(shots, obs64))

    rng = np.random.default_rng(ADJ_SEED + 1)
    fd_rows = []
    for k in range(8):
        d = [rng.standard_normal(rho.shape) for _ in range(3)]
        ana64 = sum(float(np.sum(g64[key] * dd)) for key, dd in zip(("rho", "vp", "vs"), d))
        ana32 = sum(float(np.sum(g[key] * dd)) for key, dd in zip(("rho", "vp", "vs"), d))
        row = {"adjoint_f64": ana64, "adjoint_f32": ana32, "f32_vs_f64_rel": abs(ana32 - ana64) / abs(ana64)}
        for h in (1e-3, 1e-4):
            fd = (misfit64(rho + h * d[0], vp + h * d[1], vs + h * d[2]) -
                  misfit64(rho - h * d[0], vp - h * d[1], vs - h * d[2])) / (2 * h)
            row[f"fd_h{h:g}"] = fd
            row[f"rel_err_h{h:g}"] = abs(fd - ana64) / abs(ana64)
        fd_rows.append(row)
    # dot-product identity of the state map L (initial fields -> traces), FP64, one shot, no source
    srng = np.random.default_rng(ADJ_SEED + 2)
    slots = [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
    shapes = [(n + 1, n + 1), (n, n + 1), (n + 1, n), (n, n), (n, n)]
    x = [srng.standard_normal(sh) for sh in shapes]
    s = make("f64", rho, vp, vs, None)
    for (gr, f), a in zip(slots, x):
        s.write_field(gr, f, a)
    s.run(K)
    dd = s.read_receivers()
    s.close()
    y = srng.standard_normal(dd.shape)
    y[:, 1, :] = 0.
    s = make("f64", rho, vp, vs, None)
    for (gr, f), a in zip(slots, x):
        s.write_field(gr, f, a)
    out = s.adjoint_gradient(K, dd - y, ckpt_every=50, model=False, state=True)
    s.close()
    lhs = float(np.sum(dd * y))
    rhs = float(sum(np.sum(a * out["state"][k]) for a, k in zip(x, ("NN", "MN", "NM", "MM0", "MM1"))))
    cells = n * n * K * len(shots)
    line = {"metric": METRIC, "value": cells / t_grad / 1e9, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": 0,
            "higher_is_better": True, "dtype": "f32 fields, f64 gradient accumulation", "data": "synthetic",
            "config": {"workload": f"adjoint gradient: elastic {n}x{n} FP32, {K} steps, 8 shots on MM row 16, 256 receivers "
                                   "on NM row 4, 8-layer medium, observed data from a 5 % Gaussian anomaly in vp and vs, "
                                   "checkpoints every 50 steps",
                       "value": "cell-steps of the forward problem per second of the whole gradient call "
                                "(forward sweep, segment recomputation, adjoint sweep), summed over the 8 shots"},
            "forward_ms_per_step": fwd_ms / K, "forward_gpts": n * n * K / (fwd_ms / 1e3) / 1e9,
            "gradient_seconds_per_shot": t_grad / len(shots),
            "revolve_first_shot": revolve,
            "gradient_over_forward_time": (t_grad / len(shots)) / (fwd_ms / 1e3),
            "misfit": J0, "finite_differences": {"field_precision": "f64 (FD and its adjoint); f32 adjoint compared",
                                                 "directions": fd_rows,
                                                 "max_rel_err_h1e-3": max(r["rel_err_h0.001"] for r in fd_rows),
                                                 "max_rel_err_h1e-4": max(r["rel_err_h0.0001"] for r in fd_rows),
                                                 "max_f32_vs_f64_rel": max(r["f32_vs_f64_rel"] for r in fd_rows)},
            "dot_product_test_f64": {"lhs": lhs, "rhs": rhs, "rel_err": abs(lhs - rhs) / abs(lhs)}}
    print(json.dumps(line), flush=True)


def run_variants(args):
    """The boundary variants on the elastic 2048^2 FP32 workload: the x ends joined by the SAT
    interface, free surfaces on all four sides, both; against the reference's configuration."""
    import torch
    tw = load_twave()
    torch.cuda.set_device(0)
    rho, vp, vs, dt, (sx, sy) = build_model(0)
    rx, ry = receivers()
    K = args.steps
    peak, peak_note = measured_peaks()
    out = {}
    for name, bc, sat_y in (("free_x_periodic_y", tw.SAT_FREE, False), ("interface_x", tw.SAT_INTERFACE, False),
                            ("free_all_sides", tw.SAT_FREE, True), ("interface_x_free_y", tw.SAT_INTERFACE, True)):
        s = tw.Solver(MX, MY, 1, DEN_DX, dt, physics=tw.ELASTIC, precision="f32", cpst="00", central_f=F0,
                      time_delay=DELAY, max_steps=args.warmup + K, energy=False, bc_x=bc, sat_y=sat_y)
        s.set_material_model(rho, vp, vs)
        s.set_source(tw.MM, sx, sy)
        s.add_receivers(tw.NM, rx, ry)
        stream = torch.cuda.ExternalStream(s.stream())
        s.run(args.warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(K)
        e1.record(stream)
        s.sync()
        ms = e0.elapsed_time(e1)
        s.close()
        gpts = MX * MY * K / (ms / 1e3) / 1e9
        out[name] = {"gpts": gpts, "ms_per_step": ms / K, "hbm_frac_at_60B": gpts * 60 / peak,
                     "kernels": "fused step, then the points next to the y ends recomputed (two launches)"
                                if sat_y else "fused step"}
    line = {"metric": METRIC, "value": out["free_all_sides"]["gpts"], "unit": UNIT, "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "ms_per_step": out["free_all_sides"]["ms_per_step"], "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "boundary variants of the elastic 2048x2048 FP32 workload (energy off); value: free "
                                   "surfaces on all four sides", "peak": f"{peak} GB/s {peak_note}",
                       "l2": "inputs larger than L2, no flush"},
            "variants": out}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-steps", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-target", action="store_true", help="skip the 8192^2 sub-record of the default run")
    ap.add_argument("--no-ref-gpu", action="store_true", help="reference arm: skip timing the reference's GPU program")
    ap.add_argument("--variant", default="", help="mixed workload: comma-separated variants to run "
                    "(storage-compensation[-c16], e.g. f32-00); all by default")
    ap.add_argument("--workload", choices=["elastic2048", "acoustic512", "mixed", "batch", "adjoint", "variants"],
                    default="elastic2048")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    dist = Dist()
    if args.impl == "reference":
        run_reference_arm(args, dist)
        return
    if args.workload in ("acoustic512", "mixed", "batch", "adjoint", "variants"):
        if dist.rank == 0:
            {"acoustic512": run_acoustic512, "mixed": run_mixed, "batch": run_batch,
             "adjoint": run_adjoint, "variants": run_variants}[args.workload](args)
        return
    run_ours(args, dist)


if __name__ == "__main__":
    main()
