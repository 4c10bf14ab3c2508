"""Times the reference's own GPU executable on a B200 (measurement context; test infrastructure,
never part of the product).

`oracle/_ref/twref_elastic_gpu_f32` is cuda/src/cuda_main/nvcc_device_FDM_2D.cu with the
cuda/src/cuda and cuda/src/cpp trees, unmodified and with its own main, built for sm_100a by
`make -C oracle refgpu` (FP32 fields, as the FP32 workload here). That main reads
../../data/<medium>/InputFile.txt and SrcRcv.txt relative to its working directory
(nvcc_device_FDM_2D.cu:34, :212), replaces the medium read from file by the constants rho = 1,
vp = 2, vs = 1 (:150-156), steps with the energy on (it asserts that, :47), and writes its
records and every field as text at the end (:735-843). It has no timer of its own, so this script
runs it twice on the same inputs with two step counts and takes the difference of the wall-clock
times: set-up, the final write-out and process start-up are the same in both runs and cancel,
leaving the time of the extra steps (kernel launches, the per-step energy reductions with their
host synchronisations and the receiver launches, all inside the reference's loop :449-730).

The grid: n x n M points, dx = 1/500, the source on an MM point at the centre and 16 receivers on
MM points, dt (passed in) and the Ricker parameters of the 2048^2 elastic workload, with the
program's own constant medium (stable at that dt, which was set for a faster medium; the work of
a step does not depend on the medium's values).

Usage: python oracle/ref_gpu_timing.py --n 2048 --dt 1.2e-4 --steps 200 2200 [--out file.json]
"""
import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "twref_elastic_gpu_f32")


def write_inputs(data_dir: str, n: int, den: int, dt: float, f0: float, delay: float, n_rcv: int = 16):
    """InputFile.txt and SrcRcv.txt in the reference's formats (input_processing.cpp:8-139,
    inverse.cpp:133-290): one "<name>_<value>[_<value>]" token per line; locations as
    numerator_denominator pairs, MM points at (2c + 1) / (2 den)."""
    os.makedirs(data_dir, exist_ok=True)
    lines = [f"model_{n}_{n}", f"dxM_1_{den}", f"dxS_1_{den}", f"grids_{n}_{n}", "Nt_100",
             f"MAXdt_{dt!r}", "CFL_1.0", f"frequency_{f0!r}", f"delay_{delay!r}"]
    with open(os.path.join(data_dir, "InputFile.txt"), "w") as f:
        f.write("\n\n".join(lines) + "\n")
    c = n // 2
    src = f"Src_1_MM_{2 * c + 1}_{2 * den}_{2 * c + 1}_{2 * den}"
    rcvs = []
    for k in range(n_rcv):
        r = (64 + 128 * k) % n   # the same index on both axes: the order of the pair does not matter
        rcvs.append(f"Rcv_1_{k + 1}_MM_{2 * r + 1}_{2 * den}_{2 * r + 1}_{2 * den}")
    with open(os.path.join(data_dir, "SrcRcv.txt"), "w") as f:
        f.write("\n".join([src] + rcvs) + "\n")


def run_once(root: str, medium: str, nt: int, log: str) -> float:
    cwd = os.path.join(root, "run", "bin")
    os.makedirs(cwd, exist_ok=True)
    t0 = time.perf_counter()
    with open(log, "w") as f:
        p = subprocess.run([BIN, "--medium", medium, "--Nt", str(nt), "--energy", "Y"], cwd=cwd,
                           stdout=f, stderr=subprocess.STDOUT, timeout=1800)
    t = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"reference GPU executable exited {p.returncode} (log {log})")
    return t


def energy_tail(root: str):
    """The last kinetic-energy record the run wrote (finite if the run stepped sanely)."""
    for dirpath, _, files in os.walk(os.path.join(root, "result")):
        for name in files:
            if name.startswith("E_k") or name.startswith("Energy"):
                with open(os.path.join(dirpath, name)) as f:
                    vals = [ln.split()[-1] for ln in f if ln.strip()]
                try:
                    return float(vals[-1])
                except (ValueError, IndexError):
                    return None
    return None


def time_reference_gpu(n: int, den: int, dt: float, f0: float, delay: float, steps=(200, 2200), logdir: str = "",
                       repeats: int = 2):
    """The record of one timing; None when the executable is not built. A first run of the
    shorter length is discarded (device and file-system warm-up); each length then runs
    `repeats` times and the fastest counts, since set-up and write-out vary by seconds between
    runs and would otherwise swamp the difference."""
    if not os.path.exists(BIN):
        return None
    medium = f"grid{n}"

    def one(nt, tag):
        root = tempfile.mkdtemp(prefix="twref_gpu_")
        try:
            write_inputs(os.path.join(root, "data", medium), n, den, dt, f0, delay)
            log = os.path.join(logdir or root, f"ref_gpu_{n}_{nt}_{tag}.log")
            return run_once(root, medium, nt, log), energy_tail(root)
        finally:
            shutil.rmtree(root, ignore_errors=True)

    one(steps[0], "warmup")
    times, energies = [], []
    for nt in steps:
        runs = [one(nt, str(r)) for r in range(repeats)]
        times.append(min(t for t, _ in runs))
        energies.append(runs[-1][1])
    n1, n2 = steps
    ms = (times[1] - times[0]) / (n2 - n1) * 1e3
    rec = {"program": "nvcc_device_FDM_2D.cu (reference, unmodified, sm_100a, FP32 fields)",
           "grid": f"{n}x{n}", "dt": dt, "energy": "on (the program asserts it)",
           "medium": "the program's own constant medium (rho 1, vp 2, vs 1)",
           "steps": [n1, n2], "wall_s": [round(t, 3) for t in times],
           "ms_per_step": round(ms, 4), "gpt_per_s": round(n * n / (ms * 1e-3) / 1e9, 4),
           "method": f"difference of the fastest of {repeats} runs' wall-clock times at each length, after a "
                     "discarded warm-up run (set-up and write-out cancel)",
           "last_energy_record": energies}
    if any(e is not None and not math.isfinite(e) for e in energies):
        rec["warning"] = "non-finite energy record"
    if ms <= 0:
        return {"unavailable": f"run-to-run variance exceeded the extra steps' time (wall {times})"}
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--den", type=int, default=500)
    ap.add_argument("--dt", type=float, required=True)
    ap.add_argument("--f0", type=float, default=15.0)
    ap.add_argument("--delay", type=float, default=0.1)
    ap.add_argument("--steps", type=int, nargs=2, default=[200, 2200])
    ap.add_argument("--out", default="")
    ap.add_argument("--logdir", default="")
    a = ap.parse_args()
    rec = time_reference_gpu(a.n, a.den, a.dt, a.f0, a.delay, tuple(a.steps), a.logdir)
    if rec is None:
        rec = {"unavailable": f"{BIN} not built (make -C oracle refgpu)"}
    print(json.dumps(rec))
    if a.out:
        with open(a.out, "w") as f:
            f.write(json.dumps(rec) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
