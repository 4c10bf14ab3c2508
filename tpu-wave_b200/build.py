"""Build libtwave.so (the C-ABI library with the sm_100a kernels) in-tree.

    python tpu-wave_b200/build.py            # incremental
    python tpu-wave_b200/build.py --force    # rebuild everything

Every CUDA source is compiled for sm_100a only (`-gencode arch=compute_100a,code=sm_100a`),
with -lineinfo for the profiler; objects go to tpu-wave_b200/_obj, the library to
tpu-wave_b200/lib/libtwave.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_obj")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libtwave.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-I" + os.path.join(HERE, "..", "include")]


def _headers_mtime() -> float:
    files = [f for f in glob.glob(os.path.join(CSRC, "*")) if not f.endswith(".cu")]
    files += glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return max(os.path.getmtime(f) for f in files)


def _deps_mtime() -> float:
    files = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return max(os.path.getmtime(f) for f in files)


def _obj_of(src: str) -> str:
    return os.path.join(OBJ, os.path.splitext(os.path.basename(src))[0] + ".o")


def _stale(src: str, force: bool) -> bool:
    obj = _obj_of(src)
    if force or not os.path.exists(obj):
        return True
    return os.path.getmtime(obj) < max(os.path.getmtime(src), _headers_mtime())


def _compile(src: str) -> str:
    obj = _obj_of(src)
    cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime():
        return LIB
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    # a source is recompiled when it, or any header, is newer than its object
    stale = [s for s in sources if _stale(s, force)]
    if stale:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(stale))) as ex:
            list(ex.map(_compile, stale))
    objs = [_obj_of(s) for s in sources]
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
