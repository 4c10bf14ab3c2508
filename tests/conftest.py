"""Test configuration: the `gpu` marker and one-time builds of the oracle and the product.

`-m "not gpu"` runs on any machine (oracle vs reference, golden fixtures, host logic, ABI
exports); `-m gpu` needs a B200 and calls the product through its C ABI.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    lib = os.path.join(ROOT, "tpu-wave_b200", "lib", "libtwave.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(ROOT, "tpu-wave_b200", "build.py")], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "libtwave_oracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    from oracle.refrun import REFERENCE_DIR
    ref_present = os.path.isdir(REFERENCE_DIR)
    if ref_present and not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "twref_elastic_f64")):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REFERENCE_DIR}"],
                       check=True)


_ensure_built()


@pytest.fixture(scope="session")
def tw():
    from cases import load_twave
    return load_twave()


def has_ref_binaries():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "twref_elastic_f64"))
