"""Shared test setup: repo root on sys.path, the `gpu` marker, in-tree builds.

`-m "not gpu"` runs on a CPU-only machine (oracle vs the reference's
known answers, host logic, the C-ABI library's exports); `-m gpu` needs a
CUDA device and checks the CUDA path against the oracle through the C ABI.
"""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def _ensure_built():
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(os.path.join(ROOT, "ruqu_b200", "libruqu_cuda.so")):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_rq_build", os.path.join(ROOT, "ruqu_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)   # build.py runs nvcc; it imports nothing of the package
        mod.build()


_ensure_built()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (the CUDA path vs the oracle)")
