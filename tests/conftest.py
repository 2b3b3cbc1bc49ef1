"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on any host: the oracle against the golden fixtures and
the reference's own CPU path, the library's FP64 host tables against the
oracle, and the C ABI (load, symbols, argument checks).  `-m gpu` runs the CUDA
path through the C ABI against the oracle.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "inverse-solver-gpu_b200")
for p in (PKG, os.path.dirname(os.path.abspath(__file__)), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")
