"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on a CPU-only machine: the checker against the crate's
golden values, the host-side logic and the C-ABI symbol table.  `-m gpu` runs
the parity tests proper, which call libsvdb200.so through its C ABI and compare
with the checker in oracle/.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "single-svdlib_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls libsvdb200.so")
    config.addinivalue_line("markers", "slow: long-running parity case")
