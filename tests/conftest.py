import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmatter_gpu.so")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_oracle():
    """Builds the CPU checkers if they are missing (they are build outputs)."""
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not all(os.path.exists(os.path.join(ref_dir, f"libref_{d}d_q{q}.so")) for d in (2, 3) for q in (2, 3)):
        # builds only where the reference checkout is readable (oracle/Makefile MATTER_REF)
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=False,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    if not os.path.exists(os.path.join(ref_dir, "kat", "kat")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "kat"], check=False,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


_ensure_oracle()
