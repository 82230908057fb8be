"""yannq_b200: B200 (sm_100a) backend of yannq's variational Monte Carlo step.

The product is libyannq_b200.so (C ABI in include/yannq_b200.h) with the C++
adapters in include/yannq_gpu/; this package holds its sources (csrc/) and a
ctypes binding (api.py) used by the tests and the benchmark.
"""
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    """Compile libyannq_b200.so for sm_100a with the committed Makefile."""
    out = subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), f"-j{jobs}"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libyannq_b200 build failed:\n" + out.stdout[-4000:] + out.stderr[-8000:])
    return os.path.join(_HERE, "libyannq_b200.so")
