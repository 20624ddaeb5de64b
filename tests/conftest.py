import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(ROOT, "bernasconi-krylov_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG_ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


# complex64 parity bars against complex128 / the oracle (written once, used by
# every complex64 test):
#   P_<: 1e-6 absolute, the bar the engine is built to;
#   <d_H>: 3e-6 absolute. <d_H> is ~15 at N = 28, so 1e-6 would be a relative
#   7e-8, finer than FP32 storage holds over thousands of steps: each step
#   rounds every amplitude ~n times, and the rounding (unbiased per operation)
#   random-walks through the few amplitudes that carry most of the weight.
#   Measured on a B200 with the norm-normalised estimator: 1.1e-6 (N = 24,
#   1000 steps), 1.5e-6 (N = 28, 2000 steps); an FP32 emulation of the same
#   arithmetic on the CPU gives the same size, with an exact FP64 phase too.
C64_DP_BAR = 1e-6
C64_DH_BAR = 3e-6


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test that takes more than a few seconds")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden():
    return load_golden
