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
#   <d_H>: 1.2e-5 absolute. <d_H> is 12-15 at N = 24-28, so 1e-6 would be a
#   relative 7e-8, finer than FP32 storage holds over thousands of steps: each
#   step rounds every amplitude ~n times, and the rounding (unbiased per
#   operation) random-walks through the few amplitudes that carry most of the
#   weight, so the error depends on the trap and on the order of the rounds.
#   Measured on a B200 with the norm-normalised estimator: 1.1e-6 (N = 24 trap
#   0xFAD33, 1000 steps), 4.0e-6 to 5.9e-6 (N = 24 trap of the lowest 5% of 1000
#   seeded descents, 1000 steps, every A1 kernel and schedule, with and without
#   the full phase table), 0.5e-6 to 1.5e-6 (N = 28, 2000 steps); an FP32
#   emulation of the same arithmetic on the CPU gives the same size, with an
#   exact FP64 phase too. The bar is twice the worst measurement.
C64_DP_BAR = 1e-6
C64_DH_BAR = 1.2e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test that takes more than a few seconds")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden():
    return load_golden
