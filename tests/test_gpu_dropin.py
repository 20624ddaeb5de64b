"""Runs the C++ drop-in sampler test (tests/cpp/test_sampler_dropin.cpp) on the GPU:
the reference's test_sampler.cu checks, through the header-only ISampler and the C ABI."""
import subprocess

import pytest

from test_dropin_build import build_dropin_test

pytestmark = pytest.mark.gpu


def test_dropin_sampler_cpp(tmp_path):
    out = str(tmp_path / "test_sampler_dropin")
    build_dropin_test(out)
    r = subprocess.run([out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
    assert "[Quantum Sampler] Successes / Trials" in r.stdout  # the reference's verbose summary line
