"""The C++ drop-in ISampler header builds: against this repository's own LABS types
(and links against libbk_b200.so), and — when a reference checkout is present — in
an overlay of the reference's source tree with the reference's own
labs_energy.hpp, compiled together with the connector's calling code
(src/connector/connector.cuh:629-680 restated as a snippet)."""
import os
import subprocess
import tempfile

import pytest

import bk_b200 as bk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bernasconi-krylov_b200")
REF = os.path.join(os.environ.get("BK_REFERENCE_ROOT", "/root/reference"), "src")


def build_dropin_test(out):
    bk.load_library()
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", PKG,
           os.path.join(ROOT, "tests", "cpp", "test_sampler_dropin.cpp"), "-L", os.path.join(PKG, "lib"),
           "-lbk_b200", "-Wl,-rpath," + os.path.join(PKG, "lib"), "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_dropin_header_builds_and_links(tmp_path):
    out = str(tmp_path / "test_sampler_dropin")
    build_dropin_test(out)
    assert os.path.exists(out)


CONNECTOR_SNIPPET = r'''
#include "sampling/sampler.cuh"
// the connector's use of the sampler (src/connector/connector.cuh:629-680)
int run(const SpinState& trap, int n, double g, uint64_t seed) {
    SamplerConfig s_cfg;
    s_cfg.n = n; s_cfg.g = g; s_cfg.dt = 0.05; s_cfg.t_max = 60.0; s_cfg.num_sample_points = 20;
    s_cfg.shots_per_point = 0; s_cfg.seed = seed; s_cfg.t_start = 10.0; s_cfg.dt_sample = 1.5;
    s_cfg.track_p_less = true; s_cfg.verbose = true; s_cfg.record_trajectory = true;
    s_cfg.dt_trajectory = 0.0; s_cfg.num_sampling_seeds = 3; s_cfg.seed_stride = 10007;
#if HAS_CUSTATEVEC
    auto sampler = create_sampler(n);
    SamplingResult res = sampler->sample(trap, s_cfg);
    double w = res.window_avg_dh + res.initial_rise_rate_avg + res.initial_rise_rate_max + res.p_blind
             + res.peak_p_less + res.peak_time + res.success_rate + res.per_eval_rate;
    for (const auto& ss : res.seed_stats) w += ss.success_rate + ss.mean_hamming_flips + (double)ss.best_energy;
    return (int)(res.time_points.size() + res.p_less_history.size() + res.dh_history.size() +
                 res.unique_basis.size() + (size_t)res.d_min + (size_t)w);
#else
    return -1;
#endif
}
'''


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout not present")
def test_dropin_in_reference_overlay(tmp_path):
    src = tmp_path / "src"
    (src / "sampling").mkdir(parents=True)
    os.symlink(os.path.join(REF, "labs_energy"), src / "labs_energy")
    os.symlink(os.path.join(PKG, "sampling", "sampler.cuh"), src / "sampling" / "sampler.cuh")
    tu = tmp_path / "connector_use.cpp"
    tu.write_text(CONNECTOR_SNIPPET)
    # -I src resolves "sampling/sampler.cuh"; the header's "../labs_energy/labs_energy.hpp" then
    # resolves next to the symlinked file's directory in the overlay (the reference's header)
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(src), "-I", os.path.join(ROOT, "include"),
                        str(tu)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
