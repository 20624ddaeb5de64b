"""CPU pin of the adjoint oracle: its gradient of P_<(T) and <d_H(T)> with
respect to a piecewise-constant field schedule equals central finite
differences of the oracle's own forward run (itself pinned to the reference's
golden series), and the objective equals the forward run's final measurement."""
import numpy as np
import pytest

from oracle import oracle as O


def fd_segments(n, s0, e0, gs, seg, dt, T, objective, h=1e-5):
    out = np.zeros(len(gs))
    for j in range(len(gs)):
        vals = []
        for sgn in (1.0, -1.0):
            gg = gs.copy()
            gg[j] += sgn * h
            p, d, _ = O.trotter_evolve(n, s0, e0, gg[seg], dt, T, measure=[T])
            vals.append(p[0] if objective == 0 else d[0])
        out[j] = (vals[0] - vals[1]) / (2 * h)
    return out


@pytest.mark.parametrize("n,objective", [(8, 0), (10, 0), (9, 1)])
def test_oracle_adjoint_matches_finite_differences(n, objective):
    rng = np.random.default_rng(n)
    s0 = int(O.steepest_descent(n, int(rng.integers(0, 1 << n)))[0])
    e0 = O.labs_energy(n, s0) + (4 if objective == 0 else 0)  # a threshold with P_< > 0
    nseg, T, dt = 6, 48, 0.05
    gs = rng.uniform(0.25, 0.45, nseg)
    seg = O.segment_steps(T, nseg)
    value, grad = O.trotter_adjoint(n, s0, e0, gs[seg], dt, T, objective=objective)
    p, d, _ = O.trotter_evolve(n, s0, e0, gs[seg], dt, T, measure=[T])
    assert value == pytest.approx(p[0] if objective == 0 else d[0], rel=1e-12, abs=1e-14)
    gseg = np.bincount(seg, weights=grad, minlength=nseg)
    fd = fd_segments(n, s0, e0, gs, seg, dt, T, objective)
    scale = np.max(np.abs(fd))
    assert scale > 1e-4
    # central differences with h = 1e-5: truncation ~ h^2 |O'''|, rounding ~ 1e-16 / h
    assert np.max(np.abs(gseg - fd)) <= 1e-8 * max(1.0, scale)


def test_oracle_adjoint_zero_steps_and_constant_field():
    n, s0 = 8, 0x5B
    e0 = O.labs_energy(n, s0) + 6
    value, grad = O.trotter_adjoint(n, s0, e0, [0.3], 0.05, 0)
    assert len(grad) == 0
    assert value == (1.0 if O.labs_energy(n, s0) < e0 else 0.0)
    # with a constant field the per-step gradients sum to dO/dg of the whole run
    T, dt, g, h = 40, 0.05, 0.35, 1e-5
    _, grad = O.trotter_adjoint(n, s0, e0, np.full(T, g), dt, T)
    pp = O.trotter_evolve(n, s0, e0, g + h, dt, T, measure=[T])[0][0]
    pm = O.trotter_evolve(n, s0, e0, g - h, dt, T, measure=[T])[0][0]
    assert grad.sum() == pytest.approx((pp - pm) / (2 * h), rel=1e-7, abs=1e-10)
