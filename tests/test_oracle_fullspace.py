"""The full-space Hamiltonian oracle (oracle/trotter_oracle.cpp: orc_fullspace_matvec,
orc_fullspace_lanczos, restating src/subspace/diagonalizer.cuh:60-77, 418-482)
pinned to a dense construction of H = diag(E(s)/n) - g sum_j X_j on the CPU."""
import numpy as np
import pytest
from scipy.linalg import eigh_tridiagonal

import bk_b200 as bk
from oracle import oracle as O


def dense_h(n, g, scale=None):
    N = 1 << n
    scale = 1.0 / n if scale is None else scale
    E = np.array(bk.labs_energy(n, np.arange(N, dtype=np.uint64)), dtype=np.float64)
    H = np.diag(E * scale)
    idx = np.arange(N)
    for j in range(n):
        H[idx, idx ^ (1 << j)] -= g
    return H


@pytest.mark.parametrize("n,g", [(1, 0.5), (6, 0.35), (9, 1.2)])
def test_oracle_matvec_is_the_dense_product(n, g):
    x = np.random.default_rng(n).standard_normal(1 << n)
    y = O.fullspace_matvec(n, g, x)
    ref = dense_h(n, g) @ x
    assert np.max(np.abs(y - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
    assert np.allclose(O.fullspace_matvec(n, g, x, scale=1.0), dense_h(n, g, 1.0) @ x, rtol=0, atol=1e-12)


@pytest.mark.parametrize("n,g", [(6, 0.35), (8, 0.5), (10, 0.3)])
def test_oracle_lanczos_ground_energy(n, g):
    a, b = O.fullspace_lanczos(n, g)
    assert len(a) == min(1 << n, 100) and len(b) == len(a) - 1
    lam = eigh_tridiagonal(a, b, eigvals_only=True)
    exact = np.linalg.eigvalsh(dense_h(n, g))
    assert abs(lam[0] - exact[0]) <= 1e-10 * max(1.0, abs(exact[0]))


def test_oracle_lanczos_breakdown_on_an_invariant_subspace():
    # g = 0: H is diagonal; the Krylov space of a generic start vector spans the
    # distinct diagonal values only, so beta falls below the tolerance early
    n = 6
    a, b = O.fullspace_lanczos(n, 0.0)
    distinct = len(set(bk.labs_energy(n, np.arange(1 << n, dtype=np.uint64))))
    assert len(a) <= distinct + 1
    lam = eigh_tridiagonal(a, b, eigvals_only=True) if len(a) > 1 else a
    assert abs(lam[0] - min(bk.labs_energy(n, np.arange(1 << n, dtype=np.uint64))) / n) <= 1e-10
