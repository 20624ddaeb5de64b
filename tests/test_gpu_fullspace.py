"""Full-space Hamiltonian matvec and Lanczos on the GPU (bk_fullspace_matvec,
bk_fullspace_lanczos; reference src/subspace/diagonalizer.cuh:60-77, 377-560)
against the CPU oracle, which is pinned to a dense H (tests/test_oracle_fullspace.py)."""
import numpy as np
import pytest
import torch
from scipy.linalg import eigh_tridiagonal

import bk_b200 as bk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = bk.Engine(0)
    yield e
    e.close()


# n covers: one CTA over a vector smaller than a block (5), the block pass alone
# with 0, 1, 4, 9 and 10 gathered partner bits (13, 14, 17, 22, 23), and the block
# pass plus the strided pass over the far bits (24: 1 bit, 26: 3 bits)
@pytest.mark.parametrize("n", [5, 13, 14, 17, 22, 23, 24, 26])
def test_matvec_matches_oracle(eng, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(1 << n)
    for g, scale in ((0.35, None), (1.1, 1.0)):
        ref = O.fullspace_matvec(n, g, x, scale=scale)
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty_like(xd)
        eng.fullspace_matvec(n, g, xd, yd, scale=scale)
        y = yd.cpu().numpy()
        # a different summation order: FP64 rounding of n + 1 terms
        assert np.max(np.abs(y - ref)) <= 1e-14 * (n + 1) * max(1.0, np.max(np.abs(ref))), (n, g)
        # the per-state comparison form (the reference's order; FMA contraction differs
        # between the device and host compilers, so to rounding as well)
        eng.fullspace_matvec(n, g, xd, yd, scale=scale, method=bk.BK_PLAIN)
        yp = yd.cpu().numpy()
        assert np.max(np.abs(yp - ref)) <= 1e-14 * (n + 1) * max(1.0, np.max(np.abs(ref))), (n, g)


@pytest.mark.parametrize("n,g", [(12, 0.35), (16, 0.5)])
def test_lanczos_matches_oracle(eng, n, g):
    e, vec, info = eng.fullspace_lanczos(n, g, num_eigenpairs=2, max_krylov_dim=60)
    a, b = O.fullspace_lanczos(n, g, max_krylov_dim=60)
    assert info["krylov_dim"] == len(a) == 60 and info["matvecs"] == 60
    # the same start vector and steps: the tridiagonal matrices agree to rounding
    # over the first steps; once a Ritz value converges, plain Lanczos (no
    # reorthogonalisation, as in the reference) loses orthogonality and two
    # summation orders part exponentially (x~20 per step at n = 16), so only the
    # first 12 steps and the converged Ritz values are compared
    scale_ab = max(1.0, float(np.max(np.abs(a))))
    assert np.max(np.abs(info["alphas"][:12] - a[:12])) <= 1e-10 * scale_ab
    assert np.max(np.abs(info["betas"][:12] - b[:12])) <= 1e-10 * scale_ab
    lam = eigh_tridiagonal(a, b, eigvals_only=True)
    # after 60 steps the lowest Ritz value is not converged (residual ~1e-4, so it
    # still moves at ~residual^2 / gap ~ 5e-8); plain Lanczos — like the reference,
    # without reorthogonalisation — carries the rounding differences into it
    assert abs(e[0] - lam[0]) <= 1e-8 * max(1.0, abs(lam[0]))
    # the Ritz vector: unit norm and the residual |H x - e x| of exact Lanczos,
    # |beta_m z_m| (beta_m from one more oracle step, z_m the last eigenvector entry)
    x = vec[0]
    assert abs(np.linalg.norm(x) - 1.0) <= 1e-6
    a61, b61 = O.fullspace_lanczos(n, g, max_krylov_dim=61)
    _, z = eigh_tridiagonal(a, b)
    r = O.fullspace_matvec(n, g, x) - e[0] * x
    assert np.linalg.norm(r) <= 2.0 * abs(b61[59] * z[-1, 0]) + 1e-8


def test_lanczos_ground_energy_against_dense(eng):
    n, g = 10, 0.3
    e, _, info = eng.fullspace_lanczos(n, g, vectors=False)
    N = 1 << n
    E = np.array(bk.labs_energy(n, np.arange(N, dtype=np.uint64)), dtype=np.float64)
    H = np.diag(E / n)
    idx = np.arange(N)
    for j in range(n):
        H[idx, idx ^ (1 << j)] -= g
    assert info["krylov_dim"] == 100
    assert abs(e[0] - np.linalg.eigvalsh(H)[0]) <= 1e-10


def test_fullspace_errors(eng):
    x = torch.zeros(1 << 10, dtype=torch.float64, device="cuda")
    with pytest.raises(bk.BkError):
        eng.fullspace_matvec(10, 0.3, x, x)  # aliasing
    big = torch.zeros((1 << 10) + 1, dtype=torch.float64, device="cuda")
    with pytest.raises(bk.BkError):
        eng.fullspace_matvec(10, 0.3, big[1:], x)  # x not 16-byte aligned: rejected on the host
    with pytest.raises(bk.BkError):
        eng.fullspace_lanczos(31, 0.3)  # beyond the reference's n <= 30
    with pytest.raises(bk.BkError):
        eng.fullspace_lanczos(28, 0.3, max_krylov_dim=500, vectors=False)  # 501 x 2 GB does not fit
    e, _, info = eng.fullspace_lanczos(3, 0.3, num_eigenpairs=10, vectors=False)  # m = min(2^n, 100) = 8
    assert info["krylov_dim"] <= 8 and np.isnan(e[-1])


def test_reference_lanczos_known_answer(eng):
    """The reference's own check (tests/test_lanczos.cu:10-59): n = 4, g = 0.5,
    max_krylov_dim 30 (the whole 16-state space): ground energy within 1e-6 of
    dense ED and ||H v - E v|| < 1e-5."""
    n, g = 4, 0.5
    e, vec, info = eng.fullspace_lanczos(n, g, max_krylov_dim=30)
    N = 1 << n
    E = np.array(bk.labs_energy(n, np.arange(N, dtype=np.uint64)), dtype=np.float64)
    H = np.diag(E / n)
    idx = np.arange(N)
    for j in range(n):
        H[idx, idx ^ (1 << j)] -= g
    assert info["krylov_dim"] <= N
    assert abs(e[0] - np.linalg.eigvalsh(H)[0]) < 1e-6
    v = vec[0]
    assert np.linalg.norm(H @ v - e[0] * v) < 1e-5
