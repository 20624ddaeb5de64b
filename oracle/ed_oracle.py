"""Dense exact-diagonalisation propagator — TEST INFRASTRUCTURE ONLY.

numpy/LAPACK restatement of the reference's CPU fallback for n <= 12
(src/connector/connector.cuh:683-805 with Diagonalizer::solve_fullspace_dense,
src/subspace/diagonalizer.cuh:250-294): H = diag(E(s) * scale) - g * sum_i X_i with
scale = 1/n (normalize_by_n = true), psi(t) = sum_j c_j v_j exp(-i E_j t) with
c_j = v_j[s0]. The reference builds it on Eigen, which is absent here, so this
restatement stands in for it (config: n = 12, 4096 x 4096).
"""
import numpy as np
import scipy.linalg


def hamiltonian(n, g, energies, scale=None):
    A = 1 << n
    scale = (1.0 / n) if scale is None else scale
    H = np.zeros((A, A))
    H[np.arange(A), np.arange(A)] = energies.astype(np.float64) * scale
    idx = np.arange(A)
    for q in range(n):
        H[idx, idx ^ (1 << q)] -= g
    return H


def propagate(n, g, s0, e0, times, energies, scale=None):
    """Return (p_less, d_h) at the given times, exact in the eigenbasis."""
    H = hamiltonian(n, g, energies, scale)
    w, V = scipy.linalg.eigh(H, driver="evd")
    c = V[s0, :].copy()
    below = energies.astype(np.int64) < e0
    ham = np.array([bin(s ^ s0).count("1") for s in range(1 << n)], dtype=np.float64)
    pl, dh = [], []
    for t in times:
        psi = V @ (c * np.exp(-1j * w * t))
        prob = np.abs(psi) ** 2
        pl.append(float(prob[below].sum()))
        dh.append(float((prob * ham).sum()))
    return np.array(pl), np.array(dh)
