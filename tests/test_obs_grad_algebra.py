"""The identities behind the engine's checkpointed observable gradients
(dqmc_engine_obs_grad), checked on the explicit space-time matrix O of
oracle/fermion_matrix.py (greens.c:247-264 with one slice per block):

* rotating the chain by s slices gives the inverse D P O^-1 P^T D, so the
  first block row and column of the rotated chain's inverse are row s and
  column s of O^-1, negated on the slices that wrapped;
* from O O^-1 = I and O^-1 O = I, row m+1 is B_m row m + delta_{m+1} and
  column m+1 is (column m - delta_m) B_m^-1, negated across the corner;
* propagating rows and columns from each cluster boundary s = c n_matmul
  gives every Y_m = sum_l O^-1(m, l) W_l O^-1(l, m+1)."""
import numpy as np
import pytest

import fermion_matrix as fm


def _chain(N, L, seed):
    rng = np.random.default_rng(seed)
    K = rng.standard_normal((N, N))
    K = -0.5 * (K + K.T)
    eK = np.linalg.matrix_power(np.eye(N) - 0.1 * K / 8, 8)   # a well-conditioned exp(-dt K)
    d = [np.exp(0.4 * rng.choice([-1.0, 1.0], N)) for _ in range(L)]
    return eK, d


def _blk(A, N, a, b):
    return A[a * N:(a + 1) * N, b * N:(b + 1) * N]


@pytest.mark.parametrize("N,L,nmul", [(3, 6, 2), (4, 12, 4), (5, 10, 5)])
def test_rotated_rows_and_propagated_columns_give_Y(N, L, nmul):
    eK, d = _chain(N, L, N * 100 + L)
    B = [eK * dl[None, :] for dl in d]
    G = np.linalg.inv(fm.fermion_matrix(eK, d, N, L))
    w = [np.random.default_rng(l).standard_normal(N) for l in range(L)]
    want = [sum(_blk(G, N, m, l) @ np.diag(w[l]) @ _blk(G, N, l, (m + 1) % L) for l in range(L))
            for m in range(L)]
    got = [None] * L
    for c in range(L // nmul):
        s = c * nmul
        Gr = np.linalg.inv(fm.fermion_matrix(eK, [d[(l + s) % L] for l in range(L)], N, L))
        sg = [(-1.0 if l < s else 1.0) for l in range(L)]
        R = [sg[l] * _blk(Gr, N, 0, (l - s) % L) for l in range(L)]
        X = [sg[l] * _blk(Gr, N, (l - s) % L, 0) for l in range(L)]
        for l in range(L):
            np.testing.assert_allclose(R[l], _blk(G, N, s, l), atol=1e-12)
            np.testing.assert_allclose(X[l], _blk(G, N, l, s), atol=1e-12)
        for m in range(s, s + nmul):
            X[m] = X[m] - np.eye(N)
            iB = np.linalg.inv(B[m])
            X = [(-1.0 if m == L - 1 else 1.0) * x @ iB for x in X]
            got[m] = sum(R[l] @ np.diag(w[l]) @ X[l] for l in range(L))
            if m + 1 < s + nmul:
                R = [B[m] @ r for r in R]
                R[m + 1] = R[m + 1] + np.eye(N)
    for m in range(L):
        np.testing.assert_allclose(got[m], want[m], rtol=1e-10, atol=1e-12 * np.abs(want[m]).max())
