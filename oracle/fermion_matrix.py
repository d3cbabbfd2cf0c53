"""Explicit space-time fermion matrices: the check for the fixed-field
gradients (test infrastructure, not part of the engine).

For one spin and fixed fields, O is the N L x N L block matrix with I on
the diagonal, -B_l at block (l+1, l) and +B_{L-1} at (0, L-1), B_l =
exp(-dt K) diag(lambda_{h_l}) (reference src/greens.c:247-264, calc_o with
one slice per block; exp_lambda as gen_1band_unified_hub.py:925-927).  Then
det O = det(I + B_{L-1} ... B_0), O^-1 is the space-time Green's function,
d log det O = tr[O^-1 dO] and d O^-1 = -O^-1 dO O^-1.  Derivatives of
exp(-dt K) come from scipy's expm_frechet.  Dense numpy throughout, so the
cost is that of N L x N L inverses.
"""
from __future__ import annotations

import numpy as np


def _setup(K, dK, U, dt, L, fields):
    from scipy.linalg import expm, expm_frechet
    eK = expm(-dt * K)
    dE = [expm_frechet(-dt * K, -dt * dk)[1] for dk in dK]
    lam = np.exp(0.5 * U * dt) + np.sqrt(np.expm1(U * dt))
    el = np.array([1.0 / lam, lam])
    return eK, dE, el


def _blocks(N, L):
    return [(((l + 1) % L) * N, l * N, 1.0 if l == L - 1 else -1.0) for l in range(L)]


def fermion_matrix(eK, d, N, L):
    O = np.eye(N * L)
    for l, (r, c, s) in enumerate(_blocks(N, L)):
        O[r:r + N, c:c + N] += s * (eK * d[l][None, :])
    return O


def logdet_grad(K, dK, U, dt, L, fields):
    """log |det O_up O_dn| and its gradient along every dK[k]."""
    N = K.shape[0]
    eK, dE, el = _setup(K, dK, U, dt, L, fields)
    ld, g = 0.0, np.zeros(len(dK))
    for spin in (0, 1):
        d = el[fields if spin == 0 else 1 - fields]
        O = fermion_matrix(eK, d, N, L)
        ld += np.linalg.slogdet(O)[1]
        Oi = np.linalg.inv(O)
        for k in range(len(dK)):
            tr = 0.0
            for l, (r, c, s) in enumerate(_blocks(N, L)):
                tr += np.sum(Oi[c:c + N, r:r + N].T * (s * (dE[k] * d[l][None, :])))
            g[k] += tr
    return ld, g


def obs_grad(K, dK, U, dt, L, fields):
    """(<n>, <docc>) averaged over the slices and their gradients along
    every dK[k] (2 x len(dK))."""
    N = K.shape[0]
    eK, dE, el = _setup(K, dK, U, dt, L, fields)
    G, dG = [], []
    for spin in (0, 1):
        d = el[fields if spin == 0 else 1 - fields]
        Oi = np.linalg.inv(fermion_matrix(eK, d, N, L))
        G.append(np.diag(Oi).copy())
        rows = []
        X = np.empty_like(Oi)
        for k in range(len(dK)):
            # X = dO O^-1 block row by block row; diag(O^-1 X) by rows
            for l, (r, c, s) in enumerate(_blocks(N, L)):
                X[r:r + N, :] = (s * (dE[k] * d[l][None, :])) @ Oi[c:c + N, :]
            rows.append(-np.einsum("ij,ji->i", Oi, X))
        dG.append(np.array(rows))
    NL = N * L
    obs = np.array([((1 - G[0]) + (1 - G[1])).sum() / NL, ((1 - G[0]) * (1 - G[1])).sum() / NL])
    gn = -(dG[0] + dG[1]).sum(1) / NL
    gd = (-(dG[0] * (1 - G[1])[None, :]) - ((1 - G[0])[None, :] * dG[1])).sum(1) / NL
    return obs, np.array([gn, gd])
