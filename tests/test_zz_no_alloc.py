"""dqmc_gpu_calc_eq_g_noalloc against dqmc_gpu_calc_eq_g.

The no-allocation variant serves callers that cannot call cudaMalloc: a
process whose free device memory is already held by another allocator, or
a driver that cannot take the device-wide synchronisation of cudaFree while
sweeps are queued on other streams.  It does the same computation in the
library's fixed static device scratch, so its G and phase must agree with
the allocating entry point's on the same inputs -- checked here on two calls
in a row (the second one reuses the scratch the first one left behind) for
real and complex problems, plus the size limit.

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G_TOL = 1e-10      # max abs difference of G entries (O(1)), as in the other G tests
PHASE_TOL = 1e-12


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import lib as L
    return L


def _expm_herm(h):
    w, v = np.linalg.eigh(h)
    return (v * np.exp(w)) @ v.conj().T


def _clusters(rng, Nx, L, F, U, dt, cplx, batch):
    """batch x F cluster products C_f = B_{fn+n-1} ... B_{fn} (column-major)
    of a Hubbard model on an Nx x Nx square lattice with random fields"""
    N = Nx * Nx
    K = np.zeros((N, N), np.complex128 if cplx else np.float64)
    for x in range(Nx):
        for y in range(Nx):
            i = x + Nx * y
            for j in ((x + 1) % Nx + Nx * y, x + Nx * ((y + 1) % Nx)):
                t = np.exp(1j * rng.uniform(-0.3, 0.3)) if cplx else 1.0
                K[i, j] += t
                K[j, i] += np.conj(t)
    K += 0.5 * np.eye(N)                      # chemical potential mu = -0.5
    expK = _expm_herm(dt * K)
    lam = np.arccosh(np.exp(0.5 * U * dt))
    n = L // F
    out = np.zeros((batch, F, N, N), K.dtype)
    for b in range(batch):
        s = rng.integers(0, 2, size=(L, N)) * 2 - 1
        for f in range(F):
            c = np.eye(N, dtype=K.dtype)
            for l in range(f * n, f * n + n):
                c = (expK * np.exp(lam * s[l])[None, :]) @ c
            out[b, f] = c.T                   # column-major storage
    return out


def _call(fn, torch, Cm, l):
    batch, F, N, _ = Cm.shape
    dC = torch.from_numpy(np.ascontiguousarray(Cm).reshape(-1)).cuda()
    dG = torch.full((batch * N * N,), float("nan"), dtype=dC.dtype, device="cuda")
    dph = torch.zeros(batch, dtype=dC.dtype, device="cuda")
    rc = fn(batch, N, F, l, int(np.iscomplexobj(Cm)), dC.data_ptr(), dG.data_ptr(),
            dph.data_ptr(), None)
    return rc, dG.cpu().numpy(), dph.cpu().numpy()


@pytest.mark.parametrize("cplx", [False, True])
def test_noalloc_matches_allocating(lib, cplx):
    import torch
    h = lib.load()
    rng = np.random.default_rng(20261203 + int(cplx))
    # first call: 8x8 lattice, 3 problems; second: 4x4 lattice, 5 problems,
    # another l -- smaller than the first, so the scratch holds stale data
    cases = [(_clusters(rng, 8, 40, 8, 4.0, 0.1, cplx, 3), 2),
             (_clusters(rng, 4, 48, 6, 6.0, 0.125, cplx, 5), 5)]
    for Cm, l in cases:
        rc_a, g_a, ph_a = _call(h.dqmc_gpu_calc_eq_g, torch, Cm, l)
        rc_n, g_n, ph_n = _call(h.dqmc_gpu_calc_eq_g_noalloc, torch, Cm, l)
        assert rc_a == 0 and rc_n == 0
        assert np.all(np.isfinite(g_n))
        assert np.max(np.abs(g_n - g_a)) < G_TOL
        assert np.max(np.abs(ph_n - ph_a)) < PHASE_TOL


@pytest.mark.parametrize("F,l", [(5, 3), (1, 0)])
def test_noalloc_odd_cluster_counts(lib, F, l):
    """An odd F starts the stabilised chain from one cluster read straight
    from C (no pair product in the scratch), and F = 1 is that cluster
    alone: both paths through the static scratch agree with the allocating
    entry point, again on two calls in a row."""
    import torch
    h = lib.load()
    rng = np.random.default_rng(20261204 + F)
    for cplx in (False, True):
        Cm = _clusters(rng, 6, 5 * F * 2, F, 4.0, 0.1, cplx, 3)
        for _ in range(2):
            rc_a, g_a, ph_a = _call(h.dqmc_gpu_calc_eq_g, torch, Cm, l)
            rc_n, g_n, ph_n = _call(h.dqmc_gpu_calc_eq_g_noalloc, torch, Cm, l)
            assert rc_a == 0 and rc_n == 0
            assert np.all(np.isfinite(g_n))
            assert np.max(np.abs(g_n - g_a)) < G_TOL
            assert np.max(np.abs(ph_n - ph_a)) < PHASE_TOL


def test_noalloc_rejects_oversize(lib):
    h = lib.load()
    N = 144
    per_item = 6 * 8 * N * N
    batch = lib.NOALLOC_SCRATCH_BYTES // per_item + 1
    # rejected on the host before any pointer is touched or kernel launched
    rc = h.dqmc_gpu_calc_eq_g_noalloc(batch, N, 4, 0, 0, 1, 1, 1, None)
    assert rc == lib.DQMC_E_SCRATCH
