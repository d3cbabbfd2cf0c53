"""Gradients of log |det M_up det M_dn| at fixed fields (dqmc_b200.grad):
the GPU log-determinant against numpy's slogdet of the explicit space-time
fermion matrix O (N L x N L: I on the diagonal, -B_l below it, +B_{L-1} in
the corner, greens.c:247-264 with one slice per block), the gradient against
the explicit tr[O^-1 dO] and against central differences (h = 1e-5), and
the torch.autograd.Function's backward."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LD_RTOL = 1e-10
GRAD_RTOL = 1e-8      # against the explicit fermion-matrix gradient
FD_RTOL = 1e-6        # against central differences


@pytest.fixture(scope="module")
def grad():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import grad as G, lib
    lib.load()
    return G


def _fields(n_cfg, L, N, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2, size=(n_cfg, L, N)).astype(np.int32)


def _explicit(model, theta, fields):
    """log |det O_up O_dn| and its gradient from the explicit fermion matrices"""
    import fermion_matrix as fm
    return fm.logdet_grad(model.K(theta), model.dK, model.U, model.dt, model.L, fields)


@pytest.mark.parametrize("Nx,L,nmul", [(4, 8, 4), (4, 12, 3)])
def test_logdet_and_gradient_match_fermion_matrix(grad, Nx, L, nmul):
    fields = _fields(3, L, Nx * Nx, 5)
    m = grad.SquareModel(Nx, Nx, U=4.0, dt=0.1, L=L, fields=fields, n_matmul=nmul)
    rng = np.random.default_rng(1)
    theta = np.concatenate([[1.0, -0.2, -0.3], 0.05 * rng.standard_normal(2 * Nx * Nx)])
    ld, g = m.evaluate(theta)
    for c in range(3):
        ld_x, g_x = _explicit(m, theta, fields[c])
        assert abs(ld[c] - ld_x) < LD_RTOL * max(1.0, abs(ld_x))
        np.testing.assert_allclose(g[c], g_x, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(g_x).max())


def test_gradient_matches_central_differences(grad):
    fields = _fields(2, 8, 16, 7)
    m = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(32)])
    _, g = m.evaluate(theta)
    h = 1e-5
    for k in (0, 1, 2, 3, 17):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (m.evaluate(tp)[0] - m.evaluate(tm)[0]) / (2 * h)
        np.testing.assert_allclose(g[:, k], fd, rtol=FD_RTOL, atol=FD_RTOL * np.abs(g).max())


def test_autograd_function(grad):
    import torch
    fields = _fields(4, 8, 16, 9)
    m = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
    theta = torch.tensor(np.concatenate([[1.0, -0.2, -0.3], np.zeros(32)]), dtype=torch.float64,
                         requires_grad=True)
    w = torch.arange(1, 5, dtype=torch.float64)
    y = grad.LogDet.apply(theta, m)
    (w * y).sum().backward()
    _, g = m.evaluate(theta.detach().numpy())
    np.testing.assert_allclose(theta.grad.numpy(), (w.numpy()[:, None] * g).sum(0), rtol=1e-12)


def test_full_size_configuration(grad):
    """8x8, L = 40 (N L = 2560), t' = -0.2, U = 4, mu = -0.3: one configuration
    against the explicit fermion-matrix gradient."""
    fields = _fields(1, 40, 64, 11)
    m = grad.SquareModel(8, 8, U=4.0, dt=0.1, L=40, fields=fields, n_matmul=8)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(128)])
    ld, g = m.evaluate(theta)
    ld_x, g_x = _explicit(m, theta, fields[0])
    assert abs(ld[0] - ld_x) < LD_RTOL * max(1.0, abs(ld_x))
    np.testing.assert_allclose(g[0], g_x, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(g_x).max())


def _explicit_obs(model, theta, fields):
    """<n>, <docc> and their gradients from the explicit space-time Green's
    functions of both spins"""
    import fermion_matrix as fm
    return fm.obs_grad(model.K(theta), model.dK, model.U, model.dt, model.L, fields)


@pytest.mark.parametrize("Nx,L,nmul", [(4, 8, 4), (4, 6, 3)])
def test_observable_gradients_match_fermion_matrix(grad, Nx, L, nmul):
    fields = _fields(2, L, Nx * Nx, 21)
    m = grad.SquareModel(Nx, Nx, U=4.0, dt=0.1, L=L, fields=fields, n_matmul=nmul)
    rng = np.random.default_rng(3)
    theta = np.concatenate([[1.0, -0.2, -0.3], 0.05 * rng.standard_normal(2 * Nx * Nx)])
    obs, g = m.evaluate_obs(theta)
    for c in range(2):
        ox, gx = _explicit_obs(m, theta, fields[c])
        np.testing.assert_allclose(obs[c], ox, rtol=1e-10)
        for o in range(2):
            np.testing.assert_allclose(g[c, o], gx[o], rtol=GRAD_RTOL,
                                       atol=GRAD_RTOL * np.abs(gx[o]).max())


def test_observable_gradients_match_central_differences(grad):
    fields = _fields(1, 8, 16, 23)
    m = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(32)])
    _, g = m.evaluate_obs(theta)
    h = 1e-5
    for k in (0, 1, 2, 9):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (m.evaluate_obs(tp)[0] - m.evaluate_obs(tm)[0]) / (2 * h)
        np.testing.assert_allclose(g[:, :, k], fd, rtol=FD_RTOL, atol=FD_RTOL * np.abs(g).max())


def test_reused_engine_matches_fresh_models(grad):
    """One model evaluated at theta_1, theta_2, theta_1 (the hopping replaced
    in place each time) gives what fresh models give at each theta."""
    fields = _fields(3, 8, 16, 11)
    rng = np.random.default_rng(3)
    t1 = np.concatenate([[1.0, -0.2, -0.3], 0.05 * rng.standard_normal(32)])
    t2 = np.concatenate([[0.9, -0.1, 0.2], 0.05 * rng.standard_normal(32)])
    m = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
    seq = [m.evaluate(t) + m.evaluate_obs(t) for t in (t1, t2, t1)]
    m.close()
    for t, got in zip((t1, t2), seq[:2]):
        f = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
        want = f.evaluate(t) + f.evaluate_obs(t)
        f.close()
        for a, b in zip(got, want):
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    for a, b in zip(seq[0], seq[2]):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_observables_autograd(grad):
    import torch
    fields = _fields(2, 8, 16, 13)
    m = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
    theta = torch.tensor(np.concatenate([[1.0, -0.2, -0.3], np.zeros(32)]), requires_grad=True)
    y = grad.Observables.apply(theta, m)
    wts = torch.tensor([[1.0, 2.0], [-0.5, 3.0]], dtype=torch.float64)
    (y * wts).sum().backward()
    obs, g = m.evaluate_obs(theta.detach().numpy())
    np.testing.assert_allclose(y.detach().numpy(), obs, rtol=1e-13)
    want = (wts.numpy()[:, :, None] * g).sum((0, 1))
    np.testing.assert_allclose(theta.grad.numpy(), want, rtol=1e-12, atol=1e-14)
    m.close()


def test_full_size_observable_gradients(grad):
    """8x8, L = 40, n_matmul = 8 (five rotations, eight slices propagated from
    each): <n>, <docc> and their derivatives along t, t', mu and three bond
    hoppings against the explicit space-time Green's functions."""
    import fermion_matrix as fm
    fields = _fields(1, 40, 64, 17)
    m = grad.SquareModel(8, 8, U=4.0, dt=0.1, L=40, fields=fields, n_matmul=8)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(128)])
    obs, g = m.evaluate_obs(theta)
    m.close()
    idx = [0, 1, 2, 3, 40, 130]
    dK = [m.dK[k] for k in idx]
    ox, gx = fm.obs_grad(m.K(theta), dK, m.U, m.dt, m.L, fields[0])
    np.testing.assert_allclose(obs[0], ox, rtol=1e-10)
    for o in range(2):
        np.testing.assert_allclose(g[0, o, idx], gx[o], rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(gx[o]).max())


def test_checkpointed_form_matches_dense_form(grad, monkeypatch):
    """The rotated unequal-time rows and columns against the whole inverse of
    the N L x N L matrix (DQMC_OBS_GRAD=dense), three configurations."""
    fields = _fields(3, 24, 36, 29)
    rng = np.random.default_rng(5)
    theta = np.concatenate([[1.0, -0.25, -0.5], 0.05 * rng.standard_normal(72)])
    m = grad.SquareModel(6, 6, U=6.0, dt=0.1, L=24, fields=fields, n_matmul=6)
    obs, g = m.evaluate_obs(theta)
    monkeypatch.setenv("DQMC_OBS_GRAD", "dense")
    obs_d, g_d = m.evaluate_obs(theta)
    m.close()
    np.testing.assert_allclose(obs, obs_d, rtol=1e-11)
    np.testing.assert_allclose(g, g_d, rtol=1e-9, atol=1e-9 * np.abs(g_d).max())


def test_observable_gradients_at_batched_lattice_size(grad):
    """12x12, beta = 6, dtau = 0.05 (L = 120, N L = 17280), mu = -1: the dense
    inverse would take 2 (N L)^2 numbers (4.8 GB) per configuration and spin;
    the checkpointed form stays within a few hundred MB for two
    configurations, and its derivatives along mu and t match central
    differences (h = 1e-5)."""
    import torch
    fields = _fields(2, 120, 144, 31)
    theta = np.concatenate([[1.0, 0.0, -1.0], np.zeros(288)])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    m = grad.SquareModel(12, 12, U=4.0, dt=0.05, L=120, fields=fields, n_matmul=10)
    obs, g = m.evaluate_obs(theta)
    used = free0 - torch.cuda.mem_get_info()[0]
    assert used < 2.0e9, used
    assert np.all(np.isfinite(g)) and np.all((obs[:, 0] > 0) & (obs[:, 0] < 2))
    h = 1e-5
    for k in (2, 0):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (m.evaluate_obs(tp)[0] - m.evaluate_obs(tm)[0]) / (2 * h)
        np.testing.assert_allclose(g[:, :, k], fd, rtol=FD_RTOL, atol=FD_RTOL * np.abs(g[:, :, k]).max())
    m.close()


def test_gradient_profile_counts_launches_and_keeps_results(grad):
    """dqmc_engine_profile_grad: one evaluation of each kind with per-launch
    events; the GEMM class carries time and FLOPs, the launch count is
    positive, and the evaluations after it give what they gave before."""
    fields = _fields(2, 8, 16, 37)
    m = grad.SquareModel(4, 4, U=4.0, dt=0.1, L=8, fields=fields, n_matmul=4)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(32)])
    before = m.evaluate(theta) + m.evaluate_obs(theta)
    eng = m.engine(m.K(theta))
    for which in ("logdet", "obs"):
        prof, n = eng.profile_grad(which)
        assert n > 0
        assert prof["gemm"][0] > 0 and prof["gemm"][1] > 0 and prof["gemm"][2] > 0
    after = m.evaluate(theta) + m.evaluate_obs(theta)
    m.close()
    for a, b in zip(before, after):
        np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-14)
