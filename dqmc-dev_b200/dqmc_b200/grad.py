"""Gradients of log |det M_up det M_dn| at fixed Hubbard-Stratonovich fields.

For B_l = exp(-dt K) exp(V_l) and M = I + B_{L-1} ... B_0 (one spin),

    d log det M / d theta = sum_l tr[(I - G_l) B_l^-1 dB_l/d theta]
                          = tr[S D_theta],
    S = sum_l exp(V_l) (I - G_l) exp(-V_l),
    D_theta = exp(dt K) d exp(-dt K) / d theta,

with G_l the equal-time Green's function before slice l.  The engine
accumulates S over one update-free sweep of the stabilised chain
(dqmc_engine_logdet_grad).  D_theta for every parameter comes from one
eigen-decomposition K = V diag(k) V^T: in that basis the Frechet derivative
of exp(-dt K) along E is (V^T E V) * Phi with Phi_ij the divided difference
of exp at -dt k_i, -dt k_j (computed with expm1).  The contraction over all
parameters is then a single einsum.

Parameters of the square-lattice model (periodic, as gen.hopping_square):
theta = [t, t', mu, h_0 ... h_{2N-1}], the nearest-neighbour hopping on bond
b being t + h_b.  Bonds are numbered as hopping_square adds them: site
ix + Nx iy, first the x bond to (ix+1, iy), then the y bond to (ix, iy+1).
So d/dt is the sum of the per-bond derivatives.

The same contraction gives the derivatives of the fixed-field density and
double occupancy (evaluate_obs): with Gst = O^-1 the space-time Green's
function, d <X> = sum_l tr[W_l dGst(l, l)] and dGst = -Gst dO Gst collapse to
tr[Z D_theta] with Z = sum_m s_m exp(V_m) Y_m exp(-dt K) and
Y_m = sum_l Gst(m, l) W_l Gst(l, m+1) (W_l the observable's weights).
The engine never forms Gst: the stabilised unequal-time Green's functions
of the chain rotated to each cluster boundary s give row and column s of
Gst, and one B_m or B_m^-1 product per slice gives the rows and columns in
between, so the device memory is O(N^2 L) per configuration.

LogDet and Observables wrap the log-determinant and (<n>, <docc>) in
torch.autograd.Functions: the forward runs the engine and keeps the
per-configuration gradients for the backward.  A model keeps one engine for
all its evaluations: a new theta only replaces the hopping matrices
(dqmc_engine_set_hopping), so repeated evaluations allocate no device
memory, and the parameter contraction runs on the device.
"""
from __future__ import annotations

import numpy as np

from . import gen
from .engine import Engine, SimData


def square_bonds(Nx: int, Ny: int):
    """(nearest-neighbour bonds, next-nearest pairs) as (i, j) site pairs."""
    nn, nnn = [], []
    for iy in range(Ny):
        for ix in range(Nx):
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            i = ix + Nx * iy
            nn.append((i, ix1 + Nx * iy))
            nn.append((i, ix + Nx * iy1))
            nnn.append((i, ix1 + Nx * iy1))
            nnn.append((ix1 + Nx * iy, ix + Nx * iy1))
    return nn, nnn


class SquareModel:
    """Fixed fields of `n_cfg` configurations of the square-lattice Hubbard
    model; evaluate(theta) gives log |det M_up M_dn| and its gradient."""

    def __init__(self, Nx: int, Ny: int, U: float, dt: float, L: int, fields: np.ndarray,
                 n_matmul: int = 8, device: int = 0):
        self.Nx, self.Ny, self.N = Nx, Ny, Nx * Ny
        self.U, self.dt, self.L, self.n_matmul = U, dt, L, n_matmul
        self.fields = np.ascontiguousarray(np.asarray(fields, dtype=np.int32).reshape(-1, L, self.N))
        self.n_cfg = self.fields.shape[0]
        self.device = device
        self.nn, self.nnn = square_bonds(Nx, Ny)
        self.n_params = 3 + len(self.nn)
        N = self.N
        # dK / d theta_k
        dK = np.zeros((self.n_params, N, N))
        for b, (i, j) in enumerate(self.nn):
            for k in (0, 3 + b):
                dK[k, i, j] -= 1.0
                dK[k, j, i] -= 1.0
        for i, j in self.nnn:
            dK[1, i, j] -= 1.0
            dK[1, j, i] -= 1.0
        dK[2] -= np.eye(N)
        self.dK = dK
        self._eng = None
        self._K = None
        self._dK_dev = None

    def K(self, theta: np.ndarray) -> np.ndarray:
        t, tp, mu, h = theta[0], theta[1], theta[2], theta[3:]
        N = self.N
        K = np.zeros((N, N))
        for b, (i, j) in enumerate(self.nn):
            K[i, j] -= t + h[b]
            K[j, i] -= t + h[b]
        for i, j in self.nnn:
            K[i, j] -= tp
            K[j, i] -= tp
        K -= mu * np.eye(N)
        return K

    def _hopping(self, K: np.ndarray) -> dict:
        """the eight matrices exp(-+dt K), exp(-+dt K / 2), both spins"""
        from scipy.linalg import expm
        dt = self.dt
        mats = {"exp_Ku": expm(-dt * K), "inv_exp_Ku": expm(dt * K),
                "exp_halfKu": expm(-dt / 2 * K), "inv_exp_halfKu": expm(dt / 2 * K)}
        for k in list(mats):
            mats[k[:-1] + "d"] = mats[k]
        return mats

    def _sims(self, K: np.ndarray, mats: dict) -> list[SimData]:
        d0 = gen.make_sim(Nx=self.Nx, Ny=self.Ny, U=self.U, dt=self.dt, L=self.L,
                          n_matmul=self.n_matmul, period_eqlt=self.n_matmul, n_sweep_warm=0,
                          n_sweep_meas=1)
        for k, v in mats.items():
            d0["params/" + k] = v
        d0["params/Ku"], d0["params/Kd"] = K, K.copy()
        out = []
        for c in range(self.n_cfg):
            d = dict(d0)
            d["state/hs"] = self.fields[c]
            out.append(SimData(d))
        return out

    def engine(self, K: np.ndarray) -> Engine:
        """The model's engine with hopping K: created (and its device buffers
        allocated) by the first evaluation, then only its hopping matrices
        change (dqmc_engine_set_hopping).  The same K as the previous call
        keeps everything: neither gradient evaluation changes the fields,
        the clusters or the hopping, so its successor reads the same state
        that a re-initialisation would rebuild."""
        if self._eng is not None and self._K is not None and np.array_equal(K, self._K):
            return self._eng
        mats = self._hopping(K)
        if self._eng is None:
            self._eng = Engine(self._sims(K, mats), device=self.device)
        else:
            self._eng.set_hopping(mats)
        self._K = np.array(K, copy=True)
        return self._eng

    def close(self):
        if self._eng is not None:
            self._eng.close()
            self._eng = None
        self._K = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _contract(self, V, w, X):
        """sum_ij (V^T X_c V)_ji w_ij (V^T dK_k V)_ij for every leading
        index c of X (shape [..., 2 spins, N, N], summed over the spins) and
        parameter k, on the device when one is present: two batched products
        and one (c, ij) x (ij, k) product"""
        try:
            import torch
        except ImportError:  # pragma: no cover - torch is part of the environment
            torch = None
        lead = X.shape[:-3]
        N = self.N
        if torch is not None and torch.cuda.is_available() and self.device >= 0:
            dev = torch.device("cuda", self.device)
            Vt = torch.from_numpy(V).to(dev)
            if self._dK_dev is None:
                self._dK_dev = torch.from_numpy(self.dK).to(dev)
            E = Vt.T @ self._dK_dev @ Vt                                   # [k, i, j]
            Xs = torch.from_numpy(np.ascontiguousarray(X)).to(dev).sum(-3)  # [..., a, b]
            Xp = Vt.T @ Xs.reshape(-1, N, N) @ Vt                          # [c, i, j]
            W = torch.from_numpy(w).to(dev)
            A = (Xp.transpose(-1, -2) * W).reshape(-1, N * N)             # [c, ij]
            out = (A @ E.reshape(-1, N * N).T).cpu().numpy()
        else:
            E = np.einsum("ai,kab,bj->kij", V, self.dK, V, optimize=True)
            Xp = np.einsum("ai,...sab,bj->...ij", V, X, V, optimize=True).reshape(-1, N, N)
            out = np.einsum("cji,ij,kij->ck", Xp, w, E, optimize=True)
        return out.reshape(lead + (self.n_params,))

    def d_theta(self, K: np.ndarray):
        """(V, weights) with D_theta = V [(V^T dK_theta V) * weights] V^T:
        weights_ij = -dt exp(dt k_i) Phi_ij (Phi: divided differences of
        exp at a = -dt k)."""
        k, V = np.linalg.eigh(K)
        a = -self.dt * k
        da = a[:, None] - a[None, :]
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.where(np.abs(da) > 1e-300, np.expm1(da) / da, 1.0)
        phi = np.exp(a)[None, :] * ratio                  # (e^{a_i} - e^{a_j}) / (a_i - a_j)
        w = -self.dt * np.exp(-a)[:, None] * phi          # exp(dt k_i) = exp(-a_i)
        return V, w

    def evaluate(self, theta) -> tuple[np.ndarray, np.ndarray]:
        """log |det M_up det M_dn| per configuration and its gradient
        (n_cfg x n_params) at the parameters theta."""
        theta = np.asarray(theta, dtype=np.float64)
        K = self.K(theta)
        ld, S = self.engine(K).logdet_grad()
        V, w = self.d_theta(K)
        # tr[S D_k] = sum_ij (V^T (S_up + S_dn) V)_ji w_ij (V^T dK_k V)_ij
        return ld, self._contract(V, w, S)


    def evaluate_obs(self, theta) -> tuple[np.ndarray, np.ndarray]:
        """(obs, grad): obs[c] = (<n>, <docc>) of configuration c averaged
        over the slices, grad[c, o, k] = d obs[c, o] / d theta_k, from the
        space-time Green's function (dqmc_engine_obs_grad)."""
        theta = np.asarray(theta, dtype=np.float64)
        K = self.K(theta)
        obs, Z = self.engine(K).obs_grad()
        V, w = self.d_theta(K)
        return obs, self._contract(V, w, Z)


try:
    import torch

    class LogDet(torch.autograd.Function):
        """y_c = log |det M_up det M_dn| of configuration c as a function of
        theta (a float64 tensor); the backward contracts the incoming
        gradient with the per-configuration gradients of the forward."""

        @staticmethod
        def forward(ctx, theta, model: SquareModel):
            ld, grad = model.evaluate(theta.detach().cpu().numpy())
            ctx.save_for_backward(torch.from_numpy(grad).to(theta.device))
            return torch.from_numpy(ld).to(theta.device)

        @staticmethod
        def backward(ctx, g):
            (grad,) = ctx.saved_tensors
            return (g[:, None].to(grad.dtype) * grad).sum(0), None

    class Observables(torch.autograd.Function):
        """y_c = (<n>, <docc>) of configuration c at fixed fields as a
        function of theta; the backward contracts the incoming gradient
        with the per-configuration gradients of the forward
        (SquareModel.evaluate_obs)."""

        @staticmethod
        def forward(ctx, theta, model: SquareModel):
            obs, grad = model.evaluate_obs(theta.detach().cpu().numpy())
            ctx.save_for_backward(torch.from_numpy(grad).to(theta.device))
            return torch.from_numpy(obs).to(theta.device)

        @staticmethod
        def backward(ctx, g):
            (grad,) = ctx.saved_tensors
            return (g[:, :, None].to(grad.dtype) * grad).sum((0, 1)), None
except ImportError:  # pragma: no cover - torch is part of the environment
    LogDet = Observables = None
