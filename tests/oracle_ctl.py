"""ctypes driver for the CPU oracle (oracle/liboracle_{r,c}.so).

Test infrastructure: loads a sim file, runs the oracle's sweep driver on it
and returns/saves the state and accumulators, so tests can compare the
CUDA engine with the oracle on the same inputs.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "dqmc-dev_b200"))
from dqmc_b200 import simfile  # noqa: E402

ORACLE_DIR = os.path.join(ROOT, "oracle")

_libs = {}


def oracle_lib(cplx: bool):
    key = bool(cplx)
    if key not in _libs:
        path = os.path.join(ORACLE_DIR, "liboracle_c.so" if cplx else "liboracle_r.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run make -C oracle)")
        lib = C.CDLL(path)
        lib.orc_rand_uint.restype = C.c_uint64
        lib.orc_rand_doub.restype = C.c_double
        lib.orc_flops.restype = C.c_double
        _libs[key] = lib
    return _libs[key]


class OrcSim(C.Structure):
    _fields_ = (
        [(n, C.c_int) for n in (
            "N", "L", "n_matmul", "n_delay", "F", "n_sweep_warm", "n_sweep",
            "period_eqlt", "period_uneqlt", "meas_bond_corr",
            "num_i", "num_ij", "num_b", "num_bb", "degen_i", "degen_ij", "degen_bb")]
        + [(n, C.c_void_p) for n in (
            "map_i", "map_ij", "bonds", "map_bb", "peierlsu", "peierlsd",
            "exp_Ku", "exp_Kd", "inv_exp_Ku", "inv_exp_Kd",
            "exp_halfKu", "exp_halfKd", "inv_exp_halfKu", "inv_exp_halfKd",
            "exp_lambda", "del_", "rng", "sweep", "hs",
            "eq_n_sample", "eq_sign", "density", "density_u", "density_d",
            "double_occ", "g00", "g00_u", "g00_d", "eq_nn", "eq_xx", "eq_zz",
            "eq_pair_sw", "ue_n_sample", "ue_sign", "gt0", "gt0_u", "gt0_d",
            "ue_nn", "ue_xx", "ue_zz", "ue_pair_sw", "pair_bb", "jj", "jsjs",
            "kk", "ksks")]
    )


EQ_NAMES = ["density", "density_u", "density_d", "double_occ", "g00", "g00_u",
            "g00_d", "nn", "xx", "zz", "pair_sw"]
UE_NAMES = ["gt0", "gt0_u", "gt0_d", "nn", "xx", "zz", "pair_sw"]
BOND_NAMES = ["pair_bb", "jj", "jsjs", "kk", "ksks"]


class Sim:
    """A sim file held in memory with numpy arrays the oracle works on."""

    def __init__(self, path: str):
        self.path = path
        d = simfile.read(path)
        self.d = d
        self.cplx = d["params/exp_Ku"].dtype == np.complex128
        nt = np.complex128 if self.cplx else np.float64
        self.nt = nt
        gi = lambda k: int(np.asarray(d[k]).reshape(-1)[0])  # noqa: E731
        self.N, self.L = gi("params/N"), gi("params/L")
        self.p = {k: gi("params/" + k) for k in (
            "n_matmul", "n_delay", "F", "n_sweep_warm", "n_sweep", "period_eqlt",
            "period_uneqlt", "meas_bond_corr", "num_i", "num_ij", "num_b", "num_bb",
            "degen_i", "degen_ij", "degen_bb")}
        arr = lambda k, t: np.ascontiguousarray(np.asarray(d[k], dtype=t)).reshape(-1)  # noqa: E731
        self.a = {
            "map_i": arr("params/map_i", np.int32), "map_ij": arr("params/map_ij", np.int32),
            "bonds": arr("params/bonds", np.int32), "map_bb": arr("params/map_bb", np.int32),
            "exp_lambda": arr("params/exp_lambda", np.float64),
            "del_": arr("params/del", np.float64),
        }
        for k in ("peierlsu", "peierlsd", "exp_Ku", "exp_Kd", "inv_exp_Ku", "inv_exp_Kd",
                  "exp_halfKu", "exp_halfKd", "inv_exp_halfKu", "inv_exp_halfKd"):
            self.a[k] = arr("params/" + k, nt)
        self.rng = arr("state/rng", np.uint64).copy()
        self.sweep = np.array([gi("state/sweep")], dtype=np.int32)
        self.hs = arr("state/hs", np.int32).copy()
        self.eq = {k: arr("meas_eqlt/" + k, nt).copy() for k in EQ_NAMES}
        self.eq_sign = arr("meas_eqlt/sign", nt).copy()
        self.eq_n = np.array([gi("meas_eqlt/n_sample")], dtype=np.int32)
        L, nij, nbb = self.L, self.p["num_ij"], self.p["num_bb"]
        if self.p["period_uneqlt"] > 0:
            self.ue = {k: arr("meas_uneqlt/" + k, nt).copy() for k in UE_NAMES}
            self.ue_sign = arr("meas_uneqlt/sign", nt).copy()
            self.ue_n = np.array([gi("meas_uneqlt/n_sample")], dtype=np.int32)
            if self.p["meas_bond_corr"]:
                for k in BOND_NAMES:
                    self.ue[k] = arr("meas_uneqlt/" + k, nt).copy()
        else:
            self.ue = {k: np.zeros(nij * L, nt) for k in UE_NAMES}
            self.ue_sign = np.zeros(1, nt)
            self.ue_n = np.zeros(1, np.int32)
        for k in BOND_NAMES:
            self.ue.setdefault(k, np.zeros(max(nbb, 1) * L, nt))

    def struct(self) -> OrcSim:
        s = OrcSim()
        s.N, s.L = self.N, self.L
        for k, v in self.p.items():
            setattr(s, k, v)
        ptr = lambda a: a.ctypes.data  # noqa: E731
        for k, v in self.a.items():
            setattr(s, k, ptr(v))
        s.rng, s.sweep, s.hs = ptr(self.rng), ptr(self.sweep), ptr(self.hs)
        s.eq_n_sample, s.eq_sign = ptr(self.eq_n), ptr(self.eq_sign)
        for k in EQ_NAMES:
            setattr(s, "eq_" + k if k in ("nn", "xx", "zz", "pair_sw") else k, ptr(self.eq[k]))
        s.ue_n_sample, s.ue_sign = ptr(self.ue_n), ptr(self.ue_sign)
        for k in UE_NAMES:
            setattr(s, "ue_" + k if k in ("nn", "xx", "zz", "pair_sw") else k, ptr(self.ue[k]))
        for k in BOND_NAMES:
            setattr(s, k, ptr(self.ue[k]))
        self._keep = s
        return s

    def run(self, stop_sweep: int | None = None):
        """Run the oracle up to stop_sweep (default: n_sweep); returns gu, gd, phase."""
        lib = oracle_lib(self.cplx)
        stop = self.p["n_sweep"] if stop_sweep is None else stop_sweep
        s = self.struct()
        gu = np.zeros(self.N * self.N, self.nt)
        gd = np.zeros_like(gu)
        ph = np.zeros(1, self.nt)
        lib.orc_dqmc(C.byref(s), C.c_int(stop), C.c_void_p(gu.ctypes.data),
                     C.c_void_p(gd.ctypes.data), C.c_void_p(ph.ctypes.data))
        N = self.N
        return gu.reshape(N, N).T, gd.reshape(N, N).T, ph[0]

    def hs2d(self):
        return self.hs.reshape(self.L, self.N)


_exact = {}


def exact_g(sim: "Sim", spin: int) -> np.ndarray:
    """Quad-precision G = (I + B_{L-1} ... B_0)^-1 of one spin for the sim's
    current fields (oracle/exact_g.c), as an N x N array."""
    key = bool(sim.cplx)
    if key not in _exact:
        path = os.path.join(ORACLE_DIR, "libexact_c.so" if key else "libexact_r.so")
        if not os.path.exists(path):
            raise RuntimeError(f"quad-precision G not built: {path} (run make -C oracle)")
        _exact[key] = C.CDLL(path)
    N, L = sim.N, sim.L
    ek = sim.a["exp_Ku"] if spin == 0 else sim.a["exp_Kd"]
    g = np.zeros(N * N, sim.nt)
    rc = _exact[key].exact_g(N, L, C.c_void_p(ek.ctypes.data),
                             C.c_void_p(sim.a["exp_lambda"].ctypes.data),
                             C.c_void_p(sim.hs.ctypes.data), spin, C.c_void_p(g.ctypes.data))
    if rc:
        raise RuntimeError(f"exact_g failed: {rc}")
    return g.reshape(N, N).T
