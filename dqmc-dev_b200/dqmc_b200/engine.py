"""Python front end of the GPU engine: sim files in, chains advanced on the
GPU through the C ABI, state and measurements back out.

Mirrors what the reference's data layer and driver do for one file
(src/data.c:345-789, src/dqmc.c:84-511) for any number of files that share a
parameter set; the arithmetic all happens in libdqmc_b200.so.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import lib as _lib
from . import simfile

EQ_I = ["density", "density_u", "density_d", "double_occ"]
EQ_IJ = ["g00", "g00_u", "g00_d", "nn", "xx", "zz", "pair_sw"]
UE_IJ = ["gt0", "gt0_u", "gt0_d", "nn", "xx", "zz", "pair_sw"]
UE_BB = ["pair_bb", "jj", "jsjs", "kk", "ksks"]
MATS = ["exp_Ku", "exp_Kd", "inv_exp_Ku", "inv_exp_Kd", "exp_halfKu", "exp_halfKd",
        "inv_exp_halfKu", "inv_exp_halfKd"]
INT_PARAMS = ["N", "L", "n_matmul", "n_delay", "F", "n_sweep_warm", "n_sweep", "period_eqlt",
              "period_uneqlt", "meas_bond_corr", "num_i", "num_ij", "num_b", "num_bb",
              "degen_i", "degen_ij", "degen_bb"]


def _scalar(v) -> int:
    return int(np.asarray(v).reshape(-1)[0])


def acc_datasets(p: dict):
    """The accumulated datasets after `sign`, in the engine's accumulator
    order (dqmc-dev_b200/csrc/meas.cuh), as (name, size) lists for the
    equal-time and unequal-time groups; the names and sizes are the
    reference's (data.c:441-522)."""
    L, ni, nij, nbb = p["L"], p["num_i"], p["num_ij"], p["num_bb"]
    g = lambda k: p.get(k, 0)  # noqa: E731
    eq = [(k, ni) for k in EQ_I] + [(k, nij) for k in EQ_IJ]
    if g("meas_gen_suscept"):
        eq += [(k, nij * nij) for k in ("uuuu", "dddd", "dduu", "uudd")]
    if g("meas_chiral"):
        eq += [("chi", g("num_plaq_accum"))]
    if g("meas_energy_corr"):
        eq += [("kk", nbb), ("kv", g("num_bs")), ("kn", g("num_bs")), ("vv", nij), ("vn", nij)]
    if g("meas_local_JQ"):
        eq += [("j", g("num_b_accum")), ("jn", g("num_b_accum")), ("j2", g("num_b2_accum"))]
    ue = []
    if p["period_uneqlt"] > 0:
        ue = [(k, nij * L) for k in UE_IJ]
        if g("meas_gen_suscept"):
            ue += [(k, nij * nij * L) for k in ("uuuu", "dddd", "dduu", "uudd")]
        if p["meas_bond_corr"] or g("meas_pair_bb_only"):
            ue += [("pair_bb", nbb * L)]
        if p["meas_bond_corr"]:
            ue += [(k, nbb * L) for k in UE_BB[1:]]
        if g("meas_thermal"):
            ue += [("j2jn", g("num_b2b") * L), ("jnj2", g("num_bb2") * L)]
            ue += [(k, nbb * L) for k in ("jnjn", "jnj", "jjn")]
        if g("meas_2bond_corr"):
            nb2b2 = g("num_b2b2") * L
            ue += [("pair_b2b2", nb2b2), ("j2j2", nb2b2), ("j2j", g("num_b2b") * L),
                   ("jj2", g("num_bb2") * L), ("js2js2", nb2b2), ("k2k2", nb2b2),
                   ("ks2ks2", nb2b2)]
        if g("meas_energy_corr"):
            ue += [("kv", g("num_bs") * L), ("kn", g("num_bs") * L), ("vv", nij * L),
                   ("vn", nij * L)]
        if g("meas_nematic_corr"):
            ue += [("nem_nnnn", nbb * L), ("nem_ssss", nbb * L)]
    return eq, ue


class SimData:
    """Parameters, state and accumulators of one sim file, as numpy arrays."""

    def __init__(self, d: dict, path: str | None = None):
        self.path = path
        self.cplx = np.asarray(d["params/exp_Ku"]).dtype == np.complex128
        nt = np.complex128 if self.cplx else np.float64
        self.nt = nt
        self.p = {k: _scalar(d["params/" + k]) for k in INT_PARAMS}
        self.p.update({k: _scalar(d["params/" + k]) if "params/" + k in d else 0
                       for k in _lib.TOGGLE_INTS})
        N, L = self.p["N"], self.p["L"]
        self.N, self.L = N, L
        a = lambda k, t: np.ascontiguousarray(np.asarray(d[k], dtype=t).reshape(-1))  # noqa: E731
        self.map_i = a("params/map_i", np.int32)
        self.map_ij = a("params/map_ij", np.int32)
        nb = max(self.p["num_b"], 1)
        self.bonds = a("params/bonds", np.int32) if "params/bonds" in d else np.zeros(2 * nb, np.int32)
        self.map_bb = a("params/map_bb", np.int32) if "params/map_bb" in d else np.zeros(nb * nb, np.int32)
        self.peierlsu = a("params/peierlsu", nt)
        self.peierlsd = a("params/peierlsd", nt)
        self.mats = {k: a("params/" + k, nt) for k in MATS}
        # the measurement toggles' maps and two-hop phases (absent: empty)
        self.tmaps = {}
        for k in _lib.TOGGLE_PTRS:
            t = nt if k.startswith("pp") else np.int32
            self.tmaps[k] = a("params/" + k, t) if "params/" + k in d else np.zeros(1, t)
        self.exp_lambda = a("params/exp_lambda", np.float64)
        self.del_ = a("params/del", np.float64)
        self.rng = a("state/rng", np.uint64).copy()
        self.sweep = _scalar(d["state/sweep"])
        self.hs = a("state/hs", np.int32).copy()
        self._eq_sets, self._ue_sets = acc_datasets(self.p)
        self.eq_n = _scalar(d["meas_eqlt/n_sample"])
        parts = [a("meas_eqlt/sign", nt)] + [a("meas_eqlt/" + k, nt) for k, _ in self._eq_sets]
        self.eq_acc = np.concatenate(parts).astype(nt)
        self.ue_n = 0
        self.ue_acc = np.zeros(1, nt)
        if self.p["period_uneqlt"] > 0:
            self.ue_n = _scalar(d["meas_uneqlt/n_sample"])
            parts = [a("meas_uneqlt/sign", nt)] + [a("meas_uneqlt/" + k, nt)
                                                    for k, _ in self._ue_sets]
            self.ue_acc = np.concatenate(parts).astype(nt)

    def clone(self) -> "SimData":
        """An independent copy (state and accumulators included)."""
        import copy
        return copy.deepcopy(self)

    @classmethod
    def read(cls, path: str) -> "SimData":
        d = simfile.read(path)
        if _scalar(d["state/partial_write"]):
            raise RuntimeError(f"Last checkpoint in {path} contained partial write")
        return cls(d, path)

    def params(self) -> tuple[_lib.Params, list]:
        p = _lib.Params()
        for k, v in self.p.items():
            setattr(p, k, v)
        p.cplx = int(self.cplx)
        keep = [self.map_i, self.map_ij, self.bonds, self.map_bb, self.peierlsu, self.peierlsd]
        p.map_i, p.map_ij = self.map_i.ctypes.data, self.map_ij.ctypes.data
        p.bonds, p.map_bb = self.bonds.ctypes.data, self.map_bb.ctypes.data
        p.peierlsu, p.peierlsd = self.peierlsu.ctypes.data, self.peierlsd.ctypes.data
        for k, v in self.mats.items():
            setattr(p, k, v.ctypes.data)
            keep.append(v)
        for k, v in self.tmaps.items():
            setattr(p, k, v.ctypes.data)
            keep.append(v)
        return p, keep

    def measurements(self) -> dict:
        """Accumulators as the datasets the reference writes (data.c:687-789)."""
        out = {"meas_eqlt/n_sample": self.eq_n, "meas_eqlt/sign": self.eq_acc[0]}
        o = 1
        for k, n in self._eq_sets:
            out["meas_eqlt/" + k] = self.eq_acc[o:o + n]
            o += n
        if self.p["period_uneqlt"] > 0:
            out["meas_uneqlt/n_sample"] = self.ue_n
            out["meas_uneqlt/sign"] = self.ue_acc[0]
            o = 1
            for k, n in self._ue_sets:
                out["meas_uneqlt/" + k] = self.ue_acc[o:o + n]
                o += n
        return out

    def save(self, path: str | None = None):
        """In-place update with the partial_write guard (data.c:667-789)."""
        path = path or self.path
        simfile.update(path, {"state/partial_write": 1})
        vals = {"state/rng": self.rng, "state/sweep": self.sweep,
                "state/hs": self.hs.reshape(self.L, self.N)}
        for k, v in self.measurements().items():
            vals[k] = v
        simfile.update(path, vals)
        simfile.update(path, {"state/partial_write": 0})


class Engine:
    """A group of chains with one parameter set, advanced on one GPU."""

    def __init__(self, sims: list[SimData], device: int = 0, n_delay: int | None = None,
                 lanes: int | None = None, update: str | None = None):
        """n_delay overrides the sim files' delay rank (the flush period of
        the delayed update); results then differ from the file's setting
        only by rounding.  lanes overrides the number of sub-batches with
        their own streams (else the engine's rule, or DQMC_LANES).  update
        selects the delayed update's form: "global" (G in device memory, one
        CTA per chain, k_update) or "cluster" (G on chip in a cluster of two
        CTAs per chain, one per spin, k_update_cl, where one spin's G and
        panels fit in shared memory; else "global"), else DQMC_UPDATE
        decides, else the engine's rule (on chip for real scalars with
        N >= 96 and at most 64 chains).  Results depend on neither lanes nor
        update: every form does the same arithmetic in the same order."""
        if not sims:
            raise ValueError("no chains")
        env = {}
        if lanes is not None:
            env["DQMC_LANES"] = str(int(lanes))
        if update is not None:
            if update not in ("global", "cluster"):
                raise ValueError(f"update form {update!r}: 'global' or 'cluster'")
            env["DQMC_UPDATE"] = update
        if env:
            old = {k: os.environ.get(k) for k in env}
            os.environ.update(env)
            try:
                self.__init__(sims, device, n_delay)
            finally:
                for k, v in old.items():
                    if v is None:
                        os.environ.pop(k, None)
                    else:
                        os.environ[k] = v
            return
        self.lib = _lib.load()
        self.sims = sims
        s0 = sims[0]
        self._p, self._keep = s0.params()
        if n_delay is not None:
            self._p.n_delay = int(n_delay)
        h = C.c_void_p()
        _lib.check(self.lib.dqmc_engine_create(C.byref(self._p), len(sims), device, C.byref(h)),
                   "dqmc_engine_create")
        self.h = h
        for c, s in enumerate(sims):
            _lib.check(self.lib.dqmc_engine_set_chain(
                h, c, s.exp_lambda.ctypes.data, s.del_.ctypes.data, s.rng.ctypes.data,
                s.hs.ctypes.data, s.sweep), "dqmc_engine_set_chain")
            _lib.check(self.lib.dqmc_engine_set_acc(
                h, c, s.eq_n, s.eq_acc.ctypes.data, s.ue_n, s.ue_acc.ctypes.data),
                "dqmc_engine_set_acc")

    def init(self):
        _lib.check(self.lib.dqmc_engine_init(self.h), "dqmc_engine_init")

    def push(self):
        """Upload every chain's state from its SimData again
        (dqmc_engine_set_chain); G, the cluster products and the draws follow
        the uploaded fields before the next sweep.  The accumulators stay."""
        for c, s in enumerate(self.sims):
            _lib.check(self.lib.dqmc_engine_set_chain(
                self.h, c, s.exp_lambda.ctypes.data, s.del_.ctypes.data, s.rng.ctypes.data,
                s.hs.ctypes.data, s.sweep), "dqmc_engine_set_chain")

    def sweeps(self, n: int, sync: bool = True):
        _lib.check(self.lib.dqmc_engine_sweeps(self.h, n, int(sync)), "dqmc_engine_sweeps")

    def sync(self):
        _lib.check(self.lib.dqmc_engine_sync(self.h), "dqmc_engine_sync")

    def errors(self) -> int:
        return int(self.lib.dqmc_engine_errors(self.h))

    def launches_per_sweep(self, meas_eq: bool, meas_ue: bool) -> int:
        return int(self.lib.dqmc_engine_launches_per_sweep(self.h, int(meas_eq), int(meas_ue)))

    PROFILE_CLASSES = ["gemm", "update", "qr_pivot", "uneqlt_g", "meas", "qr_presort",
                       "recombine"]

    def profile_sweep(self, meas_eq: bool, meas_ue: bool = False, n_class: int = 7):
        """One eagerly launched sweep with per-launch CUDA events; returns
        {class: (ms, launches, flops, bytes)}."""
        out = (C.c_double * (4 * n_class))()
        _lib.check(self.lib.dqmc_engine_profile_sweep(self.h, int(meas_eq), int(meas_ue), out,
                                                      n_class), "dqmc_engine_profile_sweep")
        names = self.PROFILE_CLASSES
        return {names[c]: tuple(out[4 * c:4 * c + 4]) for c in range(n_class)}

    @property
    def update_form(self) -> str:
        """"cluster" when the delayed update holds G on chip (k_update_cl),
        else "global" (dqmc_engine_update_on_chip)."""
        r = self.lib.dqmc_engine_update_on_chip(self.h)
        _lib.check(min(r, 0), "dqmc_engine_update_on_chip")
        return "cluster" if r == 1 else "global"

    def profile_grad(self, which: str, n_class: int = 7):
        """One gradient evaluation ("logdet" or "obs") with per-launch CUDA
        events, its results discarded; returns ({class: (ms, launches, flops,
        bytes)}, kernels launched) (dqmc_engine_profile_grad)."""
        out = (C.c_double * (4 * n_class))()
        n = C.c_int(0)
        _lib.check(self.lib.dqmc_engine_profile_grad(self.h, {"logdet": 0, "obs": 1}[which], out,
                                                     n_class, C.byref(n)),
                   "dqmc_engine_profile_grad")
        names = self.PROFILE_CLASSES
        return {names[c]: tuple(out[4 * c:4 * c + 4]) for c in range(n_class)}, n.value

    def logdet_grad(self):
        """(logdet per chain, S per chain and spin as N x N arrays): see
        dqmc_engine_logdet_grad; fields, RNG and sweep counts stay."""
        n, N = len(self.sims), self.sims[0].N
        ld = np.zeros(n)
        S = np.zeros(n * 2 * N * N, dtype=self.sims[0].nt)
        _lib.check(self.lib.dqmc_engine_logdet_grad(self.h, ld.ctypes.data, S.ctypes.data),
                   "dqmc_engine_logdet_grad")
        return ld, S.reshape(n, 2, N, N).transpose(0, 1, 3, 2)

    def obs_grad(self):
        """(obs per chain [n, docc], Z per chain, observable and spin as N x N
        arrays): see dqmc_engine_obs_grad."""
        n, N = len(self.sims), self.sims[0].N
        obs = np.zeros(2 * n)
        Z = np.zeros(n * 4 * N * N, dtype=self.sims[0].nt)
        _lib.check(self.lib.dqmc_engine_obs_grad(self.h, obs.ctypes.data, Z.ctypes.data),
                   "dqmc_engine_obs_grad")
        return obs.reshape(n, 2), Z.reshape(n, 2, 2, N, N).transpose(0, 1, 2, 4, 3)

    def set_hopping(self, mats: dict):
        """Replace the eight hopping matrices (names as MATS, N x N arrays of
        the engine's scalar type) of every chain in place
        (dqmc_engine_set_hopping); G follows before the next use."""
        nt = self.sims[0].nt
        col = [np.ascontiguousarray(np.asarray(mats[k], dtype=nt).T).reshape(-1) for k in MATS]
        _lib.check(self.lib.dqmc_engine_set_hopping(self.h, *[c.ctypes.data for c in col]),
                   "dqmc_engine_set_hopping")

    def check_g(self, on: bool = True, accurate: bool = False):
        """G drift self-check on or off (dqmc_engine_check_g; the runtime form
        of the reference's CHECK_G_WRP and CHECK_G_UE): every recalculation
        also compares the recalculated G with the previous slice's G wrapped
        once more.  With accurate, every recalculation also computes G from
        the L single-slice factors with a QR after each (CHECK_G_ACC)."""
        flag = (1 | (2 if accurate else 0)) if on else 0
        _lib.check(self.lib.dqmc_engine_check_g(self.h, flag), "dqmc_engine_check_g")

    def g_drift(self, unequal_time: bool = False, accurate: bool = False):
        """(max, mean, n): per chain the largest |G - G_wrapped| and its mean
        over the entries, over the n recalculations checked and both spins
        (dqmc_engine_g_drift); with unequal_time, |G - G(0,0)| of the
        unequal-time path over the n unequal-time measurements
        (dqmc_engine_g_drift_ue); with accurate, |G - G_acc| of the
        single-slice recalculation (dqmc_engine_g_drift_acc)."""
        n = len(self.sims)
        mx, mean = np.zeros(n), np.zeros(n)
        cnt = C.c_int(0)
        fn = (self.lib.dqmc_engine_g_drift_acc if accurate else
              self.lib.dqmc_engine_g_drift_ue if unequal_time else self.lib.dqmc_engine_g_drift)
        _lib.check(fn(self.h, mx.ctypes.data, mean.ctypes.data, C.addressof(cnt)),
                   "dqmc_engine_g_drift")
        return mx, mean, int(cnt.value)

    def stream(self) -> int:
        return int(self.lib.dqmc_engine_stream(self.h) or 0)

    def lanes(self) -> int:
        """Number of sub-batches (each with its own stream) the chains run in."""
        return int(self.lib.dqmc_engine_lanes(self.h))

    def pull(self):
        """Copy every chain's state and accumulators back into its SimData."""
        for c, s in enumerate(self.sims):
            sw = C.c_int()
            _lib.check(self.lib.dqmc_engine_get_chain(self.h, c, s.rng.ctypes.data,
                                                      s.hs.ctypes.data, C.byref(sw)),
                       "dqmc_engine_get_chain")
            s.sweep = sw.value
            en, un = C.c_int(), C.c_int()
            _lib.check(self.lib.dqmc_engine_get_acc(self.h, c, C.byref(en), s.eq_acc.ctypes.data,
                                                    C.byref(un), s.ue_acc.ctypes.data),
                       "dqmc_engine_get_acc")
            s.eq_n, s.ue_n = en.value, un.value

    def state_arrays(self):
        """Contiguous host arrays of every chain's state, in chain order:
        (exp_lambda [n, 2N], del [n, 2N], rng [n, 17], hs [n, L, N])."""
        return (np.ascontiguousarray(np.stack([s.exp_lambda for s in self.sims])),
                np.ascontiguousarray(np.stack([s.del_ for s in self.sims])),
                np.ascontiguousarray(np.stack([s.rng for s in self.sims])),
                np.ascontiguousarray(np.stack([s.hs for s in self.sims])))

    def set_chains(self, exp_lambda, del_, rng, hs, sweep: int):
        """Every chain's state from contiguous host arrays in one call
        (dqmc_engine_set_chains)."""
        _lib.check(self.lib.dqmc_engine_set_chains(self.h, exp_lambda.ctypes.data, del_.ctypes.data,
                                                   rng.ctypes.data, hs.ctypes.data, int(sweep)),
                   "dqmc_engine_set_chains")

    def get_chains(self, rng, hs, eq_n, eq_acc, ue_n=None, ue_acc=None) -> int:
        """Every chain's state and accumulators into contiguous host arrays
        in one call (dqmc_engine_get_chains); returns the sweep counter."""
        sw = np.zeros(1, np.int32)
        p = lambda a: None if a is None else a.ctypes.data
        _lib.check(self.lib.dqmc_engine_get_chains(self.h, p(rng), p(hs), p(sw), p(eq_n),
                                                   p(eq_acc), p(ue_n), p(ue_acc)),
                   "dqmc_engine_get_chains")
        return int(sw[0])

    def g(self, c: int):
        s = self.sims[c]
        gu = np.zeros(s.N * s.N, s.nt)
        gd = np.zeros_like(gu)
        ph = np.zeros(1, s.nt)
        _lib.check(self.lib.dqmc_engine_get_g(self.h, c, gu.ctypes.data, gd.ctypes.data,
                                              ph.ctypes.data), "dqmc_engine_get_g")
        return gu.reshape(s.N, s.N).T, gd.reshape(s.N, s.N).T, ph[0]

    def accepts(self, c: int) -> int:
        n = C.c_longlong()
        _lib.check(self.lib.dqmc_engine_accepts(self.h, c, C.byref(n)), "dqmc_engine_accepts")
        return n.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.dqmc_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_file(path: str, n_sweeps: int | None = None, device: int = 0) -> SimData:
    """Run one sim file to n_sweep (or n_sweeps more) and return its data."""
    s = SimData.read(path)
    e = Engine([s], device)
    e.init()
    e.sweeps((s.p["n_sweep"] - s.sweep) if n_sweeps is None else n_sweeps)
    e.pull()
    e.close()
    return s
