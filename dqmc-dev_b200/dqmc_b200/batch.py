"""Ragged batches: chains of different lattices, U and beta on one GPU.

The engine advances a group of chains that share every parameter it keeps
per group: the lattice and its measurement maps, L and n_matmul, the
hopping matrices, the measurement periods and the sweep counters.  U may
differ inside a group, because exp_lambda and del are per chain.  A ragged
batch therefore splits its chains into such groups.  Each group gets its own
engine and CUDA streams, and every sweep of the whole batch is one CUDA graph
launch (dqmc_batch_sweeps) that forks into all groups and joins back, so
groups of different size and length run concurrently, as the C drop-in's
dqmc_wrapper_batch runs them.

The delay rank (n_delay: rank-k updates collected before they are flushed
into G) trades per-accept work against flush traffic, and the best value
depends on N.  With `autotune`, each lattice size gets the candidate whose
timed sweep of a copy of its first group is shortest.  Changing n_delay
changes results only by rounding; without `autotune` every group keeps its
files' value.  `autotune` also times every group of 32 chains or more in
1, 2, 4 and 8 lanes (sub-batches whose launches overlap) and keeps the
fastest, and for each lattice size it times the delayed update's two forms
on the first group of that size: G in device memory with one CTA per chain
and 8-column flush tiles per warp (k_update), or G on chip in a cluster of
two CTAs per chain, one per spin (k_update_cl, where one spin's G and panels
fit in shared memory).  Neither lanes nor the update form change results.
"""
from __future__ import annotations

import hashlib
import time
from collections import OrderedDict

import numpy as np

import ctypes as C

from . import lib as _lib
from .engine import INT_PARAMS, Engine, SimData

# parameters a group shares (everything except U's exp_lambda and del)
_SHARED_ARRAYS = ("map_i", "map_ij", "bonds", "map_bb", "peierlsu", "peierlsd")


def group_key(s: SimData) -> str:
    """Digest of the parameters the chains of one group must share."""
    h = hashlib.sha1()
    h.update(repr([(k, s.p[k]) for k in INT_PARAMS if k not in ("n_delay",)]).encode())
    h.update(repr((s.cplx, s.sweep)).encode())
    for name in _SHARED_ARRAYS:
        a = getattr(s, name, None)
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    for name in sorted(s.mats):
        h.update(np.ascontiguousarray(s.mats[name]).tobytes())
    return h.hexdigest()


def time_sweep(sims: list[SimData], n_delay: int | None, device: int = 0,
               lanes: int | None = None, update: str | None = None, n: int = 1) -> float:
    """Seconds per sweep of copies of `sims` at delay rank n_delay in
    `lanes` sub-batches with the given update form, over n sweeps (after
    one untimed sweep that also captures the sweep graph)."""
    copies = [s.clone() for s in sims]
    e = Engine(copies, device=device, n_delay=n_delay, lanes=lanes, update=update)
    try:
        e.init()
        e.sweeps(1, sync=True)
        t0 = time.perf_counter()
        e.sweeps(n, sync=True)
        return (time.perf_counter() - t0) / n
    finally:
        e.close()


def update_forms(sims: list[SimData], n_delay: int | None = None, device: int = 0) -> list[str]:
    """The delayed-update forms these chains can take: "global" always,
    "cluster" where the engine places one spin's G and panels on chip."""
    e = Engine([sims[0].clone()], device=device, n_delay=n_delay, update="cluster")
    try:
        return ["global", "cluster"] if e.update_form == "cluster" else ["global"]
    finally:
        e.close()


def autotune_update(sims: list[SimData], device: int = 0, n_delay: int | None = None,
                    lanes: int | None = None) -> str:
    """The delayed-update form ("global" or "cluster") with the shorter
    timed sweeps of copies of all of `sims`.  Both forms do the same
    arithmetic in the same order, so the choice only changes the speed."""
    forms = update_forms(sims, n_delay, device)
    if len(forms) == 1:
        return forms[0]
    t = {f: time_sweep(sims, n_delay, device, lanes=lanes, update=f, n=2) for f in forms}
    return min(forms, key=lambda f: t[f])


def autotune_lanes(sims: list[SimData], candidates=(1, 2, 4, 8), device: int = 0,
                   n_delay: int | None = None) -> int:
    """The lane count (sub-batches with their own streams, whose launches
    overlap) with the shortest timed sweep of copies of all of `sims`;
    candidates above the number of chains are skipped.  Any lane count gives
    the same results, so the choice only changes the speed."""
    best, best_t = None, None
    for n in candidates:
        if n > len(sims):
            continue
        t = time_sweep(sims, n_delay, device, lanes=n)
        if best_t is None or t < best_t:
            best, best_t = n, t
    return best


def autotune_delay(sims: list[SimData], candidates=(4, 8, 16, 32), device: int = 0,
                   max_chains: int = 8) -> int:
    """The candidate delay rank with the shortest timed sweep of (up to
    max_chains of) these chains; candidates a chain cannot use are skipped."""
    probe = sims[:max_chains]
    best, best_t = None, None
    for kd in candidates:
        if kd > probe[0].N:
            continue
        t = time_sweep(probe, kd, device)
        if best_t is None or t < best_t:
            best, best_t = kd, t
    return best


class RaggedBatch:
    """Chains of any parameters advanced together; see the module docstring."""

    def __init__(self, sims: list[SimData], device: int = 0, autotune: bool = False,
                 candidates=(4, 8, 16, 32), one_graph: bool = True):
        if not sims:
            raise ValueError("no chains")
        self.sims = sims
        groups: OrderedDict[str, list[int]] = OrderedDict()
        for i, s in enumerate(sims):
            groups.setdefault(group_key(s), []).append(i)
        self.groups = list(groups.values())
        self.delay = {}
        if autotune:
            # one tuning per lattice size, on the first group of that size
            for idx in self.groups:
                n = sims[idx[0]].N
                if n not in self.delay:
                    self.delay[n] = autotune_delay([sims[i] for i in idx], candidates, device)
        # the lane count of every group large enough to split (lanes change
        # only the speed, never the results)
        self.lanes = {}
        if autotune:
            for g, idx in enumerate(self.groups):
                if len(idx) >= 32:
                    self.lanes[g] = autotune_lanes([sims[i] for i in idx], device=device,
                                                   n_delay=self.delay.get(sims[idx[0]].N))
        # the delayed update's form per lattice size, on the first group of
        # that size (the form changes only the speed)
        self.update = {}
        if autotune:
            for g, idx in enumerate(self.groups):
                n = sims[idx[0]].N
                if n not in self.update:
                    self.update[n] = autotune_update([sims[i] for i in idx], device=device,
                                                     n_delay=self.delay.get(n),
                                                     lanes=self.lanes.get(g))
        self.engines = [Engine([sims[i] for i in idx], device=device,
                               n_delay=self.delay.get(sims[idx[0]].N), lanes=self.lanes.get(g),
                               update=self.update.get(sims[idx[0]].N))
                        for g, idx in enumerate(self.groups)]
        # one CUDA graph launch per sweep of all groups (dqmc_batch), or
        # (one_graph False) every group's own sweep graph on its own stream
        self.lib = self.engines[0].lib
        self.b = None
        if one_graph:
            hs = (C.c_void_p * len(self.engines))(*[e.h for e in self.engines])
            b = C.c_void_p()
            _lib.check(self.lib.dqmc_batch_create(hs, len(self.engines), C.byref(b)),
                       "dqmc_batch_create")
            self.b = b

    def init(self):
        for e in self.engines:
            e.init()

    def sweeps(self, n: int = 1, sync: bool = True):
        """n sweeps of every chain, each one CUDA graph launch for all groups
        (captured on first use for each combination of sweep kinds) on the
        batch's stream."""
        if self.b is None:
            for _ in range(n):
                for e in self.engines:
                    e.sweeps(1, sync=False)
                for e in self.engines:
                    e.sync()
            return
        _lib.check(self.lib.dqmc_batch_sweeps(self.b, n, int(sync)), "dqmc_batch_sweeps")

    def stream(self) -> int:
        """The batch's cudaStream_t (as an integer), on which its sweeps run
        (0 without the batch graph)."""
        return int(self.lib.dqmc_batch_stream(self.b) or 0) if self.b is not None else 0

    def errors(self) -> int:
        out = 0
        for e in self.engines:
            out |= e.errors()
        return out

    def pull(self):
        for e in self.engines:
            e.pull()

    def close(self):
        if getattr(self, "b", None):
            self.lib.dqmc_batch_destroy(self.b)
            self.b = None
        for e in self.engines:
            e.close()
        self.engines = []
