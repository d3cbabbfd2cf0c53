"""Benchmark: batched DQMC chain-sweeps/s on one node.

Default workload (per GPU): 256 independent chains of the single-band
Hubbard model on a 12x12 square lattice (N = 144), t = 1, U = 4, mu = -1,
beta = 6, dtau = 0.05 (L = 120), n_matmul = 10, n_delay = 16, equal-time
measurements every 8 slices, FP64 throughout.  Chains differ by RNG stream
(splitmix64 of the seed, one 2^512 jump per chain) and so by their HS
fields.  A step is one sweep of every chain; value = chains x steps /
device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batch256|c1|uneq8x8|complex64|ragged64|grad128]

With N > 1 each rank (one process per GPU; bench.py starts them itself
through torch.distributed.run when WORLD_SIZE is unset) runs its own block
of chains (weak scaling, no collective on the data path); times are the
maximum over ranks.  `--impl reference` times the reference's own C build
(oracle/_ref/dqmc_1_{r,c}, the reference src/ compiled against OpenBLAS) on
the host cores, as the reference deploys it: one process per two cores, two
OpenMP threads each.  The other workloads are the further benchmark
configurations, one JSON line each.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import socket
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dqmc-dev_b200"))

SEED = 1000
METRIC = "chain-sweeps/s"

# single-parameter-set workloads: chains per GPU, generator arguments, the
# description, and the reference build's sweeps per process for a bounded
# CPU sample (about 5-30 s)
WORKLOADS = {
    "batch256": dict(
        chains=256,
        cfg=dict(Nx=12, Ny=12, U=4.0, mu=-1.0, tp=0.0, dt=0.05, L=120, n_matmul=10, n_delay=16,
                 period_eqlt=8),
        desc="256 chains x 12x12 square Hubbard (N=144), U=4, mu=-1, beta=6, dtau=0.05 "
             "(L=120), n_matmul=10, n_delay=16, eqlt every 8 slices, FP64",
        ref_sweeps=30),
    "c1": dict(
        chains=1,
        cfg=dict(Nx=4, Ny=4, U=4.0, mu=0.0, tp=0.0, dt=0.1, L=40, n_matmul=5, n_delay=8,
                 period_eqlt=8),
        desc="1 chain x 4x4 square Hubbard, U=4, mu=0, beta=4, dtau=0.1 (L=40), n_matmul=5, "
             "n_delay=8, eqlt every 8 slices, FP64 (the plain single-chain configuration)",
        ref_sweeps=4000),
    "uneq8x8": dict(
        chains=1,
        cfg=dict(Nx=8, Ny=8, tp=-0.25, U=6.0, mu=-0.5, dt=0.1, L=80, n_matmul=8, n_delay=16,
                 period_eqlt=8, period_uneqlt=4),
        desc="1 chain x 8x8 square Hubbard, t'=-0.25, U=6, mu=-0.5, beta=8, dtau=0.1 (L=80), "
             "n_matmul=8, n_delay=16, eqlt every 8 slices, unequal-time every 4 sweeps, FP64",
        ref_sweeps=200),
    "complex64": dict(
        chains=64,
        cfg=dict(Nx=10, Ny=10, U=4.0, mu=0.0, dt=0.1, L=50, n_matmul=5, n_delay=16, nflux=1,
                 period_eqlt=5, period_uneqlt=1, meas_bond_corr=1),
        desc="64 chains x 10x10 square Hubbard with one flux quantum (Peierls phases, "
             "complex128), U=4, mu=0, beta=5, dtau=0.1 (L=50), n_matmul=5, eqlt every 5 "
             "slices, unequal-time with current-current bond correlators every sweep",
        ref_sweeps=20),
}

# launch classes of the engine's per-launch profile whose algorithmic FLOPs
# are counted (2 M N K per GEMM; 8/3 N^3 per item for the QRs with explicit
# Q and for the recombine's LU solve; the update's flush and panel products
# from its accepts), with the kernel behind each
ROOFLINE_KERNELS = {
    "gemm": "k_gemm (batched FP64 DMMA: wraps, cluster products, half wraps, UDT products)",
    "update": "k_update (delayed rank-k Metropolis update: panel products and DMMA flush)",
    "qr_presort": "k_qrb (pre-sorted blocked Householder QR with explicit Q, calc_eq_g)",
    "qr_pivot": "k_qrp (column-pivoted Householder QR with explicit Q, calc_eq_g)",
    "recombine": "k_recb (LU solve G = (D_b^-1 Q^H + D_s T)^-1 D_b^-1 Q^H)",
}
# DRAM bytes (read + write) per chain-spin item of one launch, from ncu
# captures of these kernels on the 12x12 model (profiles/), scaled by the
# items of a launch; other workloads report null
TRAFFIC_PER_ITEM = {"batch256": {"gemm": 172580, "qr_presort": 168068, "qr_pivot": 166916,
                                 "recombine": 333636, "update": 170852}}
# the reference build's FLOPs per chain-sweep of each single-model workload,
# counted call by call with LAPACK-standard counts (python oracle/flop_tally.py
# after make -C oracle tally; averaged over an unequal-time cycle)
REF_FLOPS_PER_CHAIN_SWEEP = {"batch256": 8308315008.0, "c1": 4082880.0,
                             "uneq8x8": 700769877.3, "complex64": 14984803733.3}

T0 = time.time()


def log(msg):
    """progress line on stderr (the JSON result goes to stdout)"""
    print(f"[bench {time.time() - T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn_ranks(gpus):
    """`--gpus N` without a launcher: start N ranks of this same command
    through torch.distributed.run (one process per GPU) and return its exit
    status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1",
           f"--master-port={_free_port()}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def dist_setup():
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def dist_done(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def reduce_device():
    import torch
    return "cuda" if torch.cuda.is_available() else "cpu"


def max_over_ranks(x, world):
    from dqmc_b200 import replicas
    return replicas.max_over_ranks(x, world, device=reduce_device())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.path = tempfile.mktemp(suffix=".csv")
        self.device = device
        self.p = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device),
                                       f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()
            self.f.close()

    def summary(self):
        if not self.p or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        busy = [v for v in sm if v > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(busy)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak():
    """cuBLAS DGEMM 8192^3, best of 5 (FP64 tensor roofline denominator)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e12


# ---------------------------------------------------------------- inputs

def _restream(base, rngs):
    """copies of one sim dict with chain c's own RNG stream and fields"""
    from dqmc_b200 import gen
    N, L = int(base["params/N"]), int(base["params/L"])
    out = [base]
    for r in rngs[1:]:
        hs, rng = gen.initial_hs(r, L, N)
        d = dict(base)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rng, hs
        out.append(d)
    return out


def sim_dicts(wl, chains, n_sweep):
    """Sim data of the given global chains of the job: chain c starts from
    the master stream of SEED jumped c times (dqmc_b200.replicas)."""
    from dqmc_b200 import gen, replicas
    rngs = replicas.chain_streams(SEED, chains)
    base = gen.make_sim(init_rng=rngs[0], n_sweep_warm=0, n_sweep_meas=n_sweep, **wl["cfg"])
    return _restream(base, rngs)


# ------------------------------------------------------- reference (CPU)

def reference_rate(cfg, n_proc, sweeps, seed=1):
    """Aggregate chain-sweeps/s of the reference C build: n_proc processes of
    dqmc_1_{r,c} (2 OpenMP threads, OpenBLAS 1 thread) on independent chains
    of the model `cfg`."""
    from dqmc_b200 import gen
    cplx = cfg.get("nflux", 0) != 0
    exe = os.path.join(ROOT, "oracle", "_ref", "dqmc_1_c" if cplx else "dqmc_1_r")
    if not os.path.exists(exe):
        raise RuntimeError(f"reference build missing: {exe}")
    tmp = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        paths = gen.create_batch(Nfiles=n_proc, prefix="ref", seed=seed, n_sweep_warm=0,
                                 n_sweep_meas=sweeps, **cfg)
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="2")
        t0 = time.perf_counter()
        procs = [subprocess.Popen([exe, "-b", "-l", f"{p}.log", p], env=env,
                                  stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
                 for p in paths]
        rcs = [p.wait() for p in procs]
        t = time.perf_counter() - t0
        if any(rcs):
            raise RuntimeError(f"reference runs failed: {rcs}")
    finally:
        os.chdir(cwd)
        shutil.rmtree(tmp, ignore_errors=True)
    return n_proc * sweeps / t, t


def cpu_procs():
    return max(1, (os.cpu_count() or 2) // 2)


def ragged_reference_rate(n_proc, sweeps):
    """Aggregate chain-sweeps/s of the reference C build on a bounded sample
    of the ragged mix: n_proc chains spread evenly over the 64 (the same
    generator and seed as the GPU line), one dqmc_1_r process each (2
    OpenMP threads, OpenBLAS 1 thread), `sweeps` sweeps each.  The rate is
    that of a farm of these n_proc processes working through the mix: n_proc
    over the mean time a process spends on one chain-sweep (each process's
    wall time over its sweeps), so large and small chains weigh by their
    cost.  The files take the reference generator's layout (a params file
    per chain, linked)."""
    from dqmc_b200 import simfile
    exe = os.path.join(ROOT, "oracle", "_ref", "dqmc_1_r")
    if not os.path.exists(exe):
        raise RuntimeError(f"reference build missing: {exe}")
    dicts, _ = _ragged64(sweeps)
    step = max(1, len(dicts) // n_proc)
    dicts = dicts[::step][:n_proc]
    tmp = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        paths = []
        for c, d in enumerate(dicts):
            rel = f"r{c}.h5.params"
            simfile.write(rel, {k: v for k, v in d.items() if k.startswith(("metadata/", "params/"))})
            sim = {k: v for k, v in d.items() if not k.startswith(("metadata/", "params/"))}
            sim["params_file"] = rel
            sim["metadata"] = simfile.Link(rel)
            sim["params"] = simfile.Link(rel)
            simfile.write(f"r{c}.h5", sim)
            paths.append(f"r{c}.h5")
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="2")
        t0 = time.perf_counter()
        procs = [subprocess.Popen([exe, "-b", "-l", f"{p}.log", p], env=env,
                                  stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
                 for p in paths]
        ends = [None] * len(procs)
        while any(e is None for e in ends):
            for i, p in enumerate(procs):
                if ends[i] is None and p.poll() is not None:
                    ends[i] = time.perf_counter() - t0
            time.sleep(0.005)
        t = max(ends)
        rcs = [p.returncode for p in procs]
        if any(rcs):
            raise RuntimeError(f"reference runs failed: {rcs}")
        sides = sorted({int(round(float(np.sqrt(int(np.asarray(d["params/N"]).reshape(-1)[0])))))
                        for d in dicts})
    finally:
        os.chdir(cwd)
        shutil.rmtree(tmp, ignore_errors=True)
    n = len(paths)
    sample = (f"{n} chains spread over the ragged mix (sides {sides}), one process of the "
              f"reference dqmc_1_r each x {sweeps} sweeps (2 OpenMP threads, OpenBLAS 1 "
              f"thread), {min(ends):.1f}-{t:.1f} s per process; rate = processes / mean "
              f"seconds per chain-sweep")
    return n * sweeps / (sum(ends) / n), t, sample


def ref_sample(wl, n_proc, sweeps, t):
    cplx = wl["cfg"].get("nflux", 0) != 0
    c = wl["cfg"]
    return (f"{n_proc} processes of the reference dqmc_1_{'c' if cplx else 'r'} x {sweeps} "
            f"sweeps of one {c['Nx']}x{c['Ny']} L={c['L']} chain each (2 OpenMP threads, "
            f"OpenBLAS 1 thread), {t:.1f} s")


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    if args.workload == "grad128":
        from_grad = grad_cpu_baseline()
        print(json.dumps({
            "metric": "grad evals/s", "value": from_grad["value"], "unit": "grad evals/s",
            "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1e3 / from_grad["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": GRAD_DESC, "cpu": True}, "cpu_baseline": from_grad,
            "e2e": {"value": from_grad["value"], "unit": "grad evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "ragged64":
        n_proc = cpu_procs()
        sweeps = max(1, args.steps)
        rate, t, sample = ragged_reference_rate(n_proc, sweeps)
        print(json.dumps({
            "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / sweeps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": _ragged64(1)[1], "chains": n_proc, "cpu": True},
            "cpu_baseline": {"value": rate, "unit": METRIC, "cores": n_proc * 2,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return
    wl = WORKLOADS.get(args.workload, WORKLOADS["batch256"])
    n_proc = cpu_procs()
    sweeps = max(1, args.steps) * max(1, wl["ref_sweeps"] // 30)
    rate, t = reference_rate(wl["cfg"], n_proc, sweeps)
    line = {
        "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / sweeps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if wl["cfg"].get("nflux", 0) else "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": wl["desc"], "chains": n_proc, "cpu": True},
        "cpu_baseline": {"value": rate, "unit": METRIC, "cores": n_proc * 2, "kind": "reference",
                         "sample": ref_sample(wl, n_proc, sweeps, t)},
        "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------- GPU helpers

def plain_chain_rate(sim, device, warm=2, timed=3):
    """chain-sweeps/s of the plain single-chain GPU path: one chain of the
    same model alone in an engine (graph-replayed sweeps, CUDA events)."""
    import torch
    from dqmc_b200 import engine
    c = sim.clone()
    c.p["n_sweep"] = c.sweep + warm + timed + 2     # room for the sweeps below
    e = engine.Engine([c], device=device)
    try:
        e.init()
        e.sweeps(warm, sync=True)
        st = torch.cuda.ExternalStream(e.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        e.sweeps(timed, sync=False)
        b.record(st)
        torch.cuda.synchronize()
        return timed / (a.elapsed_time(b) / 1e3)
    finally:
        e.close()


def profile_one_lane(sims, device, period_uneqlt):
    """profile_mix of a copy of the same chains in a one-lane engine, so
    that every launch covers all chain-spin items of the workload (the
    timed engine splits them into lanes whose launches overlap; profiled
    one lane at a time, each launch would cover a fraction and underfill
    the GPU).  Returns the profile and the items of one launch."""
    from dqmc_b200 import engine
    old = os.environ.get("DQMC_LANES")
    os.environ["DQMC_LANES"] = "1"
    try:
        e1 = engine.Engine([s.clone() for s in sims], device=device)
    finally:
        if old is None:
            del os.environ["DQMC_LANES"]
        else:
            os.environ["DQMC_LANES"] = old
    try:
        e1.init()
        return profile_mix(e1, period_uneqlt), 2 * len(sims)
    finally:
        e1.close()


def profile_mix(eng, period_uneqlt):
    """Per-class (ms, launches, flops, bytes) of an average sweep: one eager
    equal-time sweep, and with unequal-time measurements every p sweeps one
    such sweep too, weighted (p - 1) / p and 1 / p."""
    prof = eng.profile_sweep(True, False)
    if period_uneqlt <= 0:
        return prof
    ue = eng.profile_sweep(True, True)
    w = 1.0 / period_uneqlt
    return {k: tuple((1 - w) * a + w * b for a, b in zip(prof[k], ue[k])) for k in prof}


def roofline(prof, items, workload, peak, ms_per_step, chains=None):
    """The dominant launch class by event time among those with counted
    FLOPs: its FLOPs over its time against the FP64 DGEMM peak, and the
    whole sweep's FLOPs over the timed sweep, by the engine's count and (for
    `chains` chains of a workload with a tally) by the reference build's."""
    cls = [k for k in ROOFLINE_KERNELS if prof[k][0] > 0 and prof[k][2] > 0]
    dom = max(cls, key=lambda k: prof[k][0])
    d_ms, d_n, d_fl, _ = prof[dom]
    achieved = d_fl / (d_ms / 1e3) / 1e12
    traffic = TRAFFIC_PER_ITEM.get(workload, {}).get(dom)
    sweep_fl = sum(prof[k][2] for k in ROOFLINE_KERNELS)
    sweep_tf = sweep_fl / (ms_per_step / 1e3) / 1e12
    out = {"bound": "tensor", "kernel": ROOFLINE_KERNELS[dom], "class": dom,
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None,
            "traffic": traffic * items if traffic else None,
            "traffic_unit": "bytes per launch (DRAM read + write)",
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json "
                           "carries no FP64 figure)",
            "launches_per_sweep": int(round(d_n)),
            "ms_per_launch": d_ms / d_n if d_n else None,
            "class_ms_per_sweep": {k: prof[k][0] for k in prof},
            "class_tflops": {k: prof[k][2] / (prof[k][0] / 1e3) / 1e12
                             for k in ROOFLINE_KERNELS if prof[k][0] > 0 and prof[k][2] > 0},
            "sweep": {"flops": sweep_fl, "achieved": sweep_tf,
                      "frac": sweep_tf / peak if peak else None,
                      "note": "counted FLOPs of every class over the timed ms_per_step"}}
    ref = REF_FLOPS_PER_CHAIN_SWEEP.get(workload)
    if ref and chains:
        ref_tf = ref * chains / (ms_per_step / 1e3) / 1e12
        out["sweep"].update({
            "reference_flops": ref * chains, "reference_achieved": ref_tf,
            "reference_frac": ref_tf / peak if peak else None,
            "reference_note": "the reference build's LAPACK-standard FLOPs per chain-sweep "
                              "(oracle/flop_tally.py) times the chains, over ms_per_step"})
    return out


def e2e_rate(engs, steps, world, sweep_all):
    """chain-sweeps/s through the C ABI with host buffers: per step, every
    engine's chains go from pinned host memory to the device in one batched
    call each (dqmc_engine_set_chains), one sweep of all of them runs
    (sweep_all, synchronised), and state plus accumulators come back in one
    call per engine (dqmc_engine_get_chains); the downloaded state is the
    next step's input."""
    import torch

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    legs, h2d, d2h, n_all = [], 0, 0, 0
    for eng in engs:
        eng.pull()          # host copies of the state the device now holds
        sims = eng.sims
        n = len(sims)
        el_h, dl_h, rg_h, hs_h = (pinned(a) for a in eng.state_arrays())
        rg_o, hs_o = pinned(np.zeros_like(rg_h)), pinned(np.zeros_like(hs_h))
        eqn_o = pinned(np.zeros(n, np.int32))
        eq_o = pinned(np.zeros((n,) + sims[0].eq_acc.shape, sims[0].eq_acc.dtype))
        ue = sims[0].p["period_uneqlt"] > 0
        uen_o = pinned(np.zeros(n, np.int32)) if ue else None
        ue_o = pinned(np.zeros((n,) + sims[0].ue_acc.shape, sims[0].ue_acc.dtype)) if ue else None
        h2d += el_h.nbytes + dl_h.nbytes + rg_h.nbytes + hs_h.nbytes
        d2h += rg_o.nbytes + hs_o.nbytes + eqn_o.nbytes + eq_o.nbytes
        if ue:
            d2h += uen_o.nbytes + ue_o.nbytes
        legs.append([eng, el_h, dl_h, rg_h, hs_h, rg_o, hs_o, eqn_o, eq_o, uen_o, ue_o, sims[0].sweep])
        n_all += n
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for lg in legs:
            lg[0].set_chains(lg[1], lg[2], lg[3], lg[4], lg[11])
        sweep_all()
        for lg in legs:
            lg[11] = lg[0].get_chains(lg[5], lg[6], lg[7], lg[8], lg[9], lg[10])
            lg[3], lg[5] = lg[5], lg[3]
            lg[4], lg[6] = lg[6], lg[4]
    t = max_over_ranks((time.perf_counter() - t0) / steps, world)
    return {"value": n_all * world / t, "unit": METRIC, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps}


def run_engine_workload(args, rank, world, local):
    """One parameter set of chains in one engine: K graph-replayed sweeps
    timed with CUDA events on the engine's stream, then the end-to-end leg,
    a per-launch profile, the roofline, and the reference build's rate."""
    import torch
    torch.cuda.set_device(local)
    from dqmc_b200 import engine, replicas
    wl = WORKLOADS[args.workload]
    nch = args.chains if args.chains else wl["chains"]
    e2e_steps = max(10, args.e2e_steps)
    total = args.warmup + args.steps + e2e_steps + 4
    dicts = sim_dicts(wl, replicas.shard(nch * world, rank, world), n_sweep=total)
    log(f"generated {nch} chains")
    sims = [engine.SimData(d) for d in dicts]
    eng = engine.Engine(sims, device=local)
    eng.init()
    log("initial G done")
    stream = torch.cuda.ExternalStream(eng.stream())
    pu = sims[0].p["period_uneqlt"]

    # warm-up (also captures the sweep graphs of every kind the timed run uses)
    for _ in range(args.warmup):
        eng.sweeps(1, sync=True)
    log("warm-up done")

    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        eng.sweeps(args.steps, sync=False)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    t_dev = ev0.elapsed_time(ev1) / 1e3
    assert eng.errors() == 0, "device error word set"
    t_max = max_over_ranks(t_dev, world)
    log(f"timed sweeps done: {1e3 * t_dev / args.steps:.2f} ms per sweep")
    value = nch * args.steps * world / t_max
    kinds = [eng.launches_per_sweep(True, False)]
    if pu > 0:
        kinds.append(eng.launches_per_sweep(True, True))
    launches = int(round(args.steps * (kinds[0] * (1 - 1 / pu) + kinds[1] / pu))) if pu > 0 \
        else kinds[0] * args.steps

    e2e = e2e_rate([eng], e2e_steps, world, lambda: eng.sweeps(1, sync=True))
    log("e2e done")
    prof, items = profile_one_lane(sims, local, pu)
    log("profile sweep done")
    peak = fp64_peak()
    rl = roofline(prof, items, args.workload, peak, 1e3 * t_max / args.steps, chains=nch)

    plain = None
    if args.workload == "batch256":
        plain = plain_chain_rate(sims[0], local)
        log("plain single-chain sweeps done")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            n_proc = cpu_procs()
            rate, t = reference_rate(wl["cfg"], n_proc, wl["ref_sweeps"])
            log("cpu baseline done")
            cpu = {"value": rate, "unit": METRIC, "cores": 2 * n_proc, "kind": "reference",
                   "sample": ref_sample(wl, n_proc, wl["ref_sweeps"], t)}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "reference",
                   "sample": f"not run: {ex}"}

    if rank == 0:
        cfg = {"workload": wl["desc"], "chains_per_gpu": nch, "lanes": eng.lanes(),
               "l2": "inputs larger than L2" if nch * 2 * 20 * sims[0].N ** 2 * 8 > 126e6
                     else "inputs fit L2 (one small chain): L2 is not flushed",
               "sweep_profile_note": "kernel ms per class over one eager sweep of a copy of "
                                     "the same chains in one lane (every launch covers all "
                                     "chain-spin items), CUDA events around each launch; the "
                                     "timed sweeps run the chains in overlapping lanes"}
        if plain is not None:
            cfg["plain_1chain_gpu"] = {"value": plain, "unit": METRIC,
                                       "batched_over_plain": value / world / plain}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "c128" if sims[0].cplx else "f64", "data": "synthetic",
            "config": cfg, "gpu_launches": launches, "e2e": e2e, "roofline": rl,
            "clocks": clk.summary(), "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    eng.close()


# ------------------------------------------------------ ragged and grad

def _ragged64(n_sweep):
    from dqmc_b200 import gen
    return gen.make_ragged(64, SEED, n_sweep_warm=0, n_sweep_meas=n_sweep, period_eqlt=10), (
        "64 ragged chains: square lattice side uniform in {6,8,10,14,16}, U uniform in [2,8], "
        "beta uniform in [2,8], dtau=0.05, L rounded to a multiple of n_matmul=10, n_delay "
        "autotuned per lattice size, eqlt every 10 slices, FP64")


def run_ragged(args, rank, world, local):
    """The ragged mix as parameter groups (one engine each), every sweep of
    all groups one CUDA graph launch on the batch's stream (dqmc_batch): K
    sweeps of every chain, timed with CUDA events on that stream; then the
    end-to-end leg (host state up, one batch sweep, host state down) and one
    profiled eager sweep of every group for the roofline."""
    import torch
    torch.cuda.set_device(local)
    from dqmc_b200 import batch
    from dqmc_b200 import engine
    dicts, desc = _ragged64(args.warmup + args.steps + args.e2e_steps + 3)
    sims = [engine.SimData(d) for d in dicts]
    log(f"generated {len(sims)} chains")
    rb = batch.RaggedBatch(sims, device=local, autotune=True)
    rb.init()
    rb.sweeps(args.warmup)
    barrier(world)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(rb.stream())
    with Clocks(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        rb.sweeps(args.steps, sync=False)
        ev1.record(stream)
        torch.cuda.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3
    barrier(world)
    assert rb.errors() == 0, "device error word set"
    t_max = max_over_ranks(t, world)
    launches = sum(e.launches_per_sweep(True, False) for e in rb.engines) * args.steps
    e2e = e2e_rate(rb.engines, args.e2e_steps, world, lambda: rb.sweeps(1, sync=True))
    # class sums of one eager sweep of every group, each launch timed alone
    profs = [e.profile_sweep(True, False) for e in rb.engines]
    prof = {k: tuple(sum(p[k][i] for p in profs) for i in range(4)) for k in profs[0]}
    rl = roofline(prof, 2 * len(sims), args.workload, fp64_peak(), 1e3 * t_max / args.steps) \
        if rank == 0 else None
    forms = {str(n): f for n, f in rb.update.items()}
    lanes = {str(g): n for g, n in rb.lanes.items()}
    rb.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_proc = cpu_procs()
        rate, _, sample = ragged_reference_rate(n_proc, 3)
        cpu = {"value": rate, "unit": METRIC, "cores": n_proc * 2, "kind": "reference",
               "sample": sample}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": len(sims) * args.steps * world / t_max, "unit": METRIC,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "chains_per_gpu": len(sims), "groups": len(rb.groups),
                       "delay_rank": {str(k): v for k, v in rb.delay.items()},
                       "update_form": forms, "lanes": lanes,
                       "timing": "CUDA events on the batch stream around the graph launches "
                                 "(one per sweep of all groups)"},
            "gpu_launches": launches, "e2e": e2e, "roofline": rl,
            "clocks": clk.summary(), "cpu_baseline": cpu,
        }))


GRAD_DESC = ("128 fixed HS field configurations, 8x8 square, t=1, t'=-0.2, U=4, mu=-0.3, "
             "beta=4, dtau=0.1 (L=40); one grad eval = log|det M_up M_dn|, <n>, <docc> and their "
             "gradients in t, t', mu and 128 bond hoppings for one configuration")


def grad_cpu_baseline():
    """the explicit fermion-matrix method on the host: one configuration
    (two 2560 x 2560 inverses per quantity), scaled to grad evals/s"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fermion_matrix as fm
    from dqmc_b200 import grad
    draw = np.random.Generator(np.random.PCG64(SEED))
    fields = draw.integers(0, 2, size=(1, 40, 64)).astype(np.int32)
    m = grad.SquareModel(8, 8, U=4.0, dt=0.1, L=40, fields=fields, n_matmul=8)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(128)])
    K = m.K(theta)
    t0 = time.perf_counter()
    fm.logdet_grad(K, m.dK, m.U, m.dt, m.L, fields[0])
    fm.obs_grad(K, m.dK, m.U, m.dt, m.L, fields[0])
    tc = time.perf_counter() - t0
    return {"value": 1.0 / tc, "unit": "grad evals/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": f"one configuration with the explicit N L x N L fermion matrices "
                      f"(numpy/OpenBLAS, {os.cpu_count()} host threads): log-det, <n>, <docc> "
                      f"and their 131-parameter gradients, {tc:.1f} s"}


def run_grad(args, rank, world, local):
    """Gradient evaluations at fixed fields: 128 field configurations
    (uniform +-1 from the seed) of the 8x8 model, t=1, t'=-0.2, U=4,
    mu=-0.3, beta=4, dtau=0.1 (L=40).  A step evaluates, for every
    configuration, log |det M_up M_dn|, <n> and <docc> and their gradients
    with respect to t, t', mu and the 128 bond hoppings (131 parameters),
    through the public Python API (host arrays in, host arrays out)."""
    import torch
    torch.cuda.set_device(local)
    from dqmc_b200 import grad, replicas
    n_cfg = 128
    blk = replicas.shard(n_cfg * world, rank, world)
    draw = np.random.Generator(np.random.PCG64(SEED + blk.start))
    fields = draw.integers(0, 2, size=(len(blk), 40, 64)).astype(np.int32)
    m = grad.SquareModel(8, 8, U=4.0, dt=0.1, L=40, fields=fields, n_matmul=8, device=local)
    theta = np.concatenate([[1.0, -0.2, -0.3], np.zeros(128)])
    for _ in range(args.warmup):
        m.evaluate(theta)
        m.evaluate_obs(theta)
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            m.evaluate(theta)
            m.evaluate_obs(theta)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
    barrier(world)
    t_max = max_over_ranks(t, world)
    # one evaluation of each kind again, with CUDA events around every
    # recorded launch and the kernels counted (outside the timed region)
    eng = m.engine(m.K(theta))
    p_ld, n_ld = eng.profile_grad("logdet")
    p_ob, n_ob = eng.profile_grad("obs")
    prof = {k: tuple(a + b for a, b in zip(p_ld[k], p_ob[k])) for k in p_ld}
    rl = None
    if rank == 0:
        rl = roofline(prof, 2 * len(blk), args.workload, fp64_peak(), 1e3 * t_max / args.steps)
        rl["launches_per_step"] = {"logdet_grad": n_ld, "obs_grad": n_ob}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = grad_cpu_baseline()
    value = n_cfg * args.steps * world / t_max
    h2d = fields.nbytes + theta.nbytes
    d2h = n_cfg * (3 + 3 * 131) * 8
    if rank == 0:
        print(json.dumps({
            "metric": "grad evals/s", "value": value,
            "unit": "grad evals/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": GRAD_DESC,
                       "timing": "host clock around the complete evaluations through the public "
                                 "API (host fields and parameters in, host values and gradients "
                                 "out)"},
            "gpu_launches": (n_ld + n_ob) * args.steps,
            "e2e": {"value": value, "unit": "grad evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "the value itself is measured end to end on the host clock"},
            "roofline": rl, "clocks": clk.summary(), "cpu_baseline": cpu,
        }))


def launch_check(rank, world):
    """The multi-rank plumbing alone (used by the CPU tests): every rank
    joins, the maximum over ranks is taken, rank 0 reports the world."""
    m = max_over_ranks(float(rank), world)
    barrier(world)
    if rank == 0:
        print(json.dumps({"n_gpus": world, "max_rank": m}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chains", type=int, default=0, help="chains per GPU (0: the workload's)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="batch256",
                    choices=sorted(WORKLOADS) + ["ragged64", "grad128"],
                    help="batch256: the headline (default); the others print their own line")
    ap.add_argument("--launch-check", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    rank, world, local = dist_setup()
    try:
        if args.launch_check:
            launch_check(rank, world)
        elif args.impl == "reference":
            run_reference_arm(args, rank, world)
        elif args.workload == "grad128":
            run_grad(args, rank, world, local)
        elif args.workload == "ragged64":
            run_ragged(args, rank, world, local)
        else:
            run_engine_workload(args, rank, world, local)
    finally:
        dist_done(world)


if __name__ == "__main__":
    main()
