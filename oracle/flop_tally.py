"""FLOPs per chain-sweep of the reference build, counted call by call.

Runs the tally variant of the reference CLI (make -C oracle tally:
_ref/dqmc_1_{r,c}_tally, whose BLAS / LAPACK shim adds each call's
LAPACK-standard operation count, ref_glue/flop_tally.c) on one chain of each
bench workload's model, for 1 and for 1 + P measured sweeps; the difference
over P sweeps removes the initial computation of G, and P, the unequal-time
period (at least 2), averages over a whole measurement cycle.  Measurement loops without
BLAS calls count nothing, as in the engine's counters.

    python oracle/flop_tally.py [workload ...]      (default: all of bench.py's
                                                     single-model workloads)

Prints one JSON object: workload -> FLOPs per chain-sweep.  Test-side tool:
it reads the reference sources only through the binaries that
oracle/Makefile built from them.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dqmc-dev_b200"))


def tally(cfg: dict, sweeps: int) -> float:
    from dqmc_b200 import gen
    cplx = cfg.get("nflux", 0) != 0
    exe = os.path.join(ROOT, "oracle", "_ref", "dqmc_1_c_tally" if cplx else "dqmc_1_r_tally")
    if not os.path.exists(exe):
        raise RuntimeError(f"tally build missing: {exe} (make -C oracle tally)")
    with tempfile.TemporaryDirectory() as tmp:
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            (path,) = gen.create_batch(Nfiles=1, prefix="t", seed=1, n_sweep_warm=0,
                                       n_sweep_meas=sweeps, **cfg)
            out = os.path.join(tmp, "flops")
            env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="2",
                       DQ_FLOP_TALLY_OUT=out)
            subprocess.run([exe, "-b", "-l", "t.log", path], env=env, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            with open(out) as f:
                return float(f.read())
        finally:
            os.chdir(cwd)


def per_sweep(cfg: dict) -> float:
    p = max(2, int(cfg.get("period_uneqlt", 0)))
    return (tally(cfg, 1 + p) - tally(cfg, 1)) / p


def main(argv):
    import bench
    names = argv or [k for k in bench.WORKLOADS]
    print(json.dumps({k: per_sweep(bench.WORKLOADS[k]["cfg"]) for k in names}))


if __name__ == "__main__":
    main(sys.argv[1:])
