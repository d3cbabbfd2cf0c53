"""Long-run statistical parity with the reference's own build.

Benchmark configuration 1 in full (4x4, U = 4, beta = 4, dtau = 0.1, L = 40,
n_matmul = 5, n_delay = 8, 100 warm-up + 400 measured sweeps, equal-time
measurements every 8 slices) for 8 chains, and a shortened configuration 2
(8x8, t' = -0.25, U = 6, mu = -0.5, L = 80, n_matmul = 8, n_delay = 16,
unequal-time every 4 sweeps; 20 + 40 sweeps) for 4 chains:

* the GPU engine is stepped one sweep at a time beside the oracle; the first
  sweep at which any chain's HS fields differ is reported (None: never);
* the reference's own C build (oracle/_ref/dqmc_1_{r}, src/*.c compiled
  against OpenBLAS) runs the same files to the end;
* every sign-weighted observable (the ratios <s O> / <s>) is compared by a
  jackknife over the chains as bins (the estimator of the reference's
  util/util.py:31-46): engine and reference agree within two standard
  errors; while no divergence occurred the final fields and RNG states are
  identical too, and the observables differ only by rounding (the summary
  reports the largest difference over sigma, which for observables whose
  spread across chains is itself at the rounding level is of order one,
  and the largest difference relative to the largest entry of its
  dataset).

The summary goes to stdout and, when DQMC_PARITY_OUT names a file, there as
JSON.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle_ctl import Sim

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import engine, lib
    lib.load()
    return engine


def jackknife(s, sx):
    """Jackknife estimate and standard error of sum(sx) / sum(s) over bins
    (first axis): leave-one-bin-out ratios r_j, estimate n r - (n-1) mean(r_j),
    error sqrt((n-1) var(r_j))."""
    n = s.shape[0]
    S, SX = s.sum(0), sx.sum(0)
    r_all = (SX.T / S.T).T.real
    r_jk = ((SX - sx).T / (S - s).T).T.real
    m = r_jk.mean(0)
    return n * r_all - (n - 1) * m, np.sqrt((n - 1) * ((r_jk - m) ** 2).mean(0))


def _run_reference(paths, cplx):
    exe = os.path.join(REF, "dqmc_1_c" if cplx else "dqmc_1_r")
    if not os.path.exists(exe):
        pytest.fail(f"reference build missing: {exe} (make -C oracle ref)")
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="2")
    procs = [subprocess.Popen([exe, "-l", p + ".log", p], env=env, stdout=subprocess.DEVNULL,
                              stderr=subprocess.DEVNULL) for p in paths]
    assert [p.wait(timeout=1200) for p in procs] == [0] * len(paths)


def _long_run(eng, tmp_path, monkeypatch, n_chain, seed, **kw):
    from dqmc_b200 import gen
    monkeypatch.chdir(tmp_path)
    paths = [str(tmp_path / p) for p in gen.create_batch(Nfiles=n_chain, prefix="lr", seed=seed,
                                                         **kw)]
    sims = [eng.SimData.read(p) for p in paths]
    oracles = [Sim(p) for p in paths]
    n_sweep = sims[0].p["n_sweep"]
    e = eng.Engine(sims)
    e.init()
    first_div = None
    hs = np.zeros((n_chain, sims[0].L * sims[0].N), np.int32)
    rng = np.zeros((n_chain, 17), np.uint64)
    for k in range(n_sweep):
        e.sweeps(1)
        if first_div is not None:
            continue
        e.get_chains(rng, hs, None, None)
        for c, o in enumerate(oracles):
            o.run(stop_sweep=k + 1)
            if not np.array_equal(hs[c], o.hs) or not np.array_equal(rng[c], o.rng):
                first_div = k + 1
                break
    e.pull()
    assert e.errors() == 0
    e.close()
    # neither the engine nor the oracle wrote the files: the reference build
    # starts from the same initial state
    _run_reference(paths, sims[0].cplx)
    refs = [eng.SimData.read(p) for p in paths]
    return sims, refs, first_div


def _compare(sims, refs, first_div, groups, worst_rel):
    worst = 0.0
    for grp in groups:
        mine, ref = [], []
        for s, r in zip(sims, refs):
            mine.append(s.measurements())
            ref.append(r.measurements())
        sign_m = np.stack([np.asarray(m[grp + "sign"]).reshape(1) for m in mine])
        sign_r = np.stack([np.asarray(m[grp + "sign"]).reshape(1) for m in ref])
        for key in mine[0]:
            if not key.startswith(grp) or key.endswith(("sign", "n_sample")):
                continue
            xm = np.stack([np.asarray(m[key]).reshape(-1) for m in mine])
            xr = np.stack([np.asarray(m[key]).reshape(-1) for m in ref])
            mu_m, err_m = jackknife(sign_m, xm)
            mu_r, err_r = jackknife(sign_r, xr)
            err = np.maximum(err_m, err_r)
            diff = np.abs(mu_m - mu_r)
            ok = diff <= 2.0 * err + 1e-9 * np.maximum(1.0, np.abs(mu_r))
            assert np.all(ok), f"{key}: engine and reference differ beyond 2 sigma"
            scale = np.where(err > 0, err, 1.0)
            worst = max(worst, float(np.max(diff / scale)))
            # relative to the dataset's largest entry (entries near zero
            # would make a per-entry ratio meaningless)
            worst_rel[0] = max(worst_rel[0],
                               float(np.max(diff) / max(np.max(np.abs(mu_r)), 1e-300)))
    if first_div is None:
        for s, r in zip(sims, refs):
            assert np.array_equal(s.hs, r.hs)
            assert np.array_equal(s.rng, r.rng)
    return worst


def _report(name, first_div, n_sweep, worst, worst_rel):
    line = {"case": name, "sweeps": n_sweep, "first_hs_divergence_sweep": first_div,
            "max_abs_diff_over_sigma": worst, "max_rel_diff": worst_rel[0]}
    print(json.dumps(line))
    out = os.environ.get("DQMC_PARITY_OUT")
    if out:
        out = os.path.join(ROOT, out) if not os.path.isabs(out) else out
        with open(out, "a") as f:
            f.write(json.dumps(line) + "\n")


def test_config1_full_run(eng, tmp_path, monkeypatch):
    sims, refs, div = _long_run(eng, tmp_path, monkeypatch, 8, 4242, Nx=4, Ny=4, U=4.0, mu=0.0,
                                tp=0.0, dt=0.1, L=40, n_matmul=5, n_delay=8, period_eqlt=8,
                                n_sweep_warm=100, n_sweep_meas=400)
    rel = [0.0]
    worst = _compare(sims, refs, div, ["meas_eqlt/"], rel)
    _report("config 1: 8 chains 4x4 L=40, 100+400 sweeps", div, 500, worst, rel)


def test_config2_short_run_uneqlt(eng, tmp_path, monkeypatch):
    sims, refs, div = _long_run(eng, tmp_path, monkeypatch, 4, 4343, Nx=8, Ny=8, U=6.0, mu=-0.5,
                                tp=-0.25, dt=0.1, L=80, n_matmul=8, n_delay=16, period_eqlt=8,
                                period_uneqlt=4, n_sweep_warm=20, n_sweep_meas=40)
    rel = [0.0]
    worst = _compare(sims, refs, div, ["meas_eqlt/", "meas_uneqlt/"], rel)
    _report("config 2: 4 chains 8x8 L=80, 20+40 sweeps, uneqlt every 4", div, 60, worst, rel)
