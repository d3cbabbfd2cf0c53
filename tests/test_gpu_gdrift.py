"""The G drift self-check (dqmc_engine_check_g / dqmc_engine_g_drift), the
runtime form of the reference's compile-time CHECK_G_WRP
(src/dqmc.c:15-16, 277-287, 339-343): at every recalculation the previous
slice's G wrapped once more against the recalculated G.

* the check leaves the sweep unchanged: HS fields, RNG state, G and every
  accumulator bit-identical with and without it (a golden case and the
  12x12 benchmark shape in two lanes);
* it counts one check per recalculation (F per sweep) and reports a drift
  that is finite, positive (the two G differ by rounding) and small (the
  wrap over n_matmul slices loses little at these well-conditioned shapes);
* dqmc_wrapper writes the drift to its log when DQMC_CHECK_G is set."""
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import engine, lib
    lib.load()
    return engine


def _headline_dicts(n):
    from dqmc_b200 import gen, replicas
    rngs = replicas.chain_streams(2024, range(n))
    base = gen.make_sim(init_rng=rngs[0], Nx=12, Ny=12, U=4.0, mu=-1.0, dt=0.05, L=120,
                        n_matmul=10, n_delay=16, period_eqlt=8, n_sweep_warm=0, n_sweep_meas=2)
    N, L = int(base["params/N"]), int(base["params/L"])
    out = [base]
    for r in rngs[1:]:
        hs, rr = gen.initial_hs(r, L, N)
        d = dict(base)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rr, hs
        out.append(d)
    return out


def _run(eng, dicts, sweeps, check):
    sims = [eng.SimData(d) for d in dicts]
    e = eng.Engine(sims)
    if check:
        e.check_g(True)
    e.init()
    e.sweeps(sweeps)
    e.pull()
    assert e.errors() == 0
    drift = e.g_drift() if check else None
    gs = [e.g(c) for c in range(len(sims))]
    e.close()
    return sims, gs, drift


@pytest.mark.parametrize("case", ["golden", "headline"])
def test_check_leaves_the_sweep_unchanged(eng, golden, case, monkeypatch):
    from dqmc_b200 import simfile
    if case == "golden":
        d = simfile.read(os.path.join(golden, "c1_small", "sim_0.h5"))
        dicts, sweeps = [d], 3
    else:
        monkeypatch.setenv("DQMC_LANES", "2")
        dicts, sweeps = _headline_dicts(4), 2
    a, ga, _ = _run(eng, dicts, sweeps, False)
    b, gb, (mx, mean, cnt) = _run(eng, dicts, sweeps, True)
    for sa, sb in zip(a, b):
        assert np.array_equal(sa.hs, sb.hs)
        assert np.array_equal(sa.rng, sb.rng)
        assert np.array_equal(sa.eq_acc, sb.eq_acc)
    for x, y in zip(ga, gb):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    F = a[0].p["L"] // a[0].p["n_matmul"]
    done = b[0].sweep - int(np.asarray(dicts[0]["state/sweep"]).reshape(-1)[0])
    assert done > 0 and cnt == F * done
    assert np.all(np.isfinite(mx)) and np.all(mx > 0) and np.all(mx < 1e-8), mx
    assert np.all(mean > 0) and np.all(mean <= mx)


def test_wrapper_logs_the_drift(eng, golden, tmp_path, monkeypatch):
    from dqmc_b200 import lib
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, "c1_small", f), tmp_path)
    monkeypatch.setenv("DQMC_CHECK_G", "1")
    log = tmp_path / "log"
    rc = lib.load().dqmc_wrapper(str(tmp_path / "sim_0.h5").encode(), str(log).encode(), 0,
                                 False, True)
    text = open(log).read()
    assert rc == 0, text
    lines = [ln for ln in text.splitlines() if "g - gwrp" in ln]
    assert len(lines) == 1, text
    mx = float(lines[0].split("max")[1].split()[0])
    assert 0 < mx < 1e-8


@pytest.mark.parametrize("case", ["uneq_small", "cplx_small"])
def test_unequal_time_check(eng, golden, case):
    """The (0, 0) block of G(tau, tau) from the unequal-time path against the
    equal-time G (the reference's CHECK_G_UE): one check per unequal-time
    measurement, a small positive difference, the sweep unchanged."""
    from dqmc_b200 import simfile
    d = simfile.read(os.path.join(golden, case, "sim_0.h5"))
    a, ga, _ = _run(eng, [d], 99, False)
    sims = [eng.SimData(d)]
    e = eng.Engine(sims)
    e.check_g(True)
    e.init()
    e.sweeps(99)
    e.pull()
    assert e.errors() == 0
    mx, mean, cnt = e.g_drift(unequal_time=True)
    gu, gd, _ = e.g(0)
    e.close()
    s = sims[0]
    assert np.array_equal(a[0].hs, s.hs) and np.array_equal(a[0].ue_acc, s.ue_acc)
    assert np.array_equal(ga[0][0], gu) and np.array_equal(ga[0][1], gd)
    assert cnt == s.ue_n > 0
    assert np.all(np.isfinite(mx)) and np.all(mx > 0) and np.all(mx < 1e-8), mx
    assert np.all(mean <= mx)


@pytest.mark.parametrize("case", ["c1_small", "cplx_small", "headline"])
def test_accurate_recalculation_check(eng, golden, case):
    """G from the L single-slice factors with a QR after each (the
    reference's CHECK_G_ACC, calc_eq_g(l, N, L, 1, B, ...)) against the G of
    the cluster chain at every recalculation: one check per recalculation
    beside the wrap check, a small positive difference, the sweep
    unchanged (a golden case, a complex one with flux, and two chains of the
    12x12, L = 120 benchmark shape)."""
    from dqmc_b200 import simfile
    if case == "headline":
        dicts, sweeps = _headline_dicts(2), 2
    else:
        dicts, sweeps = [simfile.read(os.path.join(golden, case, "sim_0.h5"))], 3
    a, ga, _ = _run(eng, dicts, sweeps, False)
    sims = [eng.SimData(d) for d in dicts]
    e = eng.Engine(sims)
    e.check_g(True, accurate=True)
    e.init()
    e.sweeps(sweeps)
    e.pull()
    assert e.errors() == 0
    mx, mean, cnt = e.g_drift(accurate=True)
    _, _, cnt_w = e.g_drift()
    gs = [e.g(c) for c in range(len(sims))]
    e.close()
    for sa, sb in zip(a, sims):
        assert np.array_equal(sa.hs, sb.hs) and np.array_equal(sa.rng, sb.rng)
        assert np.array_equal(sa.eq_acc, sb.eq_acc)
    for x, y in zip(ga, gs):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    F = sims[0].p["L"] // sims[0].p["n_matmul"]
    done = sims[0].sweep - int(np.asarray(dicts[0]["state/sweep"]).reshape(-1)[0])
    assert done > 0 and cnt == cnt_w == F * done
    bound = 1e-7 if case == "headline" else 1e-8
    assert np.all(np.isfinite(mx)) and np.all(mx > 0) and np.all(mx < bound), mx
    assert np.all(mean <= mx)


def test_wrapper_logs_the_accurate_check(eng, golden, tmp_path, monkeypatch):
    from dqmc_b200 import lib
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, "c1_small", f), tmp_path)
    monkeypatch.setenv("DQMC_CHECK_G", "acc")
    log = tmp_path / "log"
    rc = lib.load().dqmc_wrapper(str(tmp_path / "sim_0.h5").encode(), str(log).encode(), 0,
                                 False, True)
    text = open(log).read()
    assert rc == 0, text
    for key in ("g - gwrp", "g - gacc"):
        lines = [ln for ln in text.splitlines() if key in ln]
        assert len(lines) == 1, text
        mx = float(lines[0].split("max")[1].split()[0])
        assert 0 < mx < 1e-8
