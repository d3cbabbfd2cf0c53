"""Ragged batches on the GPU: chains of different lattices, U and beta in
one batch, each group on its own stream, against the oracle chain by chain;
the C drop-in's batch entry on files of different lattices against the
single-file entry."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle_ctl import Sim

pytestmark = pytest.mark.gpu

MEAS_RTOL = 1e-9


@pytest.fixture(scope="module")
def mods():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import batch, engine, gen, lib, simfile
    lib.load()
    return batch, engine, gen, simfile


def _ragged(gen, n, seed, **kw):
    return gen.make_ragged(n, seed, sides=(4, 6), U=(2.0, 6.0), beta=(0.8, 1.6), dt=0.1,
                           n_matmul=4, n_delay=4, n_sweep_warm=1, n_sweep_meas=2, **kw)


def test_ragged_batch_matches_oracle(mods, tmp_path):
    batch, engine, gen, simfile = mods
    dicts = _ragged(gen, 7, 11)
    sims = [engine.SimData(d) for d in dicts]
    rb = batch.RaggedBatch(sims)
    assert len(rb.groups) >= 3
    rb.init()
    rb.sweeps(sims[0].p["n_sweep"])
    rb.pull()
    assert rb.errors() == 0
    for c, (d, s) in enumerate(zip(dicts, sims)):
        path = str(tmp_path / f"c{c}.h5")
        simfile.write(path, d)
        o = Sim(path)
        o.run()
        assert np.array_equal(s.hs, o.hs), c
        assert np.array_equal(s.rng, o.rng), c
        m = s.measurements()
        for k, r in o.eq.items():
            np.testing.assert_allclose(np.asarray(m["meas_eqlt/" + k]).reshape(-1), r.reshape(-1),
                                       rtol=MEAS_RTOL, atol=MEAS_RTOL * max(1, np.abs(r).max()),
                                       err_msg=f"chain {c} {k}")
    rb.close()


def test_batch_graph_matches_separate_engines(mods):
    """The ragged batch's one-graph sweeps (dqmc_batch_sweeps, groups of
    different lattices and L, uneven sweep kinds: warm-up then measuring)
    against the same groups swept engine by engine: fields, RNG state and
    accumulators bit-identical; also after fields are replaced in the middle
    of the run (the re-initialisation runs before the graph)."""
    batch, engine, gen, simfile = mods
    dicts = _ragged(gen, 7, 21)
    a = [engine.SimData(d) for d in dicts]
    b = [engine.SimData(d) for d in dicts]
    rb = batch.RaggedBatch(a)
    rb.init()
    rb.sweeps(1)
    rb.pull()
    for e in rb.engines:      # replace the fields: every group re-initialises
        e.push()
    rb.sweeps(a[0].p["n_sweep"])
    rb.pull()
    assert rb.errors() == 0
    engines = [engine.Engine([b[i] for i in idx]) for idx in rb.groups]
    rb.close()
    for e in engines:
        e.init()
        e.sweeps(1)
        e.pull()
        e.push()
        e.sweeps(b[0].p["n_sweep"])
        e.pull()
        assert e.errors() == 0
        e.close()
    for c, (x, y) in enumerate(zip(a, b)):
        assert x.sweep == y.sweep == x.p["n_sweep"], c
        assert np.array_equal(x.hs, y.hs), c
        assert np.array_equal(x.rng, y.rng), c
        assert np.array_equal(x.eq_acc, y.eq_acc), c


def test_autotune_lanes_picks_a_candidate_and_keeps_results(mods):
    """The lane tuner returns one of its candidates, and an engine in the
    chosen lanes gives bit-identical results to one lane."""
    batch, engine, gen, simfile = mods
    from dqmc_b200 import replicas
    rngs = replicas.chain_streams(5, range(8))
    base = gen.make_sim(init_rng=rngs[0], Nx=4, Ny=4, U=4.0, dt=0.1, L=20, n_matmul=5,
                        n_delay=4, period_eqlt=5, n_sweep_warm=0, n_sweep_meas=3)
    dicts = [base]
    for r in rngs[1:]:
        hs, rr = gen.initial_hs(r, 20, 16)
        d = dict(base)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rr, hs
        dicts.append(d)
    sims = [engine.SimData(d) for d in dicts]
    n = batch.autotune_lanes(sims, candidates=(1, 2, 4))
    assert n in (1, 2, 4)
    runs = []
    for lanes in (1, n):
        ss = [s.clone() for s in sims]
        e = engine.Engine(ss, lanes=lanes)
        assert e.lanes() == lanes
        e.init()
        e.sweeps(3)
        e.pull()
        e.close()
        runs.append(ss)
    for a, b in zip(*runs):
        assert np.array_equal(a.hs, b.hs) and np.array_equal(a.eq_acc, b.eq_acc)


def test_autotuned_ragged_batch_runs(mods):
    batch, engine, gen, simfile = mods
    sims = [engine.SimData(d) for d in _ragged(gen, 5, 12)]
    rb = batch.RaggedBatch(sims, autotune=True, candidates=(2, 4, 8))
    assert set(rb.delay) == {s.N for s in sims}
    assert all(v in (2, 4, 8) for v in rb.delay.values())
    assert set(rb.update) == {s.N for s in sims}
    for g, idx in enumerate(rb.groups):
        assert rb.engines[g].update_form == rb.update[sims[idx[0]].N]
    rb.init()
    rb.sweeps(2)
    rb.pull()
    assert rb.errors() == 0
    for s in sims:
        assert np.all(np.isfinite(s.eq_acc))
    rb.close()


def test_wrapper_batch_ragged_equals_single(mods, tmp_path):
    batch, engine, gen, simfile = mods
    from dqmc_b200 import lib
    h = lib.load()
    dicts = _ragged(gen, 4, 13)
    single, multi = [], []
    for c, d in enumerate(dicts):
        for tag, lst in (("s", single), ("m", multi)):
            path = str(tmp_path / f"{tag}{c}.h5")
            simfile.write(path, d)
            lst.append(path)
    for p in single:
        assert h.dqmc_wrapper(p.encode(), str(tmp_path / "s.log").encode(), 0, False, False) == 0
    arr = (C.c_char_p * len(multi))(*[p.encode() for p in multi])
    st = (C.c_int * len(multi))()
    assert h.dqmc_wrapper_batch(len(multi), arr, str(tmp_path / "m.log").encode(), 0, False, st) == 0
    assert list(st) == [0] * len(multi)
    for a, b in zip(single, multi):
        da, db = simfile.read(a), simfile.read(b)
        for k in ("state/rng", "state/hs", "state/sweep", "meas_eqlt/n_sample"):
            assert np.array_equal(np.asarray(da[k]), np.asarray(db[k])), k
        for k in da:
            if k.startswith("meas_eqlt/"):
                np.testing.assert_allclose(np.asarray(db[k]), np.asarray(da[k]), rtol=1e-12,
                                           atol=1e-12, err_msg=k)


def _group(gen, n, **kw):
    """n chains of one parameter set, chain c from the master stream jumped c times"""
    from dqmc_b200 import replicas
    rngs = replicas.chain_streams(5, range(n))
    d0 = gen.make_sim(init_rng=rngs[0], **kw)
    out = [d0]
    for r in rngs[1:]:
        hs, rng = gen.initial_hs(r, kw["L"], kw["Nx"] * kw["Ny"])
        d = dict(d0)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rng, hs
        out.append(d)
    return out


def _run_lanes(engine, dicts, lanes, monkeypatch):
    monkeypatch.setenv("DQMC_LANES", str(lanes))
    sims = [engine.SimData(dict(d)) for d in dicts]
    e = engine.Engine(sims)
    e.init()
    e.sweeps(sims[0].p["n_sweep"])
    e.pull()
    assert e.errors() == 0
    gs = [e.g(c) for c in range(len(sims))]
    e.close()
    return sims, gs


def test_lanes_are_bit_identical(mods, monkeypatch):
    """An engine split into lanes (sub-batches on their own streams, forked
    from and joined to the engine's stream) gives every chain exactly the
    state and measurements of the one-lane engine; 7 chains in 3 lanes of
    3, 2 and 2, with unequal-time measurements."""
    batch, engine, gen, simfile = mods
    dicts = _group(gen, 7, Nx=4, Ny=4, U=4.0, dt=0.1, L=16, n_matmul=4, period_eqlt=4,
                   period_uneqlt=1, n_delay=4, n_sweep_warm=1, n_sweep_meas=2)
    one, g1 = _run_lanes(engine, dicts, 1, monkeypatch)
    three, g3 = _run_lanes(engine, dicts, 3, monkeypatch)
    for c, (a, b) in enumerate(zip(one, three)):
        assert np.array_equal(a.hs, b.hs), c
        assert np.array_equal(a.rng, b.rng), c
        assert np.array_equal(a.eq_acc, b.eq_acc), c
        assert np.array_equal(a.ue_acc, b.ue_acc), c
        for x, y in zip(g1[c], g3[c]):
            assert np.array_equal(x, y), c


def test_lanes_gradients_match(mods, monkeypatch):
    """logdet_grad and obs_grad of a 3-lane engine (lanes in parallel host
    threads) against the one-lane engine, configuration by configuration."""
    batch, engine, gen, simfile = mods
    dicts = _group(gen, 5, Nx=4, Ny=4, U=4.0, dt=0.1, L=8, n_matmul=4, period_eqlt=4,
                   n_sweep_warm=0, n_sweep_meas=1)
    out = {}
    for lanes in (1, 3):
        monkeypatch.setenv("DQMC_LANES", str(lanes))
        e = engine.Engine([engine.SimData(dict(d)) for d in dicts])
        out[lanes] = (e.logdet_grad(), e.obs_grad())
        e.close()
    (ld1, S1), (o1, Z1) = out[1]
    (ld3, S3), (o3, Z3) = out[3]
    assert np.array_equal(ld1, ld3) and np.array_equal(S1, S3)
    assert np.array_equal(o1, o3) and np.array_equal(Z1, Z3)


def test_batched_state_calls_match_per_chain(mods, monkeypatch):
    """dqmc_engine_set_chains / get_chains (every chain in one call, lanes
    split across) against dqmc_engine_set_chain / get_chain / get_acc chain
    by chain: the same state in, bit-identical state and accumulators out."""
    batch, engine, gen, simfile = mods
    monkeypatch.setenv("DQMC_LANES", "2")
    dicts = _group(gen, 5, Nx=4, Ny=4, U=4.0, dt=0.1, L=16, n_matmul=4, period_eqlt=4,
                   n_delay=4, n_sweep_warm=1, n_sweep_meas=4)
    one = [engine.SimData(dict(d)) for d in dicts]
    e1 = engine.Engine(one)
    e1.init()
    e1.sweeps(2)
    e1.pull()
    # a second engine takes that state in one call and both run two more sweeps
    two = [s.clone() for s in one]
    e2 = engine.Engine(two)
    assert e2.lanes() == 2
    el, dl, rg, hs = e1.state_arrays()
    e2.set_chains(el, dl, rg, hs, one[0].sweep)
    for c, s in enumerate(one):
        from dqmc_b200 import lib
        lib.check(e1.lib.dqmc_engine_set_chain(e1.h, c, s.exp_lambda.ctypes.data, s.del_.ctypes.data,
                                               s.rng.ctypes.data, s.hs.ctypes.data, s.sweep),
                  "set_chain")
        lib.check(e1.lib.dqmc_engine_set_acc(e1.h, c, 0, None, 0, None), "set_acc")
        e2.lib.dqmc_engine_set_acc(e2.h, c, 0, None, 0, None)
    e1.sweeps(2)
    e2.sweeps(2)
    e1.pull()
    n = len(one)
    rg2, hs2 = np.zeros_like(rg), np.zeros_like(hs)
    eqn2 = np.zeros(n, np.int32)
    eq2 = np.zeros((n,) + one[0].eq_acc.shape, one[0].eq_acc.dtype)
    sw = e2.get_chains(rg2, hs2, eqn2, eq2)
    assert sw == one[0].sweep
    for c, s in enumerate(one):
        assert np.array_equal(rg2[c], s.rng), c
        assert np.array_equal(hs2[c], s.hs), c
        assert eqn2[c] == s.eq_n, c
        assert np.array_equal(eq2[c], s.eq_acc), c
    assert e1.errors() == 0 and e2.errors() == 0
    e1.close()
    e2.close()


def test_update_form_option_and_autotune(mods):
    """Engine(update=...) selects the delayed update's form (G on chip in a
    two-CTA cluster, or in device memory), both give bit-identical chains,
    the tuner returns a form the chains can take, and a lattice whose G does
    not fit on chip offers only the device-memory form."""
    batch, engine, gen, simfile = mods
    from dqmc_b200 import replicas
    rngs = replicas.chain_streams(9, range(4))
    base = gen.make_sim(init_rng=rngs[0], Nx=6, Ny=6, U=4.0, dt=0.1, L=20, n_matmul=5,
                        n_delay=8, period_eqlt=5, n_sweep_warm=0, n_sweep_meas=3)
    dicts = [base]
    for r in rngs[1:]:
        hs, rr = gen.initial_hs(r, 20, 36)
        d = dict(base)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rr, hs
        dicts.append(d)
    sims = [engine.SimData(d) for d in dicts]
    assert batch.update_forms(sims) == ["global", "cluster"]
    runs = []
    for form in ("global", "cluster"):
        ss = [s.clone() for s in sims]
        e = engine.Engine(ss, update=form)
        assert e.update_form == form
        e.init()
        e.sweeps(3)
        e.pull()
        assert e.errors() == 0
        e.close()
        runs.append(ss)
    for a, b in zip(*runs):
        assert np.array_equal(a.hs, b.hs) and np.array_equal(a.rng, b.rng)
        assert np.array_equal(a.eq_acc, b.eq_acc)
    assert batch.autotune_update(sims) in ("global", "cluster")
    big = engine.SimData(gen.make_sim(Nx=16, Ny=16, U=4.0, dt=0.1, L=10, n_matmul=5, n_delay=8,
                                      period_eqlt=5, n_sweep_warm=0, n_sweep_meas=1))
    assert batch.update_forms([big]) == ["global"]
