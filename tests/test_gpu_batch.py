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


def test_autotuned_ragged_batch_runs(mods):
    batch, engine, gen, simfile = mods
    sims = [engine.SimData(d) for d in _ragged(gen, 5, 12)]
    rb = batch.RaggedBatch(sims, autotune=True, candidates=(2, 4, 8))
    assert set(rb.delay) == {s.N for s in sims}
    assert all(v in (2, 4, 8) for v in rb.delay.values())
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
