"""The delayed update with G held in shared memory (k_update_cl, selected
with DQMC_UPDATE=cluster when the engine is created) against the form with
G in device memory (k_update, DQMC_UPDATE=global): both do the arithmetic of
src/updates.c:7-84 in the same order, so fields, RNG states, G and
measurements must be bit-identical, and the fields equal the oracle's."""
import os
import shutil

import numpy as np
import pytest

from oracle_ctl import Sim

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import engine, lib
    lib.load()
    return engine


def _run(eng, dicts, n, monkeypatch, mode):
    if mode:
        monkeypatch.setenv("DQMC_UPDATE", mode)
    else:
        monkeypatch.delenv("DQMC_UPDATE", raising=False)
    sims = [eng.SimData(dict(d)) for d in dicts]
    e = eng.Engine(sims)
    e.init()
    e.sweeps(n)
    e.pull()
    assert e.errors() == 0
    gs = [e.g(c) for c in range(len(sims))]
    e.close()
    return sims, gs


def _cases(golden):
    from dqmc_b200 import gen, simfile
    out = {}
    for case in ("c1_small", "cplx_small"):
        out[case] = [simfile.read(os.path.join(golden, case, "sim_0.h5"))]
    rngs = gen.chain_rngs(77, 2)
    base = gen.make_sim(Nx=12, Ny=12, U=4.0, mu=-1.0, dt=0.05, L=40, n_matmul=10, n_delay=16,
                        period_eqlt=8, n_sweep_warm=0, n_sweep_meas=4, init_rng=rngs[0])
    d2 = dict(base)
    d2["state/hs"], d2["state/rng"] = gen.initial_hs(rngs[1], 40, 144)
    out["sq12"] = [base, d2]
    return out


@pytest.mark.parametrize("case", ["c1_small", "cplx_small", "sq12"])
def test_cluster_update_bit_identical(eng, golden, case, monkeypatch, tmp_path):
    dicts = _cases(golden)[case]
    n = 2
    a, ga = _run(eng, dicts, n, monkeypatch, "global")
    b, gb = _run(eng, dicts, n, monkeypatch, "cluster")
    for c in range(len(dicts)):
        assert np.array_equal(a[c].hs, b[c].hs)
        assert np.array_equal(a[c].rng, b[c].rng)
        assert np.array_equal(a[c].eq_acc, b[c].eq_acc)
        for x, y in zip(ga[c], gb[c]):
            assert np.array_equal(np.asarray(x), np.asarray(y))
    # and the fields are the oracle's
    from dqmc_b200 import simfile
    path = str(tmp_path / "c0.h5")
    if case in ("c1_small", "cplx_small"):
        for f in ("sim_0.h5", "sim.h5.params"):
            shutil.copy(os.path.join(golden, case, f), tmp_path)
        path = str(tmp_path / "sim_0.h5")
    else:
        simfile.write(path, dicts[0])
    o = Sim(path)
    o.run(stop_sweep=n)
    assert np.array_equal(b[0].hs, o.hs)
    assert np.array_equal(b[0].rng, o.rng)
