"""GPU parity at the shapes the benchmark reports, against the oracle.

The headline workload is many chains of the 12x12 model at L = 120,
n_matmul = 10 (F = 12 clusters), n_delay = 16, run in several lanes; the
other workload lines are the 8x8 model with unequal-time measurements and
the complex 10x10 model with one flux quantum.  Each test builds chains of
exactly that shape (own RNG streams, as the benchmark makes them), runs two
sweeps with measurements on the GPU and in the oracle, and requires:

* HS fields and RNG state bit-exact (the sweep of src/dqmc.c:247-386);
* the equal-time G of every chain within 1e-10 (max abs) of the oracle's.
  Where the two FP64 results differ by more, both are judged against the
  quad-precision G of the same fields (oracle/exact_g.c): the engine's
  error may be at most twice the oracle's, which follows the reference's
  LAPACK path.  At U = 6 and beta = 8 (the 8x8 shape) the oracle itself is
  4e-9 .. 1e-8 away from the quad G (the engine 4.6e-9 where the oracle is
  4.1e-9): no FP64 computation of this stabilisation reaches 1e-10 there,
  and the two differ by rounding only;
* the accumulated equal-time and unequal-time measurements within 1e-9
  relative of the oracle's (1e-8 where the G of the two differ by more
  than 1e-10, as at U = 6).
"""
import os

import numpy as np
import pytest

from oracle_ctl import Sim, exact_g

pytestmark = pytest.mark.gpu

G_TOL = 1e-10
MEAS_RTOL = 1e-9


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import engine, lib
    lib.load()
    return engine


def _chains(n, seed, **kw):
    """n sim dicts of one parameter set, chain c on the master stream of
    `seed` jumped c times (as the benchmark and create_batch make them)."""
    from dqmc_b200 import gen, replicas
    rngs = replicas.chain_streams(seed, range(n))
    base = gen.make_sim(init_rng=rngs[0], **kw)
    N, L = int(base["params/N"]), int(base["params/L"])
    out = [base]
    for r in rngs[1:]:
        hs, rr = gen.initial_hs(r, L, N)
        d = dict(base)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rr, hs
        out.append(d)
    return out


def _check_vs_oracle(eng, dicts, n_sweeps, lanes, tmp_path, monkeypatch):
    from dqmc_b200 import simfile
    monkeypatch.setenv("DQMC_LANES", str(lanes))
    sims = [eng.SimData(d) for d in dicts]
    e = eng.Engine(sims)
    assert e.lanes() == lanes
    e.init()
    e.sweeps(n_sweeps)
    e.pull()
    assert e.errors() == 0
    for c, d in enumerate(dicts):
        path = str(tmp_path / f"chain{c}.h5")
        simfile.write(path, d)
        o = Sim(path)
        gu_o, gd_o, ph_o = o.run(stop_sweep=n_sweeps)
        s = sims[c]
        assert np.array_equal(s.hs, o.hs), f"chain {c}: HS fields differ"
        assert np.array_equal(s.rng, o.rng), f"chain {c}: RNG state differs"
        gu, gd, ph = e.g(c)
        err = max(np.max(np.abs(gu - gu_o)), np.max(np.abs(gd - gd_o)))
        meas_rtol = MEAS_RTOL
        if err >= G_TOL:
            gu_x, gd_x = exact_g(o, 0), exact_g(o, 1)
            e_eng = max(np.max(np.abs(gu - gu_x)), np.max(np.abs(gd - gd_x)))
            e_orc = max(np.max(np.abs(gu_o - gu_x)), np.max(np.abs(gd_o - gd_x)))
            assert e_eng <= 2 * max(G_TOL, e_orc), (
                f"chain {c}: engine {e_eng:.3e} from the quad-precision G, oracle {e_orc:.3e}")
            meas_rtol = 10 * MEAS_RTOL
        assert abs(ph - ph_o) < 1e-12
        m = s.measurements()
        groups = [("meas_eqlt/", o.eq, o.eq_sign, s.eq_n, o.eq_n)]
        if s.p["period_uneqlt"] > 0:
            groups.append(("meas_uneqlt/", o.ue, o.ue_sign, s.ue_n, o.ue_n))
        for pre, ref, sign, n_mine, n_ref in groups:
            assert n_mine == int(n_ref[0]) and n_mine > 0, pre + "n_sample"
            np.testing.assert_allclose(np.asarray(m[pre + "sign"]).reshape(-1), sign.reshape(-1),
                                       rtol=meas_rtol, err_msg=pre + "sign")
            for k, r in ref.items():
                if pre + k not in m:
                    continue
                v = np.asarray(m[pre + k]).reshape(-1)
                r = r.reshape(-1)
                scale = max(np.max(np.abs(r)), 1.0)
                np.testing.assert_allclose(v, r, rtol=meas_rtol, atol=meas_rtol * scale,
                                           err_msg=f"chain {c}: {pre + k}")
    e.close()


def test_headline_shape_in_lanes(eng, tmp_path, monkeypatch):
    """12x12 (N = 144), U = 4, mu = -1, dtau = 0.05, L = 120, n_matmul = 10,
    n_delay = 16, eqlt every 8 slices: four chains in two lanes, 2 sweeps."""
    dicts = _chains(4, 1000, Nx=12, Ny=12, U=4.0, mu=-1.0, dt=0.05, L=120, n_matmul=10,
                    n_delay=16, period_eqlt=8, n_sweep_warm=0, n_sweep_meas=2)
    _check_vs_oracle(eng, dicts, 2, 2, tmp_path, monkeypatch)


def test_uneqlt_8x8_shape(eng, tmp_path, monkeypatch):
    """8x8, t' = -0.25, U = 6, mu = -0.5, dtau = 0.1, L = 80, n_matmul = 8,
    n_delay = 16, eqlt every 8 slices and unequal-time every sweep (the
    benchmark's every 4, shortened to fit two sweeps)."""
    dicts = _chains(2, 1000, Nx=8, Ny=8, tp=-0.25, U=6.0, mu=-0.5, dt=0.1, L=80, n_matmul=8,
                    n_delay=16, period_eqlt=8, period_uneqlt=1, n_sweep_warm=0, n_sweep_meas=2)
    _check_vs_oracle(eng, dicts, 2, 1, tmp_path, monkeypatch)


def test_complex_flux_10x10_shape(eng, tmp_path, monkeypatch):
    """10x10 with one flux quantum (complex128), U = 4, mu = 0, dtau = 0.1,
    L = 50, n_matmul = 5, eqlt every 5 slices, unequal-time with the bond
    (current-current) correlators every sweep: two chains in two lanes."""
    dicts = _chains(2, 1000, Nx=10, Ny=10, U=4.0, mu=0.0, dt=0.1, L=50, n_matmul=5, n_delay=16,
                    nflux=1, period_eqlt=5, period_uneqlt=1, meas_bond_corr=1, n_sweep_warm=0,
                    n_sweep_meas=2)
    _check_vs_oracle(eng, dicts, 2, 2, tmp_path, monkeypatch)
