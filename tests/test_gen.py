"""The engine's own generator (dqmc_b200/gen.py) against the reference
generator's output (fixtures made by tests/golden/make_golden.py from
util/gen_1band_unified_hub.py): every dataset it writes must have the same
dtype, shape and value; integer and map datasets exactly, matrices to the
last bit or within 1e-15 relative where expm is involved."""
import os

import numpy as np
import pytest

from dqmc_b200 import gen, simfile

CASES = {
    "gen_sq6_tp": dict(seed=1, Nx=6, Ny=6, tp=-0.25, U=6.0, mu=-0.5, dt=0.1, L=20,
                       n_matmul=5, n_delay=8, period_eqlt=5, period_uneqlt=1,
                       meas_bond_corr=1, n_sweep_warm=200, n_sweep_meas=2000),
    "gen_sq4_flux": dict(seed=2, Nx=4, Ny=4, nflux=1, U=4.0, mu=0.0, dt=0.1, L=20,
                         n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_sq6_flux": dict(seed=4, Nx=6, Ny=6, nflux=1, U=4.0, dt=0.1, L=10, n_matmul=5,
                         n_delay=8, period_eqlt=5),
    "gen_sq4_h": dict(seed=9, Nx=4, Ny=6, U=3.0, mu=0.2, h=0.1, dt=0.05, L=20,
                      n_matmul=10, n_delay=8, period_eqlt=10),
    "c1_small": dict(seed=7, Nx=4, Ny=4, U=4.0, mu=0.0, dt=0.1, L=40, n_matmul=5,
                     n_delay=8, period_eqlt=8, n_sweep_warm=10, n_sweep_meas=20),
    "uneq_small": dict(seed=11, Nx=4, Ny=4, tp=-0.25, U=6.0, mu=-0.5, dt=0.1, L=16,
                       n_matmul=4, n_delay=4, period_eqlt=4, period_uneqlt=2,
                       meas_bond_corr=1, n_sweep_warm=4, n_sweep_meas=8),
    "kat_square": dict(seed=1234, n_sweep_warm=20, n_sweep_meas=20),
    **{f"kat_{g}": dict(geometry=g, seed=1234, n_sweep_warm=20, n_sweep_meas=20)
       for g in ("triangular", "honeycomb", "kagome")},
    "gen_tri_flux": dict(geometry="triangular", seed=31, Nx=4, Ny=4, nflux=1, U=4.0, mu=-0.2,
                         dt=0.1, L=10, n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_hc_flux": dict(geometry="honeycomb", seed=32, Nx=3, Ny=3, nflux=1, U=4.0, dt=0.1,
                        L=10, n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_kag_flux": dict(geometry="kagome", seed=33, Nx=3, Ny=3, nflux=2, U=4.0, mu=0.3,
                         dt=0.1, L=10, n_matmul=5, n_delay=8, period_eqlt=5),
}
SKIP = {"metadata/commit", "params_file"}


@pytest.mark.parametrize("case", sorted(CASES))
def test_generator_matches_reference(golden, case):
    ref = simfile.read(os.path.join(golden, case, "sim_0.h5"))
    mine = gen.make_sim(**CASES[case])
    checked = 0
    for k, v in mine.items():
        if k in SKIP or k not in ref:
            continue
        r = ref[k]
        if isinstance(r, str):
            assert v == r, k
            continue
        a = np.asarray(v)
        assert a.dtype == r.dtype, (k, a.dtype, r.dtype)
        assert a.shape == r.shape, (k, a.shape, r.shape)
        if a.dtype.kind in "iu":
            assert np.array_equal(a, r), k
        else:
            np.testing.assert_allclose(a, r, rtol=1e-15, atol=1e-15, err_msg=k)
        checked += 1
    assert checked > 60
    # every dataset the engine reads is present
    for k in ("params/exp_Ku", "params/map_ij", "params/bonds", "params/map_bb", "state/hs",
              "state/rng", "params/del", "params/exp_lambda", "meas_eqlt/g00"):
        assert k in mine


def test_rand_jump_matches_reference(golden):
    ref = np.load(os.path.join(golden, "rng_ref.npz"))
    assert np.array_equal(gen.seed_splitmix64(1234), ref["seeded"])
    assert np.array_equal(gen.rand_jump(ref["seeded"]), ref["jumped"])


def test_create_batch_files(tmp_path):
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        paths = gen.create_batch(Nfiles=3, prefix="b", seed=5, Nx=4, Ny=4, L=10, n_matmul=5,
                                 period_eqlt=5)
        d = [simfile.read(p) for p in paths]
    finally:
        os.chdir(cwd)
    assert not np.array_equal(d[0]["state/hs"], d[1]["state/hs"])
    assert np.array_equal(d[0]["params/exp_Ku"], d[2]["params/exp_Ku"])
    assert np.array_equal(d[1]["state/init_rng"], gen.rand_jump(d[0]["state/init_rng"]))
