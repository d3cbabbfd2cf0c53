"""Pins the CPU oracle before anything is compared with it.

* the xorshift1024*/splitmix64/jump RNG against vectors from the reference
  generator's own helpers (util/gen_util_shared.py);
* the reference test suite's known-answer test (test_batch_seed_basic_real,
  test/test_gen_1band_hub_unified.py:119-148): final HS fields after 40 sweeps
  for four geometries must match test/hs_ref.py exactly;
* every state and measurement dataset of the reference's own C build
  (oracle/_ref, outputs committed as ref_out.npz) on the golden cases.
"""
import ctypes as C
import json
import os
import shutil

import numpy as np
import pytest

from oracle_ctl import Sim, oracle_lib

GEOMS = ["square", "triangular", "honeycomb", "kagome"]
CASES = ["c1_small", "uneq_small", "uneq_oddF", "cplx_small", "sq8_small"]


def _copy_case(golden, case, tmp_path):
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, case, f), tmp_path)
    return str(tmp_path / "sim_0.h5")


def test_rng_vectors(golden):
    ref = np.load(os.path.join(golden, "rng_ref.npz"))
    lib = oracle_lib(False)
    rng = np.zeros(17, np.uint64)
    lib.orc_seed_splitmix64(C.c_uint64(1234), C.c_void_p(rng.ctypes.data))
    assert np.array_equal(rng, ref["seeded"])
    draws = np.array([lib.orc_rand_uint(C.c_void_p(rng.ctypes.data)) for _ in range(64)],
                     dtype=np.uint64)
    assert np.array_equal(draws, ref["first_draws"])
    assert np.array_equal(rng, ref["state_after"])
    j = ref["seeded"].copy()
    lib.orc_rand_jump(C.c_void_p(j.ctypes.data))
    assert np.array_equal(j, ref["jumped"])


@pytest.mark.parametrize("geom", GEOMS)
def test_known_answer_hs(golden, geom, tmp_path):
    ref = np.load(os.path.join(golden, "hs_ref.npz"))
    s = Sim(_copy_case(golden, f"kat_{geom}", tmp_path))
    assert np.array_equal(s.hs2d(), ref[f"init_{geom}"])
    s.run()
    assert np.array_equal(s.hs2d(), ref[f"end_{geom}"])


@pytest.mark.parametrize("case", CASES + [f"kat_{g}" for g in GEOMS])
def test_oracle_matches_reference_build(golden, case, tmp_path):
    s = Sim(_copy_case(golden, case, tmp_path))
    s.run()
    ref = np.load(os.path.join(golden, case, "ref_out.npz"))
    assert np.array_equal(s.hs, ref["state__hs"].reshape(-1))
    assert np.array_equal(s.rng, ref["state__rng"])
    assert s.sweep[0] == ref["state__sweep"]
    assert s.eq_n[0] == ref["meas_eqlt__n_sample"]
    np.testing.assert_allclose(s.eq_sign, ref["meas_eqlt__sign"].reshape(-1), rtol=1e-12)
    for k, v in s.eq.items():
        np.testing.assert_allclose(v, ref[f"meas_eqlt__{k}"].reshape(-1), rtol=1e-9,
                                   atol=1e-10, err_msg=k)
    if s.p["period_uneqlt"] > 0:
        assert s.ue_n[0] == ref["meas_uneqlt__n_sample"]
        for k, v in s.ue.items():
            key = f"meas_uneqlt__{k}"
            if key in ref.files:
                np.testing.assert_allclose(v, ref[key].reshape(-1), rtol=1e-9, atol=1e-10,
                                           err_msg=k)


def test_kagome_exact_g_fixture(golden, tmp_path):
    """The 50-digit G of the kagome case after five sweeps
    (tests/golden/make_kagome_exact.py) belongs to the fields the oracle
    reaches, and it shows where the FP64 error of that ill-conditioned case
    lies: the oracle's stabilised G, which follows the reference's LAPACK
    path (greens.c:69-208), is a few 1e-9 away from it in the up spin."""
    z = np.load(os.path.join(golden, "kat_kagome", "g_exact_5.npz"))
    o = Sim(_copy_case(golden, "kat_kagome", tmp_path))
    gu, gd, _ = o.run(stop_sweep=int(z["sweeps"]))
    assert np.array_equal(o.hs.reshape(o.L, o.N), z["hs"])
    err = max(np.max(np.abs(gu - z["gu"])), np.max(np.abs(gd - z["gd"])))
    assert 1e-10 < err < 1e-8


def test_flop_tally_of_the_reference_build():
    """oracle/flop_tally.py on the c1 model (4x4, L = 40, n_matmul = 5,
    n_delay = 8): the reference build's BLAS / LAPACK calls of one sweep,
    counted with LAPACK-standard formulas, land near the analytic estimate
    (wraps 4(L-F), mul_seq 2(L-F), calc_eq_g F(3.2F + 5) and the update's
    flushes and panel products, in units of N^3 per spin), and the count is
    deterministic."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if not os.path.exists(os.path.join(root, "oracle", "_ref", "dqmc_1_r_tally")):
        pytest.skip("tally build not present (make -C oracle tally)")
    runs = []
    for _ in range(2):
        p = subprocess.run([sys.executable, os.path.join(root, "oracle", "flop_tally.py"), "c1"],
                           capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-2000:]
        runs.append(json.loads(p.stdout.strip().splitlines()[-1])["c1"])
    assert runs[0] == runs[1]
    N, L, F = 16, 40, 8
    estimate = 2 * N ** 3 * (4 * (L - F) + 2 * (L - F) + F * (3.2 * F + 5))
    assert 0.5 * estimate < runs[0] < 2.0 * estimate, (runs[0], estimate)
