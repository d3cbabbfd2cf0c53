"""GPU parity tests: the CUDA engine against the oracle and the reference's
own outputs, called through the C ABI (include/dqmc_b200.h).

* known-answer test of the reference suite (test_batch_seed_basic_real,
  test/test_gen_1band_hub_unified.py:119-148): final HS fields after 40
  sweeps must equal test/hs_ref.py exactly for all four geometries;
* every golden case: HS fields and RNG state bit-exact, measurements within
  1e-9 relative of the reference build's datasets;
* the equal-time G after a run within 1e-10 (max abs, |G| <= O(1)) of the
  oracle's, and calc_eq_g against a plain FP64 dense inverse;
* each kernel seam against the oracle function it replaces.
"""
import ctypes as C
import os
import shutil

import numpy as np
import pytest

from oracle_ctl import Sim, oracle_lib

pytestmark = pytest.mark.gpu

GEOMS = ["square", "triangular", "honeycomb", "kagome"]
EQ_CASES = ["c1_small", "sq8_small"]
UE_CASES = ["uneq_small", "uneq_oddF", "cplx_small"]
G_TOL = 1e-10      # G against the FP64 oracle (max abs; G entries are O(1))
MEAS_RTOL = 1e-9   # accumulated measurements against the reference build


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import engine, lib
    lib.load()
    return engine


def _copy(golden, case, tmp_path):
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, case, f), tmp_path)
    return str(tmp_path / "sim_0.h5")


def _run(eng, path, n=None):
    s = eng.SimData.read(path)
    e = eng.Engine([s])
    e.init()
    e.sweeps(s.p["n_sweep"] - s.sweep if n is None else n)
    e.pull()
    assert e.errors() == 0
    return s, e


def _assert_meas(s, ref, rtol=MEAS_RTOL):
    for k, v in s.measurements().items():
        key = k.replace("/", "__")
        if key not in ref.files:
            continue
        r = ref[key].reshape(-1)
        v = np.asarray(v).reshape(-1)
        scale = max(np.max(np.abs(r)), 1.0)
        np.testing.assert_allclose(v, r, rtol=rtol, atol=rtol * scale, err_msg=k)


@pytest.mark.parametrize("geom", GEOMS)
def test_known_answer_hs(eng, golden, geom, tmp_path):
    ref = np.load(os.path.join(golden, "hs_ref.npz"))
    s, e = _run(eng, _copy(golden, f"kat_{geom}", tmp_path))
    assert np.array_equal(s.hs.reshape(s.L, s.N), ref[f"end_{geom}"])
    e.close()


@pytest.mark.parametrize("case", EQ_CASES + [f"kat_{g}" for g in GEOMS])
def test_engine_matches_reference_outputs(eng, golden, case, tmp_path):
    s, e = _run(eng, _copy(golden, case, tmp_path))
    ref = np.load(os.path.join(golden, case, "ref_out.npz"))
    assert np.array_equal(s.hs, ref["state__hs"].reshape(-1))
    assert np.array_equal(s.rng, ref["state__rng"])
    assert s.sweep == int(ref["state__sweep"])
    assert s.eq_n == int(ref["meas_eqlt__n_sample"])
    _assert_meas(s, ref)
    e.close()


@pytest.mark.parametrize("case", UE_CASES)
def test_engine_uneqlt_matches_reference(eng, golden, case, tmp_path):
    s, e = _run(eng, _copy(golden, case, tmp_path))
    ref = np.load(os.path.join(golden, case, "ref_out.npz"))
    assert np.array_equal(s.hs, ref["state__hs"].reshape(-1))
    assert np.array_equal(s.rng, ref["state__rng"])
    assert s.ue_n == int(ref["meas_uneqlt__n_sample"])
    _assert_meas(s, ref)
    e.close()


def _assert_meas_oracle(s, o, rtol=MEAS_RTOL):
    m = s.measurements()
    groups = [("meas_eqlt/", o.eq, o.eq_sign)]
    if s.p["period_uneqlt"] > 0:
        groups.append(("meas_uneqlt/", o.ue, o.ue_sign))
    for pre, d, sign in groups:
        np.testing.assert_allclose(np.asarray(m[pre + "sign"]).reshape(-1), sign.reshape(-1),
                                   rtol=rtol, err_msg=pre + "sign")
        for k, r in d.items():
            v = np.asarray(m[pre + k]).reshape(-1)
            r = r.reshape(-1)
            scale = max(np.max(np.abs(r)), 1.0)
            np.testing.assert_allclose(v, r, rtol=rtol, atol=rtol * scale, err_msg=pre + k)


# more groups E = 1 + (F-1)/2 than the reference fixtures have (E = 2, 3):
# several panel QRs in bsofi, blocks two and more above the diagonal in
# R^-1, and expand_g chains of uneven length; one complex case with flux
@pytest.mark.parametrize("Nx,L,nmul,nflux", [(4, 40, 4, 0), (6, 48, 4, 0), (4, 36, 3, 0), (4, 36, 4, 0),
                                             (4, 40, 4, 1), (4, 8, 4, 0)])
def test_engine_uneqlt_matches_oracle_generated(eng, Nx, L, nmul, nflux, tmp_path):
    path = _gen_case(tmp_path, Nx, Nx, U=4.0, mu=-0.5, tp=-0.2, dt=0.1, L=L, n_matmul=nmul,
                     n_delay=4, period_eqlt=nmul, period_uneqlt=1, meas_bond_corr=1, nflux=nflux,
                     n_sweep_warm=1, n_sweep_meas=2)
    o = Sim(path)
    o.run()
    s, e = _run(eng, path)
    assert np.array_equal(s.hs, o.hs)
    assert s.ue_n == int(o.ue_n[0])
    _assert_meas_oracle(s, o)
    e.close()


# kagome at U = 6, beta = 4 is the least well-conditioned case: the oracle's
# FP64 G (the reference's LAPACK path) is itself a few 1e-9 from the exact G
# there (test_oracle.py::test_kagome_exact_g_fixture), so engine and oracle
# agree to 1e-8 only; test_kagome_g_matches_extended_precision holds the
# engine to 1e-10 against the exact G instead
@pytest.mark.parametrize("case,n,tol", [("c1_small", 3, G_TOL), ("sq8_small", 2, G_TOL),
                                        ("kat_kagome", 5, 1e-8)])
def test_g_matches_oracle(eng, golden, case, n, tol, tmp_path):
    path = _copy(golden, case, tmp_path)
    o = Sim(path)
    gu_o, gd_o, ph_o = o.run(stop_sweep=n)
    s, e = _run(eng, path, n)
    gu, gd, ph = e.g(0)
    assert np.max(np.abs(gu - gu_o)) < tol
    assert np.max(np.abs(gd - gd_o)) < tol
    assert abs(ph - ph_o) < 1e-12
    assert np.array_equal(s.hs, o.hs)
    e.close()


def test_kagome_g_matches_extended_precision(eng, golden, tmp_path):
    """The engine's G of the kagome case after five sweeps against the same
    G evaluated with 50 significant digits from the same FP64 inputs
    (tests/golden/make_kagome_exact.py).  The oracle, on the reference's
    LAPACK path, is 5.2e-9 away from it; the engine must be within 1e-10 or
    closer than the oracle (it measured 7.4e-10)."""
    z = np.load(os.path.join(golden, "kat_kagome", "g_exact_5.npz"))
    path = _copy(golden, "kat_kagome", tmp_path)
    o = Sim(path)
    gu_o, gd_o, _ = o.run(stop_sweep=int(z["sweeps"]))
    e_orc = max(np.max(np.abs(gu_o - z["gu"])), np.max(np.abs(gd_o - z["gd"])))
    s, e = _run(eng, path, int(z["sweeps"]))
    assert np.array_equal(s.hs.reshape(s.L, s.N), z["hs"])
    gu, gd, _ = e.g(0)
    err = max(np.max(np.abs(gu - z["gu"])), np.max(np.abs(gd - z["gd"])))
    assert err < max(G_TOL, e_orc), f"max |G - G_exact| = {err:.3e}, oracle {e_orc:.3e}"
    e.close()


def _clusters(o, spin, F, nmul, hs):
    """oracle cluster products C_f = B_{fn+n-1} ... B_{fn} for one spin"""
    lib = oracle_lib(o.cplx)
    N, L = o.N, o.L
    B = np.zeros(L * N * N, o.nt)
    ek = o.a["exp_Ku"] if spin == 0 else o.a["exp_Kd"]
    lib.orc_build_B(N, L, C.c_void_p(ek.ctypes.data), C.c_void_p(o.a["exp_lambda"].ctypes.data),
                    C.c_void_p(hs.ctypes.data), spin, C.c_void_p(B.ctypes.data))
    Cm = np.zeros(F * N * N, o.nt)
    alpha = np.ones(1, o.nt)
    for f in range(F):
        lib.orc_mul_seq(N, L, f * nmul, ((f + 1) * nmul) % L, C.c_void_p(alpha.ctypes.data),
                        C.c_void_p(B.ctypes.data), C.c_void_p(Cm[f * N * N:].ctypes.data), N)
    return B, Cm


@pytest.mark.parametrize("case,l", [("c1_small", 0), ("c1_small", 3), ("sq8_small", 1),
                                    ("kat_kagome", 2)])
def test_calc_eq_g_seam(eng, golden, case, l, tmp_path):
    import torch
    from dqmc_b200 import lib
    o = Sim(_copy(golden, case, tmp_path))
    N, F, nmul = o.N, o.p["F"], o.p["n_matmul"]
    B, Cm = _clusters(o, 0, F, nmul, o.hs)
    g_o = np.zeros(N * N, o.nt)
    ph_o = np.zeros(1, o.nt)
    oracle_lib(o.cplx).orc_calc_eq_g(l, N, F, 2, C.c_void_p(Cm.ctypes.data),
                                     C.c_void_p(g_o.ctypes.data), C.c_void_p(ph_o.ctypes.data))
    dC = torch.from_numpy(Cm).cuda()
    dG = torch.zeros(N * N, dtype=dC.dtype, device="cuda")
    dph = torch.zeros(1, dtype=dC.dtype, device="cuda")
    rc = lib.load().dqmc_gpu_calc_eq_g(1, N, F, l, int(o.cplx), dC.data_ptr(), dG.data_ptr(),
                                       dph.data_ptr(), None)
    assert rc == 0
    g = dG.cpu().numpy()
    assert np.max(np.abs(g - g_o)) < G_TOL
    assert abs(dph.cpu().numpy()[0] - ph_o[0]) < 1e-12
    # a short product (two clusters, beta = 2 n_matmul dtau) is well enough
    # conditioned for a plain FP64 dense inverse to be an exact reference
    g_d = np.zeros(N * N, o.nt)
    oracle_lib(o.cplx).orc_dense_g(N, 2 * nmul, 0, C.c_void_p(B.ctypes.data),
                                   C.c_void_p(g_d.ctypes.data))
    dC2 = torch.from_numpy(Cm[:2 * N * N].copy()).cuda()
    rc = lib.load().dqmc_gpu_calc_eq_g(1, N, 2, 0, int(o.cplx), dC2.data_ptr(), dG.data_ptr(),
                                       dph.data_ptr(), None)
    assert rc == 0
    g2 = dG.cpu().numpy()
    assert np.max(np.abs(g2 - g_d)) < G_TOL


@pytest.mark.parametrize("case", ["c1_small", "sq8_small", "kat_honeycomb"])
def test_update_seam(eng, golden, case, tmp_path):
    import torch
    from dqmc_b200 import lib
    path = _copy(golden, case, tmp_path)
    o = Sim(path)
    gu, gd, ph = o.run(stop_sweep=1)          # a realistic G after one sweep
    N, nd = o.N, o.p["n_delay"]
    olib = oracle_lib(o.cplx)
    for l in range(3):
        hs = o.hs.reshape(o.L, o.N)[l].copy()
        rng = o.rng.copy()
        gu_c = np.ascontiguousarray(gu.T).reshape(-1).copy()
        gd_c = np.ascontiguousarray(gd.T).reshape(-1).copy()
        phase = np.array([ph], o.nt)
        # device copies before the oracle consumes its own
        dG = torch.from_numpy(np.concatenate([gu_c, gd_c])).cuda()
        dhs = torch.from_numpy(hs.copy()).cuda()
        drng = torch.from_numpy(rng.view(np.int64).copy()).cuda()
        ddel = torch.from_numpy(o.a["del_"].copy()).cuda()
        dph = torch.from_numpy(phase.copy()).cuda()
        order = np.zeros(N, np.int32)
        olib.orc_shuffle(C.c_void_p(rng.ctypes.data), N, C.c_void_p(order.ctypes.data))
        olib.orc_update_delayed(N, nd, C.c_void_p(o.a["del_"].ctypes.data),
                                C.c_void_p(order.ctypes.data), C.c_void_p(rng.ctypes.data),
                                C.c_void_p(hs.ctypes.data), C.c_void_p(gu_c.ctypes.data),
                                C.c_void_p(gd_c.ctypes.data), C.c_void_p(phase.ctypes.data))
        rc = lib.load().dqmc_gpu_update_delayed(1, N, nd, int(o.cplx), ddel.data_ptr(),
                                                drng.data_ptr(), dhs.data_ptr(), dG.data_ptr(),
                                                dph.data_ptr(), None)
        assert rc == 0
        assert np.array_equal(dhs.cpu().numpy(), hs)
        assert np.array_equal(drng.cpu().numpy().view(np.uint64), rng)
        g = dG.cpu().numpy()
        assert np.max(np.abs(g[:N * N] - gu_c)) < G_TOL
        assert np.max(np.abs(g[N * N:] - gd_c)) < G_TOL
        assert abs(dph.cpu().numpy()[0] - phase[0]) < 1e-12


@pytest.mark.parametrize("case,spin", [("c1_small", 0), ("sq8_small", 1), ("cplx_small", 0)])
def test_mul_seq_seam(eng, golden, case, spin, tmp_path):
    import torch
    from dqmc_b200 import lib
    o = Sim(_copy(golden, case, tmp_path))
    N, nmul = o.N, o.p["n_matmul"]
    B, Cm = _clusters(o, spin, o.p["F"], nmul, o.hs)
    ek = o.a["exp_Ku"] if spin == 0 else o.a["exp_Kd"]
    dK = torch.from_numpy(ek.copy()).cuda()
    del_ = torch.from_numpy(o.a["exp_lambda"].copy()).cuda()
    dhs = torch.from_numpy(o.hs[:nmul * N].copy()).cuda()
    dC = torch.zeros(N * N, dtype=dK.dtype, device="cuda")
    rc = lib.load().dqmc_gpu_mul_seq(1, N, nmul, spin, int(o.cplx), dK.data_ptr(),
                                     del_.data_ptr(), dhs.data_ptr(), dC.data_ptr(), None)
    assert rc == 0
    c = dC.cpu().numpy()
    ref = Cm[:N * N]
    assert np.max(np.abs(c - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_wrapper_drop_in(eng, golden, tmp_path):
    """dqmc_wrapper on a sim file: the file afterwards holds the reference's
    state bit-exactly and its measurements within tolerance."""
    from dqmc_b200 import lib, simfile
    path = _copy(golden, "c1_small", tmp_path)
    rc = lib.load().dqmc_wrapper(path.encode(), str(tmp_path / "log").encode(), 0, False, False)
    assert rc == 0
    d = simfile.read(path)
    ref = np.load(os.path.join(golden, "c1_small", "ref_out.npz"))
    assert np.array_equal(d["state/hs"].reshape(-1), ref["state__hs"].reshape(-1))
    assert np.array_equal(d["state/rng"], ref["state__rng"])
    assert int(d["state/partial_write"]) == 0
    for k in ("density", "double_occ", "nn", "zz", "xx", "pair_sw", "g00"):
        np.testing.assert_allclose(d[f"meas_eqlt/{k}"], ref[f"meas_eqlt__{k}"], rtol=MEAS_RTOL,
                                   atol=1e-12)
    log = open(tmp_path / "log").read()
    assert "sim_data_save() succeeded" in log


def test_batched_chains_match_single(eng, golden, tmp_path):
    """Chains batched in one engine give the same results as each alone."""
    paths = []
    for k in range(3):
        d = tmp_path / f"c{k}"
        d.mkdir()
        paths.append(_copy(golden, "c1_small", d))
    sims = [eng.SimData.read(p) for p in paths]
    # different seeds per chain: jump the RNG of chains 1 and 2
    olib = oracle_lib(False)
    for k, s in enumerate(sims[1:], 1):
        for _ in range(k):
            olib.orc_rand_jump(C.c_void_p(s.rng.ctypes.data))
    rngs = [s.rng.copy() for s in sims]
    e = eng.Engine(sims)
    e.init()
    e.sweeps(4)
    e.pull()
    for k in range(3):
        one = eng.SimData.read(paths[k])
        one.rng[:] = rngs[k]
        e1 = eng.Engine([one])
        e1.init()
        e1.sweeps(4)
        e1.pull()
        assert np.array_equal(one.hs, sims[k].hs)
        assert np.array_equal(one.rng, sims[k].rng)
        np.testing.assert_allclose(one.eq_acc, sims[k].eq_acc, rtol=1e-12, atol=1e-12)
        e1.close()
    e.close()


# ---- larger lattices, inputs from the engine's own generator ------------------

def _gen_case(tmp_path, Nx, Ny, **kw):
    from dqmc_b200 import gen, simfile
    d = gen.make_sim(Nx=Nx, Ny=Ny, seed=17, **kw)
    path = str(tmp_path / f"g{Nx}x{Ny}.h5")
    simfile.write(path, d)
    return path


# 10x10 .. 12x12 real run the shared-memory kernels; 16x10, 14x14 and 16x16
# real and 12x12 complex the global-memory form of the same kernels
@pytest.mark.parametrize("Nx,Ny,nflux", [(10, 10, 0), (12, 12, 0), (16, 10, 0), (14, 14, 0),
                                         (16, 16, 0), (12, 12, 1)])
def test_calc_eq_g_seam_large(eng, Nx, Ny, nflux, tmp_path):
    import torch
    from dqmc_b200 import lib
    path = _gen_case(tmp_path, Nx, Ny, U=4.0, mu=-1.0, dt=0.05, L=40, n_matmul=5, n_delay=16,
                     period_eqlt=8, nflux=nflux)
    o = Sim(path)
    N, F, nmul = o.N, o.p["F"], o.p["n_matmul"]
    for spin in (0, 1):
        B, Cm = _clusters(o, spin, F, nmul, o.hs)
        for l in (0, 3):
            g_o = np.zeros(N * N, o.nt)
            ph_o = np.zeros(1, o.nt)
            oracle_lib(o.cplx).orc_calc_eq_g(l, N, F, 2, C.c_void_p(Cm.ctypes.data),
                                             C.c_void_p(g_o.ctypes.data),
                                             C.c_void_p(ph_o.ctypes.data))
            dC = torch.from_numpy(Cm).cuda()
            dG = torch.zeros(N * N, dtype=dC.dtype, device="cuda")
            dph = torch.zeros(1, dtype=dC.dtype, device="cuda")
            rc = lib.load().dqmc_gpu_calc_eq_g(1, N, F, l, int(o.cplx), dC.data_ptr(),
                                               dG.data_ptr(), dph.data_ptr(), None)
            assert rc == 0
            g = dG.cpu().numpy()
            assert np.all(np.isfinite(g))
            assert np.max(np.abs(g - g_o)) < G_TOL
            assert abs(dph.cpu().numpy()[0] - ph_o[0]) < 1e-12


@pytest.mark.parametrize("Nx,Ny,nflux", [(12, 12, 0), (16, 16, 0), (10, 10, 1), (16, 16, 1)])
def test_engine_large_matches_oracle(eng, Nx, Ny, nflux, tmp_path):
    """2 sweeps of a large chain (L = 20): HS fields and RNG bit-exact, G and
    the equal-time measurements within tolerance of the oracle.  16 x 16
    runs the delayed update in CTAs of 544 threads (its large launch form),
    real and complex."""
    path = _gen_case(tmp_path, Nx, Ny, U=4.0, mu=-1.0, dt=0.05, L=20, n_matmul=5, n_delay=16,
                     period_eqlt=5, n_sweep_warm=0, n_sweep_meas=2, nflux=nflux)
    o = Sim(path)
    gu_o, gd_o, ph_o = o.run(stop_sweep=2)
    s, e = _run(eng, path, 2)
    assert np.array_equal(s.hs, o.hs)
    assert np.array_equal(s.rng, o.rng)
    gu, gd, ph = e.g(0)
    assert np.max(np.abs(gu - gu_o)) < G_TOL
    assert np.max(np.abs(gd - gd_o)) < G_TOL
    for k, v in o.eq.items():
        mine = s.measurements()["meas_eqlt/" + k]
        np.testing.assert_allclose(mine, v, rtol=MEAS_RTOL, atol=MEAS_RTOL * max(1, np.abs(v).max()),
                                   err_msg=k)
    e.close()


def test_many_chains_stay_finite(eng, tmp_path):
    """A batch at the benchmark shape runs several sweeps without device errors
    and with finite Green's functions."""
    from dqmc_b200 import gen
    rngs = gen.chain_rngs(3, 16)
    base = gen.make_sim(Nx=12, Ny=12, U=4.0, mu=-1.0, dt=0.05, L=40, n_matmul=10, n_delay=16,
                        period_eqlt=8, n_sweep_warm=0, n_sweep_meas=6, init_rng=rngs[0])
    sims = []
    for r in rngs:
        d = dict(base)
        hs, rr = gen.initial_hs(r, 40, 144)
        d["state/hs"], d["state/rng"] = hs, rr
        sims.append(eng.SimData(d))
    e = eng.Engine(sims)
    e.init()
    e.sweeps(3, sync=False)
    e.sync()
    assert e.errors() == 0
    for c in range(len(sims)):
        gu, gd, ph = e.g(c)
        assert np.all(np.isfinite(gu)) and np.all(np.isfinite(gd))
    e.close()
