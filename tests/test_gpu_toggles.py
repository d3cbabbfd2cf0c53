"""The reference's measurement toggles on the GPU against the reference's own
build (oracle/_ref, src/meas.c compiled as is), on fixtures written by the
reference generator (tests/golden/make_golden.py):

* tog_sq: every toggle on a real 4x4 lattice with t' (the full bond and
  two-hop bond families): generalised susceptibility, chiral, energy
  (equal and unequal time), bond, thermal, two-bond and nematic
  correlators (src/meas.c:125-471, 473-714, 860-1363);
* tog_cplx: the same with one flux quantum (complex, Peierls phases), less
  the nematic correlators, which the reference has no complex form of;
* tog_local: the local heat current and pair_bb_only, which the reference
  generator allows only without translation symmetry (meas.c:214-296,
  827-858).

HS fields and RNG states bit-exact; every dataset within 1e-9 relative of
the reference build's (the generalised susceptibility is summed in another
order, see csrc/meas_x.cuh), through the Python engine and through the
drop-in dqmc_wrapper.
"""
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEAS_RTOL = 1e-9
CASES = ["tog_sq", "tog_cplx", "tog_local"]


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


def _check(values, ref):
    checked = 0
    for key in ref.files:
        if not key.startswith(("meas_eqlt__", "meas_uneqlt__")):
            continue
        v = np.asarray(values[key.replace("__", "/")]).reshape(-1)
        r = ref[key].reshape(-1)
        scale = max(np.max(np.abs(r)), 1.0)
        np.testing.assert_allclose(v, r, rtol=MEAS_RTOL, atol=MEAS_RTOL * scale, err_msg=key)
        checked += 1
    return checked


@pytest.mark.parametrize("case", CASES)
def test_toggles_match_reference_build(eng, golden, case, tmp_path):
    s = eng.SimData.read(_copy(golden, case, tmp_path))
    e = eng.Engine([s])
    e.init()
    e.sweeps(s.p["n_sweep"] - s.sweep)
    e.pull()
    assert e.errors() == 0
    e.close()
    ref = np.load(os.path.join(golden, case, "ref_out.npz"))
    assert np.array_equal(s.hs, ref["state__hs"].reshape(-1))
    assert np.array_equal(s.rng, ref["state__rng"])
    assert _check(s.measurements(), ref) >= 20


@pytest.mark.parametrize("case", CASES)
def test_toggles_through_the_wrapper(eng, golden, case, tmp_path):
    from dqmc_b200 import lib, simfile
    path = _copy(golden, case, tmp_path)
    rc = lib.load().dqmc_wrapper(path.encode(), str(tmp_path / "log").encode(), 0, False, False)
    assert rc == 0, open(tmp_path / "log").read()
    d = simfile.read(path)
    ref = np.load(os.path.join(golden, case, "ref_out.npz"))
    assert np.array_equal(d["state/hs"].reshape(-1), ref["state__hs"].reshape(-1))
    _check(d, ref)


def test_toggles_in_lanes_are_bit_identical(eng, golden, tmp_path):
    """Three chains of tog_sq (own RNG streams) in three lanes and in one:
    every accumulator bit-identical."""
    from dqmc_b200 import gen
    s0 = eng.SimData.read(_copy(golden, "tog_sq", tmp_path))
    runs = []
    for lanes in ("1", "3"):
        os.environ["DQMC_LANES"] = lanes
        try:
            sims = [s0.clone() for _ in range(3)]
            for k, s in enumerate(sims):
                for _ in range(k):
                    s.rng[:] = gen.rand_jump(s.rng)
            e = eng.Engine(sims)
            assert e.lanes() == int(lanes)
            e.init()
            e.sweeps(s0.p["n_sweep"] - s0.sweep)
            e.pull()
            e.close()
            runs.append(sims)
        finally:
            del os.environ["DQMC_LANES"]
    for a, b in zip(*runs):
        assert np.array_equal(a.eq_acc, b.eq_acc)
        assert np.array_equal(a.ue_acc, b.ue_acc)
