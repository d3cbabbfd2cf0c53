"""The C-ABI library on the host: it loads, exports every function that
include/dqmc_b200.h declares, and its host-side paths behave without
touching a GPU (sizes, argument checks, the dry run of the drop-in
dqmc_wrapper, and a clean CUDA error where no device exists)."""
import ctypes as C
import os
import re
import shutil

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dqmc_b200.h")


def _declared():
    text = open(HEADER).read()
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(dqmc_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


@pytest.fixture(scope="module")
def lib():
    from dqmc_b200 import lib as L
    L.load()
    return L


def test_header_declares_every_binding(lib):
    names = _declared()
    assert len(names) >= 20
    assert sorted(names) == sorted(lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    h = lib.load()
    for name in _declared():
        assert hasattr(h, name), name


def test_acc_sizes_match_the_layout(lib, golden):
    from dqmc_b200 import engine
    s = engine.SimData.read(os.path.join(golden, "uneq_small", "sim_0.h5"))
    p, _keep = s.params()
    eq, ue = C.c_int(), C.c_int()
    assert lib.load().dqmc_acc_sizes(C.byref(p), C.byref(eq), C.byref(ue)) == 0
    ni, nij, nbb, L = s.p["num_i"], s.p["num_ij"], s.p["num_bb"], s.L
    assert eq.value == 1 + 4 * ni + 7 * nij
    assert ue.value == 1 + 7 * nij * L + 5 * nbb * L     # meas_bond_corr is on
    assert lib.load().dqmc_acc_sizes(None, C.byref(eq), C.byref(ue)) == lib.DQMC_E_ARG


def test_dry_run_reads_no_state_and_logs_the_header(lib, golden, tmp_path):
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, "c1_small", f), tmp_path)
    sim = str(tmp_path / "sim_0.h5")
    before = open(sim, "rb").read()
    log = str(tmp_path / "log.txt")
    rc = lib.load().dqmc_wrapper(sim.encode(), log.encode(), 0, True, False)
    assert rc == 0
    text = open(log).read()
    assert "dry run" in text
    assert open(sim, "rb").read() == before


def test_argument_checks_need_no_device(lib):
    h = lib.load()
    out = C.c_void_p()
    assert h.dqmc_engine_create(None, 1, 0, C.byref(out)) == lib.DQMC_E_ARG
    # oversize no-allocation call: refused before any device work
    n = 144
    batch = lib.NOALLOC_SCRATCH_BYTES // (6 * 8 * n * n) + 1
    assert h.dqmc_gpu_calc_eq_g_noalloc(batch, n, 4, 0, 0, 1, 1, 1, None) == lib.DQMC_E_SCRATCH
    assert h.dqmc_gpu_calc_eq_g(1, 0, 4, 0, 0, 1, 1, 1, None) == lib.DQMC_E_ARG


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a CUDA device")
def test_engine_reports_missing_device(lib, golden, tmp_path):
    from dqmc_b200 import engine
    s = engine.SimData.read(os.path.join(golden, "c1_small", "sim_0.h5"))
    p, _keep = s.params()
    out = C.c_void_p()
    assert lib.load().dqmc_engine_create(C.byref(p), 1, 0, C.byref(out)) == lib.DQMC_E_CUDA
    # the drop-in fails cleanly (-1) and leaves the sim file as it was
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, "c1_small", f), tmp_path)
    sim = str(tmp_path / "sim_0.h5")
    before = open(sim, "rb").read()
    rc = lib.load().dqmc_wrapper(sim.encode(), str(tmp_path / "log.txt").encode(), 0, False,
                                 False)
    assert rc == -1
    assert open(sim, "rb").read() == before
    assert np.array_equal(np.frombuffer(before, np.uint8), np.frombuffer(open(sim, "rb").read(),
                                                                         np.uint8))


@pytest.mark.parametrize("case", ["tog_sq", "tog_cplx", "tog_local"])
def test_toggle_layout_matches_the_library(lib, golden, case):
    """With measurement toggles on, the accumulator layout the Python side
    builds (dataset by dataset, data.c:441-522 sizes) has the size the
    library computes."""
    from dqmc_b200 import engine
    s = engine.SimData.read(os.path.join(golden, case, "sim_0.h5"))
    p, _keep = s.params()
    eq, ue = C.c_int(), C.c_int()
    assert lib.load().dqmc_acc_sizes(C.byref(p), C.byref(eq), C.byref(ue)) == 0
    assert eq.value == s.eq_acc.size
    assert ue.value == s.ue_acc.size
    ref = np.load(os.path.join(golden, case, "ref_out.npz"))
    for k, v in s.measurements().items():
        key = k.replace("/", "__")
        assert key in ref.files, k
        assert np.asarray(v).size == ref[key].size, k
