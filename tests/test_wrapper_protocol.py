"""The control protocol of the drop-in dqmc_wrapper (include/dqmc_b200.h).

The reference's contract (src/dqmc.c:222-244, 525-671; src/sig.c:43-105;
src/data.c:345-357, 667-789):

* a file whose last save was interrupted (state/partial_write = 1) is
  refused: the read fails with -2 and dqmc_wrapper returns -1;
* a dry run only reports and returns 0; a finished file is left alone;
* a checkpoint is written at the start of every sweep that is a multiple of
  checkpoint_every, before the sweep runs;
* the time limit (-t) or a signal (SIGUSR1, SIGINT, SIGTERM, SIGHUP) stops
  the run at the next sweep boundary: dqmc_wrapper returns 1 ("dqmc()
  interrupted") and the file keeps the last checkpoint;
* a run resumed from that checkpoint ends bit-identical (fields, RNG,
  every accumulator) to a run that was never interrupted.

The stop flag is process-wide and stays set once raised (as in the
reference), so the runs that stop go through the dqmc_1 CLI in child
processes.  The file-level checks need no GPU; the runs are marked gpu.
"""
import os
import re
import shutil
import signal
import subprocess
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "dqmc-dev_b200", "bin", "dqmc_1")


def _copy(golden, case, tmp_path):
    for f in ("sim_0.h5", "sim.h5.params"):
        shutil.copy(os.path.join(golden, case, f), tmp_path)
    return str(tmp_path / "sim_0.h5")


def _wrapper():
    from dqmc_b200 import lib
    return lib.load().dqmc_wrapper


def test_partial_write_refused(golden, tmp_path):
    """data.c:353-357: a file whose last save did not finish is not read."""
    from dqmc_b200 import simfile
    path = _copy(golden, "c1_small", tmp_path)
    simfile.update(path, {"state/partial_write": 1})
    log = tmp_path / "log"
    rc = _wrapper()(path.encode(), str(log).encode(), 0, False, False)
    assert rc == -1
    text = log.read_text()
    assert "sim_data_read_alloc() failed: -2" in text
    # the file is left as it was
    assert int(simfile.read(path)["state/partial_write"]) == 1


def test_dry_run_and_finished_file(golden, tmp_path):
    from dqmc_b200 import simfile
    path = _copy(golden, "c1_small", tmp_path)
    log = tmp_path / "log"
    assert _wrapper()(path.encode(), str(log).encode(), 0, True, False) == 0
    assert "toggled dry run for mem check only" in log.read_text()
    d = simfile.read(path)
    simfile.update(path, {"state/sweep": int(np.asarray(d["params/n_sweep"]).reshape(-1)[0])})
    log2 = tmp_path / "log2"
    assert _wrapper()(path.encode(), str(log2).encode(), 0, False, False) == 0
    assert "already finished so don't do anything" in log2.read_text()


# ---- runs on the GPU --------------------------------------------------------

def _long_case(tmp_path, name, n_sweep_meas=4000, checkpoint_every=10):
    """8x8, L = 80 chain with many sweeps: it runs for minutes unless stopped"""
    from dqmc_b200 import gen, simfile
    d = gen.make_sim(Nx=8, Ny=8, tp=-0.25, U=6.0, mu=-0.5, dt=0.1, L=80, n_matmul=8,
                     n_delay=16, period_eqlt=8, period_uneqlt=4, n_sweep_warm=5,
                     n_sweep_meas=n_sweep_meas, checkpoint_every=checkpoint_every, seed=99)
    path = str(tmp_path / name)
    simfile.write(path, d)
    return path


def _state(path):
    from dqmc_b200 import simfile
    d = simfile.read(path)
    return {k: np.asarray(v) for k, v in d.items()
            if k.startswith(("state/", "meas_eqlt/", "meas_uneqlt/")) and k != "state/init_rng"}


def _checkpoint_calls(log_text):
    m = re.search(r"^\s*checkpoint \|.*\|\s*(\d+)\s*$", log_text, re.M)
    return int(m.group(1)) if m else 0


def _stopped_sweep(log_text):
    m = re.search(r"^(\d+)/\d+ sweeps completed \((?:measuring|warming up)\)$", log_text, re.M)
    return int(m.group(1))


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(CLI):
        pytest.fail(f"CLI not built: {CLI}")


@pytest.mark.gpu
def test_time_limit_stops_and_resume_is_bit_identical(gpu, tmp_path):
    from dqmc_b200 import simfile
    path = _long_case(tmp_path, "a.h5")
    log = tmp_path / "a.log"
    p = subprocess.run([CLI, "-t", "3", "-l", str(log), path], timeout=600)
    assert p.returncode == 1
    text = log.read_text()
    assert "stop_flag = -1, stopping" in text
    assert "dqmc() interrupted" in text
    stop = _stopped_sweep(text)
    st = _state(path)
    ck = int(st["state/sweep"])
    assert int(st["state/partial_write"]) == 0
    # a checkpoint at the start of every sweep 0, 10, 20, ... that began
    # before the stop (the stop check comes first), the last one kept
    n_ck = (stop - 1) // 10 + 1 if stop > 0 else 0
    assert _checkpoint_calls(text) == n_ck
    assert ck == 10 * (n_ck - 1) if n_ck else ck == 0

    # resume to 7 sweeps past the checkpoint, and compare with a run of the
    # same file that was never interrupted
    target = ck + 7
    fresh = _long_case(tmp_path, "b.h5")
    for f in (path, fresh):
        simfile.update(f, {"params/n_sweep": target})
    p = subprocess.run([CLI, "-l", str(tmp_path / "a2.log"), path], timeout=600)
    assert p.returncode == 0
    p = subprocess.run([CLI, "-l", str(tmp_path / "b.log"), fresh], timeout=600)
    assert p.returncode == 0
    a, b = _state(path), _state(fresh)
    assert int(a["state/sweep"]) == target
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.gpu
def test_signal_stops_at_sweep_boundary(gpu, tmp_path):
    path = _long_case(tmp_path, "s.h5")
    log = tmp_path / "s.log"
    proc = subprocess.Popen([CLI, "-l", str(log), path])
    try:
        deadline = time.time() + 120
        while time.time() < deadline:
            if log.exists() and "starting dqmc" in log.read_text():
                break
            time.sleep(0.1)
        time.sleep(1.0)
        proc.send_signal(signal.SIGUSR1)
        rc = proc.wait(timeout=120)
    finally:
        if proc.poll() is None:
            proc.kill()
            proc.wait()
    assert rc == 1
    text = log.read_text()
    assert f"stop_flag = {int(signal.SIGUSR1)}, stopping" in text
    assert "dqmc() interrupted" in text
    st = _state(path)
    assert int(st["state/partial_write"]) == 0
    assert int(st["state/sweep"]) % 10 == 0
