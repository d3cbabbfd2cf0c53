"""The dqmc_stack job board (dqmc-dev_b200/csrc/main_stack.c) against the
semantics of the reference's src/main_stack.c:56-298, 399-479:

* jobs are popped from the end of the stack file (LIFO) under the "<stack>~"
  hard-link lock, each exactly once even with several processes popping;
* a stale lock (its owner died) is released after it stays unchanged;
* an empty stack ends the process with status 0;
* a job that stops early (time limit, signal) is pushed back to the stack;
  completed and failed jobs are not.

Dry runs (-n) touch no GPU and run on the CPU; the runs with sweeps are
marked gpu.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STACK = os.path.join(ROOT, "dqmc-dev_b200", "bin", "dqmc_stack")
ENV = dict(os.environ, DQMC_STACK_SLEEP="0.01")


def _jobs(golden, tmp_path, n, case="c1_small"):
    paths = []
    for k in range(n):
        d = tmp_path / f"job{k}"
        d.mkdir()
        for f in ("sim_0.h5", "sim.h5.params"):
            shutil.copy(os.path.join(golden, case, f), d)
        paths.append(str(d / "sim_0.h5"))
    stack = tmp_path / "stack"
    stack.write_text("".join(p + "\n" for p in paths))
    return paths, str(stack)


def _run(args, timeout=300):
    if not os.path.exists(STACK):
        pytest.fail(f"CLI not built: {STACK}")
    return subprocess.run([STACK] + args, env=ENV, capture_output=True, text=True, timeout=timeout)


def _started(out):
    return re.findall(r"starting:\s+(\S+)", out)


def test_dry_run_pops_lifo_until_empty(golden, tmp_path):
    paths, stack = _jobs(golden, tmp_path, 3)
    p = _run(["-n", stack])
    assert p.returncode == 0, p.stdout + p.stderr
    assert _started(p.stdout) == paths[::-1]
    assert open(stack).read().strip() == ""
    assert "empty; idling" in p.stdout
    for f in paths:
        assert "toggled dry run for mem check only" in open(f + ".log").read()


def test_concurrent_processes_take_each_job_once(golden, tmp_path):
    paths, stack = _jobs(golden, tmp_path, 24)
    procs = [subprocess.Popen([STACK, "-n", stack], env=ENV, stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for _ in range(3)]
    outs = [pr.communicate(timeout=300)[0] for pr in procs]
    assert [pr.returncode for pr in procs] == [0, 0, 0]
    started = sum((_started(o) for o in outs), [])
    assert sorted(started) == sorted(paths)
    assert not os.path.exists(stack + "~")


def test_zombie_lock_is_released(golden, tmp_path):
    paths, stack = _jobs(golden, tmp_path, 2)
    os.link(stack, stack + "~")        # a lock left by a process that died
    p = _run(["-n", stack])
    assert p.returncode == 0, p.stdout + p.stderr
    assert "zombie lock released" in p.stdout
    assert _started(p.stdout) == paths[::-1]


def test_missing_stack_file_fails(tmp_path):
    p = _run(["-n", str(tmp_path / "nope")])
    assert p.returncode != 0
    assert "does not exist" in p.stdout


def test_batched_pops_in_dry_run(golden, tmp_path):
    paths, stack = _jobs(golden, tmp_path, 5)
    p = _run(["-n", "-k", "2", stack])
    assert p.returncode == 0, p.stdout + p.stderr
    assert _started(p.stdout) == paths[::-1]
    assert open(stack).read().strip() == ""


@pytest.fixture
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
def test_stack_runs_jobs_on_the_gpu(gpu, golden, tmp_path):
    """Three jobs, two per batch: every file ends as the reference build's
    run of that file ends (fields and RNG bit-exact)."""
    from dqmc_b200 import simfile
    paths, stack = _jobs(golden, tmp_path, 3)
    p = _run(["-k", "2", stack], timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert len(re.findall(r"completed: ", p.stdout)) == 3
    ref = np.load(os.path.join(golden, "c1_small", "ref_out.npz"))
    for f in paths:
        d = simfile.read(f)
        assert np.array_equal(d["state/hs"].reshape(-1), ref["state__hs"].reshape(-1))
        assert np.array_equal(d["state/rng"], ref["state__rng"])


@pytest.mark.gpu
def test_stack_pushes_back_a_job_stopped_by_the_time_limit(gpu, tmp_path):
    from dqmc_b200 import gen, simfile
    d = gen.make_sim(Nx=8, Ny=8, tp=-0.25, U=6.0, mu=-0.5, dt=0.1, L=80, n_matmul=8,
                     n_delay=16, period_eqlt=8, n_sweep_warm=5, n_sweep_meas=4000,
                     checkpoint_every=10, seed=5)
    job = str(tmp_path / "long.h5")
    simfile.write(job, d)
    stack = tmp_path / "stack"
    stack.write_text(job + "\n")
    p = _run(["-t", "4", str(stack)], timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"dqmc_wrapper() incomplete, pushed: {job}" in p.stdout
    assert stack.read_text().split() == [job]
    assert "stop_flag = -1, stopping" in open(job + ".log").read()
