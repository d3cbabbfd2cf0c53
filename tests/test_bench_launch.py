"""bench.py's multi-GPU plumbing on CPU: `--gpus N` without a launcher
starts N ranks itself (torch.distributed.run, one process per GPU), the
ranks join one process group (gloo here, NCCL on GPUs), and rank 0 reports
the world size and the maximum over ranks, as the timed runs do."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpus_flag_spawns_ranks():
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--launch-check"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert lines == [{"n_gpus": 2, "max_rank": 1.0}]


def test_reference_arm_times_the_ragged_mix():
    """`--impl reference --workload ragged64` runs the reference build on
    chains of the ragged mix (not the 256-chain model) and prints one line
    with its rate, the CPU baseline and an e2e of zero copies."""
    import pytest
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "dqmc_1_r")):
        pytest.skip("reference build not present")
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "ragged64", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["config"]["workload"].startswith("64 ragged chains")
    assert "ragged mix" in d["cpu_baseline"]["sample"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_roofline_carries_the_reference_flop_tally():
    """bench.roofline on a synthetic per-class profile: the dominant class,
    the engine-counted sweep fraction, and for a workload with a reference
    tally the same step measured in the reference build's FLOPs."""
    sys.path.insert(0, ROOT)
    import bench
    names = ["gemm", "update", "qr_pivot", "uneqlt_g", "meas", "qr_presort", "recombine"]
    prof = {k: (0.0, 0.0, 0.0, 0.0) for k in names}
    prof["gemm"] = (50.0, 800.0, 1.2e12, 0.0)
    prof["qr_presort"] = (60.0, 60.0, 0.3e12, 0.0)
    rl = bench.roofline(prof, 512, "batch256", 35.0, 200.0, chains=256)
    assert rl["class"] == "qr_presort" and abs(rl["achieved"] - 5.0) < 1e-9
    assert abs(rl["sweep"]["achieved"] - 7.5) < 1e-9
    ref = bench.REF_FLOPS_PER_CHAIN_SWEEP["batch256"] * 256 / 0.2 / 1e12
    assert abs(rl["sweep"]["reference_achieved"] - ref) < 1e-9
    assert abs(rl["sweep"]["reference_frac"] - ref / 35.0) < 1e-12
    rl2 = bench.roofline(prof, 128, "ragged64", 35.0, 200.0)
    assert "reference_flops" not in rl2["sweep"]
