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
