"""Multi-rank host path on CPU: two gloo ranks, as bench.py and a multi-GPU
job run (one process per GPU, chains sharded, no data-path collective).

Checks that the per-rank chain blocks partition the job, that every chain
gets the same RNG stream whatever the rank count, that the device-time
maximum and the accumulator sum over ranks are the collectives' results, and
that the summed accumulators of chains advanced on their own ranks (by the
oracle, standing in for each rank's GPU) equal the serial sum.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
N_CHAINS, SEED, SWEEPS = 5, 7, 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _chain_acc(stream, tmpdir, tag):
    """equal-time accumulators of one small chain after SWEEPS sweeps (oracle)"""
    from dqmc_b200 import gen, simfile
    from oracle_ctl import Sim
    d = gen.make_sim(Nx=4, Ny=4, U=4.0, dt=0.1, L=8, n_matmul=4, n_delay=4, period_eqlt=4,
                     n_sweep_warm=0, n_sweep_meas=SWEEPS, init_rng=stream)
    path = os.path.join(tmpdir, f"c{tag}.h5")
    simfile.write(path, d)
    o = Sim(path)
    o.run()
    return np.concatenate([o.eq_sign.reshape(-1)] + [o.eq[k].reshape(-1) for k in sorted(o.eq)])


def _worker(rank, world, port, tmpdir):
    sys.path[:0] = [HERE, os.path.join(ROOT, "dqmc-dev_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from dqmc_b200 import replicas
    blk = replicas.shard(N_CHAINS, rank, world)
    streams = replicas.chain_streams(SEED, blk)
    t = replicas.max_over_ranks(1.5 * (rank + 1), world)
    acc = sum(_chain_acc(s, tmpdir, f"{rank}_{i}") for i, s in enumerate(streams))
    total = replicas.sum_over_ranks(acc, world)
    np.savez(os.path.join(tmpdir, f"rank{rank}.npz"), blk=np.array(list(blk)),
             streams=np.array(streams), t=t, total=total)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_partitions_the_job():
    from dqmc_b200 import replicas
    for n in (0, 1, 5, 256, 257):
        for world in (1, 2, 3, 8):
            got = [c for r in range(world) for c in replicas.shard(n, r, world)]
            assert got == list(range(n))
            sizes = [len(replicas.shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_two_gloo_ranks(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                             join=False, start_method="spawn")
    while not ctx.join(timeout=120):
        pass
    from dqmc_b200 import replicas
    r = [np.load(os.path.join(tmp_path, f"rank{k}.npz")) for k in range(2)]
    assert list(r[0]["blk"]) + list(r[1]["blk"]) == list(range(N_CHAINS))
    serial = replicas.chain_streams(SEED, range(N_CHAINS))
    got = np.concatenate([r[0]["streams"], r[1]["streams"]])
    assert np.array_equal(got, np.array(serial))
    assert float(r[0]["t"]) == float(r[1]["t"]) == 3.0
    expect = sum(_chain_acc(s, str(tmp_path), f"s{i}") for i, s in enumerate(serial))
    for k in range(2):
        np.testing.assert_allclose(r[k]["total"], expect, rtol=1e-13, atol=1e-13)
