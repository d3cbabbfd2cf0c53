"""The TMA-fed form of the batched GEMM against its element-wise (cp.async)
form.  Both fill the same shared-memory tiles (zeros outside the matrix) and
read them with the same fragments in the same DMMA order, so every result
must be bit-identical: the seam GEMMs (shapes that take tensor maps and
shapes that fall back, real and complex), and whole engine sweeps of the
12x12 benchmark model and the complex 10x10 model with flux (HS fields, G,
accumulators).  DQMC_GEMM_TMA=0 selects the element-wise form; it is read
once per process, so each form runs in a process of its own."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r'''
import sys
import numpy as np
import torch
from dqmc_b200 import engine, gen, lib as L, replicas

lib = L.load()
out = {}
for cplx in (0, 1):
    for (M, N, K, batch) in [(144, 144, 144, 5), (64, 64, 64, 3), (100, 100, 100, 2),
                             (48, 96, 32, 3), (37, 53, 29, 2)]:
        g = torch.Generator().manual_seed(M + N + K + cplx)
        dt = torch.complex128 if cplx else torch.float64
        A = torch.randn(batch, K, M, dtype=dt, generator=g).cuda()
        B = torch.randn(batch, N, K, dtype=dt, generator=g).cuda()
        C = torch.randn(batch, N, M, dtype=dt, generator=g).cuda()
        nt = np.complex128 if cplx else np.float64
        alpha = np.array([0.75 + (0.25j if cplx else 0)], dtype=nt)
        beta = np.array([-0.5 + (0.1j if cplx else 0)], dtype=nt)
        rc = lib.dqmc_gpu_gemm(batch, M, N, K, cplx, alpha.ctypes.data, A.data_ptr(), M, M * K,
                               B.data_ptr(), K, K * N, beta.ctypes.data, C.data_ptr(), M, M * N,
                               None)
        assert rc == 0
        torch.cuda.synchronize()
        out[f"gemm_{cplx}_{M}_{N}_{K}"] = C.cpu().numpy()


def chains(n, seed, **kw):
    rngs = replicas.chain_streams(seed, range(n))
    base = gen.make_sim(init_rng=rngs[0], **kw)
    N, L_ = int(base["params/N"]), int(base["params/L"])
    ds = [base]
    for r in rngs[1:]:
        hs, rr = gen.initial_hs(r, L_, N)
        d = dict(base)
        d["state/init_rng"], d["state/rng"], d["state/hs"] = r, rr, hs
        ds.append(d)
    return ds


cases = {
    "real": chains(2, 77, Nx=12, Ny=12, U=4.0, mu=-1.0, dt=0.05, L=120, n_matmul=10,
                   n_delay=16, period_eqlt=8, n_sweep_warm=0, n_sweep_meas=2),
    "cplx": chains(2, 78, Nx=10, Ny=10, U=4.0, mu=0.0, dt=0.1, L=50, n_matmul=5, n_delay=16,
                   nflux=1, period_eqlt=5, period_uneqlt=1, meas_bond_corr=1,
                   n_sweep_warm=0, n_sweep_meas=2),
}
for name, dicts in cases.items():
    sims = [engine.SimData(d) for d in dicts]
    e = engine.Engine(sims)
    e.init()
    e.sweeps(2)
    e.pull()
    assert e.errors() == 0
    for c, s in enumerate(sims):
        gu, gd, ph = e.g(c)
        out[f"{name}_{c}_hs"] = s.hs
        out[f"{name}_{c}_gu"] = gu
        out[f"{name}_{c}_gd"] = gd
        out[f"{name}_{c}_eq"] = s.eq_acc
        if s.p["period_uneqlt"] > 0:
            out[f"{name}_{c}_ue"] = s.ue_acc
    e.close()
np.savez(sys.argv[1], **out)
'''


def _run(tmp_path, tag, tma):
    env = dict(os.environ)
    env.pop("DQMC_GEMM_TMA", None)
    if not tma:
        env["DQMC_GEMM_TMA"] = "0"
    env["PYTHONPATH"] = os.path.join(ROOT, "dqmc-dev_b200") + os.pathsep + env.get("PYTHONPATH", "")
    out = str(tmp_path / f"{tag}.npz")
    r = subprocess.run([sys.executable, "-c", SCRIPT, out], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


def test_tma_form_bit_identical_to_elementwise(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    a = _run(tmp_path, "tma", True)
    b = _run(tmp_path, "elementwise", False)
    assert set(a.files) == set(b.files)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
