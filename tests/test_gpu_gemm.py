"""The batched FP64 tensor-core GEMM seam (dqmc_gpu_gemm, the reference's
xgemm of src/linalg_generic.h:23-40) against torch float64 matmul on the same
inputs: relative error bounded by a small multiple of K * eps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dqmc_b200 import lib as L
    return L.load()


@pytest.mark.parametrize("cplx", [0, 1])
@pytest.mark.parametrize("M,N,K,batch", [(144, 144, 144, 7), (16, 16, 16, 3), (36, 36, 36, 5),
                                         (100, 100, 100, 2), (64, 64, 64, 4), (37, 53, 29, 3),
                                         (160, 160, 160, 2)])
def test_gemm_matches_torch(lib, cplx, M, N, K, batch):
    import ctypes as C

    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 1000 + N + K + cplx)
    dt = torch.complex128 if cplx else torch.float64
    # column-major storage: a (batch, K, M) tensor read as M x K column-major
    A = torch.randn(batch, K, M, dtype=dt, generator=g).cuda()
    B = torch.randn(batch, N, K, dtype=dt, generator=g).cuda()
    Cm = torch.randn(batch, N, M, dtype=dt, generator=g).cuda()
    alpha = np.array([0.75 + (0.25j if cplx else 0)], dtype=np.complex128 if cplx else np.float64)
    beta = np.array([-0.5 + (0.1j if cplx else 0)], dtype=np.complex128 if cplx else np.float64)
    ref = (alpha[0] * (A.transpose(1, 2) @ B.transpose(1, 2)) + beta[0] * Cm.transpose(1, 2))
    rc = lib.dqmc_gpu_gemm(batch, M, N, K, cplx, alpha.ctypes.data, A.data_ptr(), M, M * K,
                           B.data_ptr(), K, K * N, beta.ctypes.data, Cm.data_ptr(), M, M * N, None)
    assert rc == 0
    torch.cuda.synchronize()
    out = Cm.transpose(1, 2)
    err = (out - ref).abs().max().item() / max(ref.abs().max().item(), 1.0)
    assert err < 50 * K * 2.2e-16
