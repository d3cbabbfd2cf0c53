// Launchers of the dense per-matrix kernels (qr.cuh): the shared-memory or
// global-memory form by N, and the rows-per-lane instantiation.  Included by
// the launch_{qrb,qrp,rec}_{r,c}.cu translation units only.
#pragma once

#include "dqmc_b200.h"
#include "launch.cuh"

namespace dq {

// rows per lane of a warp column: 32 * RPL >= N
#define DQ_RPL(X) X(32, 1) X(64, 2) X(96, 3) X(128, 4) X(160, 5) X(192, 6) X(224, 7) X(256, 8)

// 226 KB leaves room for the kernels' static shared memory
static const size_t SMEM_FIT = 226 * 1024;

// carve: the shared-memory forms take the largest shared-memory carveout
// (room for a GEMM CTA beside them); the global-memory forms keep the
// default, whose L1 serves their working matrix
template <typename K, typename Args>
static int launch_dense(K kern, const Args &a, size_t sm, cudaStream_t st, bool carve)
{
	if (raise_smem(kern, sm, carve) != cudaSuccess) return DQMC_E_ARG;
	kern<<<a.batch, 512, sm, st>>>(a);
	return 0;
}

template <typename T, int RPL, bool GM>
static int launch_qrb_rpl(const QrArgs<T> &a, cudaStream_t st)
{
	return launch_dense(k_qrb<T, 16, 8, RPL, GM>, a, qrb_smem_bytes<T, 8>(a.N, GM), st, !GM);
}

template <typename T, int RPL, bool GM>
static int launch_qrp_rpl(const QrArgs<T> &a, cudaStream_t st)
{
	return launch_dense(k_qrp<T, 16, 8, RPL, GM>, a, qrp_smem_bytes<T, 8>(a.N, GM), st, !GM);
}

template <typename T, bool GM>
static int launch_qrb_gm(const QrArgs<T> &a, cudaStream_t st)
{
#define X(NMAX, R) if (a.N <= NMAX) return launch_qrb_rpl<T, R, GM>(a, st);
	DQ_RPL(X)
#undef X
	return DQMC_E_ARG;
}

template <typename T, bool GM>
static int launch_qrp_gm(const QrArgs<T> &a, cudaStream_t st)
{
#define X(NMAX, R) if (a.N <= NMAX) return launch_qrp_rpl<T, R, GM>(a, st);
	DQ_RPL(X)
#undef X
	return DQMC_E_ARG;
}

template <typename T>
int launch_qr_presort(const QrArgs<T> &a, cudaStream_t st)
{
	if (a.N < 1 || a.N > max_dense_n<T>()) return DQMC_E_ARG;
	if (qrb_smem_bytes<T, 8>(a.N) <= SMEM_FIT) return launch_qrb_gm<T, false>(a, st);
	if (!a.work) return DQMC_E_ARG;
	return launch_qrb_gm<T, true>(a, st);
}

template <typename T>
int launch_qr_pivot(const QrArgs<T> &a, cudaStream_t st)
{
	if (a.N < 1 || a.N > max_dense_n<T>()) return DQMC_E_ARG;
	if (qrp_smem_bytes<T, 8>(a.N) <= SMEM_FIT) return launch_qrp_gm<T, false>(a, st);
	if (!a.work) return DQMC_E_ARG;
	return launch_qrp_gm<T, true>(a, st);
}

template <typename T, int RPL, bool GM>
static int launch_rec_rpl(const RecArgs<T> &a, cudaStream_t st)
{
	return launch_dense(k_recb<T, 16, RPL, 3, GM>, a, recb_smem_bytes<T>(a.N, GM), st, !GM);
}

template <typename T, bool GM>
static int launch_rec_gm(const RecArgs<T> &a, cudaStream_t st)
{
#define X(NMAX, R) if (a.N <= NMAX) return launch_rec_rpl<T, R, GM>(a, st);
	DQ_RPL(X)
#undef X
	return DQMC_E_ARG;
}

template <typename T>
int launch_rec(const RecArgs<T> &a, cudaStream_t st)
{
	if (a.N < 1 || a.N > max_dense_n<T>()) return DQMC_E_ARG;
	if (recb_smem_bytes<T>(a.N) <= SMEM_FIT) return launch_rec_gm<T, false>(a, st);
	if (!a.work) return DQMC_E_ARG;
	return launch_rec_gm<T, true>(a, st);
}

}  // namespace dq
