// Launchers of the batched dense kernels (GEMM, pivoted and pre-sorted QR,
// recombine).  Each scalar type's launchers are compiled in a translation
// unit of their own (launch_gemm_{r,c}.cu, launch_{qrb,qrp,rec}_{r,c}.cu), so the
// kernel instantiations build in parallel; the engine and the seams call
// them through these declarations.
#pragma once

#include "gemm.cuh"
#include "qr.cuh"

namespace dq {

// The dynamic shared-memory limit of a kernel is one setting per function
// and device, shared by every engine of the process on that device: only
// ever raise it, so that a group created later with smaller needs cannot
// shrink it below what an earlier group's launches (and captured graphs)
// rely on.  Keyed by (device, kernel) under one lock: engines on other
// devices and the gradient paths' host threads launch concurrently.
// With carve, the kernel also prefers the largest shared-memory carveout,
// so that an SM configured for one such kernel (a QR CTA of one lane) can
// take CTAs of another (a GEMM of the next lane); the delayed update keeps
// the default, which leaves it the L1 cache its reads of G go through.
cudaError_t raise_smem_ptr(const void *kern, size_t bytes, bool carve);

template <typename K>
inline cudaError_t raise_smem(K kern, size_t bytes, bool carve = false)
{
	return raise_smem_ptr((const void *)kern, bytes, carve);
}

// Tensor map of one batched GEMM operand (column-major rows x cols, leading
// dimension ld, item b at base + (b / div) * hi + (b % div) * lo) for boxes
// of box_rows x box_cols elements; elem_doubles = 2 for complex128.  False
// when a tensor map cannot describe it (alignment, strides, a slice table),
// and the caller then loads element by element.
bool tma_map_operand(CUtensorMap *map, int *tz, int *tw, const void *base, int elem_doubles, int rows,
		int cols, long long ld, const Addr &ad, int batch, int box_rows, int box_cols);

// largest N the per-matrix factorisations (QR, recombine) support: the
// shared-memory form while N x N fits there, the global-memory form (working
// matrix in the caller's per-item workspace, L2-resident) up to 256
template <typename T> constexpr int max_dense_n() { return 256; }

// batched GEMM in the mode g.mode, tile chosen by least padded area
template <typename T> int launch_gemm(const GemmArgs<T> &g, cudaStream_t st);
// pre-sorted (QR_PRESORT) and column-pivoted (QR_PIVOT) QR with explicit Q
template <typename T> int launch_qr_presort(const QrArgs<T> &a, cudaStream_t st);
template <typename T> int launch_qr_pivot(const QrArgs<T> &a, cudaStream_t st);
template <typename T>
inline int launch_qr(const QrArgs<T> &a, cudaStream_t st)
{
	return a.mode == QR_PRESORT ? launch_qr_presort<T>(a, st) : launch_qr_pivot<T>(a, st);
}
// G = (D_b^-1 Q^H + D_s T)^-1 D_b^-1 Q^H and its phase
template <typename T> int launch_rec(const RecArgs<T> &a, cudaStream_t st);

extern template int launch_gemm<double>(const GemmArgs<double> &, cudaStream_t);
extern template int launch_gemm<zd>(const GemmArgs<zd> &, cudaStream_t);
extern template int launch_qr_presort<double>(const QrArgs<double> &, cudaStream_t);
extern template int launch_qr_presort<zd>(const QrArgs<zd> &, cudaStream_t);
extern template int launch_qr_pivot<double>(const QrArgs<double> &, cudaStream_t);
extern template int launch_qr_pivot<zd>(const QrArgs<zd> &, cudaStream_t);
extern template int launch_rec<double>(const RecArgs<double> &, cudaStream_t);
extern template int launch_rec<zd>(const RecArgs<zd> &, cudaStream_t);

}  // namespace dq
