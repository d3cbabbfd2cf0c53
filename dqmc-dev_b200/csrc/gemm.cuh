// Batched FP64 / complex128 GEMM on the FP64 tensor cores (DMMA m8n8k4).
//
//   C_b = alpha * opA(A_b) * opB(B_b) + beta * C_b      for b in [0, batch)
//
// The batch is the set of (chain, spin) items of a group; all items share
// M, N, K.  Operand addresses per item are base + (b / div) * hi +
// (b % div) * lo, which covers per-item matrices (div 1), per-spin shared
// parameters such as exp(-dt K_sigma) (div 2, hi 0) and per-item stacks.
//
// Operand modes fuse the diagonal factors of B_l = exp(-dt K) diag(d_l)
// (reference dqmc.c:29-59) into the tile loads instead of materialising B:
//   A_DD       A[r,k] * d[r] / d[k]     (G -> D G D^-1, the wrap prologue)
//   B_ROWD     B[k,c] * d[k]            (diag(d) X, the mul_seq step)
//   B_COLD     B[k,c] * d[c]            (X diag(d), the first factor of C_f)
//   A_UPPER    A[r,k] = 0 for r > k     (triangular A: the trmm of calc_eq_g)
//   B_GATHER   B[k,c] = B[idx[k],c]     (row permutation P^T T)
// Tiles are staged through shared memory by the CTA (register double
// buffering) with padded strides so fragment loads are bank-conflict free.
#pragma once

#include "common.cuh"

namespace dq {

enum : int {
	GM_A_DD = 1,
	GM_B_ROWD = 2,
	GM_A_UPPER = 4,
	GM_B_GATHER = 8,
	GM_B_COLD = 16,
	GM_B_IDENT = 32,   // B is the identity (C = alpha A + beta C with scaling)
};

struct Addr {
	long long hi, lo;
	int div;
	__host__ __device__ long long off(int b) const { return (long long)(b / div) * hi + (long long)(b % div) * lo; }
};

template <typename T>
struct GemmArgs {
	int M, N, K, batch;
	const T *A; Addr aA; int lda;
	const T *B; Addr aB; int ldb;
	T *C; Addr aC; int ldc;
	T alpha, beta;
	int mode;
	const double *d; const double *dinv; Addr aD;   // scaling vectors (length K or M)
	const int *gidx; Addr aG;                       // row gather for B
};

template <typename T, int BM, int BN, int BK, int WM, int WN>
struct GemmCfg {
	static constexpr int THREADS = WM * WN * 32;
	static constexpr int SA = BM + 4;      // As[k][r]
	static constexpr int SB = BK + 4;      // Bs[c][k]
	static constexpr int PLANES = is_cplx<T>::value ? 2 : 1;
	static constexpr int SMEM_A = BK * SA;
	static constexpr int SMEM_B = BN * SB;
	static constexpr int STAGE = PLANES * (SMEM_A + SMEM_B);
	static constexpr int SMEM_BYTES = 2 * STAGE * (int)sizeof(double);
	static constexpr int WTM = BM / WM, WTN = BN / WN;
	static constexpr int MT = WTM / 8, NT = WTN / 8;
	static constexpr int A_PER_T = (BM * BK + THREADS - 1) / THREADS;
	static constexpr int B_PER_T = (BK * BN + THREADS - 1) / THREADS;
	static_assert(WTM % 8 == 0 && WTN % 8 == 0, "warp tile must be a multiple of 8");
	static_assert(BK % 4 == 0, "BK multiple of 4");
};

template <typename T, int BM, int BN, int BK, int WM, int WN>
__global__ void __launch_bounds__(WM *WN * 32)
k_gemm(GemmArgs<T> g)
{
	using Cfg = GemmCfg<T, BM, BN, BK, WM, WN>;
	constexpr bool CX = is_cplx<T>::value;
	extern __shared__ double sm[];
	const int b = blockIdx.z;
	const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
	if (b >= g.batch || m0 >= g.M || n0 >= g.N) return;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wm = warp % WM, wn = warp / WM;
	const T *A = g.A + g.aA.off(b);
	const T *B = g.B + g.aB.off(b);
	T *Cp = g.C + g.aC.off(b);
	const double *d = (g.mode & (GM_A_DD | GM_B_ROWD | GM_B_COLD)) ? g.d + g.aD.off(b) : nullptr;
	const double *dinv = (g.mode & GM_A_DD) ? g.dinv + g.aD.off(b) : nullptr;
	const int *gi = (g.mode & GM_B_GATHER) ? g.gidx + g.aG.off(b) : nullptr;
	const int M = g.M, N = g.N, K = g.K;

	double acc_r[Cfg::MT][Cfg::NT][2], acc_i[CX ? Cfg::MT : 1][CX ? Cfg::NT : 1][2];
#pragma unroll
	for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
		for (int j = 0; j < Cfg::NT; j++) {
			acc_r[i][j][0] = acc_r[i][j][1] = 0.0;
			if (CX) acc_i[CX ? i : 0][CX ? j : 0][0] = acc_i[CX ? i : 0][CX ? j : 0][1] = 0.0;
		}

	int kt0 = 0;
	if (g.mode & GM_A_UPPER) kt0 = m0 / BK;
	const int nkt = (K + BK - 1) / BK;

	T ra[Cfg::A_PER_T], rb[Cfg::B_PER_T];
	auto load = [&](int kt) {
		const int k0 = kt * BK;
#pragma unroll
		for (int q = 0; q < Cfg::A_PER_T; q++) {
			const int idx = tid + q * Cfg::THREADS;
			const int r = idx % BM, k = idx / BM;
			const int gr = m0 + r, gk = k0 + k;
			T v = zero<T>();
			if (idx < BM * BK && gr < M && gk < K) {
				if (!((g.mode & GM_A_UPPER) && gr > gk)) {
					v = A[gr + (long long)gk * g.lda];
					if (g.mode & GM_A_DD) v = v * (d[gr] * dinv[gk]);
				}
			}
			ra[q] = v;
		}
#pragma unroll
		for (int q = 0; q < Cfg::B_PER_T; q++) {
			const int idx = tid + q * Cfg::THREADS;
			const int k = idx % BK, c = idx / BK;
			const int gk = k0 + k, gc = n0 + c;
			T v = zero<T>();
			if (idx < BK * BN && gk < K && gc < N) {
				if (g.mode & GM_B_IDENT) {
					v = (gk == gc) ? one<T>() : zero<T>();
				} else {
					const int row = gi ? gi[gk] : gk;
					v = B[row + (long long)gc * g.ldb];
				}
				if (g.mode & GM_B_ROWD) v = v * d[gk];
				if (g.mode & GM_B_COLD) v = v * d[gc];
			}
			rb[q] = v;
		}
	};
	auto store = [&](int stage) {
		double *As = sm + stage * Cfg::STAGE;
		double *Bs = As + Cfg::PLANES * Cfg::SMEM_A;
#pragma unroll
		for (int q = 0; q < Cfg::A_PER_T; q++) {
			const int idx = tid + q * Cfg::THREADS;
			if (idx < BM * BK) {
				const int r = idx % BM, k = idx / BM;
				double xr, xi;
				split(ra[q], xr, xi);
				As[k * Cfg::SA + r] = xr;
				if (CX) As[Cfg::SMEM_A + k * Cfg::SA + r] = xi;
			}
		}
#pragma unroll
		for (int q = 0; q < Cfg::B_PER_T; q++) {
			const int idx = tid + q * Cfg::THREADS;
			if (idx < BK * BN) {
				const int k = idx % BK, c = idx / BK;
				double xr, xi;
				split(rb[q], xr, xi);
				Bs[c * Cfg::SB + k] = xr;
				if (CX) Bs[Cfg::SMEM_B + c * Cfg::SB + k] = xi;
			}
		}
	};

	const int gq = lane >> 2, tq = lane & 3;
	int stage = 0;
	if (kt0 < nkt) {
		load(kt0);
		store(0);
	}
	__syncthreads();
	for (int kt = kt0; kt < nkt; kt++) {
		const bool more = kt + 1 < nkt;
		if (more) load(kt + 1);
		const double *As = sm + stage * Cfg::STAGE;
		const double *Bs = As + Cfg::PLANES * Cfg::SMEM_A;
#pragma unroll
		for (int kk = 0; kk < BK; kk += 4) {
			double fa[Cfg::MT], fb[Cfg::NT], fai[CX ? Cfg::MT : 1], fbi[CX ? Cfg::NT : 1];
#pragma unroll
			for (int i = 0; i < Cfg::MT; i++) {
				const int r = wm * Cfg::WTM + i * 8 + gq;
				fa[i] = As[(kk + tq) * Cfg::SA + r];
				if (CX) fai[CX ? i : 0] = As[Cfg::SMEM_A + (kk + tq) * Cfg::SA + r];
			}
#pragma unroll
			for (int j = 0; j < Cfg::NT; j++) {
				const int c = wn * Cfg::WTN + j * 8 + gq;
				fb[j] = Bs[c * Cfg::SB + kk + tq];
				if (CX) fbi[CX ? j : 0] = Bs[Cfg::SMEM_B + c * Cfg::SB + kk + tq];
			}
#pragma unroll
			for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
				for (int j = 0; j < Cfg::NT; j++) {
					dmma(acc_r[i][j][0], acc_r[i][j][1], fa[i], fb[j]);
					if (CX) {
						const int ii = CX ? i : 0, jj = CX ? j : 0;
						dmma(acc_r[i][j][0], acc_r[i][j][1], -fai[ii], fbi[jj]);
						dmma(acc_i[ii][jj][0], acc_i[ii][jj][1], fa[i], fbi[jj]);
						dmma(acc_i[ii][jj][0], acc_i[ii][jj][1], fai[ii], fb[j]);
					}
				}
		}
		if (more) store(stage ^ 1);
		__syncthreads();
		stage ^= 1;
	}

	// epilogue: lane holds C[gq][2 tq + {0,1}] of each 8x8 tile
	const bool use_beta = !(re(g.beta) == 0.0 && im(g.beta) == 0.0);
#pragma unroll
	for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
		for (int j = 0; j < Cfg::NT; j++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int r = m0 + wm * Cfg::WTM + i * 8 + gq;
				const int c = n0 + wn * Cfg::WTN + j * 8 + 2 * tq + h;
				if (r < M && c < N) {
					T v;
					if constexpr (CX) {
						v = mkz(acc_r[i][j][h], acc_i[i][j][h]);
					} else {
						v = acc_r[i][j][h];
					}
					v = g.alpha * v;
					T *dst = Cp + r + (long long)c * g.ldc;
					if (use_beta) v = v + g.beta * (*dst);
					*dst = v;
				}
			}
}

}  // namespace dq
