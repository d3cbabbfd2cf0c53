// Batched FP64 / complex128 GEMM on the FP64 tensor cores (DMMA m8n8k4).
//
//   C_b = alpha * opA(A_b) * opB(B_b) + beta * C_b      for b in [0, batch)
//
// The batch is the set of (chain, spin) items of a group; all items share
// M, N, K.  Operand addresses per item are base + (b / div) * hi +
// (b % div) * lo, which covers per-item matrices (div 1), per-spin shared
// parameters such as exp(-dt K_sigma) (div 2, hi 0) and per-item stacks.
//
// Operand modes (compile-time) fuse the diagonal factors of
// B_l = exp(-dt K) diag(d_l) (reference dqmc.c:29-59) and the other
// structure of the calc_eq_g products into the kernel instead of
// materialising them:
//   A_DD       A[r,k] * d[r] / d[k]     (G -> D G D^-1, the wrap prologue)
//   B_ROWD     B[k,c] * d[k]            (diag(d) X, the mul_seq step)
//   B_COLD     B[k,c] * d[c]            (X diag(d))
//   A_UPPER    A[r,k] = 0 for r > k     (triangular A, the trmm of calc_eq_g;
//                                        k-tiles left of the diagonal skipped)
//   B_GATHER   B[k,c] = B[idx[k],c]     (row permutation P^T T)
//   B_IDENT    B = I                    (C = alpha A + beta C)
// Tiles move global -> shared through a STAGES-deep ring, zero-filled
// outside the matrix: in the TMA form one thread loads each stage's A and B
// boxes with cp.async.bulk.tensor onto the stage's mbarrier (tensor maps over
// this GPU's memory, no multicast); otherwise (row gathers, operands whose
// address or strides a tensor map cannot take) every thread copies elements
// with cp.async.  Scale vectors are staged once per CTA and applied when
// fragments are read, so every mode keeps the same pipeline.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "mbar.cuh"

namespace dq {

enum : int {
	GM_A_DD = 1,
	GM_B_ROWD = 2,
	GM_A_UPPER = 4,
	GM_B_GATHER = 8,
	GM_B_COLD = 16,
	GM_B_IDENT = 32,
};

// off(b) = q * hi + (b % div) * lo with q = b / div, or q = tab[b / div]
// when a table is given (the slice of each group of `div` items, for the
// unequal-time slice chains, whose slices wrap around modulo L)
struct Addr {
	long long hi, lo;
	int div;
	const int *tab;
	__host__ __device__ long long off(int b) const
	{
		const int q = b / div;
		return (long long)(tab ? tab[q] : q) * hi + (long long)(b % div) * lo;
	}
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
	int b0;                                         // first item of this launch
	unsigned *err;                                  // error word (TMA wait timeouts), may be null
	// TMA form: 4-d tensor maps (rows, columns, b % div, b / div) of A and B;
	// tz / tw: whether the third / fourth coordinate is used (else 0)
	CUtensorMap tmA, tmB;
	int tzA, twA, tzB, twB;
};

__device__ inline void cp_async8(void *smem, const void *gmem, bool valid)
{
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
	             "r"(valid ? 8 : 0));
}
__device__ inline void cp_async16(void *smem, const void *gmem, bool valid)
{
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
	             "r"(valid ? 16 : 0));
}
__device__ inline void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int NPEND>
__device__ inline void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND)); }

template <typename T>
__device__ inline void cp_async_el(T *smem, const T *gmem, bool valid);
template <>
__device__ inline void cp_async_el<double>(double *smem, const double *gmem, bool valid)
{
	cp_async8(smem, gmem, valid);
}
template <>
__device__ inline void cp_async_el<zd>(zd *smem, const zd *gmem, bool valid)
{
	cp_async16(smem, gmem, valid);
}

template <typename T, int BM, int BN, int BK, int WM, int WN, int STAGES>
struct GemmCfg {
	static constexpr bool CX = is_cplx<T>::value;
	static constexpr int THREADS = WM * WN * 32;
	// padded strides: fragment reads conflict-free for 8- and 16-byte elements
	static constexpr int SA = BM + (CX ? 2 : 4);      // As[k][r]
	static constexpr int SB = BK + (CX ? 2 : 4);      // Bs[c][k]
	static constexpr int TILE_A = BK * SA;
	static constexpr int TILE_B = BN * SB;
	static constexpr int STAGE = TILE_A + TILE_B;     // elements of T
	static constexpr int KMAX = 512;                  // largest K of the scale vectors
	static constexpr int RING_BYTES = STAGES * STAGE * (int)sizeof(T);
	// TMA form: one mbarrier per stage and the CTA's abort flag
	static constexpr int MBAR_BYTES = (8 * STAGES + 8 + 15) / 16 * 16;
	// boxes land at 128-byte boundaries: every stage and tile is a multiple
	static_assert((TILE_A * (int)sizeof(T)) % 128 == 0 && (TILE_B * (int)sizeof(T)) % 128 == 0,
	              "tiles of 128-byte multiples");
	// the ring, the mbarriers (TMA form), then (modes with scale vectors or
	// a gather only) per-k scales, per-k inverse scales, per-row and
	// per-column scales and the gather rows, sized for this launch's K so
	// that the CTAs of the plain modes hold only the ring
	static constexpr int smem_bytes(int mode, int K, bool tma)
	{
		return RING_BYTES + (tma ? MBAR_BYTES : 0)
		       + ((mode & (GM_A_DD | GM_B_ROWD | GM_B_COLD | GM_B_GATHER))
		              ? (2 * K + BM + BN) * (int)sizeof(double) + K * 4
		              : 0);
	}
	static constexpr int SMEM_MAX = RING_BYTES + MBAR_BYTES + (2 * KMAX + BM + BN) * (int)sizeof(double) + KMAX * 4;
	static constexpr int WTM = BM / WM, WTN = BN / WN;
	static constexpr int MT = WTM / 8, NT = WTN / 8;
	static constexpr int A_PER_T = (BM * BK + THREADS - 1) / THREADS;
	static constexpr int B_PER_T = (BK * BN + THREADS - 1) / THREADS;
	static_assert(WTM % 8 == 0 && WTN % 8 == 0, "warp tile must be a multiple of 8");
	static_assert(BK % 4 == 0, "BK multiple of 4");
};

template <typename T, int BM, int BN, int BK, int WM, int WN, int STAGES, int MODE, bool TMA>
__global__ void __launch_bounds__(WM *WN * 32)
k_gemm(const __grid_constant__ GemmArgs<T> g)
{
	using Cfg = GemmCfg<T, BM, BN, BK, WM, WN, STAGES>;
	constexpr bool CX = Cfg::CX;
	static_assert(!(TMA && (MODE & GM_B_GATHER)), "the row gather loads element by element");
	extern __shared__ __align__(128) unsigned char gsm_raw[];
	T *sm = (T *)gsm_raw;
	uint64_t *mbar = (uint64_t *)(gsm_raw + Cfg::RING_BYTES);             // TMA: one per stage
	volatile int *abortp = (volatile int *)(mbar + STAGES);             // TMA: a wait timed out
	double *sdk = (double *)(gsm_raw + Cfg::RING_BYTES + (TMA ? Cfg::MBAR_BYTES : 0)); // per-k scale
	double *sdk2 = sdk + g.K;                                             // per-k 1/d (A_DD)
	double *sdr = sdk2 + g.K;                                             // per-row (A_DD)
	double *sdc = sdr + BM;                                               // per-column (B_COLD)
	int *sgi = (int *)(sdc + BN);                                         // gather rows
	const int b = g.b0 + blockIdx.z;
	const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
	if (b >= g.batch || m0 >= g.M || n0 >= g.N) return;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wm = warp % WM, wn = warp / WM;
	const T *A = g.A + g.aA.off(b);
	const T *B = g.B + g.aB.off(b);
	T *Cp = g.C + g.aC.off(b);
	const int M = g.M, N = g.N, K = g.K;

	// scale vectors and gather indices for this item, staged once
	if (MODE & (GM_A_DD | GM_B_ROWD | GM_B_COLD)) {
		const double *d = g.d + g.aD.off(b);
		if (MODE & GM_A_DD) {
			const double *di = g.dinv + g.aD.off(b);
			for (int q = tid; q < K; q += Cfg::THREADS) sdk2[q] = di[q];
			for (int q = tid; q < BM; q += Cfg::THREADS) sdr[q] = (m0 + q < M) ? d[m0 + q] : 0.0;
		}
		if (MODE & GM_B_ROWD)
			for (int q = tid; q < K; q += Cfg::THREADS) sdk[q] = d[q];
		if (MODE & GM_B_COLD)
			for (int q = tid; q < BN; q += Cfg::THREADS) sdc[q] = (n0 + q < N) ? d[n0 + q] : 0.0;
	}
	if (MODE & GM_B_GATHER) {
		const int *gi = g.gidx + g.aG.off(b);
		for (int q = tid; q < K; q += Cfg::THREADS) sgi[q] = gi[q];
	}
	if (MODE & (GM_A_DD | GM_B_ROWD | GM_B_COLD | GM_B_GATHER)) __syncthreads();

	int kt0 = 0;
	if (MODE & GM_A_UPPER) kt0 = m0 / BK;
	const int nkt = (K + BK - 1) / BK;

	// TMA form: the boxes of k-tile kt into ring stage `stage`, issued by one
	// thread; the stage's mbarrier completes when both boxes have landed
	constexpr int E = CX ? 2 : 1;   // doubles per element: tensor maps count doubles
	constexpr uint32_t TX = (uint32_t)((Cfg::TILE_A + ((MODE & GM_B_IDENT) ? 0 : Cfg::TILE_B)) * sizeof(T));
	const int zA = g.tzA ? b % g.aA.div : 0, wA = g.twA ? b / g.aA.div : 0;
	const int zB = g.tzB ? b % g.aB.div : 0, wB = g.twB ? b / g.aB.div : 0;
	auto issue_tma = [&](int kt, int stage) {
		T *As = sm + stage * Cfg::STAGE;
		T *Bs = As + Cfg::TILE_A;
		const uint32_t mb = smem_u32(mbar + stage);
		mbar_arrive_tx(mb, TX);
		tma_load_4d(smem_u32(As), &g.tmA, E * m0, kt * BK, zA, wA, mb);
		if (!(MODE & GM_B_IDENT)) tma_load_4d(smem_u32(Bs), &g.tmB, E * kt * BK, n0, zB, wB, mb);
	};
	if constexpr (TMA) {
		if (tid == 0) {
			for (int s = 0; s < STAGES; s++) mbar_init(smem_u32(mbar + s), 1);
			*abortp = 0;
			asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		}
		__syncthreads();
	}

	auto issue = [&](int kt, int stage) {
		T *As = sm + stage * Cfg::STAGE;
		T *Bs = As + Cfg::TILE_A;
		const int k0 = kt * BK;
#pragma unroll
		for (int q = 0; q < Cfg::A_PER_T; q++) {
			const int idx = tid + q * Cfg::THREADS;
			if (idx < BM * BK) {
				const int r = idx % BM, k = idx / BM;
				const int gr = m0 + r, gk = k0 + k;
				const bool ok = gr < M && gk < K;
				cp_async_el<T>(As + k * Cfg::SA + r, ok ? A + gr + (long long)gk * g.lda : A, ok);
			}
		}
		if (!(MODE & GM_B_IDENT)) {
#pragma unroll
			for (int q = 0; q < Cfg::B_PER_T; q++) {
				const int idx = tid + q * Cfg::THREADS;
				if (idx < BK * BN) {
					const int k = idx % BK, c = idx / BK;
					const int gk = k0 + k, gc = n0 + c;
					const bool ok = gk < K && gc < N;
					int row = gk;
					if (MODE & GM_B_GATHER) row = ok ? sgi[gk] : 0;
					cp_async_el<T>(Bs + c * Cfg::SB + k, ok ? B + row + (long long)gc * g.ldb : B, ok);
				}
			}
		}
	};

	double acc_r[Cfg::MT][Cfg::NT][2];
	double acc_i[CX ? Cfg::MT : 1][CX ? Cfg::NT : 1][2];
#pragma unroll
	for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
		for (int j = 0; j < Cfg::NT; j++) {
			acc_r[i][j][0] = acc_r[i][j][1] = 0.0;
			if constexpr (CX) acc_i[i][j][0] = acc_i[i][j][1] = 0.0;
		}

	// prologue
	if constexpr (TMA) {
		if (tid == 0)
			for (int sidx = 0; sidx < STAGES - 1; sidx++)
				if (kt0 + sidx < nkt) issue_tma(kt0 + sidx, sidx);
	} else {
#pragma unroll
		for (int sidx = 0; sidx < STAGES - 1; sidx++) {
			if (kt0 + sidx < nkt) issue(kt0 + sidx, sidx);
			cp_commit();
		}
	}
	const int gq = lane >> 2, tq = lane & 3;
	// this lane's row scales (A_DD) and column scales (B_COLD) do not change
	// along k: read once instead of at every fragment
	double srow[Cfg::MT], scol[Cfg::NT];
#pragma unroll
	for (int i = 0; i < Cfg::MT; i++) srow[i] = (MODE & GM_A_DD) ? sdr[wm * Cfg::WTM + i * 8 + gq] : 1.0;
#pragma unroll
	for (int j = 0; j < Cfg::NT; j++) scol[j] = (MODE & GM_B_COLD) ? sdc[wn * Cfg::WTN + j * 8 + gq] : 1.0;
	for (int kt = kt0; kt < nkt; kt++) {
		const int it = kt - kt0;
		// the stage written next is the one every warp finished at kt - 1
		if constexpr (TMA) {
			mbar_wait_bounded(smem_u32(mbar + it % STAGES), (it / STAGES) & 1, abortp, g.err);
			__syncthreads();
			const int nk = kt + STAGES - 1;
			if (tid == 0 && nk < nkt) issue_tma(nk, (nk - kt0) % STAGES);
		} else {
			cp_wait<STAGES - 2>();
			__syncthreads();
			const int nk = kt + STAGES - 1;
			if (nk < nkt) issue(nk, (nk - kt0) % STAGES);
			cp_commit();
		}
		const int stage = it % STAGES;
		const T *As = sm + stage * Cfg::STAGE;
		const T *Bs = As + Cfg::TILE_A;
		const int k0 = kt * BK;
#pragma unroll
		for (int kk = 0; kk < BK; kk += 4) {
			const int gk = k0 + kk + tq;
			double fa[Cfg::MT], fb[Cfg::NT], fai[CX ? Cfg::MT : 1], fbi[CX ? Cfg::NT : 1];
			double ka = 1.0, kb = 1.0;
			if (MODE & GM_A_DD) ka = (gk < K) ? sdk2[gk] : 0.0;
			if (MODE & GM_B_ROWD) kb = (gk < K) ? sdk[gk] : 0.0;
#pragma unroll
			for (int i = 0; i < Cfg::MT; i++) {
				const int r = wm * Cfg::WTM + i * 8 + gq;
				const T v = As[(kk + tq) * Cfg::SA + r];
				double xr, xi;
				split(v, xr, xi);
				double sc = ka;
				if (MODE & GM_A_DD) sc *= srow[i];
				if ((MODE & GM_A_UPPER) && (m0 + r > gk)) sc = 0.0;
				fa[i] = xr * sc;
				if constexpr (CX) fai[i] = xi * sc;
			}
#pragma unroll
			for (int j = 0; j < Cfg::NT; j++) {
				const int c = wn * Cfg::WTN + j * 8 + gq;
				double xr, xi;
				if (MODE & GM_B_IDENT) {
					xr = (gk == n0 + c) ? 1.0 : 0.0;
					xi = 0.0;
				} else {
					const T v = Bs[c * Cfg::SB + kk + tq];
					split(v, xr, xi);
				}
				double sc = kb;
				if (MODE & GM_B_COLD) sc *= scol[j];
				fb[j] = xr * sc;
				if constexpr (CX) fbi[j] = xi * sc;
			}
#pragma unroll
			for (int i = 0; i < Cfg::MT; i++)
#pragma unroll
				for (int j = 0; j < Cfg::NT; j++) {
					dmma(acc_r[i][j][0], acc_r[i][j][1], fa[i], fb[j]);
					if constexpr (CX) {
						dmma(acc_r[i][j][0], acc_r[i][j][1], -fai[i], fbi[j]);
						dmma(acc_i[i][j][0], acc_i[i][j][1], fa[i], fbi[j]);
						dmma(acc_i[i][j][0], acc_i[i][j][1], fai[i], fb[j]);
					}
				}
		}
	}
	if constexpr (!TMA) cp_wait<0>();

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
