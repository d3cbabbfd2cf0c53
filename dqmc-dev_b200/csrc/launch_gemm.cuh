// Launcher of the batched GEMM kernel (gemm.cuh): mode dispatch and tile
// choice.  Included by launch_gemm_r.cu and launch_gemm_c.cu only.
#pragma once

#include <cstdlib>

#include "dqmc_b200.h"
#include "launch.cuh"

namespace dq {

template <typename T, int BM, int BN, int BK, int WM, int WN, int ST, int MODE, bool TMA>
static int launch_gemm_form(const GemmArgs<T> &g, cudaStream_t st)
{
	using Cfg = GemmCfg<T, BM, BN, BK, WM, WN, ST>;
	if (raise_smem(k_gemm<T, BM, BN, BK, WM, WN, ST, MODE, TMA>, Cfg::SMEM_MAX, true) != cudaSuccess)
		return DQMC_E_ARG;
	// the grid's z extent is at most 65535: larger batches take several launches
	for (int b0 = 0; b0 < g.batch; b0 += 65535) {
		GemmArgs<T> gc = g;
		gc.b0 = b0;
		dim3 grid((g.M + BM - 1) / BM, (g.N + BN - 1) / BN, min(65535, g.batch - b0));
		k_gemm<T, BM, BN, BK, WM, WN, ST, MODE, TMA>
			<<<grid, Cfg::THREADS, Cfg::smem_bytes(MODE, g.K, TMA), st>>>(gc);
	}
	return 0;
}

// the TMA form wherever tensor maps describe both operands (not the row
// gather, whose rows come from a table); the element-wise form otherwise.
// DQMC_GEMM_TMA=0 in the environment selects the element-wise form always.
template <typename T, int BM, int BN, int BK, int WM, int WN, int ST, int MODE>
static int launch_gemm_mode(const GemmArgs<T> &g, cudaStream_t st)
{
	using Cfg = GemmCfg<T, BM, BN, BK, WM, WN, ST>;
	if constexpr (!(MODE & GM_B_GATHER)) {
		static const bool off = [] {
			const char *e = getenv("DQMC_GEMM_TMA");
			return e && e[0] == '0';
		}();
		constexpr int ED = is_cplx<T>::value ? 2 : 1;
		GemmArgs<T> gt = g;
		if (!off &&
		    tma_map_operand(&gt.tmA, &gt.tzA, &gt.twA, g.A, ED, g.M, g.K, g.lda, g.aA, g.batch, Cfg::SA, BK) &&
		    ((MODE & GM_B_IDENT) ||
		     tma_map_operand(&gt.tmB, &gt.tzB, &gt.twB, g.B, ED, g.K, g.N, g.ldb, g.aB, g.batch, Cfg::SB, BN)))
			return launch_gemm_form<T, BM, BN, BK, WM, WN, ST, MODE, true>(gt, st);
	}
	return launch_gemm_form<T, BM, BN, BK, WM, WN, ST, MODE, false>(g, st);
}

template <typename T, int BM, int BN, int BK, int WM, int WN, int ST>
static int launch_gemm_cfg(const GemmArgs<T> &g, cudaStream_t st)
{
	switch (g.mode) {
	case 0: return launch_gemm_mode<T, BM, BN, BK, WM, WN, ST, 0>(g, st);
	case GM_A_DD: return launch_gemm_mode<T, BM, BN, BK, WM, WN, ST, GM_A_DD>(g, st);
	case GM_B_ROWD: return launch_gemm_mode<T, BM, BN, BK, WM, WN, ST, GM_B_ROWD>(g, st);
	case GM_B_COLD: return launch_gemm_mode<T, BM, BN, BK, WM, WN, ST, GM_B_COLD>(g, st);
	case GM_B_IDENT: return launch_gemm_mode<T, BM, BN, BK, WM, WN, ST, GM_B_IDENT>(g, st);
	case GM_A_UPPER | GM_B_GATHER:
		return launch_gemm_mode<T, BM, BN, BK, WM, WN, ST, GM_A_UPPER | GM_B_GATHER>(g, st);
	default: return DQMC_E_ARG;
	}
}

// tile choice: least padded area, larger tiles on ties
template <typename T>
int launch_gemm(const GemmArgs<T> &g, cudaStream_t st)
{
	// the scale vectors and gather indices of these modes are staged per K
	const bool k_staged = g.mode & (GM_A_DD | GM_B_ROWD | GM_B_GATHER);
	if ((k_staged && g.K > 512) || g.M < 1 || g.N < 1 || g.K < 1 || g.batch < 1) return DQMC_E_ARG;
	auto pad = [&](int t) { return (long long)((g.M + t - 1) / t * t) * ((g.N + t - 1) / t * t); };
	const long long p64 = pad(64), p48 = pad(48), p32 = pad(32);
	if constexpr (is_cplx<T>::value) {
		if (p64 <= p48 && p64 <= p32) return launch_gemm_cfg<T, 64, 64, 8, 4, 2, 3>(g, st);
		if (p48 <= p32) return launch_gemm_cfg<T, 48, 48, 8, 2, 2, 3>(g, st);
		return launch_gemm_cfg<T, 32, 32, 8, 2, 2, 3>(g, st);
	} else {
		if (p64 <= p48 && p64 <= p32) return launch_gemm_cfg<T, 64, 64, 16, 2, 2, 3>(g, st);
		// k-depth 8: 24-28 KB per CTA, 7-8 CTAs per SM (2-5% over k-depth 16
		// with its 4-5 CTAs at 512 x 144^3)
		if (p48 <= p32) return launch_gemm_cfg<T, 48, 48, 8, 2, 2, 3>(g, st);
		return launch_gemm_cfg<T, 32, 32, 16, 2, 2, 4>(g, st);
	}
}

}  // namespace dq
