// Measurement contractions of the (half-wrapped) Green's functions into the
// per-chain accumulators, reference src/meas.c:66-120 (measure_eqlt,
// always-on part), 728-801 (measure_uneqlt, always-on part) and 860-964
// (the meas_bond_corr block of measure_uneqlt).
//
// Each output class r (a distance class of map_ij or a bond-pair class of
// map_bb) is owned by one thread, which sums its (i, j) pairs in the
// reference's loop order from an inverse map built on the host: no atomics,
// and the accumulated value depends on nothing but the inputs.
#pragma once

#include "common.cuh"
#include "dqmc_b200.h"

namespace dq {

// accumulator layout, per chain (each group only when its toggle is on)
//   eqlt:   sign | density, density_u, density_d, double_occ [num_i]
//           | g00, g00_u, g00_d, nn, xx, zz, pair_sw [num_ij]
//           | uuuu, dddd, dduu, uudd [num_ij^2]                 (gen_suscept)
//           | chi [num_plaq_accum]                              (chiral)
//           | kk [num_bb], kv, kn [num_bs], vv, vn [num_ij]     (energy_corr)
//           | j, jn [num_b_accum], j2 [num_b2_accum]            (local_JQ)
//   uneqlt: sign | gt0, gt0_u, gt0_d, nn, xx, zz, pair_sw [L][num_ij]
//           | uuuu, dddd, dduu, uudd [L][num_ij^2]              (gen_suscept)
//           | pair_bb [L][num_bb]                   (bond_corr or pair_bb_only)
//           | jj, jsjs, kk, ksks [L][num_bb]                    (bond_corr)
//           | j2jn [L][num_b2b], jnj2 [L][num_bb2], jnjn, jnj, jjn [L][num_bb]
//                                                               (thermal)
//           | pair_b2b2, j2j2 [L][num_b2b2], j2j [L][num_b2b], jj2 [L][num_bb2],
//             js2js2, k2k2, ks2ks2 [L][num_b2b2]                (2bond_corr)
//           | kv, kn [L][num_bs], vv, vn [L][num_ij]            (energy_corr)
//           | nem_nnnn, nem_ssss [L][num_bb]                    (nematic_corr)
// The dataset names and sizes are those of the reference's data.c:441-522.
struct AccLayout {
	long long eq_size, ue_size;
	long long gs, chi, energy, jq;                                   // eqlt groups
	long long ue_gs, pair_bb, bond, thermal, two_bond, ue_energy, nem;  // uneqlt groups
};

inline AccLayout acc_layout(const dqmc_params &p)
{
	AccLayout a;
	const long long L = p.L, ni = p.num_i, nij = p.num_ij, nbb = p.num_bb, nbs = p.num_bs;
	long long o = 1 + 4 * ni + 7 * nij;
	a.gs = o;     o += p.meas_gen_suscept ? 4 * nij * nij : 0;
	a.chi = o;    o += p.meas_chiral ? p.num_plaq_accum : 0;
	a.energy = o; o += p.meas_energy_corr ? nbb + 2 * nbs + 2 * nij : 0;
	a.jq = o;     o += p.meas_local_JQ ? 2LL * p.num_b_accum + p.num_b2_accum : 0;
	a.eq_size = o;
	o = 1 + 7 * nij * L;
	a.ue_gs = o;     o += p.meas_gen_suscept ? 4 * nij * nij * L : 0;
	a.pair_bb = o;   o += (p.meas_bond_corr || p.meas_pair_bb_only) ? nbb * L : 0;
	a.bond = o;      o += p.meas_bond_corr ? 4 * nbb * L : 0;
	a.thermal = o;   o += p.meas_thermal ? ((long long)p.num_b2b + p.num_bb2 + 3 * nbb) * L : 0;
	a.two_bond = o;  o += p.meas_2bond_corr ? (5LL * p.num_b2b2 + p.num_b2b + p.num_bb2) * L : 0;
	a.ue_energy = o; o += p.meas_energy_corr ? (2 * nbs + 2 * nij) * L : 0;
	a.nem = o;       o += p.meas_nematic_corr ? 2 * nbb * L : 0;
	a.ue_size = p.period_uneqlt > 0 ? o : 0;
	return a;
}

template <typename T>
struct MeasArgs {
	int N, L, nchain, num_i, num_ij, num_b, num_bb;
	int degen_i, degen_ij, degen_bb;
	const T *G;            // eqlt: [chain][2][N*N]
	const T *G0t, *Gtt, *Gt0;   // uneqlt: [chain][2][L][N*N]
	const T *phase;        // [chain]
	const int *i_off, *i_idx;   // inverse of map_i
	const int *ij_off, *ij_idx; // inverse of map_ij, entries i + N*j
	const int *bb_off, *bb_idx; // inverse of map_bb, entries b + num_b*c
	const int *bonds;      // [2][num_b]
	const T *peu, *ped;    // Peierls phases (complex path)
	T *acc;                // per chain, stride acc_stride
	long long acc_stride;
	int *n_sample;         // [chain]
	int bond;              // accumulate the bond correlators
	// the measurement toggles (meas.c:125-714, 827-858, 966-1363) and the
	// inverse maps of their classes; `lay` holds the group offsets
	int energy, thermal, two_bond, nematic, chiral, local_jq, gen_suscept, pair_bb_only;
	int Nx, Ny, num_bs, num_b2, num_b2b, num_bb2, num_b2b2, num_plaq;
	int degen_bs, degen_b2b, degen_bb2, degen_b2b2, degen_plaq, degen_b, degen_b2;
	int num_plaq_accum, num_b_accum, num_b2_accum;
	const int *bs_off, *bs_idx;      // inverse of map_bs, entries b + num_b*j
	const int *bb2_off, *bb2_idx;    // inverse of map_bb2, entries b + num_b2*c
	const int *b2b_off, *b2b_idx;    // inverse of map_b2b, entries b + num_b*c
	const int *b2b2_off, *b2b2_idx;  // inverse of map_b2b2, entries b + num_b2*c
	const int *nem_off, *nem_idx;    // inverse of map_bb over b, c < 2N
	const int *plaq_off, *plaq_idx;  // inverse of map_plaq
	const int *b_off, *b_idx;        // inverse of map_b
	const int *b2_off, *b2_idx;      // inverse of map_b2
	const int *plaqs, *bond2s;       // [3][num_plaq], [2][num_b2]
	const T *pp_u, *pp_d, *ppr_u, *ppr_d;  // two-hop phases [num_b2]
	AccLayout lay;
};

template <typename T>
__device__ inline T peierls(const T *p, int idx)
{
	if constexpr (is_cplx<T>::value) return p[idx];
	else return 1.0;
}

template <typename T>
__global__ void k_meas_eqlt(MeasArgs<T> a)
{
	// grid (chain, class chunk): each warp sums whole classes, its lanes
	// striding over the class's entries, reduced by a fixed butterfly (a
	// deterministic order); the chunks split a chain's classes
	const int c = blockIdx.x, chunk = blockIdx.y;
	if (c >= a.nchain) return;
	const int lane = threadIdx.x & 31, gw = chunk * (blockDim.x >> 5) + (threadIdx.x >> 5);
	const int ngw = gridDim.y * (blockDim.x >> 5);
	const int N = a.N;
	const size_t NN = (size_t)N * N;
	const T *gu = a.G + (size_t)(2 * c) * NN, *gd = gu + NN;
	extern __shared__ __align__(16) unsigned char smraw[];
	T *du = (T *)smraw, *dd = du + N;
	for (int i = threadIdx.x; i < N; i += blockDim.x) {
		du[i] = gu[i + (size_t)N * i];
		dd[i] = gd[i + (size_t)N * i];
	}
	__syncthreads();
	const T phase = a.phase[c];
	T *acc = a.acc + (size_t)c * a.acc_stride;
	const int ni = a.num_i, nij = a.num_ij;
	if (chunk == 0 && threadIdx.x == 0) {
		acc[0] = acc[0] + phase;
		a.n_sample[c] += 1;
	}
	const T pre_i = phase / (double)a.degen_i;
	for (int r = gw; r < ni; r += ngw) {
		T s0 = zero<T>(), s1 = zero<T>(), s2 = zero<T>(), s3 = zero<T>();
		for (int q = a.i_off[r] + lane; q < a.i_off[r + 1]; q += 32) {
			const int i = a.i_idx[q];
			const T guii = du[i], gdii = dd[i];
			s0 += 2.0 - guii - gdii;
			s1 += 1.0 - guii;
			s2 += 1.0 - gdii;
			s3 += (1.0 - guii) * (1.0 - gdii);
		}
		s0 = warp_sum(s0);
		s1 = warp_sum(s1);
		s2 = warp_sum(s2);
		s3 = warp_sum(s3);
		if (lane == 0) {
			acc[1 + r] += pre_i * s0;
			acc[1 + ni + r] += pre_i * s1;
			acc[1 + 2 * ni + r] += pre_i * s2;
			acc[1 + 3 * ni + r] += pre_i * s3;
		}
	}
	const T pre = phase / (double)a.degen_ij;
	T *a2 = acc + 1 + 4 * ni;
	for (int r = gw; r < nij; r += ngw) {
		T g00 = zero<T>(), g00u = zero<T>(), g00d = zero<T>(), nn = zero<T>();
		T xx = zero<T>(), zz = zero<T>(), ps = zero<T>(), vv = zero<T>(), vn = zero<T>();
		for (int q = a.ij_off[r] + lane; q < a.ij_off[r + 1]; q += 32) {
			const int e = a.ij_idx[q];
			const int i = e % N, j = e / N;
			const double delta = (i == j) ? 1.0 : 0.0;
			const T guii = du[i], gdii = dd[i], gujj = du[j], gdjj = dd[j];
			const T guij = gu[i + (size_t)N * j], gdij = gd[i + (size_t)N * j];
			const T guji = gu[j + (size_t)N * i], gdji = gd[j + (size_t)N * i];
			const T pu = guij * peierls(a.peu, j + N * i), pd = gdij * peierls(a.ped, j + N * i);
			g00 += 0.5 * (pu + pd);
			g00u += pu;
			g00d += pd;
			const T x = delta * (guii + gdii) - (guji * guij + gdji * gdij);
			nn += (2.0 - guii - gdii) * (2.0 - gujj - gdjj) + x;
			xx += 0.25 * (delta * (guii + gdii) - (guji * gdij + gdji * guij));
			zz += 0.25 * ((gdii - guii) * (gdjj - gujj) + x);
			ps += guij * gdij;
			if (a.energy) {
				// meas.c:113-118
				const T nun = (1.0 - guii) * (1.0 - gujj) + (delta - guji) * guij;
				const T ndn = (1.0 - gdii) * (1.0 - gdjj) + (delta - gdji) * gdij;
				vv += nun * ndn;
				vn += nun * (1.0 - gdii) + (1.0 - guii) * ndn;
			}
		}
		g00 = warp_sum(g00);
		g00u = warp_sum(g00u);
		g00d = warp_sum(g00d);
		nn = warp_sum(nn);
		xx = warp_sum(xx);
		zz = warp_sum(zz);
		ps = warp_sum(ps);
		if (a.energy) {
			vv = warp_sum(vv);
			vn = warp_sum(vn);
		}
		if (lane != 0) continue;
		if (a.energy) {
			T *ae = acc + a.lay.energy + a.num_bb + 2 * (size_t)a.num_bs;
			ae[r] += pre * vv;
			ae[nij + r] += pre * vn;
		}
		a2[r] += pre * g00;
		a2[nij + r] += pre * g00u;
		a2[2 * nij + r] += pre * g00d;
		a2[3 * nij + r] += pre * nn;
		a2[4 * nij + r] += pre * xx;
		a2[5 * nij + r] += pre * zz;
		a2[6 * nij + r] += pre * ps;
	}
}

// grid (chain, t); at most 128 registers a thread for complex (two CTAs per
// SM instead of one at 132), 64 for real (four CTAs, as the compiler chooses)
template <typename T>
__global__ void __launch_bounds__(256, is_cplx<T>::value ? 2 : 4) k_meas_uneqlt(MeasArgs<T> a)
{
	const int c = blockIdx.x, t = blockIdx.y;
	if (c >= a.nchain || t >= a.L) return;
	const int N = a.N, L = a.L;
	const size_t NN = (size_t)N * N;
	// slice-major stacks: slice t of item b at (t * 2 nchain + b) N^2
	const size_t su = ((size_t)t * 2 * a.nchain + 2 * c) * NN, sd = su + NN;
	const T *u0t = a.G0t + su, *utt = a.Gtt + su, *ut0 = a.Gt0 + su;
	const T *d0t = a.G0t + sd, *dtt = a.Gtt + sd, *dt0 = a.Gt0 + sd;
	const T *u00 = a.Gtt + (size_t)2 * c * NN, *d00 = u00 + NN;
	const T phase = a.phase[c];
	T *acc = a.acc + (size_t)c * a.acc_stride;
	const int nij = a.num_ij;
	if (t == 0 && threadIdx.x == 0) {
		acc[0] = acc[0] + phase;
		a.n_sample[c] += 1;
	}
	const double dt = (t == 0) ? 1.0 : 0.0;
	const T pre = phase / (double)a.degen_ij;
	T *a2 = acc + 1;
	for (int r = threadIdx.x; r < nij; r += blockDim.x) {
		T g0 = zero<T>(), g0u = zero<T>(), g0d = zero<T>(), nn = zero<T>();
		T xx = zero<T>(), zz = zero<T>(), ps = zero<T>(), vv = zero<T>(), vn = zero<T>();
		for (int q = a.ij_off[r]; q < a.ij_off[r + 1]; q++) {
			const int e = a.ij_idx[q];
			const int i = e % N, j = e / N;
			const double dtij = (i == j) ? dt : 0.0;
			const T guii = utt[i + (size_t)N * i], guij = ut0[i + (size_t)N * j];
			const T guji = u0t[j + (size_t)N * i], gujj = u00[j + (size_t)N * j];
			const T gdii = dtt[i + (size_t)N * i], gdij = dt0[i + (size_t)N * j];
			const T gdji = d0t[j + (size_t)N * i], gdjj = d00[j + (size_t)N * j];
			const T pu = guij * peierls(a.peu, j + N * i), pd = gdij * peierls(a.ped, j + N * i);
			g0 += 0.5 * (pu + pd);
			g0u += pu;
			g0d += pd;
			const T x = dtij * (guii + gdii) - (guji * guij + gdji * gdij);
			nn += (2.0 - guii - gdii) * (2.0 - gujj - gdjj) + x;
			xx += 0.25 * (dtij * (guii + gdii) - (guji * gdij + gdji * guij));
			zz += 0.25 * ((gdii - guii) * (gdjj - gujj) + x);
			ps += guij * gdij;
			if (a.energy) {
				// meas.c:791-798
				const T nun = (1.0 - guii) * (1.0 - gujj) + (dtij - guji) * guij;
				const T ndn = (1.0 - gdii) * (1.0 - gdjj) + (dtij - gdji) * gdij;
				vv += nun * ndn;
				vn += nun * (1.0 - gdii) + (1.0 - guii) * ndn;
			}
		}
		const size_t o = (size_t)nij * t + r, st = (size_t)nij * L;
		if (a.energy) {
			T *ae = acc + a.lay.ue_energy + 2 * (size_t)a.num_bs * L;
			ae[o] += pre * vv;
			ae[st + o] += pre * vn;
		}
		a2[o] += pre * g0;
		a2[st + o] += pre * g0u;
		a2[2 * st + o] += pre * g0d;
		a2[3 * st + o] += pre * nn;
		a2[4 * st + o] += pre * xx;
		a2[5 * st + o] += pre * zz;
		a2[6 * st + o] += pre * ps;
	}
	if (!a.bond && !a.pair_bb_only) return;
	const int nb = a.num_b, nbb = a.num_bb;
	T *a3 = acc + a.lay.pair_bb;
	const T preb = phase / (double)a.degen_bb;
	for (int bb = threadIdx.x; bb < nbb; bb += blockDim.x) {
		T pbb = zero<T>(), jj = zero<T>(), jsjs = zero<T>(), kk = zero<T>(), ksks = zero<T>();
		for (int q = a.bb_off[bb]; q < a.bb_off[bb + 1]; q++) {
			const int e = a.bb_idx[q];
			const int b = e % nb, cc = e / nb;
			const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
			const int j0 = a.bonds[cc], j1 = a.bonds[cc + nb];
			const T pui0i1 = peierls(a.peu, i0 + N * i1), pui1i0 = peierls(a.peu, i1 + N * i0);
			const T pdi0i1 = peierls(a.ped, i0 + N * i1), pdi1i0 = peierls(a.ped, i1 + N * i0);
			const T puj0j1 = peierls(a.peu, j0 + N * j1), puj1j0 = peierls(a.peu, j1 + N * j0);
			const T pdj0j1 = peierls(a.ped, j0 + N * j1), pdj1j0 = peierls(a.ped, j1 + N * j0);
			const T gui1i0 = utt[i1 + i0 * N], gui0i1 = utt[i0 + i1 * N];
			const T gui0j0 = ut0[i0 + j0 * N], gui1j0 = ut0[i1 + j0 * N];
			const T gui0j1 = ut0[i0 + j1 * N], gui1j1 = ut0[i1 + j1 * N];
			const T guj0i0 = u0t[j0 + i0 * N], guj1i0 = u0t[j1 + i0 * N];
			const T guj0i1 = u0t[j0 + i1 * N], guj1i1 = u0t[j1 + i1 * N];
			const T guj1j0 = u00[j1 + j0 * N], guj0j1 = u00[j0 + j1 * N];
			const T gdi1i0 = dtt[i1 + i0 * N], gdi0i1 = dtt[i0 + i1 * N];
			const T gdi0j0 = dt0[i0 + j0 * N], gdi1j0 = dt0[i1 + j0 * N];
			const T gdi0j1 = dt0[i0 + j1 * N], gdi1j1 = dt0[i1 + j1 * N];
			const T gdj0i0 = d0t[j0 + i0 * N], gdj1i0 = d0t[j1 + i0 * N];
			const T gdj0i1 = d0t[j0 + i1 * N], gdj1i1 = d0t[j1 + i1 * N];
			const T gdj1j0 = d00[j1 + j0 * N], gdj0j1 = d00[j0 + j1 * N];
			pbb += 0.5 * (gui0j0 * gdi1j1 + gui1j0 * gdi0j1 + gui0j1 * gdi1j0 + gui1j1 * gdi0j0);
			if (!a.bond) continue;   // pair_bb_only (meas.c:827-858)
			const double e00 = (i0 == j0) ? dt : 0.0, e10 = (i1 == j0) ? dt : 0.0;
			const double e01 = (i0 == j1) ? dt : 0.0, e11 = (i1 == j1) ? dt : 0.0;
			// the eight exchange terms of meas.c:932-941, with their phases
			const T x = pdi0i1 * pdj0j1 * ((e01 - gdj1i0) * gdi1j0) + pdi1i0 * pdj1j0 * ((e10 - gdj0i1) * gdi0j1)
			          + pui0i1 * puj0j1 * ((e01 - guj1i0) * gui1j0) + pui1i0 * puj1j0 * ((e10 - guj0i1) * gui0j1);
			const T y = pdi0i1 * pdj1j0 * ((e00 - gdj0i0) * gdi1j1) + pdi1i0 * pdj0j1 * ((e11 - gdj1i1) * gdi0j0)
			          + pui0i1 * puj1j0 * ((e00 - guj0i0) * gui1j1) + pui1i0 * puj0j1 * ((e11 - guj1i1) * gui0j0);
			const T t0 = pui1i0 * gui0i1, t1 = pui0i1 * gui1i0, t2 = pdi1i0 * gdi0i1, t3 = pdi0i1 * gdi1i0;
			const T t4 = puj1j0 * guj0j1, t5 = puj0j1 * guj1j0, t6 = pdj1j0 * gdj0j1, t7 = pdj0j1 * gdj1j0;
			jj += (t0 - t1 + t2 - t3) * (t4 - t5 + t6 - t7) + x - y;
			jsjs += (t0 - t1 - t2 + t3) * (t4 - t5 - t6 + t7) + x - y;
			kk += (t0 + t1 + t2 + t3) * (t4 + t5 + t6 + t7) + x + y;
			ksks += (t0 + t1 - t2 - t3) * (t4 + t5 - t6 - t7) + x + y;
		}
		const size_t o = (size_t)nbb * t + bb, st = (size_t)nbb * L;
		a3[o] += preb * pbb;
		if (!a.bond) continue;
		a3[st + o] += preb * jj;
		a3[2 * st + o] += preb * jsjs;
		a3[3 * st + o] += preb * kk;
		a3[4 * st + o] += preb * ksks;
	}
}

}  // namespace dq
