// The reference's optional measurements (src/meas.c:125-471, 473-714,
// 827-858, 966-1363): generalised susceptibility, chiral, energy, local heat
// current (equal time) and energy, generalised susceptibility, thermal,
// two-bond and nematic correlators (unequal time).  The always-on parts,
// vv / vn and pair_bb_only ride in k_meas_eqlt / k_meas_uneqlt (meas.cuh).
//
// As there, every output class is owned by one thread that sums its members
// in the reference's loop order (inverse maps built on the host), so the
// results do not depend on scheduling.  The Wick contractions are the
// reference's, term for term: they are the physics of each correlator.
//
// The generalised susceptibility of the reference is a four-site loop
// (O(N^4) per sample) whose summand is a product f(i1, j2) g(i2, j1) of a
// pair in class k1 and a pair in class k2; its class sum is therefore the
// product of the two class sums, which is how it is computed here (O(N^2)).
#pragma once

#include "meas.cuh"

namespace dq {

// G[i + N j] of a column-major N x N matrix
template <typename T>
struct Gm {
	const T *p;
	int N;
	__device__ T operator()(int i, int j) const { return p[i + (size_t)N * j]; }
};

// ---------------------------------------------------------------- eqlt

// grid: one block per chain; gs_tmp: [chain][4][num_ij] class sums
template <typename T>
__global__ void k_meas_eqlt_x(MeasArgs<T> a, T *gs_tmp)
{
	const int c = blockIdx.x;
	if (c >= a.nchain) return;
	const int N = a.N;
	const size_t NN = (size_t)N * N;
	const Gm<T> gu{a.G + (size_t)(2 * c) * NN, N}, gd{a.G + (size_t)(2 * c + 1) * NN, N};
	const T phase = a.phase[c];
	T *acc = a.acc + (size_t)c * a.acc_stride;
	const int nij = a.num_ij;

	if (a.gen_suscept) {
		// meas.c:125-156: A[k] = sum over (i1, j2) of class k of
		// (delta - G[j2, i1]), B[k] = sum over (i2, j1) of class k of G[j1, i2]
		T *S = gs_tmp + (size_t)c * 4 * nij;
		for (int k = threadIdx.x; k < nij; k += blockDim.x) {
			T au = zero<T>(), bu = zero<T>(), ad = zero<T>(), bd = zero<T>();
			for (int q = a.ij_off[k]; q < a.ij_off[k + 1]; q++) {
				const int e = a.ij_idx[q];
				const int i = e % N, j = e / N;
				const double dl = (i == j) ? 1.0 : 0.0;
				const T u = gu(j, i), d = gd(j, i);
				au += dl - u;
				ad += dl - d;
				bu += u;
				bd += d;
			}
			S[k] = au; S[nij + k] = bu; S[2 * nij + k] = ad; S[3 * nij + k] = bd;
		}
		__syncthreads();
		const T pre = phase / ((double)a.Nx * a.Ny * a.Nx * a.Ny);
		const size_t n2 = (size_t)nij * nij;
		T *o = acc + a.lay.gs;
		for (size_t r = threadIdx.x; r < n2; r += blockDim.x) {
			const int k1 = (int)(r % nij), k2 = (int)(r / nij);
			const T au = S[k1], ad = S[2 * nij + k1], bu = S[nij + k2], bd = S[3 * nij + k2];
			o[r] += pre * (au * bu);            // uuuu
			o[n2 + r] += pre * (ad * bd);       // dddd
			o[2 * n2 + r] += pre * (ad * bu);   // dduu
			o[3 * n2 + r] += pre * (au * bd);   // uudd
		}
	}

	if (a.chiral) {
		// meas.c:163-208
		const int np = a.num_plaq;
		const T pre = phase / (double)a.degen_plaq;
		for (int r = threadIdx.x; r < a.num_plaq_accum; r += blockDim.x) {
			T s = zero<T>();
			for (int q = a.plaq_off[r]; q < a.plaq_off[r + 1]; q++) {
				const int pa = a.plaq_idx[q];
				const int i0 = a.plaqs[pa], i1 = a.plaqs[pa + np], i2 = a.plaqs[pa + 2 * np];
				const T gui0i0 = gu(i0, i0), gui1i1 = gu(i1, i1), gui2i2 = gu(i2, i2);
				const T gdi0i0 = gd(i0, i0), gdi1i1 = gd(i1, i1), gdi2i2 = gd(i2, i2);
				const T gui0i1 = gu(i0, i1), gui1i0 = gu(i1, i0), gui0i2 = gu(i0, i2);
				const T gui2i0 = gu(i2, i0), gui1i2 = gu(i1, i2), gui2i1 = gu(i2, i1);
				const T gdi0i1 = gd(i0, i1), gdi1i0 = gd(i1, i0), gdi0i2 = gd(i0, i2);
				const T gdi2i0 = gd(i2, i0), gdi1i2 = gd(i1, i2), gdi2i1 = gd(i2, i1);
				const T x =
				    gdi1i1 * gdi2i0 * gui0i2 - gdi0i2 * gdi2i1 * gui1i0 + gdi0i1 * gdi2i2 * gui1i0 -
				    gdi2i1 * gui0i2 * gui1i0 - gdi2i0 * gui0i2 * gui1i1 + gdi0i1 * gdi2i0 * gui1i2 -
				    gdi0i0 * gdi2i1 * gui1i2 + gdi2i1 * gui0i0 * gui1i2 + gdi2i0 * gui0i1 * gui1i2 -
				    gdi0i2 * gdi1i1 * gui2i0 + gdi0i2 * gui1i1 * gui2i0 + gdi0i1 * gui1i2 * gui2i0 -
				    gdi0i2 * gui1i0 * gui2i1 +
				    gdi1i2 * (gdi2i0 * gui0i1 + (gdi0i1 + gui0i1) * gui2i0 + (gdi0i0 - gui0i0) * gui2i1) -
				    gdi1i0 * (gdi2i1 * gui0i2 + (gdi0i2 + gui0i2) * gui2i1 + gui0i1 * (gdi2i2 - gui2i2)) -
				    gdi0i1 * gui1i0 * gui2i2;
				s += x;
			}
			acc[a.lay.chi + r] += pre * s;
		}
	}

	if (a.energy) {
		const int nb = a.num_b;
		T *ae = acc + a.lay.energy;   // kk [num_bb] | kv, kn [num_bs] | vv, vn (meas.cuh)
		// 1 bond - 1 site: kv, kn (meas.c:303-343)
		const T pre_bs = phase / (double)a.degen_bs;
		for (int r = threadIdx.x; r < a.num_bs; r += blockDim.x) {
			T kv = zero<T>(), kn = zero<T>();
			for (int q = a.bs_off[r]; q < a.bs_off[r + 1]; q++) {
				const int e = a.bs_idx[q];
				const int b = e % nb, j = e / nb;
				const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
				const T pui0i1 = peierls(a.peu, i0 + N * i1), pui1i0 = peierls(a.peu, i1 + N * i0);
				const T pdi0i1 = peierls(a.ped, i0 + N * i1), pdi1i0 = peierls(a.ped, i1 + N * i0);
				const double di0j = (i0 == j) ? 1.0 : 0.0, di1j = (i1 == j) ? 1.0 : 0.0;
				const T gui0j = gu(i0, j), guji0 = gu(j, i0), gdi0j = gd(i0, j), gdji0 = gd(j, i0);
				const T gui1j = gu(i1, j), guji1 = gu(j, i1), gdi1j = gd(i1, j), gdji1 = gd(j, i1);
				const T gui0i1 = gu(i0, i1), gui1i0 = gu(i1, i0);
				const T gdi0i1 = gd(i0, i1), gdi1i0 = gd(i1, i0);
				const T gujj = gu(j, j), gdjj = gd(j, j);
				const T ku = pui1i0 * (0.0 - gui0i1) + pui0i1 * (0.0 - gui1i0);
				const T kd = pdi1i0 * (0.0 - gdi0i1) + pdi0i1 * (0.0 - gdi1i0);
				const T xu = pui0i1 * (di0j - guji0) * gui1j + pui1i0 * (di1j - guji1) * gui0j;
				const T xd = pdi0i1 * (di0j - gdji0) * gdi1j + pdi1i0 * (di1j - gdji1) * gdi0j;
				kv += (ku * (1.0 - gujj) + xu) * (1.0 - gdjj) + (kd * (1.0 - gdjj) + xd) * (1.0 - gujj);
				kn += (ku + kd) * (2.0 - gujj - gdjj) + xu + xd;
			}
			ae[a.num_bb + r] += pre_bs * kv;
			ae[a.num_bb + a.num_bs + r] += pre_bs * kn;
		}
		// 1 bond - 1 bond: kk (meas.c:345-406)
		const T pre_bb = phase / (double)a.degen_bb;
		for (int r = threadIdx.x; r < a.num_bb; r += blockDim.x) {
			T kk = zero<T>();
			for (int q = a.bb_off[r]; q < a.bb_off[r + 1]; q++) {
				const int e = a.bb_idx[q];
				const int b = e % nb, cc = e / nb;
				const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
				const int j0 = a.bonds[cc], j1 = a.bonds[cc + nb];
				const T pui0i1 = peierls(a.peu, i0 + N * i1), pui1i0 = peierls(a.peu, i1 + N * i0);
				const T pdi0i1 = peierls(a.ped, i0 + N * i1), pdi1i0 = peierls(a.ped, i1 + N * i0);
				const T puj0j1 = peierls(a.peu, j0 + N * j1), puj1j0 = peierls(a.peu, j1 + N * j0);
				const T pdj0j1 = peierls(a.ped, j0 + N * j1), pdj1j0 = peierls(a.ped, j1 + N * j0);
				const double di0j0 = (i0 == j0) ? 1.0 : 0.0, di1j0 = (i1 == j0) ? 1.0 : 0.0;
				const double di0j1 = (i0 == j1) ? 1.0 : 0.0, di1j1 = (i1 == j1) ? 1.0 : 0.0;
				const T gui1i0 = gu(i1, i0), gui0i1 = gu(i0, i1), gui0j0 = gu(i0, j0);
				const T gui1j0 = gu(i1, j0), gui0j1 = gu(i0, j1), gui1j1 = gu(i1, j1);
				const T guj0i0 = gu(j0, i0), guj1i0 = gu(j1, i0), guj0i1 = gu(j0, i1);
				const T guj1i1 = gu(j1, i1), guj1j0 = gu(j1, j0), guj0j1 = gu(j0, j1);
				const T gdi1i0 = gd(i1, i0), gdi0i1 = gd(i0, i1), gdi0j0 = gd(i0, j0);
				const T gdi1j0 = gd(i1, j0), gdi0j1 = gd(i0, j1), gdi1j1 = gd(i1, j1);
				const T gdj0i0 = gd(j0, i0), gdj1i0 = gd(j1, i0), gdj0i1 = gd(j0, i1);
				const T gdj1i1 = gd(j1, i1), gdj1j0 = gd(j1, j0), gdj0j1 = gd(j0, j1);
				const T x = pui0i1 * puj0j1 * (di0j1 - guj1i0) * gui1j0 +
				            pui1i0 * puj1j0 * (di1j0 - guj0i1) * gui0j1 +
				            pdi0i1 * pdj0j1 * (di0j1 - gdj1i0) * gdi1j0 +
				            pdi1i0 * pdj1j0 * (di1j0 - gdj0i1) * gdi0j1;
				const T y = pui0i1 * puj1j0 * (di0j0 - guj0i0) * gui1j1 +
				            pui1i0 * puj0j1 * (di1j1 - guj1i1) * gui0j0 +
				            pdi0i1 * pdj1j0 * (di0j0 - gdj0i0) * gdi1j1 +
				            pdi1i0 * pdj0j1 * (di1j1 - gdj1i1) * gdi0j0;
				kk += (pui1i0 * gui0i1 + pui0i1 * gui1i0 + pdi1i0 * gdi0i1 + pdi0i1 * gdi1i0) *
				          (puj1j0 * guj0j1 + puj0j1 * guj1j0 + pdj1j0 * gdj0j1 + pdj0j1 * gdj1j0) +
				      x + y;
			}
			ae[r] += pre_bb * kk;
		}
	}

	if (a.local_jq) {
		// meas.c:214-296: jn, j per bond class, j2 per two-bond class
		const int nb = a.num_b;
		T *aj = acc + a.lay.jq;       // j, jn [num_b_accum] | j2 [num_b2_accum]
		const T pre_b = phase / (double)a.degen_b;
		for (int r = threadIdx.x; r < a.num_b_accum; r += blockDim.x) {
			T jn = zero<T>(), jj = zero<T>();
			for (int q = a.b_off[r]; q < a.b_off[r + 1]; q++) {
				const int cb = a.b_idx[q];
				const int i0 = a.bonds[cb], i1 = a.bonds[cb + nb];
				const T pui0i1 = peierls(a.peu, i0 + N * i1), pui1i0 = peierls(a.peu, i1 + N * i0);
				const T pdi0i1 = peierls(a.ped, i0 + N * i1), pdi1i0 = peierls(a.ped, i1 + N * i0);
				const double d01 = (i0 == i1) ? 1.0 : 0.0;
				const T gui0i1 = gu(i0, i1), gui1i0 = gu(i1, i0), gdi0i1 = gd(i0, i1), gdi1i0 = gd(i1, i0);
				const T gui0i0 = gu(i0, i0), gdi0i0 = gd(i0, i0), gui1i1 = gu(i1, i1), gdi1i1 = gd(i1, i1);
				jn += pui0i1 * (1.0 - gui0i0) * (d01 - gdi1i0) + pdi0i1 * (1.0 - gdi0i0) * (d01 - gui1i0) +
				      pui0i1 * (1.0 - gui1i1) * (d01 - gdi1i0) + pdi0i1 * (1.0 - gdi1i1) * (d01 - gui1i0) -
				      pui1i0 * (1.0 - gui0i0) * (d01 - gdi0i1) - pdi1i0 * (1.0 - gdi0i0) * (d01 - gui0i1) -
				      pui1i0 * (1.0 - gui1i1) * (d01 - gdi0i1) - pdi1i0 * (1.0 - gdi1i1) * (d01 - gui0i1);
				jj += pui0i1 * (d01 - gui1i0) + pdi0i1 * (d01 - gdi1i0) - pui1i0 * (d01 - gui0i1) -
				      pdi1i0 * (d01 - gdi0i1);
			}
			aj[a.num_b_accum + r] += pre_b * jn;
			aj[r] += pre_b * jj;
		}
		const int nb2 = a.num_b2;
		const T pre_b2 = phase / (double)a.degen_b2;
		for (int r = threadIdx.x; r < a.num_b2_accum; r += blockDim.x) {
			T s = zero<T>();
			for (int q = a.b2_off[r]; q < a.b2_off[r + 1]; q++) {
				const int cb = a.b2_idx[q];
				const T ppui0i2 = a.pp_u[cb], ppui2i0 = a.ppr_u[cb];
				const T ppdi0i2 = a.pp_d[cb], ppdi2i0 = a.ppr_d[cb];
				const int i0 = a.bond2s[cb], i2 = a.bond2s[cb + nb2];
				const double d02 = (i0 == i2) ? 1.0 : 0.0;
				s += ppui0i2 * (d02 - gu(i2, i0)) + ppdi0i2 * (d02 - gd(i2, i0)) -
				     ppui2i0 * (d02 - gu(i0, i2)) - ppdi2i0 * (d02 - gd(i0, i2));
			}
			aj[2 * a.num_b_accum + r] += pre_b2 * s;
		}
	}
}

// -------------------------------------------------------------- uneqlt

// the six unequal-time matrices of chain c at slice t (slice-major stacks,
// slice t of item b at (t 2 nchain + b) N^2) and G(0,0) = Gtt at t = 0
template <typename T>
struct UeSlice {
	Gm<T> u0t, utt, ut0, u00, d0t, dtt, dt0, d00;
	double dt;   // 1 at t = 0 (the equal-time contact terms), else 0
	__device__ UeSlice(const MeasArgs<T> &a, int c, int t)
	{
		const int N = a.N;
		const size_t NN = (size_t)N * N;
		const size_t su = ((size_t)t * 2 * a.nchain + 2 * c) * NN, sd = su + NN;
		u0t = Gm<T>{a.G0t + su, N}; utt = Gm<T>{a.Gtt + su, N}; ut0 = Gm<T>{a.Gt0 + su, N};
		d0t = Gm<T>{a.G0t + sd, N}; dtt = Gm<T>{a.Gtt + sd, N}; dt0 = Gm<T>{a.Gt0 + sd, N};
		u00 = Gm<T>{a.Gtt + (size_t)2 * c * NN, N};
		d00 = Gm<T>{a.Gtt + (size_t)(2 * c + 1) * NN, N};
		dt = (t == 0) ? 1.0 : 0.0;
	}
};

// site-class toggles at slice t: the generalised susceptibility
// (meas.c:473-516) and kv, kn of the energy correlators (meas.c:409-471);
// grid (chain, t), gs_tmp: [chain][L][4][num_ij] class sums
template <typename T>
__global__ void k_meas_uneqlt_xs(MeasArgs<T> a, T *gs_tmp)
{
	const int c = blockIdx.x, t = blockIdx.y;
	if (c >= a.nchain || t >= a.L) return;
	const int N = a.N, L = a.L, nij = a.num_ij;
	const UeSlice<T> g(a, c, t);
	const T phase = a.phase[c];
	T *acc = a.acc + (size_t)c * a.acc_stride;
	if (a.gen_suscept) {
		T *S = gs_tmp + ((size_t)c * L + t) * 4 * nij;
		for (int k = threadIdx.x; k < nij; k += blockDim.x) {
			T au = zero<T>(), bu = zero<T>(), ad = zero<T>(), bd = zero<T>();
			for (int q = a.ij_off[k]; q < a.ij_off[k + 1]; q++) {
				const int e = a.ij_idx[q];
				const int i = e % N, j = e / N;
				const double dl = (i == j) ? g.dt : 0.0;
				au += dl - g.u0t(j, i);
				ad += dl - g.d0t(j, i);
				bu += g.ut0(j, i);
				bd += g.dt0(j, i);
			}
			S[k] = au; S[nij + k] = bu; S[2 * nij + k] = ad; S[3 * nij + k] = bd;
		}
		__syncthreads();
		const T pre = phase / ((double)a.Nx * a.Ny * a.Nx * a.Ny);
		const size_t n2 = (size_t)nij * nij, st = n2 * L;
		T *o = acc + a.lay.ue_gs + n2 * t;
		for (size_t r = threadIdx.x; r < n2; r += blockDim.x) {
			const int k1 = (int)(r % nij), k2 = (int)(r / nij);
			const T au = S[k1], ad = S[2 * nij + k1], bu = S[nij + k2], bd = S[3 * nij + k2];
			o[r] += pre * (au * bu);            // uuuu
			o[st + r] += pre * (ad * bd);       // dddd
			o[2 * st + r] += pre * (ad * bu);   // dduu
			o[3 * st + r] += pre * (au * bd);   // uudd
		}
	}
	if (a.energy) {
		const int nb = a.num_b, nbs = a.num_bs;
		const T pre = phase / (double)a.degen_bs;
		T *ae = acc + a.lay.ue_energy;   // kv, kn [L][num_bs] | vv, vn (meas.cuh)
		for (int r = threadIdx.x; r < nbs; r += blockDim.x) {
			T kv = zero<T>(), kn = zero<T>();
			for (int q = a.bs_off[r]; q < a.bs_off[r + 1]; q++) {
				const int e = a.bs_idx[q];
				const int b = e % nb, j = e / nb;
				const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
				const T pui0i1 = peierls(a.peu, i0 + N * i1), pui1i0 = peierls(a.peu, i1 + N * i0);
				const T pdi0i1 = peierls(a.ped, i0 + N * i1), pdi1i0 = peierls(a.ped, i1 + N * i0);
				const double di0j = (i0 == j) ? g.dt : 0.0, di1j = (i1 == j) ? g.dt : 0.0;
				const T gui0j = g.ut0(i0, j), guji0 = g.u0t(j, i0);
				const T gdi0j = g.dt0(i0, j), gdji0 = g.d0t(j, i0);
				const T gui1j = g.ut0(i1, j), guji1 = g.u0t(j, i1);
				const T gdi1j = g.dt0(i1, j), gdji1 = g.d0t(j, i1);
				const T gui0i1 = g.utt(i0, i1), gui1i0 = g.utt(i1, i0);
				const T gdi0i1 = g.dtt(i0, i1), gdi1i0 = g.dtt(i1, i0);
				const T gujj = g.u00(j, j), gdjj = g.d00(j, j);
				const T ku = pui1i0 * (0.0 - gui0i1) + pui0i1 * (0.0 - gui1i0);
				const T kd = pdi1i0 * (0.0 - gdi0i1) + pdi0i1 * (0.0 - gdi1i0);
				const T xu = pui0i1 * (di0j - guji0) * gui1j + pui1i0 * (di1j - guji1) * gui0j;
				const T xd = pdi0i1 * (di0j - gdji0) * gdi1j + pdi1i0 * (di1j - gdji1) * gdi0j;
				kv += (ku * (1.0 - gujj) + xu) * (1.0 - gdjj) + (kd * (1.0 - gdjj) + xd) * (1.0 - gujj);
				kn += (ku + kd) * (2.0 - gujj - gdjj) + xu + xd;
			}
			const size_t o = (size_t)nbs * t + r;
			ae[o] += pre * kv;
			ae[(size_t)nbs * L + o] += pre * kn;
		}
	}
}

// the Green's functions and Peierls phases of one bond pair (i0 i1), (j0 j1)
// at slice t, with the contact terms delta_t (i == j)
template <typename T>
struct BondPair {
	T pui0i1, pui1i0, pdi0i1, pdi1i0, puj0j1, puj1j0, pdj0j1, pdj1j0;
	T gui1i0, gui0i1, gui0j0, gui1j0, gui0j1, gui1j1, guj0i0, guj1i0, guj0i1, guj1i1, guj1j0, guj0j1;
	T gdi1i0, gdi0i1, gdi0j0, gdi1j0, gdi0j1, gdi1j1, gdj0i0, gdj1i0, gdj0i1, gdj1i1, gdj1j0, gdj0j1;
	double e00, e10, e01, e11;   // delta_t (i0 == j0), (i1 == j0), (i0 == j1), (i1 == j1)
	__device__ BondPair(const MeasArgs<T> &a, const UeSlice<T> &g, int i0, int i1, int j0, int j1)
	{
		const int N = a.N;
		pui0i1 = peierls(a.peu, i0 + N * i1); pui1i0 = peierls(a.peu, i1 + N * i0);
		pdi0i1 = peierls(a.ped, i0 + N * i1); pdi1i0 = peierls(a.ped, i1 + N * i0);
		puj0j1 = peierls(a.peu, j0 + N * j1); puj1j0 = peierls(a.peu, j1 + N * j0);
		pdj0j1 = peierls(a.ped, j0 + N * j1); pdj1j0 = peierls(a.ped, j1 + N * j0);
		gui1i0 = g.utt(i1, i0); gui0i1 = g.utt(i0, i1);
		gui0j0 = g.ut0(i0, j0); gui1j0 = g.ut0(i1, j0); gui0j1 = g.ut0(i0, j1); gui1j1 = g.ut0(i1, j1);
		guj0i0 = g.u0t(j0, i0); guj1i0 = g.u0t(j1, i0); guj0i1 = g.u0t(j0, i1); guj1i1 = g.u0t(j1, i1);
		guj1j0 = g.u00(j1, j0); guj0j1 = g.u00(j0, j1);
		gdi1i0 = g.dtt(i1, i0); gdi0i1 = g.dtt(i0, i1);
		gdi0j0 = g.dt0(i0, j0); gdi1j0 = g.dt0(i1, j0); gdi0j1 = g.dt0(i0, j1); gdi1j1 = g.dt0(i1, j1);
		gdj0i0 = g.d0t(j0, i0); gdj1i0 = g.d0t(j1, i0); gdj0i1 = g.d0t(j0, i1); gdj1i1 = g.d0t(j1, i1);
		gdj1j0 = g.d00(j1, j0); gdj0j1 = g.d00(j0, j1);
		e00 = (i0 == j0) ? g.dt : 0.0; e10 = (i1 == j0) ? g.dt : 0.0;
		e01 = (i0 == j1) ? g.dt : 0.0; e11 = (i1 == j1) ? g.dt : 0.0;
	}
};

// thermal correlators of bond pairs at slice t: jnjn, jnj, jjn
// (meas.c:966-1062); grid (chain, t)
template <typename T>
__global__ void k_meas_uneqlt_xb(MeasArgs<T> a)
{
	const int c = blockIdx.x, t = blockIdx.y;
	if (c >= a.nchain || t >= a.L) return;
	const int L = a.L, nb = a.num_b, nbb = a.num_bb;
	const UeSlice<T> g(a, c, t);
	const T pre = a.phase[c] / (double)a.degen_bb;
	T *at = a.acc + (size_t)c * a.acc_stride + a.lay.thermal +
	        ((size_t)a.num_b2b + a.num_bb2) * L;   // jnjn, jnj, jjn [L][num_bb]
	for (int r = threadIdx.x; r < nbb; r += blockDim.x) {
		T s_jnjn = zero<T>(), s_jnj = zero<T>(), s_jjn = zero<T>();
		for (int q = a.bb_off[r]; q < a.bb_off[r + 1]; q++) {
			const int e = a.bb_idx[q];
			const int b = e % nb, cc = e / nb;
			const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
			const int j0 = a.bonds[cc], j1 = a.bonds[cc + nb];
			const BondPair<T> p(a, g, i0, i1, j0, j1);
			const T gui0i0 = g.utt(i0, i0), gdi0i0 = g.dtt(i0, i0);
			const T gui1i1 = g.utt(i1, i1), gdi1i1 = g.dtt(i1, i1);
			const T guj0j0 = g.u00(j0, j0), gdj0j0 = g.d00(j0, j0);
			const T guj1j1 = g.u00(j1, j1), gdj1j1 = g.d00(j1, j1);
			const T arr[8] = {
			    (p.e01 - p.gdj1i0) * p.gdi1j0, (p.e00 - p.gdj0i0) * p.gdi1j1,
			    (p.e11 - p.gdj1i1) * p.gdi0j0, (p.e10 - p.gdj0i1) * p.gdi0j1,
			    (p.e01 - p.guj1i0) * p.gui1j0, (p.e00 - p.guj0i0) * p.gui1j1,
			    (p.e11 - p.guj1i1) * p.gui0j0, (p.e10 - p.guj0i1) * p.gui0j1};
			const T arrp[8] = {p.pdi0i1 * p.pdj0j1 * arr[0], p.pdi0i1 * p.pdj1j0 * arr[1],
			                   p.pdi1i0 * p.pdj0j1 * arr[2], p.pdi1i0 * p.pdj1j0 * arr[3],
			                   p.pui0i1 * p.puj0j1 * arr[4], p.pui0i1 * p.puj1j0 * arr[5],
			                   p.pui1i0 * p.puj0j1 * arr[6], p.pui1i0 * p.puj1j0 * arr[7]};
			const T ta[8] = {
			    (p.e01 - p.guj1i0) * p.gui0j0, (p.e11 - p.guj1i1) * p.gui1j0,
			    (p.e00 - p.guj0i0) * p.gui0j1, (p.e10 - p.guj0i1) * p.gui1j1,
			    (p.e01 - p.gdj1i0) * p.gdi0j0, (p.e11 - p.gdj1i1) * p.gdi1j0,
			    (p.e00 - p.gdj0i0) * p.gdi0j1, (p.e10 - p.gdj0i1) * p.gdi1j1};
			const T tb[8] = {
			    (p.e00 - p.guj0i0) * p.gui1j0, (p.e01 - p.guj1i0) * p.gui1j1,
			    (p.e10 - p.guj0i1) * p.gui0j0, (p.e11 - p.guj1i1) * p.gui0j1,
			    (p.e00 - p.gdj0i0) * p.gdi1j0, (p.e01 - p.gdj1i0) * p.gdi1j1,
			    (p.e10 - p.gdj0i1) * p.gdi0j0, (p.e11 - p.gdj1i1) * p.gdi0j1};
			const T d[4] = {p.pdi0i1 * p.gdi1i0 - p.pdi1i0 * p.gdi0i1,
			                p.pui0i1 * p.gui1i0 - p.pui1i0 * p.gui0i1,
			                p.pdj0j1 * p.gdj1j0 - p.pdj1j0 * p.gdj0j1,
			                p.puj0j1 * p.guj1j0 - p.puj1j0 * p.guj0j1};
			const T mt[4] = {2.0 - gui0i0 - gui1i1, 2.0 - gdi0i0 - gdi1i1, 2.0 - guj0j0 - guj1j1,
			                 2.0 - gdj0j0 - gdj1j1};
			// jn(i0 i1) j(j0 j1)
			const T wjn_i = mt[0] * d[0] + mt[1] * d[1];
			const T wj_i = d[2] + d[3];
			T t2 = ((ta[2] + ta[3]) * p.puj1j0 - (ta[0] + ta[1]) * p.puj0j1) * d[0];
			T t4 = ((ta[6] + ta[7]) * p.pdj1j0 - (ta[4] + ta[5]) * p.pdj0j1) * d[1];
			T t5 = mt[0] * (arrp[0] - arrp[1] - arrp[2] + arrp[3]);
			T t6 = mt[1] * (arrp[4] - arrp[5] - arrp[6] + arrp[7]);
			s_jnj += wj_i * wjn_i + t2 + t4 + t5 + t6;
			// j(i0 i1) jn(j0 j1)
			const T wjn_j = mt[2] * d[2] + mt[3] * d[3];
			const T wj_j = d[0] + d[1];
			t2 = ((tb[2] + tb[3]) * p.pui1i0 - (tb[0] + tb[1]) * p.pui0i1) * d[2];
			t4 = ((tb[6] + tb[7]) * p.pdi1i0 - (tb[4] + tb[5]) * p.pdi0i1) * d[3];
			t5 = mt[2] * (arrp[0] - arrp[1] - arrp[2] + arrp[3]);
			t6 = mt[3] * (arrp[4] - arrp[5] - arrp[6] + arrp[7]);
			s_jjn += wj_j * wjn_j + t2 + t4 + t5 + t6;
			// jn(i0 i1) jn(j0 j1)
			const T c1 = ((p.e00 - p.guj0i0) * p.gui0j0 + (p.e10 - p.guj0i1) * p.gui1j0 +
			              (p.e01 - p.guj1i0) * p.gui0j1 + (p.e11 - p.guj1i1) * p.gui1j1) *
			             (p.pdi0i1 * p.pdj0j1 * (p.gdi1i0 * p.gdj1j0 + arr[0]) -
			              p.pdi0i1 * p.pdj1j0 * (p.gdi1i0 * p.gdj0j1 + arr[1]) -
			              p.pdi1i0 * p.pdj0j1 * (p.gdi0i1 * p.gdj1j0 + arr[2]) +
			              p.pdi1i0 * p.pdj1j0 * (p.gdi0i1 * p.gdj0j1 + arr[3]));
			const T c3 = ((p.e00 - p.gdj0i0) * p.gdi0j0 + (p.e10 - p.gdj0i1) * p.gdi1j0 +
			              (p.e01 - p.gdj1i0) * p.gdi0j1 + (p.e11 - p.gdj1i1) * p.gdi1j1) *
			             (+p.pui0i1 * p.puj0j1 * (p.gui1i0 * p.guj1j0 + arr[4]) -
			              p.pui0i1 * p.puj1j0 * (p.gui1i0 * p.guj0j1 + arr[5]) -
			              p.pui1i0 * p.puj0j1 * (p.gui0i1 * p.guj1j0 + arr[6]) +
			              p.pui1i0 * p.puj1j0 * (p.gui0i1 * p.guj0j1 + arr[7]));
			const T c2 = mt[0] * mt[2] * (arrp[0] - arrp[1] - arrp[2] + arrp[3]);
			const T c4 = mt[1] * mt[3] * (arrp[4] - arrp[5] - arrp[6] + arrp[7]);
			const T b1 = (+p.pdi0i1 * (-p.gdi1i0 * mt[3] + tb[4] + tb[5]) -
			              p.pdi1i0 * (-p.gdi0i1 * mt[3] + tb[6] + tb[7])) *
			             (+p.puj0j1 * (ta[0] + ta[1]) - p.puj1j0 * (ta[2] + ta[3]));
			const T b3 = (+p.pui0i1 * (-p.gui1i0 * mt[2] + tb[0] + tb[1]) -
			              p.pui1i0 * (-p.gui0i1 * mt[2] + tb[2] + tb[3])) *
			             (+p.pdj0j1 * (ta[4] + ta[5]) - p.pdj1j0 * (ta[6] + ta[7]));
			const T b2 = mt[0] * (-p.puj0j1 * p.guj1j0 + p.puj1j0 * p.guj0j1) *
			             (+p.pdi0i1 * (tb[4] + tb[5]) - p.pdi1i0 * (tb[6] + tb[7]));
			const T b4 = mt[1] * (-p.pdj0j1 * p.gdj1j0 + p.pdj1j0 * p.gdj0j1) *
			             (+p.pui0i1 * (tb[0] + tb[1]) - p.pui1i0 * (tb[2] + tb[3]));
			s_jnjn += wjn_i * wjn_j + c1 + c2 + c3 + c4 + b1 + b2 + b3 + b4;
		}
		const size_t o = (size_t)nbb * t + r, st = (size_t)nbb * L;
		at[o] += pre * s_jnjn;
		at[st + o] += pre * s_jnj;
		at[2 * st + o] += pre * s_jjn;
	}
}

// two-hop bond correlators at slice t (meas.c:1063-1360): per class of
// map_bb2 (two-hop bond b, bond c) j2jn and j2j, of map_b2b2 (two-hop bonds
// b, c) pair_b2b2, j2j2, js2js2, k2k2, ks2ks2, of map_b2b (bond b, two-hop
// bond c) jnj2 and jj2; grid (chain, t)
template <typename T>
__global__ void k_meas_uneqlt_x2(MeasArgs<T> a)
{
	const int c = blockIdx.x, t = blockIdx.y;
	if (c >= a.nchain || t >= a.L) return;
	const int N = a.N, L = a.L, nb = a.num_b, nb2 = a.num_b2;
	const UeSlice<T> g(a, c, t);
	const T phase = a.phase[c];
	T *acc = a.acc + (size_t)c * a.acc_stride;
	const size_t nb2b = a.num_b2b, nbb2 = a.num_bb2, nb2b2 = a.num_b2b2;
	T *th = acc + a.lay.thermal;    // j2jn [L][num_b2b], jnj2 [L][num_bb2], ...
	T *tw = acc + a.lay.two_bond;   // pair_b2b2, j2j2 | j2j | jj2 | js2js2, k2k2, ks2ks2
	const double dt = g.dt;

	// two-hop bond (i0 i2) with bond (j0 j1)
	const T pre_bb2 = phase / (double)a.degen_bb2;
	for (int r = threadIdx.x; r < (int)nbb2; r += blockDim.x) {
		T s_j2jn = zero<T>(), s_j2j = zero<T>();
		for (int q = a.bb2_off[r]; q < a.bb2_off[r + 1]; q++) {
			const int e = a.bb2_idx[q];
			const int b = e % nb2, cc = e / nb2;
			const int j0 = a.bonds[cc], j1 = a.bonds[cc + nb];
			const T puj0j1 = peierls(a.peu, j0 + N * j1), puj1j0 = peierls(a.peu, j1 + N * j0);
			const T pdj0j1 = peierls(a.ped, j0 + N * j1), pdj1j0 = peierls(a.ped, j1 + N * j0);
			const T ppui0i2 = a.pp_u[b], ppui2i0 = a.ppr_u[b];
			const T ppdi0i2 = a.pp_d[b], ppdi2i0 = a.ppr_d[b];
			const int i0 = a.bond2s[b], i2 = a.bond2s[b + nb2];
			const double di0j0 = (i0 == j0) ? dt : 0.0, di2j0 = (i2 == j0) ? dt : 0.0;
			const double di0j1 = (i0 == j1) ? dt : 0.0, di2j1 = (i2 == j1) ? dt : 0.0;
			const T gui2i0 = g.utt(i2, i0), gui0i2 = g.utt(i0, i2);
			const T gui0j0 = g.ut0(i0, j0), gui2j0 = g.ut0(i2, j0), gui0j1 = g.ut0(i0, j1), gui2j1 = g.ut0(i2, j1);
			const T guj0i0 = g.u0t(j0, i0), guj1i0 = g.u0t(j1, i0), guj0i2 = g.u0t(j0, i2), guj1i2 = g.u0t(j1, i2);
			const T guj1j0 = g.u00(j1, j0), guj0j1 = g.u00(j0, j1);
			const T gdi2i0 = g.dtt(i2, i0), gdi0i2 = g.dtt(i0, i2);
			const T gdi0j0 = g.dt0(i0, j0), gdi2j0 = g.dt0(i2, j0), gdi0j1 = g.dt0(i0, j1), gdi2j1 = g.dt0(i2, j1);
			const T gdj0i0 = g.d0t(j0, i0), gdj1i0 = g.d0t(j1, i0), gdj0i2 = g.d0t(j0, i2), gdj1i2 = g.d0t(j1, i2);
			const T gdj1j0 = g.d00(j1, j0), gdj0j1 = g.d00(j0, j1);
			const T arr[4] = {puj1j0 * guj0j1, puj0j1 * guj1j0, pdj1j0 * gdj0j1, pdj0j1 * gdj1j0};
			const T dd[8] = {di0j1 - guj1i0, di0j0 - guj0i0, di2j1 - guj1i2, di2j0 - guj0i2,
			                 di0j1 - gdj1i0, di0j0 - gdj0i0, di2j1 - gdj1i2, di2j0 - gdj0i2};
			const T term[8] = {
			    ppui0i2 * puj0j1 * dd[0] * gui2j0, ppui0i2 * puj1j0 * dd[1] * gui2j1,
			    ppui2i0 * puj0j1 * dd[2] * gui0j0, ppui2i0 * puj1j0 * dd[3] * gui0j1,
			    ppdi0i2 * pdj0j1 * dd[4] * gdi2j0, ppdi0i2 * pdj1j0 * dd[5] * gdi2j1,
			    ppdi2i0 * pdj0j1 * dd[6] * gdi0j0, ppdi2i0 * pdj1j0 * dd[7] * gdi0j1};
			const T wj = -ppui2i0 * gui0i2 + ppui0i2 * gui2i0 - ppdi2i0 * gdi0i2 + ppdi0i2 * gdi2i0;
			if (a.thermal) {
				const T md[2] = {2.0 - g.u00(j0, j0) - g.u00(j1, j1), 2.0 - g.d00(j0, j0) - g.d00(j1, j1)};
				const T wjn = md[0] * (arr[3] - arr[2]) + md[1] * (arr[1] - arr[0]);
				const T t5 = md[1] * (+term[0] - term[1] - term[2] + term[3]);
				const T t6 = md[0] * (+term[4] - term[5] - term[6] + term[7]);
				const T t1 = (-(dd[1] * gui2j0 + dd[0] * gui2j1) * ppui0i2 +
				              (dd[3] * gui0j0 + dd[2] * gui0j1) * ppui2i0) * (arr[3] - arr[2]);
				const T t3 = (-(dd[5] * gdi2j0 + dd[4] * gdi2j1) * ppdi0i2 +
				              (dd[7] * gdi0j0 + dd[6] * gdi0j1) * ppdi2i0) * (arr[1] - arr[0]);
				s_j2jn += wj * wjn + t1 + t3 + t5 + t6;
			}
			if (a.two_bond) {
				const T x = term[0] + term[3] + term[4] + term[7];
				const T y = term[1] + term[2] + term[5] + term[6];
				s_j2j += -wj * (arr[0] - arr[1] + arr[2] - arr[3]) + x - y;
			}
		}
		const size_t o = nbb2 * t + r;
		if (a.thermal) th[o] += pre_bb2 * s_j2jn;
		if (a.two_bond) tw[2 * nb2b2 * L + o] += pre_bb2 * s_j2j;
	}

	// two-hop bond (i0 i2) with two-hop bond (j0 j2)
	if (a.two_bond) {
		const T pre = phase / (double)a.degen_b2b2;
		for (int r = threadIdx.x; r < (int)nb2b2; r += blockDim.x) {
			T pb = zero<T>(), jj = zero<T>(), jsjs = zero<T>(), kk = zero<T>(), ksks = zero<T>();
			for (int q = a.b2b2_off[r]; q < a.b2b2_off[r + 1]; q++) {
				const int e = a.b2b2_idx[q];
				const int b = e % nb2, cc = e / nb2;
				const T ppuj0j2 = a.pp_u[cc], ppuj2j0 = a.ppr_u[cc];
				const T ppdj0j2 = a.pp_d[cc], ppdj2j0 = a.ppr_d[cc];
				const int j0 = a.bond2s[cc], j2 = a.bond2s[cc + nb2];
				const T ppui0i2 = a.pp_u[b], ppui2i0 = a.ppr_u[b];
				const T ppdi0i2 = a.pp_d[b], ppdi2i0 = a.ppr_d[b];
				const int i0 = a.bond2s[b], i2 = a.bond2s[b + nb2];
				const double di0j0 = (i0 == j0) ? dt : 0.0, di2j0 = (i2 == j0) ? dt : 0.0;
				const double di0j2 = (i0 == j2) ? dt : 0.0, di2j2 = (i2 == j2) ? dt : 0.0;
				const T gui2i0 = g.utt(i2, i0), gui0i2 = g.utt(i0, i2);
				const T gui0j0 = g.ut0(i0, j0), gui2j0 = g.ut0(i2, j0), gui0j2 = g.ut0(i0, j2), gui2j2 = g.ut0(i2, j2);
				const T guj0i0 = g.u0t(j0, i0), guj2i0 = g.u0t(j2, i0), guj0i2 = g.u0t(j0, i2), guj2i2 = g.u0t(j2, i2);
				const T guj2j0 = g.u00(j2, j0), guj0j2 = g.u00(j0, j2);
				const T gdi2i0 = g.dtt(i2, i0), gdi0i2 = g.dtt(i0, i2);
				const T gdi0j0 = g.dt0(i0, j0), gdi2j0 = g.dt0(i2, j0), gdi0j2 = g.dt0(i0, j2), gdi2j2 = g.dt0(i2, j2);
				const T gdj0i0 = g.d0t(j0, i0), gdj2i0 = g.d0t(j2, i0), gdj0i2 = g.d0t(j0, i2), gdj2i2 = g.d0t(j2, i2);
				const T gdj2j0 = g.d00(j2, j0), gdj0j2 = g.d00(j0, j2);
				pb += 0.5 * (gui0j0 * gdi2j2 + gui2j0 * gdi0j2 + gui0j2 * gdi2j0 + gui2j2 * gdi0j0);
				const T x = ppui0i2 * ppuj0j2 * (di0j2 - guj2i0) * gui2j0 +
				            ppui2i0 * ppuj2j0 * (di2j0 - guj0i2) * gui0j2 +
				            ppdi0i2 * ppdj0j2 * (di0j2 - gdj2i0) * gdi2j0 +
				            ppdi2i0 * ppdj2j0 * (di2j0 - gdj0i2) * gdi0j2;
				const T y = ppui0i2 * ppuj2j0 * (di0j0 - guj0i0) * gui2j2 +
				            ppui2i0 * ppuj0j2 * (di2j2 - guj2i2) * gui0j0 +
				            ppdi0i2 * ppdj2j0 * (di0j0 - gdj0i0) * gdi2j2 +
				            ppdi2i0 * ppdj0j2 * (di2j2 - gdj2i2) * gdi0j0;
				const T tt[8] = {ppui2i0 * gui0i2, ppui0i2 * gui2i0, ppdi2i0 * gdi0i2, ppdi0i2 * gdi2i0,
				                 ppuj2j0 * guj0j2, ppuj0j2 * guj2j0, ppdj2j0 * gdj0j2, ppdj0j2 * gdj2j0};
				jj += (tt[0] - tt[1] + tt[2] - tt[3]) * (tt[4] - tt[5] + tt[6] - tt[7]) + x - y;
				jsjs += (tt[0] - tt[1] - tt[2] + tt[3]) * (tt[4] - tt[5] - tt[6] + tt[7]) + x - y;
				kk += (tt[0] + tt[1] + tt[2] + tt[3]) * (tt[4] + tt[5] + tt[6] + tt[7]) + x + y;
				ksks += (tt[0] + tt[1] - tt[2] - tt[3]) * (tt[4] + tt[5] - tt[6] - tt[7]) + x + y;
			}
			const size_t o = nb2b2 * t + r, st = nb2b2 * L;
			const size_t rest = (2 * nb2b2 + nb2b + nbb2) * L;
			tw[o] += pre * pb;
			tw[st + o] += pre * jj;
			tw[rest + o] += pre * jsjs;
			tw[rest + st + o] += pre * kk;
			tw[rest + 2 * st + o] += pre * ksks;
		}
	}

	// bond (i0 i1) with two-hop bond (j0 j2)
	const T pre_b2b = phase / (double)a.degen_b2b;
	for (int r = threadIdx.x; r < (int)nb2b; r += blockDim.x) {
		T s_jnj2 = zero<T>(), s_jj2 = zero<T>();
		for (int q = a.b2b_off[r]; q < a.b2b_off[r + 1]; q++) {
			const int e = a.b2b_idx[q];
			const int b = e % nb, cc = e / nb;
			const T ppuj0j2 = a.pp_u[cc], ppuj2j0 = a.ppr_u[cc];
			const T ppdj0j2 = a.pp_d[cc], ppdj2j0 = a.ppr_d[cc];
			const int j0 = a.bond2s[cc], j2 = a.bond2s[cc + nb2];
			const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
			const T pui0i1 = peierls(a.peu, i0 + N * i1), pui1i0 = peierls(a.peu, i1 + N * i0);
			const T pdi0i1 = peierls(a.ped, i0 + N * i1), pdi1i0 = peierls(a.ped, i1 + N * i0);
			const double di0j0 = (i0 == j0) ? dt : 0.0, di1j0 = (i1 == j0) ? dt : 0.0;
			const double di0j2 = (i0 == j2) ? dt : 0.0, di1j2 = (i1 == j2) ? dt : 0.0;
			const T gui1i0 = g.utt(i1, i0), gui0i1 = g.utt(i0, i1);
			const T gui0j0 = g.ut0(i0, j0), gui1j0 = g.ut0(i1, j0), gui0j2 = g.ut0(i0, j2), gui1j2 = g.ut0(i1, j2);
			const T guj0i0 = g.u0t(j0, i0), guj2i0 = g.u0t(j2, i0), guj0i1 = g.u0t(j0, i1), guj2i1 = g.u0t(j2, i1);
			const T guj2j0 = g.u00(j2, j0), guj0j2 = g.u00(j0, j2);
			const T gdi1i0 = g.dtt(i1, i0), gdi0i1 = g.dtt(i0, i1);
			const T gdi0j0 = g.dt0(i0, j0), gdi1j0 = g.dt0(i1, j0), gdi0j2 = g.dt0(i0, j2), gdi1j2 = g.dt0(i1, j2);
			const T gdj0i0 = g.d0t(j0, i0), gdj2i0 = g.d0t(j2, i0), gdj0i1 = g.d0t(j0, i1), gdj2i1 = g.d0t(j2, i1);
			const T gdj2j0 = g.d00(j2, j0), gdj0j2 = g.d00(j0, j2);
			const T arr[4] = {pui1i0 * gui0i1, pui0i1 * gui1i0, pdi1i0 * gdi0i1, pdi0i1 * gdi1i0};
			const T dd[8] = {di0j2 - gdj2i0, di0j0 - gdj0i0, di1j2 - gdj2i1, di1j0 - gdj0i1,
			                 di0j2 - guj2i0, di0j0 - guj0i0, di1j2 - guj2i1, di1j0 - guj0i1};
			const T term[8] = {
			    pdi0i1 * ppdj0j2 * dd[0] * gdi1j0, pdi0i1 * ppdj2j0 * dd[1] * gdi1j2,
			    pdi1i0 * ppdj0j2 * dd[2] * gdi0j0, pdi1i0 * ppdj2j0 * dd[3] * gdi0j2,
			    pui0i1 * ppuj0j2 * dd[4] * gui1j0, pui0i1 * ppuj2j0 * dd[5] * gui1j2,
			    pui1i0 * ppuj0j2 * dd[6] * gui0j0, pui1i0 * ppuj2j0 * dd[7] * gui0j2};
			const T wj = -ppuj2j0 * guj0j2 + ppuj0j2 * guj2j0 - ppdj2j0 * gdj0j2 + ppdj0j2 * gdj2j0;
			if (a.thermal) {
				const T md[2] = {2.0 - g.utt(i0, i0) - g.utt(i1, i1), 2.0 - g.dtt(i0, i0) - g.dtt(i1, i1)};
				const T wjn = md[0] * (arr[3] - arr[2]) + md[1] * (arr[1] - arr[0]);
				const T t1 = (-(dd[4] * gui0j0 + dd[6] * gui1j0) * ppuj0j2 +
				              (dd[5] * gui0j2 + dd[7] * gui1j2) * ppuj2j0) * (arr[3] - arr[2]);
				const T t3 = (-(dd[0] * gdi0j0 + dd[2] * gdi1j0) * ppdj0j2 +
				              (dd[1] * gdi0j2 + dd[3] * gdi1j2) * ppdj2j0) * (arr[1] - arr[0]);
				const T t5 = md[0] * (term[0] - term[1] - term[2] + term[3]);
				const T t6 = md[1] * (term[4] - term[5] - term[6] + term[7]);
				s_jnj2 += wj * wjn + t1 + t3 + t5 + t6;
			}
			if (a.two_bond) {
				const T x = term[4] + term[7] + term[0] + term[3];
				const T y = term[5] + term[6] + term[1] + term[2];
				s_jj2 += (arr[0] - arr[1] + arr[2] - arr[3]) * (-wj) + x - y;
			}
		}
		const size_t o = nb2b * t + r;
		if (a.thermal) th[nb2b * L + o] += pre_b2b * s_jnj2;
		if (a.two_bond) tw[(2 * nb2b2 + nb2b) * L + o] += pre_b2b * s_jj2;
	}
}

// 4-site nematic correlators nem_nnnn, nem_ssss of bond pairs among the
// first NEM_BONDS N = 2 N bonds (meas.c:518-714), the sixteen spin terms
// with every contact term zero, as the reference writes them (it has no
// complex form); grid (chain, t)
template <typename T>
__global__ void k_meas_uneqlt_xn(MeasArgs<T> a)
{
	const int c = blockIdx.x, t = blockIdx.y;
	if (c >= a.nchain || t >= a.L) return;
	const int L = a.L, nb = a.num_b, nbb = a.num_bb;
	const UeSlice<T> g(a, c, t);
	const T pre = a.phase[c] / (double)a.degen_bb;
	T *an = a.acc + (size_t)c * a.acc_stride + a.lay.nem;
	const double delta_i0i1 = 0.0, delta_j0j1 = 0.0, delta_i0j0 = 0.0, delta_i1j0 = 0.0;
	const double delta_i0j1 = 0.0, delta_i1j1 = 0.0;
	for (int r = threadIdx.x; r < nbb; r += blockDim.x) {
		T snn = zero<T>(), sss = zero<T>();
		for (int q = a.nem_off[r]; q < a.nem_off[r + 1]; q++) {
			const int e = a.nem_idx[q];
			const int b = e % nb, cc = e / nb;
			const int i0 = a.bonds[b], i1 = a.bonds[b + nb];
			const int j0 = a.bonds[cc], j1 = a.bonds[cc + nb];
			const T gui0i0 = g.utt(i0, i0), gui1i0 = g.utt(i1, i0), gui0i1 = g.utt(i0, i1), gui1i1 = g.utt(i1, i1);
			const T gui0j0 = g.ut0(i0, j0), gui1j0 = g.ut0(i1, j0), gui0j1 = g.ut0(i0, j1), gui1j1 = g.ut0(i1, j1);
			const T guj0i0 = g.u0t(j0, i0), guj1i0 = g.u0t(j1, i0), guj0i1 = g.u0t(j0, i1), guj1i1 = g.u0t(j1, i1);
			const T guj0j0 = g.u00(j0, j0), guj1j0 = g.u00(j1, j0), guj0j1 = g.u00(j0, j1), guj1j1 = g.u00(j1, j1);
			const T gdi0i0 = g.dtt(i0, i0), gdi1i0 = g.dtt(i1, i0), gdi0i1 = g.dtt(i0, i1), gdi1i1 = g.dtt(i1, i1);
			const T gdi0j0 = g.dt0(i0, j0), gdi1j0 = g.dt0(i1, j0), gdi0j1 = g.dt0(i0, j1), gdi1j1 = g.dt0(i1, j1);
			const T gdj0i0 = g.d0t(j0, i0), gdj1i0 = g.d0t(j1, i0), gdj0i1 = g.d0t(j0, i1), gdj1i1 = g.d0t(j1, i1);
			const T gdj0j0 = g.d00(j0, j0), gdj1j0 = g.d00(j1, j0), gdj0j1 = g.d00(j0, j1), gdj1j1 = g.d00(j1, j1);
			// all four operators of one spin (meas.c:578-602, 683-707), contact terms zero
			auto same = [&](T gi0i0, T gi1i0, T gi0i1, T gi1i1, T gi0j0, T gi1j0, T gi0j1, T gi1j1,
			                T gj0i0, T gj1i0, T gj0i1, T gj1i1, T gj0j0, T gj1j0, T gj0j1, T gj1j1) -> T {
				return +(1.0 - gi0i0) * (1.0 - gi1i1) * (1.0 - gj0j0) * (1.0 - gj1j1) +
				       (1.0 - gi0i0) * (1.0 - gi1i1) * (delta_j0j1 - gj1j0) * gj0j1 +
				       (1.0 - gi0i0) * (delta_i1j0 - gj0i1) * gi1j0 * (1.0 - gj1j1) -
				       (1.0 - gi0i0) * (delta_i1j0 - gj0i1) * gi1j1 * (delta_j0j1 - gj1j0) +
				       (1.0 - gi0i0) * (delta_i1j1 - gj1i1) * gi1j0 * gj0j1 +
				       (1.0 - gi0i0) * (delta_i1j1 - gj1i1) * gi1j1 * (1.0 - gj0j0) +
				       (delta_i0i1 - gi1i0) * gi0i1 * (1.0 - gj0j0) * (1.0 - gj1j1) +
				       (delta_i0i1 - gi1i0) * gi0i1 * (delta_j0j1 - gj1j0) * gj0j1 -
				       (delta_i0i1 - gi1i0) * gi0j0 * (delta_i1j0 - gj0i1) * (1.0 - gj1j1) -
				       (delta_i0i1 - gi1i0) * gi0j0 * (delta_i1j1 - gj1i1) * gj0j1 +
				       (delta_i0i1 - gi1i0) * gi0j1 * (delta_i1j0 - gj0i1) * (delta_j0j1 - gj1j0) -
				       (delta_i0i1 - gi1i0) * gi0j1 * (delta_i1j1 - gj1i1) * (1.0 - gj0j0) +
				       (delta_i0j0 - gj0i0) * gi0i1 * gi1j0 * (1.0 - gj1j1) -
				       (delta_i0j0 - gj0i0) * gi0i1 * gi1j1 * (delta_j0j1 - gj1j0) +
				       (delta_i0j0 - gj0i0) * gi0j0 * (1.0 - gi1i1) * (1.0 - gj1j1) +
				       (delta_i0j0 - gj0i0) * gi0j0 * (delta_i1j1 - gj1i1) * gi1j1 -
				       (delta_i0j0 - gj0i0) * gi0j1 * (1.0 - gi1i1) * (delta_j0j1 - gj1j0) -
				       (delta_i0j0 - gj0i0) * gi0j1 * (delta_i1j1 - gj1i1) * gi1j0 +
				       (delta_i0j1 - gj1i0) * gi0i1 * gi1j0 * gj0j1 +
				       (delta_i0j1 - gj1i0) * gi0i1 * gi1j1 * (1.0 - gj0j0) +
				       (delta_i0j1 - gj1i0) * gi0j0 * (1.0 - gi1i1) * gj0j1 -
				       (delta_i0j1 - gj1i0) * gi0j0 * (delta_i1j0 - gj0i1) * gi1j1 +
				       (delta_i0j1 - gj1i0) * gi0j1 * (1.0 - gi1i1) * (1.0 - gj0j0) +
				       (delta_i0j1 - gj1i0) * gi0j1 * (delta_i1j0 - gj0i1) * gi1j0;
			};
			const T uuuu = same(gui0i0, gui1i0, gui0i1, gui1i1, gui0j0, gui1j0, gui0j1, gui1j1,
			                    guj0i0, guj1i0, guj0i1, guj1i1, guj0j0, guj1j0, guj0j1, guj1j1);
			const T dddd = same(gdi0i0, gdi1i0, gdi0i1, gdi1i1, gdi0j0, gdi1j0, gdi0j1, gdi1j1,
			                    gdj0i0, gdj1i0, gdj0i1, gdj1i1, gdj0j0, gdj1j0, gdj0j1, gdj1j1);
			const T uuud = +(1.0 - gui0i0) * (1.0 - gui1i1) * (1.0 - guj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gui0i0) * (delta_i1j0 - guj0i1) * gui1j0 * (1.0 - gdj1j1) +
			               (delta_i0i1 - gui1i0) * gui0i1 * (1.0 - guj0j0) * (1.0 - gdj1j1) -
			               (delta_i0i1 - gui1i0) * gui0j0 * (delta_i1j0 - guj0i1) * (1.0 - gdj1j1) +
			               (delta_i0j0 - guj0i0) * gui0i1 * gui1j0 * (1.0 - gdj1j1) +
			               (delta_i0j0 - guj0i0) * gui0j0 * (1.0 - gui1i1) * (1.0 - gdj1j1);
			const T uudu = +(1.0 - gui0i0) * (1.0 - gui1i1) * (1.0 - gdj0j0) * (1.0 - guj1j1) +
			               (1.0 - gui0i0) * (delta_i1j1 - guj1i1) * gui1j1 * (1.0 - gdj0j0) +
			               (delta_i0i1 - gui1i0) * gui0i1 * (1.0 - gdj0j0) * (1.0 - guj1j1) -
			               (delta_i0i1 - gui1i0) * gui0j1 * (delta_i1j1 - guj1i1) * (1.0 - gdj0j0) +
			               (delta_i0j1 - guj1i0) * gui0i1 * gui1j1 * (1.0 - gdj0j0) +
			               (delta_i0j1 - guj1i0) * gui0j1 * (1.0 - gui1i1) * (1.0 - gdj0j0);
			const T uudd = +(1.0 - gui0i0) * (1.0 - gui1i1) * (1.0 - gdj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gui0i0) * (1.0 - gui1i1) * (delta_j0j1 - gdj1j0) * gdj0j1 +
			               (delta_i0i1 - gui1i0) * gui0i1 * (1.0 - gdj0j0) * (1.0 - gdj1j1) +
			               (delta_i0i1 - gui1i0) * gui0i1 * (delta_j0j1 - gdj1j0) * gdj0j1;
			const T uduu = +(1.0 - gui0i0) * (1.0 - gdi1i1) * (1.0 - guj0j0) * (1.0 - guj1j1) +
			               (1.0 - gui0i0) * (1.0 - gdi1i1) * (delta_j0j1 - guj1j0) * guj0j1 +
			               (delta_i0j0 - guj0i0) * gui0j0 * (1.0 - gdi1i1) * (1.0 - guj1j1) -
			               (delta_i0j0 - guj0i0) * gui0j1 * (1.0 - gdi1i1) * (delta_j0j1 - guj1j0) +
			               (delta_i0j1 - guj1i0) * gui0j0 * (1.0 - gdi1i1) * guj0j1 +
			               (delta_i0j1 - guj1i0) * gui0j1 * (1.0 - gdi1i1) * (1.0 - guj0j0);
			const T udud = +(1.0 - gui0i0) * (1.0 - gdi1i1) * (1.0 - guj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gui0i0) * (delta_i1j1 - gdj1i1) * gdi1j1 * (1.0 - guj0j0) +
			               (delta_i0j0 - guj0i0) * gui0j0 * (1.0 - gdi1i1) * (1.0 - gdj1j1) +
			               (delta_i0j0 - guj0i0) * gui0j0 * (delta_i1j1 - gdj1i1) * gdi1j1;
			const T uddu = +(1.0 - gui0i0) * (1.0 - gdi1i1) * (1.0 - gdj0j0) * (1.0 - guj1j1) +
			               (1.0 - gui0i0) * (delta_i1j0 - gdj0i1) * gdi1j0 * (1.0 - guj1j1) +
			               (delta_i0j1 - guj1i0) * gui0j1 * (1.0 - gdi1i1) * (1.0 - gdj0j0) +
			               (delta_i0j1 - guj1i0) * gui0j1 * (delta_i1j0 - gdj0i1) * gdi1j0;
			const T uddd = +(1.0 - gui0i0) * (1.0 - gdi1i1) * (1.0 - gdj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gui0i0) * (1.0 - gdi1i1) * (delta_j0j1 - gdj1j0) * gdj0j1 +
			               (1.0 - gui0i0) * (delta_i1j0 - gdj0i1) * gdi1j0 * (1.0 - gdj1j1) -
			               (1.0 - gui0i0) * (delta_i1j0 - gdj0i1) * gdi1j1 * (delta_j0j1 - gdj1j0) +
			               (1.0 - gui0i0) * (delta_i1j1 - gdj1i1) * gdi1j0 * gdj0j1 +
			               (1.0 - gui0i0) * (delta_i1j1 - gdj1i1) * gdi1j1 * (1.0 - gdj0j0);
			const T duuu = +(1.0 - gdi0i0) * (1.0 - gui1i1) * (1.0 - guj0j0) * (1.0 - guj1j1) +
			               (1.0 - gdi0i0) * (1.0 - gui1i1) * (delta_j0j1 - guj1j0) * guj0j1 +
			               (1.0 - gdi0i0) * (delta_i1j0 - guj0i1) * gui1j0 * (1.0 - guj1j1) -
			               (1.0 - gdi0i0) * (delta_i1j0 - guj0i1) * gui1j1 * (delta_j0j1 - guj1j0) +
			               (1.0 - gdi0i0) * (delta_i1j1 - guj1i1) * gui1j0 * guj0j1 +
			               (1.0 - gdi0i0) * (delta_i1j1 - guj1i1) * gui1j1 * (1.0 - guj0j0);
			const T duud = +(1.0 - gdi0i0) * (1.0 - gui1i1) * (1.0 - guj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gdi0i0) * (delta_i1j0 - guj0i1) * gui1j0 * (1.0 - gdj1j1) +
			               (delta_i0j1 - gdj1i0) * gdi0j1 * (1.0 - gui1i1) * (1.0 - guj0j0) +
			               (delta_i0j1 - gdj1i0) * gdi0j1 * (delta_i1j0 - guj0i1) * gui1j0;
			const T dudu = +(1.0 - gdi0i0) * (1.0 - gui1i1) * (1.0 - gdj0j0) * (1.0 - guj1j1) +
			               (1.0 - gdi0i0) * (delta_i1j1 - guj1i1) * gui1j1 * (1.0 - gdj0j0) +
			               (delta_i0j0 - gdj0i0) * gdi0j0 * (1.0 - gui1i1) * (1.0 - guj1j1) +
			               (delta_i0j0 - gdj0i0) * gdi0j0 * (delta_i1j1 - guj1i1) * gui1j1;
			const T dudd = +(1.0 - gdi0i0) * (1.0 - gui1i1) * (1.0 - gdj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gdi0i0) * (1.0 - gui1i1) * (delta_j0j1 - gdj1j0) * gdj0j1 +
			               (delta_i0j0 - gdj0i0) * gdi0j0 * (1.0 - gui1i1) * (1.0 - gdj1j1) -
			               (delta_i0j0 - gdj0i0) * gdi0j1 * (1.0 - gui1i1) * (delta_j0j1 - gdj1j0) +
			               (delta_i0j1 - gdj1i0) * gdi0j0 * (1.0 - gui1i1) * gdj0j1 +
			               (delta_i0j1 - gdj1i0) * gdi0j1 * (1.0 - gui1i1) * (1.0 - gdj0j0);
			const T dduu = +(1.0 - gdi0i0) * (1.0 - gdi1i1) * (1.0 - guj0j0) * (1.0 - guj1j1) +
			               (1.0 - gdi0i0) * (1.0 - gdi1i1) * (delta_j0j1 - guj1j0) * guj0j1 +
			               (delta_i0i1 - gdi1i0) * gdi0i1 * (1.0 - guj0j0) * (1.0 - guj1j1) +
			               (delta_i0i1 - gdi1i0) * gdi0i1 * (delta_j0j1 - guj1j0) * guj0j1;
			const T ddud = +(1.0 - gdi0i0) * (1.0 - gdi1i1) * (1.0 - guj0j0) * (1.0 - gdj1j1) +
			               (1.0 - gdi0i0) * (delta_i1j1 - gdj1i1) * gdi1j1 * (1.0 - guj0j0) +
			               (delta_i0i1 - gdi1i0) * gdi0i1 * (1.0 - guj0j0) * (1.0 - gdj1j1) -
			               (delta_i0i1 - gdi1i0) * gdi0j1 * (delta_i1j1 - gdj1i1) * (1.0 - guj0j0) +
			               (delta_i0j1 - gdj1i0) * gdi0i1 * gdi1j1 * (1.0 - guj0j0) +
			               (delta_i0j1 - gdj1i0) * gdi0j1 * (1.0 - gdi1i1) * (1.0 - guj0j0);
			const T dddu = +(1.0 - gdi0i0) * (1.0 - gdi1i1) * (1.0 - gdj0j0) * (1.0 - guj1j1) +
			               (1.0 - gdi0i0) * (delta_i1j0 - gdj0i1) * gdi1j0 * (1.0 - guj1j1) +
			               (delta_i0i1 - gdi1i0) * gdi0i1 * (1.0 - gdj0j0) * (1.0 - guj1j1) -
			               (delta_i0i1 - gdi1i0) * gdi0j0 * (delta_i1j0 - gdj0i1) * (1.0 - guj1j1) +
			               (delta_i0j0 - gdj0i0) * gdi0i1 * gdi1j0 * (1.0 - guj1j1) +
			               (delta_i0j0 - gdj0i0) * gdi0j0 * (1.0 - gdi1i1) * (1.0 - guj1j1);
			snn += uuuu + uuud + uudu + uudd + uduu + udud + uddu + uddd + duuu + duud + dudu +
			       dudd + dduu + ddud + dddu + dddd;
			sss += uuuu - uuud - uudu + uudd - uduu + udud + uddu - uddd - duuu + duud + dudu -
			       dudd + dduu - ddud - dddu + dddd;
		}
		const size_t o = (size_t)nbb * t + r;
		an[o] += pre * snn;
		an[(size_t)nbb * L + o] += pre * sss;
	}
}

}  // namespace dq
