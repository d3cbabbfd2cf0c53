// Delayed rank-k Sherman-Morrison Metropolis updates of one imaginary-time
// slice (reference src/updates.c:7-84, with the shuffle of src/rand.h:25-31
// and the draws of rand.h:6-22 that dqmc.c:249-253 makes before it).
//
// One CTA per chain handles both spins: threads [0, NP) work on spin up,
// [NP, 2NP) on spin down, thread j of a spin owning site/row j, and one more
// warp runs the chain's xorshift1024* stream.
//   * The number of draws of a slice depends only on its fields at slice
//     start (one uniform per site whose delta is non-zero), so the site
//     permutation and uniforms of slice l+1 can be drawn while slice l is
//     being updated: the extra warp does exactly that, off the critical path,
//     and the next kernel reads them.  rng_ckpt keeps the state as it was
//     before the look-ahead, which is the state the reference has at that
//     point (dqmc.c:249).
//   * every Metropolis thread evaluates the accept test from shared memory,
//     so rejected sites cost no barrier; an accept builds the new columns
//     a_k, b_k of the panels (rows of A, B and the G row/column from L2), and
//     the running diagonal changes only between two named barriers, when no
//     thread can still be testing an earlier site;
//   * every n_delay accepts the panels are flushed, G += A B^T, with FP64
//     tensor-core MMAs reading the panels from shared memory, several G
//     tiles in flight per warp.
#pragma once

#include "common.cuh"

namespace dq {

template <typename T>
struct UpdArgs {
	int N, L, n_delay;     // n_delay: flush period used by the kernel
	int nchain;
	int slice;
	int ldp;               // panel leading dimension in shared memory
	const double *del;     // [chain][2][N]
	const double *exp_lambda; // [chain][2][N]
	uint64_t *rng;         // [chain][17] working state (ahead by the look-ahead draws)
	uint64_t *rng_ckpt;    // [chain][17] state before the look-ahead draws
	int *hs;               // [chain][L][N]
	T *G;                  // [chain][2][N*N]
	T *phase;              // [chain]
	double *dv, *dvi;      // [chain][2][L][N]: d_l and 1/d_l of every slice (optional)
	int *n_accept;         // [chain] running accept count (optional)
	int *order;            // [chain][2][N] site permutations, by slice parity
	double *u;             // [chain][2][N] uniforms in visiting order (2: never accept)
	int next_slice;        // slice whose draws the look-ahead warp takes (-1: none)
	unsigned *err;
};

__device__ inline uint64_t xs1024_next(uint64_t *s)
{
	const uint64_t a = s[s[16]];
	const int p = (int)((s[16] + 1) & 15);
	s[16] = (uint64_t)p;
	uint64_t b = s[p];
	b ^= b << 31;
	s[p] = b ^ a ^ (b >> 11) ^ (a >> 30);
	return s[p] * 1181783497276652981ULL;
}

// x mod m for x < 2^61 and m < 2^10, with 32-bit divisions only
__device__ inline unsigned mod_small(uint64_t x, unsigned m)
{
	unsigned r = (unsigned)(x >> 44) % m;
	r = ((r << 22) | (unsigned)((x >> 22) & 0x3FFFFFu)) % m;
	r = ((r << 22) | (unsigned)(x & 0x3FFFFFu)) % m;
	return r;
}

__device__ inline double u01_from(uint64_t r)
{
	return __longlong_as_double((long long)((0x3FFULL << 52) | (r >> 12))) - 1.0;
}

// The draws of one slice, in the reference's order: the inside-out
// Fisher-Yates permutation (rand.h:25-31), then one uniform per visited site
// whose delta is non-zero (updates.c:19-26).  Single thread; rs in memory.
__device__ inline void draw_slice(uint64_t *rs, int N, const int *hs_row, const double *del,
		int *order, double *u)
{
	for (int i = 0; i < N; i++) {
		const unsigned jj = mod_small(xs1024_next(rs) >> 3, (unsigned)(i + 1));
		if ((int)jj != i) order[i] = order[jj];
		order[jj] = i;
	}
	for (int ii = 0; ii < N; ii++) {
		const int i = order[ii];
		const int h = hs_row[i];
		const double du = del[i + N * h], dd = del[i + N * (1 - h)];
		u[ii] = (du == 0.0 && dd == 0.0) ? 2.0 : u01_from(xs1024_next(rs));
	}
}

// draws of slice `slice` for every chain, one thread per chain (start of a run)
__global__ void k_draws(int N, int L, int nchain, int slice, const double *del, uint64_t *rng,
		uint64_t *rng_ckpt, const int *hs, int *order, double *u)
{
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= nchain) return;
	uint64_t s[17];
	for (int k = 0; k < 17; k++) s[k] = rng[(size_t)c * 17 + k];
	for (int k = 0; k < 17; k++) rng_ckpt[(size_t)c * 17 + k] = s[k];
	const int par = slice & 1;
	draw_slice(s, N, hs + ((size_t)c * L + slice) * N, del + (size_t)c * 2 * N,
	           order + ((size_t)c * 2 + par) * N, u + ((size_t)c * 2 + par) * N);
	for (int k = 0; k < 17; k++) rng[(size_t)c * 17 + k] = s[k];
}

template <typename T>
size_t update_smem_bytes(int N, int kd, int ldp)
{
	const int planes = is_cplx<T>::value ? 2 : 1;
	// rng, order, hsl, u, del, dg, each padded to 16 bytes, then the panels
	return sizeof(uint64_t) * 17 + sizeof(int) * 2 * (size_t)N + sizeof(double) * 3 * (size_t)N
	       + sizeof(T) * 2 * (size_t)N + 6 * 16 + sizeof(double) * planes * 4 * (size_t)ldp * kd;
}

// Named barrier 1 over the Metropolis threads only (the look-ahead warp never
// joins it).  The non-aligned form: threads of a warp may arrive apart, which
// happens in the warps that straddle N (their threads j >= N skip the row
// work), and the aligned form (bar.sync) is undefined in that case.
__device__ inline void bar_metro(int nthreads)
{
	asm volatile("barrier.sync 1, %0;\n" ::"r"(nthreads) : "memory");
}

template <typename T>
__device__ __forceinline__ void update_chain(const UpdArgs<T> &a)
{
	constexpr bool CX = is_cplx<T>::value;
	constexpr int PL = CX ? 2 : 1;
	constexpr int FT = 4;          // G tiles in flight per warp (flushes of more than 4 FKS columns)
	constexpr int FKS = 4;         // k steps of 4 held in registers by the flush
	constexpr int FRT = 4;         // row tiles per DMMA group in the flush
	const int c = blockIdx.x;
	if (c >= a.nchain) return;
	const int N = a.N, KD = a.n_delay, LDP = a.ldp;
	const int NP = (N + 31) / 32 * 32;
	const int NM = 2 * NP;                 // Metropolis threads
	const int tid = threadIdx.x;
	const bool metro = tid < NM;
	const int s = tid < NP ? 0 : 1;        // spin of this thread
	const int j = tid - s * NP;            // row/site of this thread
	const size_t NN = (size_t)N * N;
	const int par = a.slice & 1;

	extern __shared__ __align__(16) unsigned char smraw[];
	auto al16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
	size_t off = 0;
	uint64_t *rs = (uint64_t *)(smraw + off);  off = al16(off + 17 * sizeof(uint64_t));
	int *order = (int *)(smraw + off);         off = al16(off + N * sizeof(int));
	int *hsl = (int *)(smraw + off);           off = al16(off + N * sizeof(int));
	double *u = (double *)(smraw + off);       off = al16(off + N * sizeof(double));
	double *dl = (double *)(smraw + off);      off = al16(off + 2 * N * sizeof(double));
	T *dg = (T *)(smraw + off);                off = al16(off + 2 * N * sizeof(T));
	double *pan = (double *)(smraw + off);     // [spin][A/B][plane][LDP*KD]
	auto P = [&](int sp, int ab, int pl) -> double * {
		return pan + ((size_t)((sp * 2 + ab) * PL + pl)) * LDP * KD;
	};
	__shared__ T s_phase;
	__shared__ int s_nacc;

	T *Gs = a.G + (size_t)(2 * c + s) * NN;
	int *hs = a.hs + ((size_t)c * a.L + a.slice) * N;

	for (int q = tid; q < N; q += blockDim.x) {
		hsl[q] = hs[q];
		order[q] = a.order[((size_t)c * 2 + par) * N + q];
		u[q] = a.u[((size_t)c * 2 + par) * N + q];
	}
	for (int q = tid; q < 2 * N; q += blockDim.x) dl[q] = a.del[(size_t)c * 2 * N + q];
	if (tid < 17) rs[tid] = a.rng[(size_t)c * 17 + tid];
	if (tid == 0) {
		s_phase = a.phase[c];
		s_nacc = 0;
	}
	if (metro && j < N) dg[s * N + j] = Gs[j + (size_t)N * j];
	__syncthreads();

	if (!metro) {
		// look-ahead warp: the draws of the next slice
		if (tid == NM && a.next_slice >= 0) {
			for (int k = 0; k < 17; k++) a.rng_ckpt[(size_t)c * 17 + k] = rs[k];
			const int np = a.next_slice & 1;
			draw_slice(rs, N, a.hs + ((size_t)c * a.L + a.next_slice) * N, dl,
			           a.order + ((size_t)c * 2 + np) * N, a.u + ((size_t)c * 2 + np) * N);
			for (int k = 0; k < 17; k++) a.rng[(size_t)c * 17 + k] = rs[k];
		}
	} else {
		int k = 0;
		auto flush = [&](int kc) {
			// G_s += A_s B_s^T for both spins.  Each warp takes an 8-column
			// tile of one spin, holds its B fragments (k < 4 FKS) in registers
			// and sweeps the row tiles FRT at a time, independent DMMA chains
			// per row tile; the k order per tile is ascending as before.
			const int nt = (N + 7) / 8;
			const int lane = tid & 31, warp = tid >> 5, nwarp = NM >> 5;
			const int gq = lane >> 2, tq = lane & 3;
			if (kc <= 4 * FKS) {
				for (int task = warp; task < 2 * nt; task += nwarp) {
					const int sp = task >= nt ? 1 : 0;
					const int c0 = (task - sp * nt) * 8;
					T *Gt = a.G + (size_t)(2 * c + sp) * NN;
					const double *Ar = P(sp, 0, 0), *Br = P(sp, 1, 0);
					const double *Ai = P(sp, 0, PL - 1), *Bi = P(sp, 1, PL - 1);
					const int cb = c0 + gq, cc0 = c0 + 2 * tq;
					double bre[FKS], bim[FKS];
#pragma unroll
					for (int q = 0; q < FKS; q++) {
						const int kk = 4 * q + tq;
						const bool ok = kk < kc && cb < N;
						bre[q] = ok ? Br[cb + LDP * kk] : 0.0;
						bim[q] = (CX && ok) ? Bi[cb + LDP * kk] : 0.0;
					}
					for (int r0 = 0; r0 < N; r0 += 8 * FRT) {
						T gv[FRT][2];
						double cr[FRT][2], ci[FRT][2];
#pragma unroll
						for (int u = 0; u < FRT; u++) {
							const int rr = r0 + 8 * u + gq;
#pragma unroll
							for (int h = 0; h < 2; h++) {
								gv[u][h] = (rr < N && cc0 + h < N) ? Gt[rr + (size_t)N * (cc0 + h)] : zero<T>();
								cr[u][h] = 0.0;
								ci[u][h] = 0.0;
							}
						}
#pragma unroll
						for (int q = 0; q < FKS; q++) {
							if (4 * q < kc) {
								const int kk = 4 * q + tq;
#pragma unroll
								for (int u = 0; u < FRT; u++) {
									const int ra = r0 + 8 * u + gq;
									const bool ok = kk < kc && ra < N;
									const double ar = ok ? Ar[ra + LDP * kk] : 0.0;
									dmma(cr[u][0], cr[u][1], ar, bre[q]);
									if (CX) {
										const double ai = ok ? Ai[ra + LDP * kk] : 0.0;
										dmma(cr[u][0], cr[u][1], -ai, bim[q]);
										dmma(ci[u][0], ci[u][1], ar, bim[q]);
										dmma(ci[u][0], ci[u][1], ai, bre[q]);
									}
								}
							}
						}
#pragma unroll
						for (int u = 0; u < FRT; u++) {
							const int rr = r0 + 8 * u + gq;
#pragma unroll
							for (int h = 0; h < 2; h++) {
								if (rr < N && cc0 + h < N) {
									if constexpr (CX) {
										Gt[rr + (size_t)N * (cc0 + h)] = gv[u][h] + mkz(cr[u][h], ci[u][h]);
									} else {
										Gt[rr + (size_t)N * (cc0 + h)] = gv[u][h] + cr[u][h];
									}
								}
							}
						}
					}
				}
			} else {
				const int ntt = nt * nt;
				for (int t0 = warp * FT; t0 < 2 * ntt; t0 += nwarp * FT) {
					T gv[FT][2];
					int r_[FT], c_[FT], sp_[FT];
	#pragma unroll
					for (int f = 0; f < FT; f++) {
						const int tile = t0 + f;
						const int sp = tile / ntt, tt = tile - sp * ntt;
						const int r0 = (tt % nt) * 8, c0 = (tt / nt) * 8;
						sp_[f] = sp;
						r_[f] = r0;
						c_[f] = c0;
						const T *Gt = a.G + (size_t)(2 * c + (sp & 1)) * NN;
	#pragma unroll
						for (int h = 0; h < 2; h++) {
							const int rr = r0 + gq, cc = c0 + 2 * tq + h;
							gv[f][h] = (tile < 2 * ntt && rr < N && cc < N) ? Gt[rr + (size_t)N * cc] : zero<T>();
						}
					}
	#pragma unroll
					for (int f = 0; f < FT; f++) {
						const int tile = t0 + f;
						if (tile >= 2 * ntt) break;
						const int sp = sp_[f], r0 = r_[f], c0 = c_[f];
						const double *Ar = P(sp, 0, 0), *Br = P(sp, 1, 0);
						const double *Ai = P(sp, 0, PL - 1), *Bi = P(sp, 1, PL - 1);
						double cr[2] = {0.0, 0.0}, ci[2] = {0.0, 0.0};
						const int ra = r0 + gq, cb = c0 + gq;
						for (int k0 = 0; k0 < kc; k0 += 4) {
							const int kk = k0 + tq;
							const bool okk = kk < kc;
							const double ar = (okk && ra < N) ? Ar[ra + LDP * kk] : 0.0;
							const double br = (okk && cb < N) ? Br[cb + LDP * kk] : 0.0;
							dmma(cr[0], cr[1], ar, br);
							if (CX) {
								const double ai = (okk && ra < N) ? Ai[ra + LDP * kk] : 0.0;
								const double bi = (okk && cb < N) ? Bi[cb + LDP * kk] : 0.0;
								dmma(cr[0], cr[1], -ai, bi);
								dmma(ci[0], ci[1], ar, bi);
								dmma(ci[0], ci[1], ai, br);
							}
						}
						T *Gt = a.G + (size_t)(2 * c + sp) * NN;
	#pragma unroll
						for (int h = 0; h < 2; h++) {
							const int rr = r0 + gq, cc = c0 + 2 * tq + h;
							if (rr < N && cc < N) {
								if constexpr (CX) {
									Gt[rr + (size_t)N * cc] = gv[f][h] + mkz(cr[h], ci[h]);
								} else {
									Gt[rr + (size_t)N * cc] = gv[f][h] + cr[h];
								}
							}
						}
					}
				}
			}
			bar_metro(NM);
			if (j < N) dg[s * N + j] = Gs[j + (size_t)N * j];
			bar_metro(NM);
		};

		for (int ii = 0; ii < N; ii++) {
			if (u[ii] >= 1.0) continue;   // never accepted (both deltas zero)
			const int i = order[ii];
			const int h = hsl[i];
			const double delu = dl[i + N * h], deld = dl[i + N * (1 - h)];
			const T ru = 1.0 + (1.0 - dg[i]) * delu;
			const T rd = 1.0 + (1.0 - dg[N + i]) * deld;
			const T prob = ru * rd;
			const double aprob = absv(prob);
			if (!(u[ii] < aprob)) continue;
			// Accept.  Rejected sites do not synchronise, so a thread can be
			// several sites behind, still testing an earlier site against the
			// diagonal.  No diagonal entry may therefore change until every
			// thread has reached this accept (first barrier), and the next
			// test must see all of them (second barrier).
			T nd = zero<T>();
			if (j < N) {
				double *Ar = P(s, 0, 0), *Br = P(s, 1, 0);
				T av = Gs[j + (size_t)N * i];
				T bv = Gs[i + (size_t)N * j];
				if constexpr (CX) {
					double *Ai = P(s, 0, 1), *Bi = P(s, 1, 1);
					for (int m = 0; m < k; m++) {
						const zd aj = mkz(Ar[j + LDP * m], Ai[j + LDP * m]);
						const zd bi = mkz(Br[i + LDP * m], Bi[i + LDP * m]);
						const zd bj = mkz(Br[j + LDP * m], Bi[j + LDP * m]);
						const zd ai = mkz(Ar[i + LDP * m], Ai[i + LDP * m]);
						av = fma_(aj, bi, av);
						bv = fma_(bj, ai, bv);
					}
				} else {
					for (int m = 0; m < k; m++) {
						av = fma(Ar[j + LDP * m], Br[i + LDP * m], av);
						bv = fma(Br[j + LDP * m], Ar[i + LDP * m], bv);
					}
				}
				if (j == i) av = av - 1.0;
				av = av * ((s == 0 ? delu : deld) / (s == 0 ? ru : rd));
				nd = dg[s * N + j] + av * bv;
				// panel column k: nobody reads column k before the barrier
				double xr, xi;
				split(av, xr, xi);
				Ar[j + LDP * k] = xr;
				if (CX) P(s, 0, PL - 1)[j + LDP * k] = xi;
				split(bv, xr, xi);
				Br[j + LDP * k] = xr;
				if (CX) P(s, 1, PL - 1)[j + LDP * k] = xi;
			}
			bar_metro(NM);
			if (j < N) dg[s * N + j] = nd;
			if (tid == 0) {
				hsl[i] = 1 - h;
				s_phase = s_phase * (prob / aprob);
				s_nacc++;
			}
			bar_metro(NM);
			k++;
			if (k == KD) {
				flush(k);
				k = 0;
			}
		}
		if (k > 0) flush(k);
	}
	__syncthreads();
	for (int q = tid; q < N; q += blockDim.x) {
		const int hq = hsl[q];
		hs[q] = hq;
		if (!a.dv) continue;
		for (int sp = 0; sp < 2; sp++) {
			const double el = a.exp_lambda[(size_t)c * 2 * N + q + N * (hq ^ sp)];
			const size_t o = (((size_t)c * 2 + sp) * a.L + a.slice) * N + q;
			a.dv[o] = el;
			a.dvi[o] = 1.0 / el;
		}
	}
	if (tid == 0) {
		a.phase[c] = s_phase;
		if (a.n_accept) a.n_accept[c] += s_nacc;
	}
}

// The delayed update, one CTA per chain.  k_update leaves the register
// count to the compiler (two CTAs of N <= 160 share an SM); k_update_big
// bounds it so that CTAs of up to 544 threads (N <= 256) can launch.
template <typename T>
__global__ void k_update(UpdArgs<T> a)
{
	update_chain(a);
}

template <typename T>
__global__ void __launch_bounds__(544, 1) k_update_big(UpdArgs<T> a)
{
	update_chain(a);
}

}  // namespace dq
