// Delayed rank-k Sherman-Morrison Metropolis updates of one imaginary-time
// slice (reference src/updates.c:7-84, with the shuffle of src/rand.h:25-31
// and the draws of rand.h:6-22 that dqmc.c:249-253 makes before it).
//
// One CTA per chain handles both spins: threads [0, NP) work on spin up,
// [NP, 2NP) on spin down, thread j of a spin owning site/row j.
//   * thread 0 runs the chain's xorshift1024* stream: the site permutation
//     and then one uniform per site whose delta is non-zero.  The number of
//     draws depends only on the fields at slice start, so all draws are taken
//     before the Metropolis loop and the loop consumes them in order;
//   * every thread evaluates the accept test from shared memory, so rejected
//     sites cost no barrier; an accept builds the new columns a_k, b_k of the
//     panels (rows of A, B and the G row/column from L2) and updates the
//     running diagonal;
//   * every n_delay accepts the panels are flushed, G += A B^T, with FP64
//     tensor-core MMAs reading the panels from shared memory.
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
	uint64_t *rng;         // [chain][17]
	int *hs;               // [chain][L][N]
	T *G;                  // [chain][2][N*N]
	T *phase;              // [chain]
	double *dv, *dvi;      // [chain][2][L][N]: d_l and 1/d_l of every slice
	int *n_accept;         // [chain] running accept count (statistics)
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

template <typename T>
size_t update_smem_bytes(int N, int kd, int ldp)
{
	const int planes = is_cplx<T>::value ? 2 : 1;
	// the six arrays before the panels, each padded to 16 bytes
	return sizeof(uint64_t) * 17 + sizeof(int) * 2 * (size_t)N + sizeof(double) * 3 * (size_t)N
	       + sizeof(T) * 2 * (size_t)N + 6 * 16 + sizeof(double) * planes * 4 * (size_t)ldp * kd;
}

template <typename T>
__global__ void k_update(UpdArgs<T> a)
{
	constexpr bool CX = is_cplx<T>::value;
	constexpr int PL = CX ? 2 : 1;
	const int c = blockIdx.x;
	if (c >= a.nchain) return;
	const int N = a.N, KD = a.n_delay, LDP = a.ldp;
	const int NP = blockDim.x / 2;
	const int tid = threadIdx.x;
	const int s = tid < NP ? 0 : 1;     // spin of this thread
	const int j = tid - s * NP;         // row/site of this thread
	const size_t NN = (size_t)N * N;

	extern __shared__ __align__(16) unsigned char smraw[];
	// every array starts on a 16-byte boundary (complex loads need it)
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

	for (int q = tid; q < N; q += blockDim.x) hsl[q] = hs[q];
	for (int q = tid; q < 2 * N; q += blockDim.x) dl[q] = a.del[(size_t)c * 2 * N + q];
	if (tid < 17) rs[tid] = a.rng[(size_t)c * 17 + tid];
	if (tid == 0) {
		s_phase = a.phase[c];
		s_nacc = 0;
	}
	__syncthreads();
	if (tid == 0) {
		// shuffle (rand.h:25-31), then the accept draws in visiting order
		for (int i = 0; i < N; i++) {
			const unsigned jj = mod_small(xs1024_next(rs) >> 3, (unsigned)(i + 1));
			if ((int)jj != i) order[i] = order[jj];
			order[jj] = i;
		}
		for (int ii = 0; ii < N; ii++) {
			const int i = order[ii];
			const int h = hsl[i];
			const double du_ = dl[i + N * h], dd_ = dl[i + N * (1 - h)];
			u[ii] = (du_ == 0.0 && dd_ == 0.0) ? 2.0 : u01_from(xs1024_next(rs));
		}
	}
	if (j < N) dg[s * N + j] = Gs[j + (size_t)N * j];
	__syncthreads();
	if (tid < 17) a.rng[(size_t)c * 17 + tid] = rs[tid];

	int k = 0;
	auto flush = [&](int kc) {
		// G_s += A_s B_s^T for both spins; 8x8 output tiles per warp
		const int nt = (N + 7) / 8;
		const int lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
		const int gq = lane >> 2, tq = lane & 3;
		for (int tile = warp; tile < 2 * nt * nt; tile += nwarp) {
			const int sp = tile / (nt * nt);
			const int tt = tile % (nt * nt);
			const int r0 = (tt % nt) * 8, c0 = (tt / nt) * 8;
			T *Gt = a.G + (size_t)(2 * c + sp) * NN;
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
			const int r = r0 + gq;
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int cc = c0 + 2 * tq + h;
				if (r < N && cc < N) {
					T *dst = Gt + r + (size_t)N * cc;
					if constexpr (CX) {
						*dst = *dst + mkz(cr[h], ci[h]);
					} else {
						*dst = *dst + cr[h];
					}
				}
			}
		}
		__syncthreads();
		if (j < N) dg[s * N + j] = Gs[j + (size_t)N * j];
		__syncthreads();
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
		// accept: new panel column k for both spins.  dg[i] and hsl[i] are
		// still being read by slower warps for this site's test, so their
		// writes wait for the barrier; every other diagonal entry is safe.
		T dnew = zero<T>();
		bool defer = false;
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
			const T nd = dg[s * N + j] + av * bv;
			if (j == i) {
				dnew = nd;
				defer = true;
			} else {
				dg[s * N + j] = nd;
			}
			double xr, xi;
			split(av, xr, xi);
			Ar[j + LDP * k] = xr;
			if (CX) P(s, 0, PL - 1)[j + LDP * k] = xi;
			split(bv, xr, xi);
			Br[j + LDP * k] = xr;
			if (CX) P(s, 1, PL - 1)[j + LDP * k] = xi;
		}
		__syncthreads();
		if (defer) dg[s * N + i] = dnew;
		if (tid == 0) {
			hsl[i] = 1 - h;
			s_phase = s_phase * (prob / aprob);
			s_nacc++;
		}
		k++;
		if (k == KD) {
			flush(k);
			k = 0;
		}
	}
	if (k > 0) flush(k);
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

}  // namespace dq
