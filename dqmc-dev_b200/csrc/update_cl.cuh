// Delayed rank-k Metropolis updates of one slice with the Green's function
// held on chip (reference src/updates.c:7-84; draws of src/rand.h:6-31 as in
// update.cuh).
//
// One CTA per (chain, spin), the two spins of a chain forming a cluster of
// two CTAs.  Each CTA loads its spin's G (N x N) into shared memory once per
// slice, keeps the rank-k panels A, B beside it, and writes G back once at
// the end: the flushes G += A B^T and the row/column reads of every accept
// stay in shared memory instead of going through L2.
//
// The Metropolis test of a site needs both spins' diagonal entries G_ii.
// Each CTA keeps both spins' running diagonals, double-buffered by exchange
// parity.  At every exchange (an accept, or the diagonal refresh after a
// flush) thread j of each CTA writes its spin's new entry j into the copy of
// the next parity, locally and into the peer CTA through st.async, which
// completes the transaction bytes on the peer's mbarrier of that parity.
// Every Metropolis thread then arrives on its own CTA's mbarrier and waits
// for the phase: it completes when all local threads have arrived (their
// panel columns and local entries written) and the peer's N entries have
// landed.  Because the copy written at exchange e is only read by tests
// after exchange e, and was last read before exchange e - 1 (which every
// thread of both CTAs has passed), one synchronisation per accept suffices.
// Both CTAs see the same fields, uniforms and diagonals, so they take the
// same decisions.
//
// Every wait inside the Metropolis loop is an mbarrier wait with a time
// limit (no bar.sync), so a CTA whose peer stops answering sets
// DQ_ERR_TIMEOUT and finishes in bounded time instead of hanging.
//
// The arithmetic (test, panel columns, flush, diagonal refresh) is that of
// update_chain in update.cuh, operation for operation, so both kernels give
// bit-identical fields, RNG states and G.
#pragma once

#include "mbar.cuh"
#include "update.cuh"

namespace dq {

// ------------------------------------------------------------ PTX helpers

__device__ inline uint32_t cluster_rank()
{
	uint32_t r;
	asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
	return r;
}

// address of the same shared-memory location in CTA `rank` of the cluster
__device__ inline uint32_t peer_smem(uint32_t a, uint32_t rank)
{
	uint32_t r;
	asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
	return r;
}

__device__ inline void st_cluster_f64(uint32_t a, double v)
{
	asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}

// asynchronous 8-byte store into a peer CTA's shared memory, completing 8
// transaction bytes on the peer's mbarrier at `mbar`
__device__ inline void st_async_f64(uint32_t a, double v, uint32_t mbar)
{
	asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];"
	             ::"r"(a), "d"(v), "r"(mbar) : "memory");
}

// cluster-wide barrier of all threads of both CTAs, with release/acquire
// ordering of shared-memory accesses across the cluster
__device__ inline void cluster_sync_all()
{
	asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// ------------------------------------------------------ shared-memory plan

// leading dimension of G in shared memory: >= N with ld = 2 (mod 4), so
// that the flush's accumulator fragments (rows gq, columns 2 tq + h) of a
// half-warp fall in distinct banks
__host__ __device__ inline int cl_ldg(int N) { return N + ((6 - N % 4) % 4); }
// panel leading dimension: >= N, = 4 (mod 16) for conflict-free fragments
__host__ __device__ inline int cl_ldp(int N) { return N + ((20 - N % 16) % 16); }

struct ClPlan {
	size_t mb, rs, order, hsl, u, dl, dgc, pan, g, total;
};

template <typename T>
__host__ __device__ inline ClPlan cl_plan(int N, int kd)
{
	const int NP = (N + 31) / 32 * 32, planes = is_cplx<T>::value ? 2 : 1;
	auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
	ClPlan p;
	size_t off = 0;
	p.mb = off;    off = al(off + 3 * sizeof(uint64_t));
	p.rs = off;    off = al(off + 17 * sizeof(uint64_t));
	p.order = off; off = al(off + (size_t)N * sizeof(int));
	p.hsl = off;   off = al(off + (size_t)N * sizeof(int));
	p.u = off;     off = al(off + (size_t)N * sizeof(double));
	p.dl = off;    off = al(off + 2 * (size_t)N * sizeof(double));
	p.dgc = off;   off = al(off + 4 * (size_t)NP * sizeof(T));
	p.pan = off;   off = al(off + sizeof(double) * planes * 2 * (size_t)cl_ldp(N) * kd);
	p.g = off;     off = al(off + sizeof(T) * (size_t)N * cl_ldg(N));
	p.total = off;
	return p;
}

// ------------------------------------------------------------------ kernel

template <typename T>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(512, 1) k_update_cl(UpdArgs<T> a)
{
	constexpr bool CX = is_cplx<T>::value;
	constexpr int PL = CX ? 2 : 1;
	constexpr int FT = 4, FKS = 4, FRT = 4;   // flush shape, as update_chain
	const int c = blockIdx.x >> 1;             // chain (the grid is 2 nchain)
	const int s = (int)cluster_rank();          // spin = rank in the cluster
	const int N = a.N, KD = a.n_delay;
	const int LDP = cl_ldp(N), LDG = cl_ldg(N);
	const int NP = (N + 31) / 32 * 32;
	const int tid = threadIdx.x, j = tid;
	const bool metro = tid < NP;
	const size_t NN = (size_t)N * N;
	const int par = a.slice & 1;
	const ClPlan pl = cl_plan<T>(N, KD);

	extern __shared__ __align__(16) unsigned char smraw[];
	uint64_t *mb = (uint64_t *)(smraw + pl.mb);     // [0], [1] exchange parity, [2] flush done
	uint64_t *rs = (uint64_t *)(smraw + pl.rs);
	int *order = (int *)(smraw + pl.order);
	int *hsl = (int *)(smraw + pl.hsl);
	double *u = (double *)(smraw + pl.u);
	double *dl = (double *)(smraw + pl.dl);
	T *dgc = (T *)(smraw + pl.dgc);                 // [copy][spin][NP]
	double *pan = (double *)(smraw + pl.pan);       // [A/B][plane][LDP * KD]
	T *Gs = (T *)(smraw + pl.g);                    // G of this spin, ld LDG
	auto P = [&](int ab, int pl_) -> double * { return pan + (size_t)(ab * PL + pl_) * LDP * KD; };
	__shared__ T s_phase;
	__shared__ int s_nacc;
	__shared__ volatile int s_abort;

	const T *Gg = a.G + (size_t)(2 * c + s) * NN;
	int *hs = a.hs + ((size_t)c * a.L + a.slice) * N;
	const int lane = tid & 31, warp = tid >> 5, nwarp_all = blockDim.x >> 5;
	for (int col = warp; col < N; col += nwarp_all)
		for (int r = lane; r < N; r += 32) Gs[r + (size_t)LDG * col] = Gg[r + (size_t)N * col];
	for (int q = tid; q < N; q += blockDim.x) {
		hsl[q] = hs[q];
		order[q] = a.order[((size_t)c * 2 + par) * N + q];
		u[q] = a.u[((size_t)c * 2 + par) * N + q];
	}
	for (int q = tid; q < 2 * N; q += blockDim.x) dl[q] = a.del[(size_t)c * 2 * N + q];
	if (s == 0 && tid < 17) rs[tid] = a.rng[(size_t)c * 17 + tid];
	if (tid == 0) {
		s_phase = a.phase[c];
		s_nacc = 0;
		s_abort = 0;
		mbar_init(smem_u32(&mb[0]), NP);
		mbar_init(smem_u32(&mb[1]), NP);
		mbar_init(smem_u32(&mb[2]), NP);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	const uint32_t peer = (uint32_t)(s ^ 1);
	// copy 0 of this spin's diagonal, here and in the peer
	if (metro) {
		const T d = j < N ? Gs[j + (size_t)LDG * j] : zero<T>();
		T *dst = dgc + (size_t)s * NP + j;
		*dst = d;
		double xr, xi;
		split(d, xr, xi);
		const uint32_t ra = peer_smem(smem_u32(dst), peer);
		st_cluster_f64(ra, xr);
		if (CX) st_cluster_f64(ra + 8, xi);
	}
	cluster_sync_all();

	if (!metro) {
		// look-ahead warp of the spin-up CTA: the draws of the next slice
		if (s == 0 && tid == NP && a.next_slice >= 0) {
			for (int q = 0; q < 17; q++) a.rng_ckpt[(size_t)c * 17 + q] = rs[q];
			const int np = a.next_slice & 1;
			draw_slice(rs, N, a.hs + ((size_t)c * a.L + a.next_slice) * N, dl,
			           a.order + ((size_t)c * 2 + np) * N, a.u + ((size_t)c * 2 + np) * N);
			for (int q = 0; q < 17; q++) a.rng[(size_t)c * 17 + q] = rs[q];
		}
	} else {
		int k = 0, e = 0, nflush = 0;
		const uint32_t mb_loc0 = smem_u32(&mb[0]), mb_loc1 = smem_u32(&mb[1]);
		const uint32_t mb_peer0 = peer_smem(mb_loc0, peer), mb_peer1 = peer_smem(mb_loc1, peer);
		const uint32_t mb_flush = smem_u32(&mb[2]);
		const uint32_t tx_bytes = (uint32_t)(NP * sizeof(T));

		// exchange e + 1: this thread's entry of its spin's new diagonal
		auto exchange = [&](const T &v) {
			const int ex = e + 1, cp = ex & 1;
			T *dst = dgc + ((size_t)cp * 2 + s) * NP + j;
			*dst = v;
			double xr, xi;
			split(v, xr, xi);
			const uint32_t ra = peer_smem(smem_u32(dst), peer);
			const uint32_t mpeer = cp ? mb_peer1 : mb_peer0, mloc = cp ? mb_loc1 : mb_loc0;
			st_async_f64(ra, xr, mpeer);
			if (CX) st_async_f64(ra + 8, xi, mpeer);
			if (j == 0) mbar_arrive_tx(mloc, tx_bytes);
			else mbar_arrive(mloc);
			mbar_wait_bounded(mloc, (uint32_t)(((ex - 1) >> 1) & 1), &s_abort, a.err);
			e = ex;
		};

		auto flush = [&](int kc) {
			// G_s += A_s B_s^T, as update_chain's flush for one spin, G in
			// shared memory with leading dimension LDG
			const int nt = (N + 7) / 8;
			const int nwarp = NP >> 5;
			const int gq = lane >> 2, tq = lane & 3;
			const double *Ar = P(0, 0), *Br = P(1, 0);
			const double *Ai = P(0, PL - 1), *Bi = P(1, PL - 1);
			if (kc <= 4 * FKS) {
				for (int task = warp; task < nt; task += nwarp) {
					const int c0 = task * 8;
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
						for (int uu = 0; uu < FRT; uu++) {
							const int rr = r0 + 8 * uu + gq;
#pragma unroll
							for (int h = 0; h < 2; h++) {
								gv[uu][h] = (rr < N && cc0 + h < N) ? Gs[rr + (size_t)LDG * (cc0 + h)] : zero<T>();
								cr[uu][h] = 0.0;
								ci[uu][h] = 0.0;
							}
						}
#pragma unroll
						for (int q = 0; q < FKS; q++) {
							if (4 * q < kc) {
								const int kk = 4 * q + tq;
#pragma unroll
								for (int uu = 0; uu < FRT; uu++) {
									const int ra = r0 + 8 * uu + gq;
									const bool ok = kk < kc && ra < N;
									const double ar = ok ? Ar[ra + LDP * kk] : 0.0;
									dmma(cr[uu][0], cr[uu][1], ar, bre[q]);
									if (CX) {
										const double ai = ok ? Ai[ra + LDP * kk] : 0.0;
										dmma(cr[uu][0], cr[uu][1], -ai, bim[q]);
										dmma(ci[uu][0], ci[uu][1], ar, bim[q]);
										dmma(ci[uu][0], ci[uu][1], ai, bre[q]);
									}
								}
							}
						}
#pragma unroll
						for (int uu = 0; uu < FRT; uu++) {
							const int rr = r0 + 8 * uu + gq;
#pragma unroll
							for (int h = 0; h < 2; h++) {
								if (rr < N && cc0 + h < N) {
									if constexpr (CX) {
										Gs[rr + (size_t)LDG * (cc0 + h)] = gv[uu][h] + mkz(cr[uu][h], ci[uu][h]);
									} else {
										Gs[rr + (size_t)LDG * (cc0 + h)] = gv[uu][h] + cr[uu][h];
									}
								}
							}
						}
					}
				}
			} else {
				const int ntt = nt * nt;
				for (int t0 = warp * FT; t0 < ntt; t0 += nwarp * FT) {
#pragma unroll
					for (int f = 0; f < FT; f++) {
						const int tile = t0 + f;
						if (tile >= ntt) break;
						const int r0 = (tile % nt) * 8, c0 = (tile / nt) * 8;
						T gv[2];
#pragma unroll
						for (int h = 0; h < 2; h++) {
							const int rr = r0 + gq, cc = c0 + 2 * tq + h;
							gv[h] = (rr < N && cc < N) ? Gs[rr + (size_t)LDG * cc] : zero<T>();
						}
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
#pragma unroll
						for (int h = 0; h < 2; h++) {
							const int rr = r0 + gq, cc = c0 + 2 * tq + h;
							if (rr < N && cc < N) {
								if constexpr (CX) {
									Gs[rr + (size_t)LDG * cc] = gv[h] + mkz(cr[h], ci[h]);
								} else {
									Gs[rr + (size_t)LDG * cc] = gv[h] + cr[h];
								}
							}
						}
					}
				}
			}
		};

		for (int ii = 0; ii < N; ii++) {
			if (u[ii] >= 1.0) continue;   // never accepted (both deltas zero)
			const int i = order[ii];
			const int h = hsl[i];
			const double delu = dl[i + N * h], deld = dl[i + N * (1 - h)];
			const T *D = dgc + (size_t)(e & 1) * 2 * NP;
			const T ru = 1.0 + (1.0 - D[i]) * delu;
			const T rd = 1.0 + (1.0 - D[NP + i]) * deld;
			const T prob = ru * rd;
			const double aprob = absv(prob);
			if (!(u[ii] < aprob)) continue;
			// accept: this spin's panel columns a_k, b_k and diagonal
			T nd = zero<T>();
			if (j < N) {
				double *Ar = P(0, 0), *Br = P(1, 0);
				T av = Gs[j + (size_t)LDG * i];
				T bv = Gs[i + (size_t)LDG * j];
				if constexpr (CX) {
					double *Ai = P(0, 1), *Bi = P(1, 1);
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
				nd = D[(size_t)s * NP + j] + av * bv;
				// panel column k: nobody reads it before the exchange completes
				double xr, xi;
				split(av, xr, xi);
				Ar[j + LDP * k] = xr;
				if (CX) P(0, PL - 1)[j + LDP * k] = xi;
				split(bv, xr, xi);
				Br[j + LDP * k] = xr;
				if (CX) P(1, PL - 1)[j + LDP * k] = xi;
			}
			exchange(nd);
			// after the exchange: every local thread has finished its test of
			// site i, which reads hsl[i]
			if (tid == 0) {
				hsl[i] = 1 - h;
				s_phase = s_phase * (prob / aprob);
				s_nacc++;
			}
			k++;
			if (k == KD) {
				flush(k);
				k = 0;
				// every warp's tiles are written before the diagonal is read
				mbar_arrive(mb_flush);
				mbar_wait_bounded(mb_flush, (uint32_t)(nflush & 1), &s_abort, a.err);
				nflush++;
				exchange(j < N ? Gs[j + (size_t)LDG * j] : zero<T>());
			}
		}
		if (k > 0) flush(k);
	}
	__syncthreads();
	// this spin's G back to global memory
	T *Gw = a.G + (size_t)(2 * c + s) * NN;
	for (int col = warp; col < N; col += nwarp_all)
		for (int r = lane; r < N; r += 32) Gw[r + (size_t)N * col] = Gs[r + (size_t)LDG * col];
	if (s == 0) {
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
	// neither CTA leaves while the other may still address its shared memory
	cluster_sync_all();
}

template <typename T>
size_t update_cl_smem_bytes(int N, int kd)
{
	return cl_plan<T>(N, kd).total;
}

}  // namespace dq
