// Unequal-time Green's functions G(0,t), G(t,t), G(t,0) for every slice t
// (reference src/greens.c:247-494, calc_ue_g), batched over the (chain,
// spin) items of a group.
//
//   calc_o   (greens.c:247-264)  block-cyclic O of the E = 1 + (F-1)/2
//                                pair products of the cluster matrices
//   bsofi    (greens.c:266-337)  O = Q R by Householder QRs of 2N-row
//                                panels, R^-1 by blocks, O^-1 = R^-1 Q^H
//   expand_g (greens.c:339-469)  the E x E blocks of O^-1 seed G at every
//                                2 n_matmul-th slice; chains of B_l / B_l^-1
//                                products fill the slices between
//
// Layouts: O and O^-1 are NE x NE per item (NE = N E), column-major.  The
// slice stacks (G0t, Gtt, Gt0 and the materialised B_l, B_l^-1) are
// slice-major, stack[l][item] N x N, so that one launch can take the same
// step of every group's chain through a table of slice indices.
#pragma once

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "gemm.cuh"

namespace dq {

// B_l = exp_K diag(d_l) and B_l^-1 = diag(1/d_l) inv_exp_K for every slice
// and item (reference calcBu/iBu, dqmc.c:29-59); d per item [L][N]
template <typename T>
__global__ void k_build_bib(int N, int L, int NB, const T *expK, const T *iexpK,
		const double *dv, const double *dvi, T *Bs, T *iBs)
{
	const long long NN = (long long)N * N, tot = NN * NB * L;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long e = q % NN, sb = q / NN;
		const int item = (int)(sb % NB), l = (int)(sb / NB);
		const int r = (int)(e % N), c = (int)(e / N);
		const long long s = (long long)(item & 1) * NN;
		const size_t dof = ((size_t)item * L + l) * N;
		Bs[q] = expK[s + e] * dv[dof + c];
		iBs[q] = iexpK[s + e] * dvi[dof + r];
	}
}

// dst_b = alpha src_b (rows x cols, leading dimensions lds / ldd), or the
// identity when src is null
template <typename T>
__global__ void k_copy2d(int rows, int cols, int NB, const T *src, long long ss, int lds, T *dst,
		long long ds, int ldd, T alpha)
{
	const long long per = (long long)rows * cols, tot = per * NB;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const int b = (int)(q / per);
		const long long e = q % per;
		const int r = (int)(e % rows), c = (int)(e / rows);
		T v;
		if (src) v = alpha * src[b * ss + r + (long long)lds * c];
		else v = (r == c) ? one<T>() : zero<T>();
		dst[b * ds + r + (long long)ldd * c] = v;
	}
}

// diag += 1 on NB matrices n x n, item stride s
template <typename T>
__global__ void k_add_diag(int n, int NB, T *A, long long s)
{
	const long long tot = (long long)n * NB;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const int b = (int)(q / n), i = (int)(q % n);
		T *p = A + b * s + i + (long long)n * i;
		*p = *p + 1.0;
	}
}

// ------------------------------------------------ Householder QR with Q^H
//
// One CTA per item factors an M x n panel (M >= n) in place, A = Q R,
// leaving R in the top n rows (zeros below), writing Q^H (M x M) and
// applying Q^H to `nx1` columns right of the panel and `nx2` columns at X
// (rows of the panel).  The reflectors are LAPACK's geqrf convention
// (zgeqr2/zlarfg: beta = -sign(Re alpha) ||x||); NBK of them at a time are
// factored in shared memory and applied to the trailing columns as one
// block reflector I - V T^H V^H (larft forward, columnwise), so every
// trailing column is read and written once per block.

template <typename T>
struct HqrArgs {
	int M, n, batch;
	T *A; Addr aA; int lda;
	int nx1, nx2;
	T *X; Addr aX;            // nx2 extra columns, leading dimension lda
	T *Qh; Addr aQ;           // M x M, leading dimension M
	unsigned *err;
};

template <typename T, int NBK, int NW>
size_t hqr_smem_bytes(int M)
{
	return sizeof(T) * ((size_t)M * NBK + NBK * NBK + NBK) + sizeof(double) * NW + 64;
}

template <typename T, int NBK, int MAXR, int NW>
__global__ void __launch_bounds__(NW * 32) k_hqr(HqrArgs<T> a)
{
	const int item = blockIdx.x;
	if (item >= a.batch) return;
	const int M = a.M, n = a.n, lda = a.lda;
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	extern __shared__ __align__(16) unsigned char smraw[];
	T *V = (T *)smraw;                    // rows j0.. of the panel, ld M
	T *Tt = V + (size_t)M * NBK;          // NBK x NBK block-reflector factor
	T *tau = Tt + NBK * NBK;
	double *red = (double *)(tau + NBK);
	T *A = a.A + a.aA.off(item);
	T *Q = a.Qh + a.aQ.off(item);
	T *X2 = a.nx2 ? a.X + a.aX.off(item) : nullptr;
	if (M > 32 * MAXR || n > M) {
		if (tid == 0) atomicOr(a.err, DQ_ERR_SIZE);
		return;
	}
	for (long long q = tid; q < (long long)M * M; q += NW * 32) {
		const int r = (int)(q % M), c = (int)(q / M);
		Q[q] = (r == c) ? one<T>() : zero<T>();
	}
	bool bad = false;
	__syncthreads();
	for (int j0 = 0; j0 < n; j0 += NBK) {
		const int nb = min(NBK, n - j0);
		const int mr = M - j0;
		for (int q = tid; q < mr * nb; q += NW * 32) {
			const int r = q % mr, c = q / mr;
			V[r + (size_t)M * c] = A[(j0 + r) + (size_t)lda * (j0 + c)];
		}
		__syncthreads();
		// unblocked QR of the panel (zgeqr2), reflectors stored below the diagonal
		for (int k = 0; k < nb; k++) {
			double s = 0.0;
			for (int r = k + 1 + tid; r < mr; r += NW * 32) s += abs2(V[r + (size_t)M * k]);
			s = warp_sum(s);
			if (lane == 0) red[w] = s;
			__syncthreads();
			double sig = 0.0;
			for (int q = 0; q < NW; q++) sig += red[q];
			const T alpha = V[k + (size_t)M * k];
			T tk, scal;
			double beta;
			if (sig == 0.0 && im(alpha) == 0.0) {
				tk = zero<T>();
				beta = re(alpha);
				scal = zero<T>();
			} else {
				beta = -copysign(sqrt(abs2(alpha) + sig), re(alpha));
				tk = (from_re<T>(beta) - alpha) / beta;
				scal = one<T>() / (alpha - beta);
			}
			if (!(beta == beta)) bad = true;
			__syncthreads();
			for (int r = k + 1 + tid; r < mr; r += NW * 32) V[r + (size_t)M * k] *= scal;
			if (tid == 0) {
				V[k + (size_t)M * k] = from_re<T>(beta);
				tau[k] = tk;
			}
			__syncthreads();
			const T ct = conjv(tk);
			for (int c = k + 1 + w; c < nb; c += NW) {
				T dot = zero<T>();
				for (int r = k + lane; r < mr; r += 32) {
					const T v = (r == k) ? one<T>() : V[r + (size_t)M * k];
					dot += conjv(v) * V[r + (size_t)M * c];
				}
				dot = warp_sum(dot);
				const T f = ct * dot;
				for (int r = k + lane; r < mr; r += 32) {
					const T v = (r == k) ? one<T>() : V[r + (size_t)M * k];
					V[r + (size_t)M * c] -= v * f;
				}
			}
			__syncthreads();
		}
		// R rows of the panel back to A, zeros below the diagonal
		for (int q = tid; q < mr * nb; q += NW * 32) {
			const int r = q % mr, c = q / mr;
			A[(j0 + r) + (size_t)lda * (j0 + c)] = (r <= c) ? V[r + (size_t)M * c] : zero<T>();
		}
		// y[p][k] = v_p^H v_k (p < k), then T by the larft recurrence
		for (int pk = w; pk < nb * nb; pk += NW) {
			const int p = pk % nb, k = pk / nb;
			if (p >= k) continue;
			T dot = zero<T>();
			for (int r = k + lane; r < mr; r += 32) {
				const T vk = (r == k) ? one<T>() : V[r + (size_t)M * k];
				dot += conjv(V[r + (size_t)M * p]) * vk;
			}
			dot = warp_sum(dot);
			if (lane == 0) Tt[p + NBK * k] = dot;
		}
		__syncthreads();
		if (tid == 0) {
			for (int k = 0; k < nb; k++) {
				T tmp[NBK];
#pragma unroll
				for (int p = 0; p < NBK; p++) {
					T s = zero<T>();
					if (p < k)
						for (int q = p; q < k; q++) s += Tt[p + NBK * q] * Tt[q + NBK * k];
					tmp[p] = -tau[k] * s;
				}
#pragma unroll
				for (int p = 0; p < NBK; p++)
					if (p < k) Tt[p + NBK * k] = tmp[p];
				Tt[k + NBK * k] = tau[k];
			}
		}
		__syncthreads();
		// trailing columns: col -= V T^H (V^H col), rows j0..M-1
		const int nA = n - j0 - nb;
		const int ntot = nA + a.nx1 + a.nx2 + M;
		for (int t = w; t < ntot; t += NW) {
			T *col;
			if (t < nA) col = A + (size_t)lda * (j0 + nb + t);
			else if (t < nA + a.nx1) col = A + (size_t)lda * (n + t - nA);
			else if (t < nA + a.nx1 + a.nx2) col = X2 + (size_t)lda * (t - nA - a.nx1);
			else col = Q + (size_t)M * (t - nA - a.nx1 - a.nx2);
			T x[MAXR], wv[NBK];
#pragma unroll
			for (int k = 0; k < NBK; k++) wv[k] = zero<T>();
#pragma unroll
			for (int p = 0; p < MAXR; p++) {
				const int r = lane + 32 * p;
				x[p] = (r < mr) ? col[j0 + r] : zero<T>();
				if (r < mr) {
#pragma unroll
					for (int k = 0; k < NBK; k++) {
						if (k < nb && r >= k) {
							const T v = (r == k) ? one<T>() : V[r + (size_t)M * k];
							wv[k] += conjv(v) * x[p];
						}
					}
				}
			}
#pragma unroll
			for (int o = 16; o > 0; o >>= 1)
#pragma unroll
				for (int k = 0; k < NBK; k++) wv[k] += shfl_xor(wv[k], o);
			T wp[NBK];
#pragma unroll
			for (int k = 0; k < NBK; k++) {
				T s = zero<T>();
#pragma unroll
				for (int p = 0; p < NBK; p++)
					if (p <= k && k < nb) s += conjv(Tt[p + NBK * k]) * wv[p];
				wp[k] = s;
			}
#pragma unroll
			for (int p = 0; p < MAXR; p++) {
				const int r = lane + 32 * p;
				if (r < mr) {
					T y = x[p];
#pragma unroll
					for (int k = 0; k < NBK; k++) {
						if (k < nb && r >= k) {
							const T v = (r == k) ? one<T>() : V[r + (size_t)M * k];
							y -= v * wp[k];
						}
					}
					col[j0 + r] = y;
				}
			}
		}
		__syncthreads();
	}
	if (bad && tid == 0) atomicOr(a.err, DQ_ERR_NAN);
}

// ------------------------------------------------ triangular block inverse
//
// One CTA per (item, diagonal block e): X_ee = R_ee^-1 for the N x N upper
// triangular diagonal blocks of R (NE x NE per item, leading dimension NE),
// column by column: X[0:j, j] = -X[0:j, 0:j] R[0:j, j] / R[j, j].

template <typename T>
struct TriArgs {
	int N, NE, E, batch;
	const T *R;
	T *X;
	unsigned *err;
};

template <typename T>
size_t trtri_smem_bytes(int N)
{
	return sizeof(T) * ((size_t)N * N + N) + 64;
}

template <typename T>
__global__ void __launch_bounds__(256) k_trtri(TriArgs<T> a)
{
	const int item = blockIdx.x / a.E, e = blockIdx.x % a.E;
	if (item >= a.batch) return;
	const int N = a.N;
	const long long NE = a.NE;
	const size_t off = (size_t)item * NE * NE + (size_t)e * N * (1 + NE);
	const T *R = a.R + off;
	T *X = a.X + off;
	extern __shared__ __align__(16) unsigned char smraw[];
	T *S = (T *)smraw;
	T *rc = S + (size_t)N * N;
	bool bad = false;
	for (int j = 0; j < N; j++) {
		for (int i = threadIdx.x; i <= j; i += blockDim.x) rc[i] = R[i + NE * j];
		__syncthreads();
		const T xjj = one<T>() / rc[j];
		for (int i = threadIdx.x; i < N; i += blockDim.x) {
			T v;
			if (i < j) {
				T s = zero<T>();
				for (int k = i; k < j; k++) s += S[i + (size_t)N * k] * rc[k];
				v = -s * xjj;
			} else {
				v = (i == j) ? xjj : zero<T>();
			}
			S[i + (size_t)N * j] = v;
		}
		__syncthreads();
	}
	for (int q = threadIdx.x; q < N * N; q += blockDim.x) {
		const T v = S[q];
		if (!(abs2(v) == abs2(v)) || abs2(v) > 1e300) bad = true;
		X[(q % N) + NE * (q / N)] = v;
	}
	if (bad) atomicOr(a.err, DQ_ERR_SINGULAR);
}

// the blocks of O^-1 that seed the slice stacks (greens.c:353-357, 404-409,
// 437-442): G0t[e nme] = (0, e), Gtt[e nme] = (e, e), Gt0[e nme] = (e, 0)
template <typename T>
__global__ void k_ue_seed(int N, int E, int NB, int nme, const T *Gred, T *G0t, T *Gtt, T *Gt0)
{
	const long long NN = (long long)N * N, NE = (long long)N * E, tot = NN * E * NB;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long el = q % NN;
		const int item = (int)((q / NN) % NB), e = (int)(q / (NN * NB));
		const int r = (int)(el % N), c = (int)(el / N);
		const T *g = Gred + (size_t)item * NE * NE;
		const size_t d = ((size_t)e * nme * NB + item) * NN + el;
		G0t[d] = g[r + NE * (c + (long long)N * e)];
		Gtt[d] = g[(r + (long long)N * e) + NE * (c + (long long)N * e)];
		Gt0[d] = g[(r + (long long)N * e) + NE * c];
	}
}

// ------------------------------------------------ the expand_g step plan
//
// Six chain kinds, each a sequence of (m, next) slice pairs per group:
//   0 G0t left   G0t[n] = a G0t[m] B[n]               a = -1 at m = 0
//   1 G0t right  G0t[n] = a G0t[m] iB[m] + b iB[m]     b = -1 at m = 0
//   2 Gtt up     Gtt[n] = iB[n] (Gtt[m] B[n])
//   3 Gtt down   Gtt[n] = B[m] (Gtt[m] iB[m])
//   4 Gt0 up     Gt0[n] = a iB[n] Gt0[m] + b iB[n]     a = -1, b = 1 at m = 0
//   5 Gt0 down   Gt0[n] = a B[m] Gt0[m] (+ I)          a = -1, + I at n = 0
// The steps with the ordinary coefficients of all groups go in one batched
// launch per (step, kind), through tables of slice indices; the few steps
// with other coefficients get launches of their own.

struct UeOp {
	int kind, nact;     // nact groups in this launch (1 for a special step)
	int tab;            // offset of 4 * nact ints: slices of A, B, C, D (D: 2nd GEMM's A)
	bool special;
	int m, next;
	double alpha, beta; // special steps only
	int prefill;        // special: 0 none, 1 iB[m], 2 iB[next], 3 identity
};

struct UePlan {
	int E = 0, nme = 0;
	std::vector<UeOp> ops;
	std::vector<int> tabs;

	static void coef(int kind, int m, int next, double &alpha, double &beta, int &prefill)
	{
		alpha = 1.0; beta = 0.0; prefill = 0;
		switch (kind) {
		case 0: if (m == 0) alpha = -1.0; break;
		case 1:
			if (next == 0) alpha = -1.0;
			if (m == 0) { beta = -alpha; prefill = 1; }
			break;
		case 4:
			if (m == 0) { alpha = -1.0; beta = 1.0; prefill = 2; }
			break;
		case 5:
			if (next == 0) { alpha = -1.0; beta = 1.0; prefill = 3; }
			break;
		default: break;
		}
	}

	// reference expand_g bounds (greens.c:339-352), with E = 1 + (F-1)/2
	// groups of nme = 2 L/F slices
	void build(int L, int F)
	{
		E = 1 + (F - 1) / 2;
		nme = (L / F) * 2;
		const int n_left = (nme - 1) / 2, n_right = nme / 2;
		const int rstop_last = ((E - 1) * nme + L) / 2;
		const int lstop_first = (rstop_last + 1) % L;
		// chains[kind][group] = (m, next) pairs
		std::vector<std::vector<std::pair<int, int>>> ch[6];
		int maxlen = 0;
		for (int kind = 0; kind < 6; kind++) {
			ch[kind].resize(E);
			const bool left = (kind % 2 == 0);
			for (int f = 0; f < E; f++) {
				const int l = f * nme;
				const int stop = left ? ((f == 0) ? lstop_first : l - n_left)
				                      : ((f == E - 1) ? rstop_last : l + n_right);
				int m = l;
				for (int it = 0; it < L && m != stop; it++) {
					const int nx = left ? (m - 1 + L) % L : (m + 1) % L;
					ch[kind][f].push_back({m, nx});
					m = nx;
				}
				maxlen = std::max(maxlen, (int)ch[kind][f].size());
			}
		}
		ops.clear();
		tabs.clear();
		for (int s = 0; s < maxlen; s++)
			for (int kind = 0; kind < 6; kind++) {
				std::vector<std::pair<int, int>> norm, spec;
				for (int f = 0; f < E; f++) {
					if ((int)ch[kind][f].size() <= s) continue;
					const auto pr = ch[kind][f][s];
					double al, be;
					int pf;
					coef(kind, pr.first, pr.second, al, be, pf);
					((al == 1.0 && be == 0.0) ? norm : spec).push_back(pr);
				}
				if (!norm.empty()) {
					UeOp o{};
					o.kind = kind; o.nact = (int)norm.size(); o.tab = (int)tabs.size();
					o.special = false;
					for (int k = 0; k < 4; k++)
						for (const auto &pr : norm) tabs.push_back(slice_of(kind, k, pr.first, pr.second));
					ops.push_back(o);
				}
				for (const auto &pr : spec) {
					UeOp o{};
					o.kind = kind; o.nact = 1; o.tab = -1; o.special = true;
					o.m = pr.first; o.next = pr.second;
					coef(kind, o.m, o.next, o.alpha, o.beta, o.prefill);
					ops.push_back(o);
				}
			}
	}

	// slice of operand k (0 A, 1 B, 2 C, 3 D) of a step of this kind
	static int slice_of(int kind, int k, int m, int nx)
	{
		switch (kind) {
		case 0: { const int s[4] = {m, nx, nx, 0}; return s[k]; }
		case 1: { const int s[4] = {m, m, nx, 0}; return s[k]; }
		case 2: { const int s[4] = {m, nx, nx, nx}; return s[k]; }
		case 3: { const int s[4] = {m, m, nx, m}; return s[k]; }
		case 4: { const int s[4] = {nx, m, nx, 0}; return s[k]; }
		default: { const int s[4] = {m, m, nx, 0}; return s[k]; }
		}
	}
};

// device buffers of the unequal-time computation of one group
template <typename T>
struct UneqState {
	// sizes the kernels here take: trtri keeps an N x N block in shared
	// memory, k_hqr holds 2N rows in MAXR = 10 registers per lane
	static bool supported(int N, int F, int L)
	{
		const int nmax = is_cplx<T>::value ? 112 : 160;
		return N >= 1 && N <= nmax && F >= 1 && L >= 2 && L % F == 0;
	}
	struct Buf {
		T *p = nullptr;
		int alloc(size_t n)
		{
			if (cudaMalloc(&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) { p = nullptr; return 1; }
			return 0;
		}
		void release() { if (p) cudaFree(p); p = nullptr; }
	};
	Buf G0t, Gtt, Gt0, Bs, iBs, O, Gr, Qh, Tw, Rw, Cw;
	int *dtab = nullptr;
	UePlan plan;
	int N = 0, L = 0, F = 0, NB = 0, E = 0, NE = 0;

	int alloc(int N_, int L_, int F_, int NB_)
	{
		N = N_; L = L_; F = F_; NB = NB_;
		plan.build(L, F);
		E = plan.E;
		NE = N * E;
		const size_t NN = (size_t)N * N, st = (size_t)L * NB * NN;
		int rc = 0;
		rc |= G0t.alloc(st); rc |= Gtt.alloc(st); rc |= Gt0.alloc(st);
		rc |= Bs.alloc(st); rc |= iBs.alloc(st);
		rc |= O.alloc((size_t)NB * NE * NE); rc |= Gr.alloc((size_t)NB * NE * NE);
		rc |= Qh.alloc((size_t)NB * std::max(E - 1, 1) * 4 * NN);
		rc |= Tw.alloc((size_t)NB * E * NN);
		rc |= Rw.alloc((size_t)NB * NE * 2 * N);
		rc |= Cw.alloc((size_t)NB * E * NN);
		if (rc) return 1;
		const size_t nt = plan.tabs.size();
		if (cudaMalloc(&dtab, sizeof(int) * (nt ? nt : 1)) != cudaSuccess) { dtab = nullptr; return 1; }
		if (nt && cudaMemcpy(dtab, plan.tabs.data(), sizeof(int) * nt, cudaMemcpyHostToDevice) != cudaSuccess)
			return 1;
		return 0;
	}
	void release()
	{
		Buf *b[] = {&G0t, &Gtt, &Gt0, &Bs, &iBs, &O, &Gr, &Qh, &Tw, &Rw, &Cw};
		for (Buf *x : b) x->release();
		if (dtab) cudaFree(dtab);
		dtab = nullptr;
	}
};

}  // namespace dq
