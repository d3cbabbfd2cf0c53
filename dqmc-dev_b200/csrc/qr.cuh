// The dense factorisations of the stabilised equal-time Green's function
// (reference src/greens.c:69-208, calc_eq_g), one CTA of 16 warps per
// (chain, spin) matrix, the N x N working matrix in shared memory (or, where
// it does not fit, in a per-item global workspace):
//
// k_qrp   Householder QR with column pivoting by the largest remaining
//         partial column norm, downdated and recomputed as LAPACK geqp3 does
//         (greens.c:89, QR_PIVOT);
// k_qrb   Householder QR of the columns in order of decreasing norm, computed
//         once after scaling by d (the norm pre-pivoting of greens.c:112-135,
//         QR_PRESORT), blocked by 8 with DMMA block-reflector updates;
//         both form Q explicitly (so that a later g*Q is a plain GEMM and
//         diag(v) Q^H is elementwise), with the phase of det Q;
// k_recb  G = (D_b^-1 Q^H + D_s T)^-1 D_b^-1 Q^H (greens.c:157-178) by LU
//         with partial row pivoting and two triangular solves, plus the
//         phase of det G (greens.c:194-207).
#pragma once

#include "common.cuh"

namespace dq {

enum : int { QR_PIVOT = 1, QR_PRESORT = 2 };

template <typename T>
struct QrArgs {
	int N, batch, mode;
	const T *X; long long x_stride;       // input matrices (ld N)
	const double *dcol; long long d_stride; // PRESORT: columns scaled by d on load
	T *Q; long long q_stride;             // explicit Q out
	T *Tout; long long t_stride;          // PIVOT: T = D^-1 R P^T
	T *Rs; long long r_stride;            // PRESORT: D^-1 R in pivot order
	int *pvt; long long p_stride;         // pivot order (column chosen at step j)
	double *dout; long long dout_stride;  // diag(R), 0 -> 1 (real: Householder beta)
	T *qdet;                              // phase of det Q per item
	T *work; long long w_stride;          // N x N per item: working matrix of the
	                                      // shared-memory kernels' global-memory form
	unsigned *err;
};

// ----------------------------------------------- blocked QR, pre-sorted
//
// The QR_PRESORT factorisation (greens.c:119-146: columns scaled by
// the previous D, ordered by descending norm, then geqrf and the explicit
// Q), with the matrix in shared memory and the reflectors taken NBK = 8 at
// a time.  Warps 0-7 factor a panel of 8 columns (one column each, named
// barriers) and form its block-reflector factor T (larft, forward
// columnwise); warps 8-15 meanwhile apply the previous panel's block
// reflector I - V T^H V^H to the trailing columns (one-panel look-ahead), 8
// columns per warp as FP64 tensor-core (DMMA m8n8k4) tiles in the real case.
// Q is then accumulated backwards, block by block, in the same memory.
// Outputs: Q, D^-1 R in position order (Rs), diag(R) and the order.

// leading dimension: N rounded so that ld = 4 (mod 16) doubles, which keeps
// the 8 x 4 DMMA fragment loads of neighbouring columns bank-conflict free
__host__ __device__ inline int qrb_ld(int N) { return (N + 11) / 16 * 16 + 4; }

// In the global-memory form (GM) the N x N working matrix lives in the
// caller's per-item workspace with leading dimension N, and shared memory
// keeps only the small arrays; otherwise it is the first part of shared memory.
template <typename T, int NBK>
size_t qrb_smem_bytes(int N, bool gm = false)
{
	const int np = (N + NBK - 1) / NBK, ld = gm ? N : qrb_ld(N);
	return sizeof(T) * ((gm ? 0 : (size_t)ld * N) + (size_t)ld * NBK + N + (size_t)np * NBK * NBK)
	       + sizeof(double) * 3 * (size_t)N + sizeof(int) * (size_t)N + 64;
}

// reflector k of a panel at global row r (< N): unit diagonal, zero above
template <typename T>
__device__ inline T qrb_v(const T *Vp, int ld, int r, int j0, int k, int nb)
{
	const int rr = r - j0;
	return (k < nb && rr >= k) ? ((rr == k) ? one<T>() : Vp[r + (size_t)ld * k]) : zero<T>();
}

// col[j0..N-1] -= V W (V^H col), W = T^H (HERM) or T, one warp, one column
template <typename T, int NBK, int RPL, bool HERM>
__device__ inline void qrb_apply(T *col, const T *Vp, int ld, const T *Tp, int N, int j0, int nb,
		int lane)
{
	T x[RPL], wv[NBK];
#pragma unroll
	for (int k = 0; k < NBK; k++) wv[k] = zero<T>();
#pragma unroll
	for (int q = 0; q < RPL; q++) {
		const int r = j0 + lane + 32 * q;
		x[q] = (r < N) ? col[r] : zero<T>();
		if (r < N) {
#pragma unroll
			for (int k = 0; k < NBK; k++) wv[k] += conjv(qrb_v(Vp, ld, r, j0, k, nb)) * x[q];
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
		for (int m = 0; m < NBK; m++) {
			if (m >= nb) continue;
			if (HERM) {
				if (m <= k) s += conjv(Tp[m + NBK * k]) * wv[m];
			} else {
				if (m >= k) s += Tp[k + NBK * m] * wv[m];
			}
		}
		wp[k] = s;
	}
#pragma unroll
	for (int q = 0; q < RPL; q++) {
		const int r = j0 + lane + 32 * q;
		if (r < N) {
			T y = x[q];
#pragma unroll
			for (int k = 0; k < NBK; k++) y -= qrb_v(Vp, ld, r, j0, k, nb) * wp[k];
			col[r] = y;
		}
	}
}

// The same for the 8 real columns c0 .. c0+7 (those < cend) on the FP64
// tensor cores, one warp: W = V^T C, W' = op(T) W, C -= V W'.  Fragment
// layouts of m8n8k4: lane l holds A[l/4][l%4], B[l%4][l/4] and
// C[l/4][2(l%4) + {0,1}]; W moves from the C to the B layout by shuffles.
template <int NBK, bool HERM>
__device__ inline void qrb_apply8(double *A, int ld, int c0, int cend, const double *Vp,
		const double *Tp, int N, int j0, int nb, int lane)
{
	static_assert(NBK == 8, "one m8n8k4 tile of reflectors");
	const int lr = lane & 3, lq = lane >> 2;
	const int cb = c0 + lq;
	const bool cbok = cb < cend;
	// W: four independent accumulator pairs over row quads r0, r0+4, ...
	double w[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
	for (int r0 = j0; r0 < N; r0 += 16) {
		double av[4], bv[4];
#pragma unroll
		for (int u = 0; u < 4; u++) {
			const int r = r0 + 4 * u + lr;
			const bool rok = r < N;
			av[u] = rok ? qrb_v(Vp, ld, r, j0, lq, nb) : 0.0;
			bv[u] = (rok && cbok) ? A[r + (size_t)ld * cb] : 0.0;
		}
#pragma unroll
		for (int u = 0; u < 4; u++) dmma(w[u][0], w[u][1], av[u], bv[u]);
	}
	const double w0 = (w[0][0] + w[1][0]) + (w[2][0] + w[3][0]);
	const double w1 = (w[0][1] + w[1][1]) + (w[2][1] + w[3][1]);
	double u0 = 0.0, u1 = 0.0;
#pragma unroll
	for (int s = 0; s < 2; s++) {
		const int kk = 4 * s + lr, src = 4 * kk + (lq >> 1);
		const double v0 = __shfl_sync(0xffffffffu, w0, src), v1 = __shfl_sync(0xffffffffu, w1, src);
		const double b = (lq & 1) ? v1 : v0;
		double a;
		if (HERM) a = (kk <= lq && lq < nb) ? Tp[kk + NBK * lq] : 0.0;
		else a = (lq <= kk && kk < nb) ? Tp[lq + NBK * kk] : 0.0;
		dmma(u0, u1, a, b);
	}
	double bw[2];
#pragma unroll
	for (int s = 0; s < 2; s++) {
		const int kk = 4 * s + lr, src = 4 * kk + (lq >> 1);
		const double v0 = __shfl_sync(0xffffffffu, u0, src), v1 = __shfl_sync(0xffffffffu, u1, src);
		bw[s] = -((lq & 1) ? v1 : v0);
	}
	// C -= V W', three row tiles of 8 at a time
	const int cc = c0 + 2 * lr;
	const bool ok0 = cc < cend, ok1 = cc + 1 < cend;
	for (int r0 = j0; r0 < N; r0 += 24) {
		double x0[3], x1[3], va[3][2];
#pragma unroll
		for (int u = 0; u < 3; u++) {
			const int r = r0 + 8 * u + lq;
			const bool rok = r < N;
			const double *p0 = A + r + (size_t)ld * cc;
			x0[u] = (rok && ok0) ? p0[0] : 0.0;
			x1[u] = (rok && ok1) ? p0[ld] : 0.0;
#pragma unroll
			for (int s = 0; s < 2; s++) va[u][s] = rok ? qrb_v(Vp, ld, r, j0, 4 * s + lr, nb) : 0.0;
		}
#pragma unroll
		for (int s = 0; s < 2; s++)
#pragma unroll
			for (int u = 0; u < 3; u++) dmma(x0[u], x1[u], va[u][s], bw[s]);
#pragma unroll
		for (int u = 0; u < 3; u++) {
			const int r = r0 + 8 * u + lq;
			if (r < N) {
				double *p0 = A + r + (size_t)ld * cc;
				if (ok0) p0[0] = x0[u];
				if (ok1) p0[ld] = x1[u];
			}
		}
	}
}

// columns [cfirst, N) in groups of 8 (real, tensor cores) or one by one
// (complex), group g taken by warp `slot` when g % nslots == slot
template <typename T, int NBK, int RPL, bool HERM>
__device__ inline void qrb_apply_cols(T *A, int ld, int cfirst, const T *Vp, const T *Tp, int N,
		int j0, int nb, int slot, int nslots, int lane)
{
	if constexpr (is_cplx<T>::value) {
		for (int c = cfirst + slot; c < N; c += nslots)
			qrb_apply<T, NBK, RPL, HERM>(A + (size_t)ld * c, Vp, ld, Tp, N, j0, nb, lane);
	} else {
		for (int c = cfirst + 8 * slot; c < N; c += 8 * nslots)
			qrb_apply8<NBK, HERM>(A, ld, c, N, Vp, Tp, N, j0, nb, lane);
	}
}

// T of the block of reflectors j0 .. j0+nb-1 stored below the diagonal of
// A (larft, forward columnwise): one warp
template <typename T, int NBK>
__device__ inline void qrb_block_t(const T *A, int ld, const T *tau, T *Tp, int N, int j0, int nb,
		int lane)
{
	for (int k = 0; k < nb; k++) {
		const int jk = j0 + k;
		T y[NBK];
#pragma unroll
		for (int m = 0; m < NBK; m++) y[m] = zero<T>();
		for (int r = jk + lane; r < N; r += 32) {
			const T vk = (r == jk) ? one<T>() : A[r + (size_t)ld * jk];
#pragma unroll
			for (int m = 0; m < NBK; m++)
				if (m < k) y[m] += conjv(A[r + (size_t)ld * (j0 + m)]) * vk;
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
#pragma unroll
			for (int m = 0; m < NBK; m++) y[m] += shfl_xor(y[m], o);
		const T tk = tau[jk];
		if (lane < k) {
			T sm = zero<T>();
#pragma unroll
			for (int m = 0; m < NBK; m++)
				if (m >= lane && m < k) sm += Tp[lane + NBK * m] * y[m];
			Tp[lane + NBK * k] = -tk * sm;
		}
		if (lane == k) Tp[k + NBK * k] = tk;
		__syncwarp();
	}
}

// Q = H_0 ... H_{N-1} from the reflectors below the diagonal of A and the
// block factors Ts, accumulated backwards by blocks in place of A (block p
// acts on rows and columns >= j0 of the partial product, whose panel
// columns are still e_c there and whose rows j0..j1-1 are zero), then Q to
// global memory and the phase of det Q.  All warps of the CTA.  Per block:
// each thread moves its elements of the block's reflectors into Vb and
// resets them to e_c in the same pass; one barrier; the apply; one barrier.
// (A second buffer, filled while the previous block is applied, saves the
// first barrier but takes 9.5 KB more shared memory, which keeps a GEMM CTA
// of another lane from sharing the SM.)
template <typename T, int NW, int NBK, int RPL>
__device__ inline void qrb_form_q(const QrArgs<T> &a, int item, T *A, int ld, T *Vb, const T *Ts,
		const T *tau, const double *vv, int N)
{
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	const int np = (N + NBK - 1) / NBK;
	for (int p = np - 1; p >= 0; p--) {
		const int j0 = p * NBK, nb = min(NBK, N - j0), j1 = j0 + nb, mr = N - j0;
		// element (j0 + q % mr, j0 + q / mr) of the panel, copied then reset
		for (int q = tid; q < nb * mr; q += blockDim.x) {
			const int k = q / mr, r = j0 + q - k * mr;
			T *e = A + r + (size_t)ld * (j0 + k);
			Vb[r + (size_t)ld * k] = *e;
			*e = (r == j0 + k) ? one<T>() : zero<T>();
		}
		for (int q = tid; q < nb * (N - j1); q += blockDim.x) {
			const int c = q / nb;
			A[j0 + q - c * nb + (size_t)ld * (j1 + c)] = zero<T>();
		}
		__syncthreads();
		qrb_apply_cols<T, NBK, RPL, false>(A, ld, j0, Vb, Ts + (size_t)p * NBK * NBK, N, j0, nb, w, NW,
		                                   lane);
		__syncthreads();
	}
	T *Q = a.Q + (size_t)item * a.q_stride;
	for (int c = w; c < N; c += NW)
		for (int r = lane; r < N; r += 32) Q[r + (size_t)N * c] = A[r + (size_t)ld * c];
	if (tid == 0 && a.qdet) {
		T ph = one<T>();
		for (int j = 0; j < N; j++) ph = ph * phase_of(one<T>() - tau[j] * vv[j]);
		a.qdet[item] = ph;
	}
}

template <typename T, int NW, int NBK, int RPL, bool GM>
__global__ void __launch_bounds__(NW * 32) k_qrb(QrArgs<T> a)
{
	const int item = blockIdx.x;
	if (item >= a.batch) return;
	const int N = a.N, ld = GM ? N : qrb_ld(N);
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	const int np = (N + NBK - 1) / NBK;
	extern __shared__ __align__(16) unsigned char smraw[];
	// N columns, leading dimension ld, position order
	T *A = GM ? a.work + (size_t)item * a.w_stride : (T *)smraw;
	T *Vb = GM ? (T *)smraw : A + (size_t)ld * N;   // copy of one panel's V (ld x NBK)
	T *tau = Vb + (size_t)ld * NBK;             // N
	T *Ts = tau + N;                            // np blocks of NBK x NBK
	double *dsh = (double *)(Ts + (size_t)np * NBK * NBK);
	double *vv = dsh + N;                       // v^H v
	double *vn = vv + N;                        // squared column norms
	int *pvt = (int *)(vn + N);
	if (N > 32 * RPL) {
		if (tid == 0 && a.err) atomicOr(a.err, DQ_ERR_SIZE);
		return;
	}
	const T *X = a.X + (size_t)item * a.x_stride;
	const double *dc = a.dcol + (size_t)item * a.d_stride;

	for (int c = w; c < N; c += NW) {
		const double sc = dc[c];
		double s = 0.0;
		for (int r = lane; r < N; r += 32) s += abs2(X[r + (size_t)N * c] * sc);
		s = warp_sum(s);
		if (lane == 0) vn[c] = s;
	}
	__syncthreads();
	// stable descending order of the squared norms (greens.c:123-129); a NaN
	// norm ranks last so that the order stays a permutation
	for (int c = tid; c < N; c += blockDim.x) {
		double v = vn[c];
		if (!(v >= 0.0)) {
			v = -1.0;
			if (a.err) atomicOr(a.err, DQ_ERR_NAN);
		}
		int rank = 0;
		for (int o = 0; o < N; o++) {
			double u = vn[o];
			if (!(u >= 0.0)) u = -1.0;
			rank += (u > v) || (u == v && o < c);
		}
		pvt[rank] = c;
	}
	__syncthreads();
	for (int j = w; j < N; j += NW) {
		const int c = pvt[j];
		const double sc = dc[c];
		for (int r = lane; r < N; r += 32) A[r + (size_t)ld * j] = X[r + (size_t)N * c] * sc;
	}
	__syncthreads();

	// panel p by warps 0..NBK-1, warp c holding column j0 + c in registers
	// (rows j0 + lane + 32 t).  Per reflector k: its owner (warp k) forms it
	// (zlarfg convention) and publishes v; the later columns' warps update
	// themselves, the earlier ones give y_c = v_c^H v_k for T (larft); two
	// named barriers of the panel warps per reflector.  The next owner's
	// norm below its diagonal is taken in the same pass as its update.
	static_assert(NW == 2 * NBK, "NBK panel warps and NBK trailing warps");
	__shared__ T ybuf[NBK];
	auto bar_panel = []() { asm volatile("barrier.sync 1, %0;\n" ::"r"(NBK * 32) : "memory"); };
	auto panel = [&](int p) {
		const int j0 = p * NBK, nb = min(NBK, N - j0);
		T *Tp = Ts + (size_t)p * NBK * NBK;
		const int c = w, jc = j0 + c;
		T *colc = A + (size_t)ld * jc;
		T x[RPL];
#pragma unroll
		for (int t = 0; t < RPL; t++) {
			const int r = j0 + lane + 32 * t;
			x[t] = (c < nb && r < N) ? colc[r] : zero<T>();
		}
		double sig = 0.0;
		if (c == 0) {
#pragma unroll
			for (int t = 0; t < RPL; t++)
				if (j0 + lane + 32 * t > j0) sig += abs2(x[t]);
			sig = warp_sum(sig);
		}
		for (int k = 0; k < nb; k++) {
			const int j = j0 + k;
			T tk = zero<T>();
			if (c == k) {
				const T alpha = shfl(x[0], k);
				T scal;
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
#pragma unroll
				for (int t = 0; t < RPL; t++) {
					const int r = j0 + lane + 32 * t;
					if (r > j) x[t] *= scal;
					else if (r == j) x[t] = from_re<T>(beta);
					if (r < N) colc[r] = x[t];
				}
				if (lane == 0) {
					tau[j] = tk;
					dsh[j] = beta;
					vv[j] = 1.0 + sig * abs2(scal);
				}
			}
			bar_panel();
			if (c != k && c < nb) {
				const T *vk = A + (size_t)ld * j;
				T vr[RPL];
				T d = zero<T>();
#pragma unroll
				for (int t = 0; t < RPL; t++) {
					const int r = j0 + lane + 32 * t;
					vr[t] = (r > j && r < N) ? vk[r] : ((r == j) ? one<T>() : zero<T>());
					d += conjv(vr[t]) * x[t];
				}
				d = warp_sum(d);
				if (c > k) {
					const T f = conjv(tau[j]) * d;
					double s2 = 0.0;
#pragma unroll
					for (int t = 0; t < RPL; t++) {
						x[t] -= vr[t] * f;
						if (j0 + lane + 32 * t > j + 1) s2 += abs2(x[t]);
					}
					if (c == k + 1) sig = warp_sum(s2);
				} else if (lane == 0) {
					ybuf[c] = conjv(d);
				}
			}
			bar_panel();
			// T[0:k, k] = -tau_k T[0:k, 0:k] y, T[k, k] = tau_k
			if (c == k) {
				if (lane < k) {
					T sm = zero<T>();
#pragma unroll
					for (int m = 0; m < NBK; m++)
						if (m >= lane && m < k) sm += Tp[lane + NBK * m] * ybuf[m];
					Tp[lane + NBK * k] = -tk * sm;
				}
				if (lane == k) Tp[k + NBK * k] = tk;
			}
		}
		if (c < nb) {
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = j0 + lane + 32 * t;
				if (r < N) colc[r] = x[t];
			}
		}
	};

	if (w < NBK) panel(0);
	__syncthreads();
	for (int p = 0; p < np; p++) {
		const int j0 = p * NBK, nb = min(NBK, N - j0), j1 = j0 + nb;
		const T *Vp = A + (size_t)ld * j0;
		const T *Tp = Ts + (size_t)p * NBK * NBK;
		if (w < NBK) {
			if (j1 < N) {
				// the next panel's columns first, then that panel
				if constexpr (is_cplx<T>::value) {
					if (j1 + w < N)
						qrb_apply<T, NBK, RPL, true>(A + (size_t)ld * (j1 + w), Vp, ld, Tp, N, j0, nb, lane);
				} else {
					if (w == 0) qrb_apply8<NBK, true>(A, ld, j1, min(j1 + NBK, N), Vp, Tp, N, j0, nb, lane);
				}
				bar_panel();
				panel(p + 1);
			}
		} else {
			qrb_apply_cols<T, NBK, RPL, true>(A, ld, j1 + NBK, Vp, Tp, N, j0, nb, w - NBK, NW - NBK, lane);
		}
		__syncthreads();
	}

	// D^-1 R in position order, diag(R) (0 -> 1) and the order
	for (int j = w; j < N; j += NW)
		for (int r = lane; r < N; r += 32) {
			const double dr = dsh[r] == 0.0 ? 1.0 : dsh[r];
			a.Rs[(size_t)item * a.r_stride + r + (size_t)N * j] =
				(r <= j) ? A[r + (size_t)ld * j] / dr : zero<T>();
		}
	for (int r = tid; r < N; r += blockDim.x) {
		a.dout[(size_t)item * a.dout_stride + r] = dsh[r] == 0.0 ? 1.0 : dsh[r];
		if (a.pvt) a.pvt[(size_t)item * a.p_stride + r] = pvt[r];
	}
	__syncthreads();

	qrb_form_q<T, NW, NBK, RPL>(a, item, A, ld, Vb, Ts, tau, vv, N);
}

// ----------------------------------------------- column-pivoted QR
//
// The QR_PIVOT factorisation (geqp3 as greens.c:97-101 calls it:
// column pivoting by the largest partial column norm, norms downdated as
// LAPACK dlaqp2 does and recomputed when cancellation makes the downdate
// unreliable), with the matrix in shared memory and columns swapped in
// place so that column j holds pivot position j.  Step j: warp 0 picks
// the pivot (first largest norm in position order, as idamax) from the
// per-warp first largest norms of the last update, exchanges the two
// columns with the pivot column kept in registers and forms the reflector
// there; all warps then update the remaining columns and their norms
// (qrp_update) and leave their own first largest norm for the next step.
// Q is formed from blocks of NBK reflectors as in k_qrb.
// Outputs: Q, T = D^-1 R P^T, diag(R) and the pivot order.

template <typename T, int NBK>
size_t qrp_smem_bytes(int N, bool gm = false)
{
	return qrb_smem_bytes<T, NBK>(N, gm) + sizeof(double) * (size_t)N + 16;
}

// Householder step j of the pivoted QR on the columns j+1 .. N-1: one column
// per 8 lanes, 4 columns per warp at a time (lane = 4 g + s: column slot s,
// rows j + g + 8 i), so that a column's products need three exchange levels;
// then each column's partial norm is downdated from its updated row j as
// LAPACK dlaqp2 does, or recomputed below row j when the downdate has lost
// too much.  The downdate n1 sqrt(1 - (|a_j| / n1)^2) is taken as
// sqrt((n1 - |a_j|)(n1 + |a_j|)) and its test tt (n1 / n2)^2 <= tol3z as
// (n1 - |a_j|)(n1 + |a_j|) <= tol3z n2^2: the same quantities without a
// division.  The loops over a lane's rows stop at the last row (a
// warp-uniform test), so late steps issue only the rows that remain.
// Returns this warp's first largest new norm among its columns (NaN ranks
// below every number, as -0.5) and its position, in every lane.
// MAXI >= ceil(N / 8); the real shared-memory forms keep the column in
// registers between the two passes (v is read again: its loads are shared by
// the four column slots of a warp).
template <typename T, int NW, int MAXI>
__device__ inline void qrp_update(T *A, int ld, int N, int j, T ct, double *vn1, double *vn2,
		double tol3z, double &best, int &bi, bool &nan_seen)
{
	constexpr bool CACHE = !is_cplx<T>::value && MAXI <= 20;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, s = lane & 3, g = lane >> 2;
	const T *vj = A + (size_t)ld * j;
	auto vrow = [&](int r) { return (r < N) ? ((r == j) ? one<T>() : vj[r]) : zero<T>(); };
	best = -1.0;
	bi = N;
	const int nc = N - j - 1;
	for (int q0 = 4 * w; q0 < nc; q0 += 4 * NW) {
		const int q = q0 + s, c = j + 1 + q;
		const bool act = q < nc;
		// an idle slot reads column j+1 and writes nothing
		T *col = A + (size_t)ld * (act ? c : j + 1);
		T d0 = zero<T>(), d1 = zero<T>(), aj;
		double s2a = 0.0, s2b = 0.0;
		if constexpr (CACHE) {
			T x[MAXI];
#pragma unroll
			for (int i = 0; i < MAXI; i++) {
				if (j + 8 * i >= N) break;
				const int r = j + g + 8 * i;
				x[i] = (r < N) ? col[r] : zero<T>();
				if (i & 1) d1 += conjv(vrow(r)) * x[i];
				else d0 += conjv(vrow(r)) * x[i];
			}
			T d = d0 + d1;
			d += shfl_xor(d, 4);
			d += shfl_xor(d, 8);
			d += shfl_xor(d, 16);
			const T f = ct * d;
#pragma unroll
			for (int i = 0; i < MAXI; i++) {
				if (j + 8 * i >= N) break;
				const int r = j + g + 8 * i;
				x[i] -= vrow(r) * f;
				if (r < N) {
					if (act) col[r] = x[i];
					if (r > j) {
						if (i & 1) s2b += abs2(x[i]);
						else s2a += abs2(x[i]);
					}
				}
			}
			aj = shfl(x[0], s);
		} else {
			for (int r = j + g; r < N; r += 8) d0 += conjv(vrow(r)) * col[r];
			T d = d0;
			d += shfl_xor(d, 4);
			d += shfl_xor(d, 8);
			d += shfl_xor(d, 16);
			const T f = ct * d;
			T x0 = zero<T>();
			for (int r = j + g; r < N; r += 8) {
				const T y = col[r] - vrow(r) * f;
				if (act) col[r] = y;
				if (r > j) s2a += abs2(y);
				else x0 = y;
			}
			aj = shfl(x0, s);
		}
		double s2 = s2a + s2b;
		s2 += __shfl_xor_sync(0xffffffffu, s2, 4);
		s2 += __shfl_xor_sync(0xffffffffu, s2, 8);
		s2 += __shfl_xor_sync(0xffffffffu, s2, 16);
		if (act) {
			// every lane of the column computes the new norm; lane g = 0 stores it
			const double n1 = vn1[c], n2 = vn2[c];
			double nv = n1;
			if (n1 != 0.0) {
				const double aa = absv(aj);
				const double d2 = fmax(0.0, (n1 - aa) * (n1 + aa));
				if (d2 <= tol3z * n2 * n2) {
					nv = sqrt(s2);
					if (g == 0) vn2[c] = nv;
				} else {
					nv = sqrt(d2);
				}
				if (g == 0) vn1[c] = nv;
			}
			if (!(nv >= 0.0)) {
				nv = -0.5;
				nan_seen = true;
			}
			if (nv > best) {
				best = nv;
				bi = c;
			}
		}
	}
	// first largest over the warp's four column slots
#pragma unroll
	for (int o = 1; o <= 2; o <<= 1) {
		const double ob = __shfl_xor_sync(0xffffffffu, best, o);
		const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
		if (ob > best || (ob == best && oi < bi)) {
			best = ob;
			bi = oi;
		}
	}
}

// at most 96 registers a thread (48 K of the SM's 64 K for 512 threads), so
// that a GEMM CTA of another lane can share the SM with this one
template <typename T, int NW, int NBK, int RPL, bool GM>
__global__ void __maxnreg__(96) k_qrp(QrArgs<T> a)
{
	const int item = blockIdx.x;
	if (item >= a.batch) return;
	const int N = a.N, ld = GM ? N : qrb_ld(N);
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	const int np = (N + NBK - 1) / NBK;
	extern __shared__ __align__(16) unsigned char smraw[];
	T *A = GM ? a.work + (size_t)item * a.w_stride : (T *)smraw;
	T *Vb = GM ? (T *)smraw : A + (size_t)ld * N;
	T *tau = Vb + (size_t)ld * NBK;
	T *Ts = tau + N;
	double *dsh = (double *)(Ts + (size_t)np * NBK * NBK);
	double *vv = dsh + N;
	double *vn1 = vv + N;                       // partial column norms
	int *pvt = (int *)(vn1 + N);                // original column at each position
	const size_t o2 = ((size_t)((unsigned char *)(pvt + N) - smraw) + 15) & ~(size_t)15;
	double *vn2 = (double *)(smraw + o2);       // norms at the last recompute
	if (N > 32 * RPL) {
		if (tid == 0 && a.err) atomicOr(a.err, DQ_ERR_SIZE);
		return;
	}
	// per warp: first largest candidate norm of its columns and its position
	__shared__ double s_best[NW];
	__shared__ int s_bi[NW];
	bool nan_seen = false;
	const T *X = a.X + (size_t)item * a.x_stride;
	{
		double best = -1.0;
		int bi = N;
		for (int c = w; c < N; c += NW) {
			double s = 0.0;
			for (int r = lane; r < N; r += 32) {
				const T v = X[r + (size_t)N * c];
				A[r + (size_t)ld * c] = v;
				s += abs2(v);
			}
			s = sqrt(warp_sum(s));
			if (lane == 0) {
				vn1[c] = s;
				vn2[c] = s;
				pvt[c] = c;
			}
			if (!(s >= 0.0)) {
				s = -0.5;
				nan_seen = true;
			}
			if (s > best) {
				best = s;
				bi = c;
			}
		}
		if (lane == 0) {
			s_best[w] = best;
			s_bi[w] = bi;
		}
	}
	__syncthreads();
	const double tol3z = sqrt(2.220446049250313e-16);
	for (int j = 0; j < N; j++) {
		if (w == 0) {
			// pivot: the first largest partial norm among positions j..N-1 (a
			// NaN norm ranks below every number but stays a candidate), from
			// the warps' partial results of the last update
			double best = lane < NW ? s_best[lane] : -1.0;
			int bi = lane < NW ? s_bi[lane] : N;
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) {
				const double ob = __shfl_xor_sync(0xffffffffu, best, o);
				const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
				if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
			}
			const int pj = bi;
			// columns pj and j exchange places; the pivot column stays in
			// registers and becomes the reflector (dlarfg convention)
			T xp[RPL], xj[RPL];
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				xp[t] = (r < N) ? A[r + (size_t)ld * pj] : zero<T>();
				xj[t] = (r < N) ? A[r + (size_t)ld * j] : zero<T>();
			}
			if (pj != j) {
#pragma unroll
				for (int t = 0; t < RPL; t++) {
					const int r = lane + 32 * t;
					if (r < N) A[r + (size_t)ld * pj] = xj[t];
				}
				if (lane == 0) {
					const double t1 = vn1[j]; vn1[j] = vn1[pj]; vn1[pj] = t1;
					const double t2 = vn2[j]; vn2[j] = vn2[pj]; vn2[pj] = t2;
					const int t3 = pvt[j]; pvt[j] = pvt[pj]; pvt[pj] = t3;
				}
			}
			double sig = 0.0;
			T al = zero<T>();
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				if (r > j && r < N) sig += abs2(xp[t]);
				if (t == (j >> 5)) al = xp[t];
			}
			sig = warp_sum(sig);
			const T alpha = shfl(al, j & 31);
			T tj, scal;
			double beta;
			if (sig == 0.0 && im(alpha) == 0.0) {
				tj = zero<T>();
				beta = re(alpha);
				scal = zero<T>();
			} else {
				beta = -copysign(sqrt(abs2(alpha) + sig), re(alpha));
				tj = (from_re<T>(beta) - alpha) / beta;
				scal = one<T>() / (alpha - beta);
			}
			T *vj = A + (size_t)ld * j;
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				if (r < N) vj[r] = (r > j) ? xp[t] * scal : ((r == j) ? from_re<T>(beta) : xp[t]);
			}
			if (lane == 0) {
				tau[j] = tj;
				dsh[j] = beta;
				vv[j] = 1.0 + sig * abs2(scal);
			}
		}
		__syncthreads();
		// H_j^H = I - conj(tau) v v^H on every remaining column, then the
		// norm downdate from the updated row j
		double best;
		int bi;
		qrp_update<T, NW, 4 * RPL>(A, ld, N, j, conjv(tau[j]), vn1, vn2, tol3z, best, bi, nan_seen);
		if (lane == 0) {
			s_best[w] = best;
			s_bi[w] = bi;
		}
		__syncthreads();
	}
	if (nan_seen && a.err) atomicOr(a.err, DQ_ERR_NAN);
	// T = D^-1 R P^T: position j is original column pvt[j]
	for (int j = w; j < N; j += NW) {
		const int c = pvt[j];
		for (int r = lane; r < N; r += 32) {
			const double dr = dsh[r] == 0.0 ? 1.0 : dsh[r];
			a.Tout[(size_t)item * a.t_stride + r + (size_t)N * c] =
				(r <= j) ? A[r + (size_t)ld * j] / dr : zero<T>();
		}
	}
	for (int r = tid; r < N; r += blockDim.x) {
		a.dout[(size_t)item * a.dout_stride + r] = dsh[r] == 0.0 ? 1.0 : dsh[r];
		if (a.pvt) a.pvt[(size_t)item * a.p_stride + r] = pvt[r];
	}
	for (int p = w; p < np; p += NW)
		qrb_block_t<T, NBK>(A, ld, tau, Ts + (size_t)p * NBK * NBK, N, p * NBK, min(NBK, N - p * NBK), lane);
	__syncthreads();
	qrb_form_q<T, NW, NBK, RPL>(a, item, A, ld, Vb, Ts, tau, vv, N);
}

template <typename T>
struct RecArgs {
	int N, batch;
	const T *Q; long long q_stride;
	const T *Tm; long long t_stride;
	const double *d; long long d_stride;
	const T *qdet;
	T *G; long long g_stride;
	T *phase;                 // per item: 1 / phase(det G)
	double *logdet;           // per item, optional: log |det(I + B...B)| = -log |det G|
	T *work; long long w_stride;   // N x N per item, global-memory form only
	unsigned *err;
};

// The two triangular solves of the recombine for 8 real right-hand sides
// c0 .. c0+7 (those < N) on the FP64 tensor cores, one warp: Y = D_b^-1 Q^H
// with the LU's row order (perm), then L (unit lower) and U from M.  Rows go
// by tiles of 8; the product of a tile's row of L (or U) with the tiles
// already solved is a chain of m8n8k4 DMMAs (two accumulators), the 8 x 8
// diagonal block is solved with shuffles.  Solved tiles are kept in the
// B-fragment layout (lane: rows 4s + l%4, column l/4) for the later products.
// ys: this warp's slab of 64 ceil(N/8) doubles in shared memory.  Tile t
// of the solution is kept there in B layout (ys[64 t + 32 s + lane], k-step
// s), each lane reading back only what it wrote, so the slab needs no
// synchronisation; holding the tiles in registers instead spills.
__device__ inline void recb_solve8(const double *M, int ld, const int *perm, const double *vsh,
		const double *Q, double *G, int N, int c0, int lane, double *ys)
{
	const int lr = lane & 3, lq = lane >> 2;
	const int nt = (N + 7) / 8;
	auto yb = [&](int u, int sgrp) -> double & { return ys[64 * u + 32 * sgrp + lane]; };
	// C layout -> B layout of one tile: element (row r, col c) sits in lane
	// 4 c + r % 4, k-step r / 4; lane (lq, lr) of the C layout holds rows lq,
	// columns 2 lr + e
	auto c_to_b = [&](double x0, double x1, double &b0, double &b1) {
#pragma unroll
		for (int sgrp = 0; sgrp < 2; sgrp++) {
			// B lane (lr', lq') wants row 4 sgrp + lr', column lq': in C it is
			// lane 4 (4 sgrp + lr') + lq' / 2, element lq' % 2
			const int src = 4 * (4 * sgrp + lr) + (lq >> 1);
			const double v0 = __shfl_sync(0xffffffffu, x0, src), v1 = __shfl_sync(0xffffffffu, x1, src);
			const double v = (lq & 1) ? v1 : v0;
			if (sgrp == 0) b0 = v; else b1 = v;
		}
	};
	auto b_to_c = [&](double b0, double b1, double &x0, double &x1) {
		// C lane (lq, lr), element e: row lq, column 2 lr + e, held by B lane
		// 4 (2 lr + e) + lq % 4 in k-step lq / 4
#pragma unroll
		for (int e = 0; e < 2; e++) {
			const int src = 4 * (2 * lr + e) + (lq & 3);
			const double v0 = __shfl_sync(0xffffffffu, b0, src), v1 = __shfl_sync(0xffffffffu, b1, src);
			const double v = (lq < 4) ? v0 : v1;
			if (e == 0) x0 = v; else x1 = v;
		}
	};
	const int cc = c0 + 2 * lr;
	// forward: L y = P Y
#pragma unroll 1
	for (int t = 0; t < nt; t++) {
		const int r = 8 * t + lq;
		double x[2];
#pragma unroll
		for (int e = 0; e < 2; e++) {
			const int c = cc + e;
			const int pr = (r < N) ? perm[r] : 0;
			x[e] = (r < N && c < N) ? Q[c + (size_t)N * pr] * vsh[pr] : 0.0;
		}
		double a0[2] = {x[0], x[1]}, a1[2] = {0.0, 0.0};
#pragma unroll 4
		for (int u = 0; u < t; u++) {
#pragma unroll
			for (int sgrp = 0; sgrp < 2; sgrp++) {
				const int k = 8 * u + 4 * sgrp + lr;
				const double l = (r < N) ? -M[r + (size_t)ld * k] : 0.0;
				if (sgrp == 0) dmma(a0[0], a0[1], l, yb(u, 0));
				else dmma(a1[0], a1[1], l, yb(u, 1));
			}
		}
		x[0] = a0[0] + a1[0];
		x[1] = a0[1] + a1[1];
		// unit lower 8 x 8 block
#pragma unroll
		for (int q = 0; q < 7; q++) {
			const double y0 = __shfl_sync(0xffffffffu, x[0], 4 * q + lr);
			const double y1 = __shfl_sync(0xffffffffu, x[1], 4 * q + lr);
			if (lq > q && r < N) {
				const double l = M[r + (size_t)ld * (8 * t + q)];
				x[0] -= l * y0;
				x[1] -= l * y1;
			}
		}
		c_to_b(x[0], x[1], yb(t, 0), yb(t, 1));
	}
	// backward: U g = y
#pragma unroll 1
	for (int t = nt - 1; t >= 0; t--) {
		const int r = 8 * t + lq;
		double x[2];
		b_to_c(yb(t, 0), yb(t, 1), x[0], x[1]);
		double a0[2] = {x[0], x[1]}, a1[2] = {0.0, 0.0};
#pragma unroll 4
		for (int u = t + 1; u < nt; u++) {
#pragma unroll
			for (int sgrp = 0; sgrp < 2; sgrp++) {
				const int k = 8 * u + 4 * sgrp + lr;
				const double uv = (r < N && k < N) ? -M[r + (size_t)ld * k] : 0.0;
				if (sgrp == 0) dmma(a0[0], a0[1], uv, yb(u, 0));
				else dmma(a1[0], a1[1], uv, yb(u, 1));
			}
		}
		x[0] = a0[0] + a1[0];
		x[1] = a0[1] + a1[1];
		// upper 8 x 8 block, bottom up
#pragma unroll
		for (int q = 7; q >= 0; q--) {
			const int jq = 8 * t + q;
			double ujj = (jq < N) ? M[jq + (size_t)ld * jq] : 1.0;
			if (ujj == 0.0) ujj = 1.0;
			if (lq == q) {
				x[0] /= ujj;
				x[1] /= ujj;
			}
			const double y0 = __shfl_sync(0xffffffffu, x[0], 4 * q + lr);
			const double y1 = __shfl_sync(0xffffffffu, x[1], 4 * q + lr);
			if (lq < q && r < N && jq < N) {
				const double uv = M[r + (size_t)ld * jq];
				x[0] -= uv * y0;
				x[1] -= uv * y1;
			}
		}
		if (r < N) {
			if (cc < N) G[r + (size_t)N * cc] = x[0];
			if (cc + 1 < N) G[r + (size_t)N * (cc + 1)] = x[1];
		}
		c_to_b(x[0], x[1], yb(t, 0), yb(t, 1));
	}
}

// ----------------------------------------------- recombine in shared memory
//
// G = (D_b^-1 Q^H + D_s T)^-1 D_b^-1 Q^H (greens.c:157-178)
// with M in shared memory: LU with partial pivoting and physical row swaps
// (getrf: the first largest |M[r, j]| of the column, as idamax); warp 0
// picks, swaps and scales, all warps update the trailing columns.  Then
// each warp solves for its right-hand sides, CB at a time held in
// registers (permutation, unit-lower forward, upper backward), and the
// phase 1/phase(det G) = phase(det Q) phase(det M) sign(prod v).

// the recombine's shared memory: M (unless in global memory), the scale
// vectors and pivots, then (real M in shared memory) the solve slabs of
// recb_solve_warps warps, as many as fit under RECB_SMEM_CAP, at least one
constexpr size_t RECB_SMEM_CAP = 226 * 1024;

template <typename T>
__host__ __device__ inline size_t recb_base_bytes(int N, bool gm)
{
	// a multiple of 16 bytes, where the solve slabs start
	return ((gm ? 0 : sizeof(T) * (size_t)qrb_ld(N) * N) + sizeof(double) * 2 * (size_t)N
	        + sizeof(int) * 2 * (size_t)N + 64 + 15) & ~(size_t)15;
}

__host__ __device__ inline size_t recb_slab_bytes(int N) { return sizeof(double) * 64 * (size_t)((N + 7) / 8); }

template <typename T>
__host__ __device__ inline int recb_solve_warps(int N, bool gm)
{
	if (is_cplx<T>::value || gm) return 0;
	const size_t base = recb_base_bytes<T>(N, gm), slab = recb_slab_bytes(N);
	const size_t fit = base < RECB_SMEM_CAP ? (RECB_SMEM_CAP - base) / slab : 0;
	return fit < 1 ? 1 : (fit > 16 ? 16 : (int)fit);
}

template <typename T>
size_t recb_smem_bytes(int N, bool gm = false)
{
	return recb_base_bytes<T>(N, gm) + recb_slab_bytes(N) * recb_solve_warps<T>(N, gm);
}

template <typename T, int NW, int RPL, int CB, bool GM>
__global__ void __launch_bounds__(NW * 32) k_recb(RecArgs<T> a)
{
	const int item = blockIdx.x;
	if (item >= a.batch) return;
	const int N = a.N, ld = GM ? N : qrb_ld(N);
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	extern __shared__ __align__(16) unsigned char smraw[];
	// N columns, leading dimension ld
	T *M = GM ? a.work + (size_t)item * a.w_stride : (T *)smraw;
	double *vsh = GM ? (double *)smraw : (double *)(M + (size_t)ld * N);   // D_b^-1
	double *dss = vsh + N;                      // D_s
	int *ipiv = (int *)(dss + N);               // row swapped with row j at step j
	int *perm = ipiv + N;                       // row r of P Y is row perm[r] of Y
	if (N > 32 * RPL) {
		if (tid == 0 && a.err) atomicOr(a.err, DQ_ERR_SIZE);
		return;
	}
	const T *Q = a.Q + (size_t)item * a.q_stride;
	const T *Tm = a.Tm + (size_t)item * a.t_stride;
	const double *d = a.d + (size_t)item * a.d_stride;
	for (int r = tid; r < N; r += blockDim.x) {
		const double dr = d[r];
		if (fabs(dr) > 1.0) { vsh[r] = 1.0 / dr; dss[r] = 1.0; }
		else { vsh[r] = 1.0; dss[r] = dr; }
	}
	__syncthreads();
	for (int c = w; c < N; c += NW)
		for (int r = lane; r < N; r += 32)
			M[r + (size_t)ld * c] = conjv(Q[c + (size_t)N * r]) * vsh[r] + Tm[r + (size_t)N * c] * dss[r];
	__syncthreads();

	bool nan_seen = false, sing = false;
	// Pivot of column j (warp 0): the first largest |M[r, j]|, r >= j, as
	// idamax; rows j and the pivot row swapped in column j only (the other
	// columns swap them when step j reaches them); multipliers scaled.
	auto pivot_col = [&](int j) {
		double best = -1.0;
		int br = N;
		for (int r = j + lane; r < N; r += 32) {
			double m = absv(M[r + (size_t)ld * j]);
			if (!(m >= 0.0)) {
				m = -0.5;
				nan_seen = true;
			}
			if (m > best) { best = m; br = r; }
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			const double ob = __shfl_xor_sync(0xffffffffu, best, o);
			const int orr = __shfl_xor_sync(0xffffffffu, br, o);
			if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
		}
		if (lane == 0) {
			if (br != j) {
				const T t0 = M[j + (size_t)ld * j];
				M[j + (size_t)ld * j] = M[br + (size_t)ld * j];
				M[br + (size_t)ld * j] = t0;
			}
			ipiv[j] = br;
		}
		__syncwarp();
		T piv = M[j + (size_t)ld * j];
		if (re(piv) == 0.0 && im(piv) == 0.0) {
			sing = true;
			piv = one<T>();
		}
		const T ip = one<T>() / piv;
		for (int r = j + 1 + lane; r < N; r += 32) M[r + (size_t)ld * j] *= ip;
	};
	// Step j on column c > j (one warp): the row swap of step j, then the
	// rank-1 update with the multipliers l of column j
	auto update_col = [&](int j, int pj, int c, const T (&l)[RPL]) {
		T *col = M + (size_t)ld * c;
		if (lane == 0 && pj != j) {
			const T t0 = col[j];
			col[j] = col[pj];
			col[pj] = t0;
		}
		__syncwarp();
		const T u = col[j];
#pragma unroll
		for (int t = 0; t < RPL; t++) {
			const int r = j + 1 + lane + 32 * t;
			if (r < N) col[r] -= l[t] * u;
		}
	};
	// One barrier per step: warp 0 updates column j + 1 and pivots it for
	// the next step (look-ahead) while warps 1.. update the other columns and
	// apply the step's row swap to the columns left of j (the L factor).
	if (w == 0) pivot_col(0);
	__syncthreads();
	for (int j = 0; j < N; j++) {
		const int pj = ipiv[j];
		T l[RPL];
#pragma unroll
		for (int t = 0; t < RPL; t++) {
			const int r = j + 1 + lane + 32 * t;
			l[t] = (r < N) ? M[r + (size_t)ld * j] : zero<T>();
		}
		if (w == 0) {
			if (j + 1 < N) {
				update_col(j, pj, j + 1, l);
				__syncwarp();
				pivot_col(j + 1);
			}
		} else {
			if (pj != j)
				for (int c = tid - 32; c < j; c += blockDim.x - 32) {
					const T t0 = M[j + (size_t)ld * c];
					M[j + (size_t)ld * c] = M[pj + (size_t)ld * c];
					M[pj + (size_t)ld * c] = t0;
				}
			for (int c = j + 1 + w; c < N; c += NW - 1) update_col(j, pj, c, l);
		}
		__syncthreads();
	}
	nan_seen = __any_sync(0xffffffffu, nan_seen);
	sing = __any_sync(0xffffffffu, sing);
	if (tid == 0) {
		for (int r = 0; r < N; r++) perm[r] = r;
		for (int j = 0; j < N; j++) {
			const int q = ipiv[j];
			const int t0 = perm[j];
			perm[j] = perm[q];
			perm[q] = t0;
		}
	}
	if (w == 0 && lane == 0) {
		if (nan_seen && a.err) atomicOr(a.err, DQ_ERR_NAN);
		if (sing && a.err) atomicOr(a.err, DQ_ERR_SINGULAR);
	}
	__syncthreads();

	// right-hand sides Y = D_b^-1 Q^H, CB columns per pass of a warp
	T *G = a.G + (size_t)item * a.g_stride;
	constexpr bool TC = !is_cplx<T>::value && !GM;   // real, shared memory: DMMA tiles
	if constexpr (TC) {
		const int nws = min(NW, recb_solve_warps<T>(N, GM));
		double *ys = (double *)(smraw + recb_base_bytes<T>(N, GM))
		             + (size_t)64 * ((N + 7) / 8) * w;
		for (int c0 = 8 * w; w < nws && c0 < N; c0 += 8 * nws)
			recb_solve8((const double *)M, ld, perm, vsh, (const double *)Q, (double *)G, N, c0,
			                     lane, ys);
	}
	for (int c0 = w * CB; !TC && c0 < N; c0 += NW * CB) {
		T y[CB][RPL];
#pragma unroll
		for (int b = 0; b < CB; b++) {
			const int c = c0 + b;
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				const int pr = (r < N) ? perm[r] : 0;
				y[b][t] = (c < N && r < N) ? conjv(Q[c + (size_t)N * pr]) * vsh[pr] : zero<T>();
			}
		}
		// L (unit lower)
		for (int k = 0; k < N - 1; k++) {
			const int tk = k >> 5, lk = k & 31;
			T yk[CB];
#pragma unroll
			for (int b = 0; b < CB; b++) {
				T v = zero<T>();
#pragma unroll
				for (int t = 0; t < RPL; t++)
					if (t == tk) v = y[b][t];
				yk[b] = shfl(v, lk);
			}
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				if (r > k && r < N) {
					const T lv = M[r + (size_t)ld * k];
#pragma unroll
					for (int b = 0; b < CB; b++) y[b][t] -= lv * yk[b];
				}
			}
		}
		// U
		for (int k = N - 1; k >= 0; k--) {
			const int tk = k >> 5, lk = k & 31;
			T ukk = M[k + (size_t)ld * k];
			if (re(ukk) == 0.0 && im(ukk) == 0.0) ukk = one<T>();
			const T iu = one<T>() / ukk;
			T yk[CB];
#pragma unroll
			for (int b = 0; b < CB; b++) {
				T v = zero<T>();
#pragma unroll
				for (int t = 0; t < RPL; t++)
					if (t == tk) v = y[b][t];
				yk[b] = shfl(v, lk) * iu;
			}
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				if (r < k) {
					const T uv = M[r + (size_t)ld * k];
#pragma unroll
					for (int b = 0; b < CB; b++) y[b][t] -= uv * yk[b];
				} else if (r == k) {
#pragma unroll
					for (int b = 0; b < CB; b++) y[b][t] = yk[b];
				}
			}
		}
#pragma unroll
		for (int b = 0; b < CB; b++) {
			const int c = c0 + b;
			if (c >= N) continue;
#pragma unroll
			for (int t = 0; t < RPL; t++) {
				const int r = lane + 32 * t;
				if (r < N) G[r + (size_t)N * c] = y[b][t];
			}
		}
	}
	if (w == 0) {
		// phase(det) = phase(det Q) prod phase(U_jj) sign(prod v_j) (-1)^swaps,
		// each lane taking every 32nd j, then a butterfly over the warp
		T ph = one<T>();
		int neg = 0;
		double l = 0.0;
		for (int j = lane; j < N; j += 32) {
			const T u = M[j + (size_t)ld * j];
			ph = ph * phase_of(u);
			neg ^= (vsh[j] < 0.0) ^ (ipiv[j] != j);
			// G = M^-1 diag(v) Q^H: log |det G| = sum log |v_j| - sum log |U_jj|
			if (a.logdet) l += log(absv(u)) - log(fabs(vsh[j]));
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			ph = ph * shfl_xor(ph, o);
			neg ^= __shfl_xor_sync(0xffffffffu, neg, o);
			l += __shfl_xor_sync(0xffffffffu, l, o);
		}
		if (lane == 0) {
			if (a.qdet) ph = a.qdet[item] * ph;
			a.phase[item] = neg ? ph * -1.0 : ph;
			if (a.logdet) a.logdet[item] = l;
		}
	}
}

}  // namespace dq
