// The dense factorisations of the stabilised equal-time Green's function
// (reference src/greens.c:69-208, calc_eq_g), one CTA per (chain, spin)
// matrix with the working matrix held in registers:
//
//   warp w owns columns c = w + NW*q (q < CPW), lane l owns rows l + 32*p
//   (p < RPL); Householder vectors and scalars live in shared memory.
//
// k_qr      Householder QR that picks, at each step, which remaining column
//           to eliminate next, so no columns are moved:
//             QR_PIVOT   largest remaining partial column norm, with the norm
//                        downdating and recomputation rule of LAPACK geqp3
//                        (greens.c:89);
//             QR_PRESORT columns in order of decreasing norm, computed once
//                        after scaling by d (the norm pre-pivoting of
//                        greens.c:112-135), then unpivoted.
//           Q is formed explicitly (so that later g*Q is a plain GEMM and
//           diag(v) Q^H is elementwise), with the phase of det Q.
// k_recombine  G = (D_b^-1 Q^H + D_s T)^-1 D_b^-1 Q^H (greens.c:157-178) by
//           LU with partial (implicit) row pivoting and a two-sided solve,
//           plus the phase of det G (greens.c:194-207).
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
	unsigned *err;
};

template <typename T, int RPL, int CPW, int NW>
struct QrShape {
	static constexpr int NMAX = 32 * RPL < NW * CPW ? 32 * RPL : NW * CPW;
	static constexpr int THREADS = NW * 32;
};

template <typename T>
size_t qr_smem_bytes(int N, int nw)
{
	return sizeof(T) * ((size_t)N * N + N) + sizeof(double) * (4 * (size_t)N + 2 * nw)
	       + sizeof(int) * (3 * (size_t)N + 2 * nw) + 64;
}

// select slot q of a register array with a compile-time bound
template <typename T, int NQ>
__device__ inline T pick(const T (&arr)[NQ], int q)
{
	T v = arr[0];
#pragma unroll
	for (int i = 1; i < NQ; i++)
		if (i == q) v = arr[i];
	return v;
}

template <typename T, int RPL, int CPW, int NW>
__global__ void __launch_bounds__(NW * 32) k_qr(QrArgs<T> a)
{
	const int item = blockIdx.x;
	if (item >= a.batch) return;
	const int N = a.N;
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	extern __shared__ __align__(16) unsigned char smraw[];
	T *V = (T *)smraw;                          // N*N reflectors, column j = v_j
	T *tau = V + (size_t)N * N;                 // N
	double *vn1 = (double *)(tau + N);          // N partial norms
	double *vn2 = vn1 + N;                      // N norms at last recompute
	double *dsh = vn2 + N;                      // N diag(R)
	double *vv = dsh + N;                       // N  v^H v
	double *cval = vv + N;                      // NW candidate norms
	int *used = (int *)(cval + NW);             // N  column eliminated?
	int *pvt = used + N;                        // N  column chosen at step j
	int *pos = pvt + N;                         // N  step at which column c was chosen
	int *ccol = pos + N;                        // NW candidate columns
	__shared__ int s_col;

	const T *X = a.X + (size_t)item * a.x_stride;
	T x[CPW][RPL];
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
		const double sc = (a.mode == QR_PRESORT && c < N) ? a.dcol[(size_t)item * a.d_stride + c] : 1.0;
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			x[q][p] = (c < N && r < N) ? X[r + (size_t)N * c] * sc : zero<T>();
		}
	}
	for (int c = tid; c < N; c += blockDim.x) used[c] = 0;
	// column norms
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		double s = 0.0;
#pragma unroll
		for (int p = 0; p < RPL; p++) s += abs2(x[q][p]);
		s = warp_sum(s);
		const int c = w + NW * q;
		if (lane == 0 && c < N) {
			vn1[c] = (a.mode == QR_PIVOT) ? sqrt(s) : s;
			vn2[c] = vn1[c];
		}
	}
	__syncthreads();
	if (a.mode == QR_PRESORT) {
		// stable descending order of the squared norms (greens.c:123-129)
		for (int c = tid; c < N; c += blockDim.x) {
			const double v = vn1[c];
			int rank = 0;
			for (int o = 0; o < N; o++) {
				const double u = vn1[o];
				rank += (u > v) || (u == v && o < c);
			}
			pvt[rank] = c;
			pos[c] = rank;
		}
		__syncthreads();
	}

	const double tol3z = sqrt(2.220446049250313e-16);
	for (int j = 0; j < N; j++) {
		int cj;
		if (a.mode == QR_PIVOT) {
			// warp candidates: largest partial norm among remaining columns
			double best = -1.0;
			int bc = N;
#pragma unroll
			for (int q = 0; q < CPW; q++) {
				const int c = w + NW * q;
				if (c < N && !used[c]) {
					const double v = vn1[c];
					if (v > best || (v == best && c < bc)) { best = v; bc = c; }
				}
			}
			if (lane == 0) { cval[w] = best; ccol[w] = bc; }
			__syncthreads();
			if (tid == 0) {
				double bb = -1.0;
				int bcol = N;
				for (int q = 0; q < NW; q++)
					if (cval[q] > bb || (cval[q] == bb && ccol[q] < bcol)) { bb = cval[q]; bcol = ccol[q]; }
				s_col = bcol;
				pvt[j] = bcol;
				pos[bcol] = j;
				used[bcol] = 1;
			}
			__syncthreads();
			cj = s_col;
		} else {
			cj = pvt[j];
			if (tid == 0) used[cj] = 1;
		}
		const int ow = cj % NW, oq = cj / NW;
		if (w == ow) {
			T col[RPL];
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				T v = x[0][p];
#pragma unroll
				for (int q = 1; q < CPW; q++)
					if (q == oq) v = x[q][p];
				col[p] = v;
			}
			// alpha = row j, sigma = sum over rows > j
			double sig = 0.0;
			T alpha = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				const int r = lane + 32 * p;
				if (r > j && r < N) sig += abs2(col[p]);
				if (r == j) alpha = col[p];
			}
			sig = warp_sum(sig);
			alpha = shfl(alpha, j & 31);
			const double anorm2 = abs2(alpha);
			T tj, scal;
			double beta;
			if (sig == 0.0 && im(alpha) == 0.0) {
				tj = zero<T>();
				beta = re(alpha);
				scal = zero<T>();
			} else {
				beta = -copysign(sqrt(anorm2 + sig), re(alpha));
				tj = (from_re<T>(beta) - alpha) / beta;
				scal = one<T>() / (alpha - beta);
			}
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				const int r = lane + 32 * p;
				if (r < N) {
					T v;
					if (r < j) v = zero<T>();
					else if (r == j) v = one<T>();
					else v = col[p] * scal;
					V[r + (size_t)N * j] = v;
					if (r == j) col[p] = from_re<T>(beta);
					else if (r > j) col[p] = zero<T>();
				}
			}
			if (lane == 0) {
				tau[j] = tj;
				dsh[j] = beta;
				vv[j] = 1.0 + sig * abs2(scal);
			}
#pragma unroll
			for (int q = 0; q < CPW; q++)
				if (q == oq)
#pragma unroll
					for (int p = 0; p < RPL; p++) x[q][p] = col[p];
		}
		__syncthreads();
		// apply H_j^H = I - conj(tau) v v^H to the remaining columns
		const T ct = conjv(tau[j]);
		T vr[RPL];
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			vr[p] = (r < N) ? V[r + (size_t)N * j] : zero<T>();
		}
#pragma unroll
		for (int q = 0; q < CPW; q++) {
			const int c = w + NW * q;
			if (c >= N || c == cj) continue;
			if (a.mode == QR_PIVOT ? used[c] : (pos[c] <= j)) continue;
			T s = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++) s = fma_(conjv(vr[p]), x[q][p], s);
			s = warp_sum(s);
			const T f = ct * s;
#pragma unroll
			for (int p = 0; p < RPL; p++) x[q][p] = x[q][p] - vr[p] * f;
			if (a.mode == QR_PIVOT && vn1[c] != 0.0) {
				// partial norm downdate (LAPACK dlaqp2)
				T xj = zero<T>();
#pragma unroll
				for (int p = 0; p < RPL; p++)
					if (lane + 32 * p == j) xj = x[q][p];
				xj = shfl(xj, j & 31);
				double t = absv(xj) / vn1[c];
				t = fmax(0.0, 1.0 - t * t);
				const double t2 = t * (vn1[c] / vn2[c]) * (vn1[c] / vn2[c]);
				double nv;
				const bool recompute = t2 <= tol3z;
				if (recompute) {
					double s2 = 0.0;
#pragma unroll
					for (int p = 0; p < RPL; p++)
						if (lane + 32 * p > j && lane + 32 * p < N) s2 += abs2(x[q][p]);
					s2 = warp_sum(s2);
					nv = sqrt(s2);
				} else {
					nv = vn1[c] * sqrt(t);
				}
				__syncwarp();
				if (lane == 0) {
					vn1[c] = nv;
					if (recompute) vn2[c] = nv;
				}
				__syncwarp();
			}
		}
	}
	__syncthreads();

	// R outputs: the register column of original index c holds R[:, pos[c]]
	const size_t NN = (size_t)N * N;
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
		if (c >= N) continue;
		const int jc = pos[c];
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			if (r >= N) continue;
			const double dr = dsh[r] == 0.0 ? 1.0 : dsh[r];
			const T v = (r <= jc) ? x[q][p] / dr : zero<T>();
			if (a.mode == QR_PIVOT) a.Tout[(size_t)item * a.t_stride + r + (size_t)N * c] = v;
			else a.Rs[(size_t)item * a.r_stride + r + (size_t)N * jc] = v;
		}
	}
	for (int r = tid; r < N; r += blockDim.x) {
		a.dout[(size_t)item * a.dout_stride + r] = dsh[r] == 0.0 ? 1.0 : dsh[r];
		if (a.pvt) a.pvt[(size_t)item * a.p_stride + r] = pvt[r];
	}
	(void)NN;

	// explicit Q = H_0 H_1 ... H_{N-1}: columns by position, reflectors backwards
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
#pragma unroll
		for (int p = 0; p < RPL; p++) x[q][p] = (lane + 32 * p == c) ? one<T>() : zero<T>();
	}
	for (int j = N - 1; j >= 0; j--) {
		const T tj = tau[j];
		T vr[RPL];
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			vr[p] = (r < N) ? V[r + (size_t)N * j] : zero<T>();
		}
#pragma unroll
		for (int q = 0; q < CPW; q++) {
			const int c = w + NW * q;
			if (c < j || c >= N) continue;
			T s = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++) s = fma_(conjv(vr[p]), x[q][p], s);
			s = warp_sum(s);
			const T f = tj * s;
#pragma unroll
			for (int p = 0; p < RPL; p++) x[q][p] = x[q][p] - vr[p] * f;
		}
	}
	T *Q = a.Q + (size_t)item * a.q_stride;
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
		if (c >= N) continue;
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			if (r < N) Q[r + (size_t)N * c] = x[q][p];
		}
	}
	if (tid == 0 && a.qdet) {
		T ph = one<T>();
		for (int j = 0; j < N; j++) ph = ph * phase_of(one<T>() - tau[j] * vv[j]);
		a.qdet[item] = ph;
	}
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
	unsigned *err;
};

template <typename T>
size_t rec_smem_bytes(int N)
{
	return sizeof(T) * ((size_t)N * N + N) + sizeof(int) * 3 * (size_t)N + sizeof(double) * 2 * N + 64;
}

template <typename T, int RPL, int CPW, int NW>
__global__ void __launch_bounds__(NW * 32) k_recombine(RecArgs<T> a)
{
	const int item = blockIdx.x;
	if (item >= a.batch) return;
	const int N = a.N;
	const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
	extern __shared__ __align__(16) unsigned char smraw[];
	T *LU = (T *)smraw;                 // N*N
	T *lcol = LU + (size_t)N * N;       // N current multipliers
	double *vsh = (double *)(lcol + N); // N  v = D_b^-1
	double *dss = vsh + N;              // N  D_s
	int *prow = (int *)(dss + N);       // N pivot row of step j
	int *stepof = prow + N;             // N step at which row r became pivot
	int *rused = stepof + N;            // N
	__shared__ int s_prow;

	const T *Q = a.Q + (size_t)item * a.q_stride;
	const T *Tm = a.Tm + (size_t)item * a.t_stride;
	const double *d = a.d + (size_t)item * a.d_stride;
	for (int r = tid; r < N; r += blockDim.x) {
		const double dr = d[r];
		if (fabs(dr) > 1.0) { vsh[r] = 1.0 / dr; dss[r] = 1.0; }
		else { vsh[r] = 1.0; dss[r] = dr; }
		rused[r] = 0;
	}
	__syncthreads();
	// M = diag(v) Q^H + diag(ds) T
	T x[CPW][RPL];
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			x[q][p] = (c < N && r < N) ? conjv(Q[c + (size_t)N * r]) * vsh[r] + Tm[r + (size_t)N * c] * dss[r]
			                           : zero<T>();
		}
	}
	// LU, implicit partial pivoting: rows stay put, prow[j] is the pivot row
	for (int j = 0; j < N; j++) {
		const int ow = j % NW, oq = j / NW;
		if (w == ow) {
			T col[RPL];
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				T v = x[0][p];
#pragma unroll
				for (int q = 1; q < CPW; q++)
					if (q == oq) v = x[q][p];
				col[p] = v;
			}
			double best = -1.0;
			int br = N;
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				const int r = lane + 32 * p;
				if (r < N && !rused[r]) {
					const double m = absv(col[p]);
					if (m > best || (m == best && r < br)) { best = m; br = r; }
				}
			}
			for (int o = 16; o > 0; o >>= 1) {
				const double ob = __shfl_xor_sync(0xffffffffu, best, o);
				const int orr = __shfl_xor_sync(0xffffffffu, br, o);
				if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
			}
			T piv = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++)
				if (lane + 32 * p == br) piv = col[p];
			piv = shfl(piv, br & 31);
			if (re(piv) == 0.0 && im(piv) == 0.0) {
				if (lane == 0 && a.err) atomicOr(a.err, DQ_ERR_SINGULAR);
				piv = one<T>();
			}
			const T ipiv = one<T>() / piv;
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				const int r = lane + 32 * p;
				if (r < N) {
					const T l = (!rused[r] && r != br) ? col[p] * ipiv : zero<T>();
					lcol[r] = l;
					if (!rused[r] && r != br) LU[r + (size_t)N * j] = l;
				}
			}
			if (lane == 0) {
				s_prow = br;
				prow[j] = br;
				stepof[br] = j;
			}
		}
		__syncthreads();
		const int pr = s_prow;
		if (tid == 0) rused[pr] = 1;
		T lr[RPL];
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			lr[p] = (r < N) ? lcol[r] : zero<T>();
		}
#pragma unroll
		for (int q = 0; q < CPW; q++) {
			const int c = w + NW * q;
			if (c <= j || c >= N) continue;
			T xp = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++)
				if (lane + 32 * p == pr) xp = x[q][p];
			xp = shfl(xp, pr & 31);
#pragma unroll
			for (int p = 0; p < RPL; p++) x[q][p] = x[q][p] - lr[p] * xp;
		}
		__syncthreads();
	}
	// U entries: row r holds U[stepof[r]][c] for c >= stepof[r]
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
		if (c >= N) continue;
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			if (r < N && stepof[r] <= c) LU[r + (size_t)N * c] = x[q][p];
		}
	}
	__syncthreads();

	// right-hand sides Y = diag(v) Q^H, solve M G = Y
	int sr[RPL];
#pragma unroll
	for (int p = 0; p < RPL; p++) {
		const int r = lane + 32 * p;
		sr[p] = r < N ? stepof[r] : -1;
	}
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			x[q][p] = (c < N && r < N) ? conjv(Q[c + (size_t)N * r]) * vsh[r] : zero<T>();
		}
	}
	// forward: eliminate below the pivots in step order
	for (int j = 0; j < N; j++) {
		const int pr = prow[j];
		T m[RPL];
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			m[p] = (r < N && sr[p] > j) ? LU[r + (size_t)N * j] : zero<T>();
		}
#pragma unroll
		for (int q = 0; q < CPW; q++) {
			T yp = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++)
				if (lane + 32 * p == pr) yp = x[q][p];
			yp = shfl(yp, pr & 31);
#pragma unroll
			for (int p = 0; p < RPL; p++) x[q][p] = x[q][p] - m[p] * yp;
		}
	}
	// backward: x_j = y[prow j] / U_jj, then remove it from earlier pivot rows
	for (int j = N - 1; j >= 0; j--) {
		const int pr = prow[j];
		const T ujj = LU[pr + (size_t)N * j];
		const T iu = (re(ujj) == 0.0 && im(ujj) == 0.0) ? one<T>() : one<T>() / ujj;
		T u[RPL];
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			u[p] = (r < N && sr[p] < j) ? LU[r + (size_t)N * j] : zero<T>();
		}
#pragma unroll
		for (int q = 0; q < CPW; q++) {
			T yp = zero<T>();
#pragma unroll
			for (int p = 0; p < RPL; p++)
				if (lane + 32 * p == pr) yp = x[q][p];
			yp = shfl(yp, pr & 31) * iu;
#pragma unroll
			for (int p = 0; p < RPL; p++) {
				if (lane + 32 * p == pr) x[q][p] = yp;
				else x[q][p] = x[q][p] - u[p] * yp;
			}
		}
	}
	T *G = a.G + (size_t)item * a.g_stride;
#pragma unroll
	for (int q = 0; q < CPW; q++) {
		const int c = w + NW * q;
		if (c >= N) continue;
#pragma unroll
		for (int p = 0; p < RPL; p++) {
			const int r = lane + 32 * p;
			if (r < N) G[sr[p] + (size_t)N * c] = x[q][p];
		}
	}
	if (tid == 0) {
		// 1/phase(det G) = phase(det M) conj(phase(prod v)) phase(det Q)
		T ph = a.qdet ? a.qdet[item] : one<T>();
		double vs = 1.0;
		for (int j = 0; j < N; j++) {
			ph = ph * phase_of(LU[prow[j] + (size_t)N * j]);
			vs *= (vsh[j] < 0.0) ? -1.0 : 1.0;
		}
		// sign of the permutation j -> prow[j]
		int parity = 0;
		for (int j = 0; j < N; j++) rused[j] = 0;
		for (int j = 0; j < N; j++) {
			if (rused[j]) continue;
			int len = 0, q = j;
			while (!rused[q]) { rused[q] = 1; q = prow[q]; len++; }
			parity ^= (len - 1) & 1;
		}
		if (parity) ph = ph * -1.0;
		a.phase[item] = ph * vs;
	}
}

}  // namespace dq
