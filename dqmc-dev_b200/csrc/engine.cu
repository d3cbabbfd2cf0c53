// Host side of the GPU engine: device state of a group of chains, the
// sequencing of one sweep (reference src/dqmc.c:222-459) as batched kernel
// launches, CUDA-graph capture per sweep kind, and the C ABI of
// include/dqmc_b200.h.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <unistd.h>
#include <cstring>
#include <map>
#include <new>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "dqmc_b200.h"
#include "launch.cuh"
#include "meas.cuh"
#include "meas_x.cuh"
#include "update.cuh"
#include "update_cl.cuh"
#include "uneq.cuh"

namespace dq {

#define CK(x)                                                                      \
	do {                                                                           \
		cudaError_t e_ = (x);                                                      \
		if (e_ != cudaSuccess) {                                                   \
			fprintf(stderr, "dqmc_b200: %s failed: %s (%s:%d)\n", #x,              \
			        cudaGetErrorString(e_), __FILE__, __LINE__);                   \
			return DQMC_E_CUDA;                                                    \
		}                                                                          \
	} while (0)

static inline Addr per_item(long long stride) { return Addr{stride, 0, 1}; }
static inline Addr per_spin(long long stride) { return Addr{0, stride, 2}; }

// ------------------------------------------------------------------ launches

template <typename T>
static GemmArgs<T> gargs(int M, int N, int K, int batch, const T *A, Addr aA, int lda,
		const T *B, Addr aB, int ldb, T *C, Addr aC, int ldc, T alpha = one<T>(),
		T beta = zero<T>(), int mode = 0)
{
	GemmArgs<T> g;
	memset(&g, 0, sizeof(g));
	g.M = M; g.N = N; g.K = K; g.batch = batch;
	g.A = A; g.aA = aA; g.lda = lda;
	g.B = B; g.aB = aB; g.ldb = ldb;
	g.C = C; g.aC = aC; g.ldc = ldc;
	g.alpha = alpha; g.beta = beta; g.mode = mode;
	g.aD = Addr{0, 0, 1};
	g.aG = Addr{0, 0, 1};
	return g;
}

// ------------------------------------------------------- small helper kernels

// G drift of one recalculation, one block per item: the largest and the
// mean |G - G_wrapped| over the N x N entries (the reference's matdiff,
// dqmc.c:61-71), folded into the item's running maximum (non-negative
// doubles order as their bit patterns) and running sum of means; block 0
// counts the recalculations
template <typename T>
__global__ void k_gdrift(int N, const T *G, const T *Gw, long long w_stride,
		unsigned long long *dmax, double *dsum, int *count)
{
	const int b = blockIdx.x;
	const long long NN = (long long)N * N;
	const T *g = G + b * NN, *w = Gw + b * w_stride;
	double mx = 0.0, sm = 0.0;
	for (long long q = threadIdx.x; q < NN; q += blockDim.x) {
		const double d = absv(g[q] - w[q]);
		mx = (mx != mx) ? mx : ((d != d) ? d : fmax(mx, d));   // a NaN stays
		sm += d;
	}
	__shared__ double smx[8], ssm[8];
	for (int o = 16; o > 0; o >>= 1) {
		const double om = __shfl_xor_sync(0xffffffffu, mx, o);
		mx = (mx != mx) ? mx : ((om != om) ? om : fmax(mx, om));
		sm += __shfl_xor_sync(0xffffffffu, sm, o);
	}
	const int lane = threadIdx.x & 31, w8 = threadIdx.x >> 5;
	if (lane == 0) {
		smx[w8] = mx;
		ssm[w8] = sm;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
			mx = (mx != mx) ? mx : ((smx[k] != smx[k]) ? smx[k] : fmax(mx, smx[k]));
			sm += ssm[k];
		}
		atomicMax(dmax + b, (unsigned long long)__double_as_longlong(mx));
		dsum[b] += sm / (double)NN;
		if (b == 0) count[0] += 1;
	}
}

// d_l and 1/d_l of every slice from the fields: spin s uses exp_lambda[i + N*(h^s)]
__global__ void k_diag_all(int N, int L, int nchain, const double *el, const int *hs,
		double *dv, double *dvi)
{
	const long long total = (long long)nchain * 2 * L * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
	     q += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(q % N);
		const int l = (int)((q / N) % L);
		const int s = (int)((q / ((long long)N * L)) % 2);
		const int c = (int)(q / (2LL * N * L));
		const int h = hs[((size_t)c * L + l) * N + i];
		const double v = el[(size_t)c * 2 * N + i + N * (h ^ s)];
		dv[q] = v;
		dvi[q] = 1.0 / v;
	}
}

// out[b] = in[b] * diag(d[b])  (N x N)
template <typename T>
__global__ void k_colscale(int N, int batch, const T *in, Addr ain, const double *d, Addr ad,
		T *out, Addr aout)
{
	const long long NN = (long long)N * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < NN * batch;
	     q += (long long)gridDim.x * blockDim.x) {
		const int b = (int)(q / NN);
		const long long e = q % NN;
		const int c = (int)(e / N);
		out[aout.off(b) + e] = in[ain.off(b) + e] * d[ad.off(b) + c];
	}
}

template <typename T>
__global__ void k_copy(long long n, const T *in, T *out)
{
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
	     q += (long long)gridDim.x * blockDim.x)
		out[q] = in[q];
}

template <typename T>
__global__ void k_combine_phase(int nchain, const T *phi, T *phase)
{
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c < nchain) phase[c] = phi[2 * c] * phi[2 * c + 1];
}

static int grid_for(long long n, int threads = 256)
{
	long long g = (n + threads - 1) / threads;
	if (g > 148 * 16) g = 148 * 16;
	return (int)(g < 1 ? 1 : g);
}

// ------------------------------------------------- calc_eq_g as launches

// device buffers the stabilised G computation works in, NB items each
template <typename T>
struct EqWork {
	int N, F, NB;
	const T *Cl; long long cl_stride;  // cluster matrices: item b, cluster f at
	                                   // Cl + b*cl_stride + f*N*N
	T *Qm, *Tm, *Tm2, *Rs, *X, *W;     // NB x N*N each
	double *dR;                        // NB x N
	int *pvt;                          // NB x N
	T *qdet;                           // NB
	T *G; long long g_stride;          // output
	T *phi;                            // NB output phases
	double *logdet;                    // NB, optional: log |det(I + C...C)|
	const T *Pr; long long pr_stride;  // optional cache of the pair products
	                                   // C_{(m+1)%F} C_m at Pr + b*pr_stride + m*N*N
	unsigned *err;
};

// per-launch timing of an eager sweep: begin() before a launch, end() after
// it with the launch class and its algorithmic FLOPs and operand bytes
struct ProfHook {
	virtual void begin() = 0;
	virtual void end(int cls, double flops, double bytes) = 0;
};

// launch classes of the per-launch profile (dqmc_engine_profile_sweep)
enum : int {
	PC_GEMM = 0, PC_UPDATE = 1, PC_QR_PIVOT = 2, PC_UNEQ = 3, PC_MEAS = 4, PC_QR_PRESORT = 5,
	PC_RECOMBINE = 6, PC_COUNT = 7
};

template <typename T>
static double gemm_flops(const GemmArgs<T> &g)
{
	double fl = 2.0 * g.M * g.N * g.K * g.batch * (is_cplx<T>::value ? 4.0 : 1.0);
	return (g.mode & GM_A_UPPER) ? 0.5 * fl : fl;
}

template <typename T>
static double gemm_bytes(const GemmArgs<T> &g)
{
	return (double)sizeof(T) * ((double)g.M * g.K + (double)g.K * g.N + (double)g.M * g.N) * g.batch;
}

// QR with explicit Q (geqrf 4/3 N^3 + orgqr 4/3 N^3) and the recombine's
// LU with N right-hand sides (2/3 N^3 + 2 N^3): both 8/3 N^3 per item
template <typename T>
static double dense_flops(int N, int batch)
{
	return 8.0 / 3.0 * (double)N * N * N * batch * (is_cplx<T>::value ? 4.0 : 1.0);
}

template <typename T>
static int eq_gemm(const GemmArgs<T> &g, cudaStream_t st, int *count, ProfHook *ph = nullptr,
		unsigned *err = nullptr)
{
	if (ph) ph->begin();
	GemmArgs<T> ge = g;
	if (!ge.err) ge.err = err;
	const int rc = launch_gemm<T>(ge, st);
	if (ph) ph->end(PC_GEMM, gemm_flops(g), gemm_bytes(g));
	if (count) (*count)++;
	return rc;
}

// G = (I + C_{l0-1} ... C_{l0})^-1 over the F clusters (cyclic), grouped two
// clusters at a time as calc_eq_g(l0, N, F, 2, C, ...) does (greens.c:69-208),
// or one at a time (group 1: calc_eq_g(l0, N, L, 1, B, ...), a QR after every
// factor, as the reference's CHECK_G_ACC calls it, dqmc.c:283-287)
template <typename T>
static int run_calc_eq_g(const EqWork<T> &w, int l0, cudaStream_t st, int *count,
		ProfHook *ph = nullptr, int group = 2)
{
	const int N = w.N, F = w.F, NB = w.NB;
	const size_t NN = (size_t)N * N;
	const Addr aCl = Addr{w.cl_stride, 0, 1}, aI = Addr{(long long)NN, 0, 1};
	auto clu = [&](int f) { return w.Cl + (size_t)(((f % F) + F) % F) * NN; };
	if (group != 1 && group != 2) return DQMC_E_ARG;
	int m = (l0 + 1 + (F - 1) % group) % F;
	QrArgs<T> q;
	memset(&q, 0, sizeof(q));
	q.N = N; q.batch = NB; q.err = w.err;
	q.Q = w.Qm; q.q_stride = NN;
	q.dout = w.dR; q.dout_stride = N;
	q.qdet = w.qdet;
	q.pvt = w.pvt; q.p_stride = N;
	q.work = w.W; q.w_stride = NN;     // free while a QR runs
	// factors in the first group: 1 + (F - 1) % group
	const int first = 1 + (F - 1) % group;
	if (first == 2 && w.Pr) {
		q.X = w.Pr + (size_t)l0 * NN; q.x_stride = w.pr_stride;
	} else if (first == 2) {
		eq_gemm(gargs<T>(N, N, N, NB, clu(l0 + 1), aCl, N, clu(l0), aCl, N, w.X, aI, N), st, count, ph, w.err);
		q.X = w.X; q.x_stride = NN;
	} else {
		q.X = clu(l0); q.x_stride = w.cl_stride;
	}
	q.mode = QR_PIVOT;
	q.Tout = w.Tm; q.t_stride = NN;
	const double qfl = dense_flops<T>(N, NB), qby = 3.0 * sizeof(T) * NN * NB;
	if (ph) ph->begin();
	if (launch_qr<T>(q, st)) return DQMC_E_ARG;
	if (ph) ph->end(PC_QR_PIVOT, qfl, qby);
	if (count) (*count)++;
	T *Tc = w.Tm, *Tn = w.Tm2;
	while (m != l0) {
		const int next = (m + group) % F;
		if (group == 1) {
			eq_gemm(gargs<T>(N, N, N, NB, clu(m), aCl, N, w.Qm, aI, N, w.X, aI, N), st, count, ph, w.err);
		} else if (w.Pr) {
			eq_gemm(gargs<T>(N, N, N, NB, w.Pr + (size_t)m * NN, Addr{w.pr_stride, 0, 1}, N, w.Qm, aI, N,
			                 w.X, aI, N), st, count, ph, w.err);
		} else {
			eq_gemm(gargs<T>(N, N, N, NB, clu(m + 1), aCl, N, clu(m), aCl, N, w.W, aI, N), st, count, ph, w.err);
			eq_gemm(gargs<T>(N, N, N, NB, w.W, aI, N, w.Qm, aI, N, w.X, aI, N), st, count, ph, w.err);
		}
		m = next;
		QrArgs<T> r = q;
		r.mode = QR_PRESORT;
		r.X = w.X; r.x_stride = NN;
		r.dcol = w.dR; r.d_stride = N;
		r.Tout = nullptr;
		r.Rs = w.Rs; r.r_stride = NN;
		if (ph) ph->begin();
		if (launch_qr<T>(r, st)) return DQMC_E_ARG;
		if (ph) ph->end(PC_QR_PRESORT, qfl, qby);
		if (count) (*count)++;
		GemmArgs<T> g = gargs<T>(N, N, N, NB, w.Rs, aI, N, Tc, aI, N, Tn, aI, N, one<T>(),
		                         zero<T>(), GM_A_UPPER | GM_B_GATHER);
		g.gidx = w.pvt;
		g.aG = Addr{(long long)N, 0, 1};
		eq_gemm(g, st, count, ph, w.err);
		T *t = Tc; Tc = Tn; Tn = t;
	}
	RecArgs<T> ra;
	memset(&ra, 0, sizeof(ra));
	ra.N = N; ra.batch = NB;
	ra.Q = w.Qm; ra.q_stride = NN;
	ra.Tm = Tc; ra.t_stride = NN;
	ra.d = w.dR; ra.d_stride = N;
	ra.qdet = w.qdet;
	ra.G = w.G; ra.g_stride = w.g_stride;
	ra.phase = w.phi;
	ra.work = w.W; ra.w_stride = NN;
	ra.logdet = w.logdet;
	ra.err = w.err;
	if (ph) ph->begin();
	if (launch_rec<T>(ra, st)) return DQMC_E_ARG;
	if (ph) ph->end(PC_RECOMBINE, dense_flops<T>(N, NB), qby);
	if (count) (*count)++;
	return 0;
}

// C = B_{l0+n-1} ... B_{l0} with B_l = exp_K diag(d_l) (mul_seq, greens.c:8-41,
// over B's that are never materialised).  d_l for item b at d + b*d_stride +
// l*N; exp_K per spin (item parity); X, W: NB x N*N scratch.
template <typename T>
static void run_mul_seq(int N, int n, int NB, const T *expK, Addr aK, const double *d,
		long long d_stride, T *out, Addr aout, T *X, T *W, cudaStream_t st, int *count,
		unsigned *err = nullptr)
{
	const size_t NN = (size_t)N * N;
	const Addr aI = Addr{(long long)NN, 0, 1};
	T *src = (n == 1) ? out : W;
	Addr as = (n == 1) ? aout : aI;
	k_colscale<T><<<grid_for((long long)NB * NN), 256, 0, st>>>(N, NB, expK, aK, d,
	        Addr{d_stride, 0, 1}, src, as);
	if (count) (*count)++;
	for (int m = 1; m < n; m++) {
		const bool last = (m == n - 1);
		T *dst = last ? out : (src == W ? X : W);
		const Addr ad = last ? aout : aI;
		GemmArgs<T> g = gargs<T>(N, N, N, NB, expK, aK, N, src, as, N, dst, ad, N, one<T>(),
		                         zero<T>(), GM_B_ROWD);
		g.d = d + (size_t)m * N;
		g.aD = Addr{d_stride, 0, 1};
		eq_gemm(g, st, count, nullptr, err);
		src = dst;
		as = ad;
	}
}

// -------------------------------------------------------------- the group

template <typename T>
struct DevBuf {
	T *p = nullptr;
	size_t n = 0;
	int alloc(size_t count)
	{
		n = count;
		if (count == 0) return 0;
		if (cudaMalloc(&p, sizeof(T) * count) != cudaSuccess) {
			p = nullptr;
			return DQMC_E_NOMEM;
		}
		cudaMemset(p, 0, sizeof(T) * count);
		return 0;
	}
	void release()
	{
		if (p) cudaFree(p);
		p = nullptr;
	}
};

// inverse of a class map: CSR offsets over classes, entries in loop order;
// entries with keep(e) false are left out.  Returns false when an entry's
// class is outside [0, n_class).
template <typename K>
static bool invert_map_if(const int *map, long long n_entries, int n_class, K keep,
		std::vector<int> &off, std::vector<int> &idx)
{
	off.assign(n_class + 1, 0);
	for (long long e = 0; e < n_entries; e++) {
		if (!keep(e)) continue;
		if (map[e] < 0 || map[e] >= n_class) return false;
		off[map[e] + 1]++;
	}
	for (int r = 0; r < n_class; r++) off[r + 1] += off[r];
	idx.resize(off[n_class]);
	std::vector<int> fill(off.begin(), off.end() - 1);
	for (long long e = 0; e < n_entries; e++)
		if (keep(e)) idx[fill[map[e]]++] = (int)e;
	return true;
}

static void invert_map(const int *map, int n_entries, int n_class, std::vector<int> &off,
		std::vector<int> &idx)
{
	invert_map_if(map, n_entries, n_class, [](long long) { return true; }, off, idx);
}

// S_b += diag(d_l) (I - G_b) diag(1/d_l): the slice-l term of the log-det
// gradient sums, d_l = exp(V_l) of item b
template <typename T>
__global__ void k_grad_acc(int N, int NB, int L, int l, const T *G, const double *dv,
		const double *dvi, T *S)
{
	const long long NN = (long long)N * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < NN * NB;
	     q += (long long)gridDim.x * blockDim.x) {
		const int b = (int)(q / NN);
		const long long e = q % NN;
		const int i = (int)(e % N), j = (int)(e / N);
		const size_t o = ((size_t)b * L + l) * N;
		const T g = G[q];
		const T x = (i == j) ? one<T>() - g : -g;
		S[q] = S[q] + x * (dv[o + i] * dvi[o + j]);
	}
}

// B_l = exp_K diag(d_l) of every slice and item, item-major (out[item][l],
// N x N each): the single-slice factors of the accurate recalculation
// check (the reference's CHECK_G_ACC builds them as calcBu, dqmc.c:29-59)
template <typename T>
__global__ void k_build_b_items(int N, int L, int NB, const T *expK, const double *dv, T *out)
{
	const long long NN = (long long)N * N, tot = NN * L * NB;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long e = q % NN, bl = q / NN;   // bl = item L + l
		const int item = (int)(bl / L), c = (int)(e / N);
		out[q] = expK[(long long)(item & 1) * NN + e] * dv[bl * N + c];
	}
}

// O of every item with one slice per block (greens.c:247-264 for
// n_matmul = 1): identity, -B_e at block (e+1, e), +B_{L-1} at (0, L-1),
// B_e = exp_K diag(d_e); leading dimension NL, item stride NL^2; O must
// hold the identity on entry (the corner adds to it when L = 1)
template <typename T>
__global__ void k_build_o(int N, int L, int NB, const T *expK, const double *dv, T *O)
{
	const long long NN = (long long)N * N, NL = (long long)N * L, tot = NN * L * NB;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long el = q % NN;
		const int e = (int)((q / NN) % L), b = (int)(q / (NN * L));
		const int i = (int)(el % N), j = (int)(el / N);
		const double sg = (e == L - 1) ? 1.0 : -1.0;
		const T v = expK[(size_t)(b & 1) * NN + el] * (sg * dv[((size_t)b * L + e) * N + j]);
		T *p = O + (size_t)b * NL * NL + ((e + 1) % L) * (long long)N + i + NL * ((long long)e * N + j);
		*p = *p + v;
	}
}

// diagonal of every item's N L x N L matrix
template <typename T>
__global__ void k_diag_of(long long n, int NB, const T *A, T *out)
{
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n * NB;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long r = q % n, b = q / n;
		out[q] = A[b * n * n + r * (n + 1)];
	}
}

// out_b = diag(w_b) A_b for n x n matrices
template <typename T>
__global__ void k_rowscale(long long n, int NB, const T *A, const double *w, T *out)
{
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n * n * NB;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long b = q / (n * n), r = (q % (n * n)) % n;
		out[q] = A[q] * w[b * n + r];
	}
}

// Yh_b = sum_m s_m diag(d_m) Y_{b,m}, s_m = +1 (m < L-1), -1 (m = L-1)
template <typename T>
__global__ void k_yhat(int N, int L, int NB, const T *Y, const double *dv, T *Yh)
{
	const long long NN = (long long)N * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < NN * NB;
	     q += (long long)gridDim.x * blockDim.x) {
		const int b = (int)(q / NN);
		const long long el = q % NN;
		const int i = (int)(el % N);
		T s = zero<T>();
		for (int m = 0; m < L; m++) {
			const double f = dv[((size_t)b * L + m) * N + i] * (m == L - 1 ? -1.0 : 1.0);
			s = s + Y[((size_t)b * L + m) * NN + el] * f;
		}
		Yh[q] = s;
	}
}

// ---------------------------------- checkpointed observable gradients
//
// Rows and columns of the space-time Green's function Gst = O^-1 without
// forming it.  For the chain rotated by s slices (slice l' of the rotated
// chain is slice (l' + s) mod L) the rotated O is D P O P^T D, D = -1 on
// the slices that wrapped, so the unequal-time stacks of the rotated chain
// hold row and column s: Gst(s, l) = sg G0t'[l - s], Gst(l, s) =
// sg Gt0'[l - s], sg = -1 for l < s.  From O Gst = I and Gst O = I the
// next row and column follow by one product each:
//   Gst(m+1, .) = B_m Gst(m, .) + delta_{m+1}
//   Gst(., m+1) = (Gst(., m) - delta_m) B_m^-1     (negated for m = L-1)
// which the engine takes across one cluster of n_matmul slices from each
// rotation s = c n_matmul, the within-cluster propagation of expand_g
// (greens.c:339-469).

// diagonals of the equal-time blocks G(l, l) from a slice-major stack
// Gtt[l][item]: out[item][l N + i]
template <typename T>
__global__ void k_stack_diag(int N, int L, int NB, const T *Gtt, T *out)
{
	const long long NN = (long long)N * N, tot = (long long)NB * L * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(q % N);
		const long long bl = q / N;
		const int l = (int)(bl % L), b = (int)(bl / L);
		out[q] = Gtt[((size_t)l * NB + b) * NN + (long long)i * (N + 1)];
	}
}

// row s (R_b, N x NL, block l at columns l N) and column s (X_b, NL x N,
// block l at rows l N) of Gst from the rotated chain's stacks
template <typename T>
__global__ void k_seed_rowcol(int N, int L, int NB, int s, const T *G0t, const T *Gt0, T *R, T *X)
{
	const long long NN = (long long)N * N, NL = (long long)N * L, tot = NN * L * NB;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const long long e = q % NN, bl = q / NN;
		const int l = (int)(bl % L), b = (int)(bl / L);
		const int r = (int)(e % N), c = (int)(e / N);
		const size_t src = ((size_t)((l - s + L) % L) * NB + b) * NN + e;
		const double sg = l < s ? -1.0 : 1.0;
		R[(size_t)b * NN * L + (size_t)l * NN + e] = G0t[src] * sg;
		X[(size_t)b * NN * L + (size_t)l * N + r + NL * c] = Gt0[src] * sg;
	}
}

// A_b[i step] += v for i < N, item stride s: the identity added to one
// N x N block of a row (step N + 1) or a column (step N L + 1)
template <typename T>
__global__ void k_shift_diag(int N, int NB, T *A, long long s, long long step, double v)
{
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)N * NB;
	     q += (long long)gridDim.x * blockDim.x) {
		T *p = A + (q / N) * s + (q % N) * step;
		*p = *p + v;
	}
}

// Yh_b += s_m diag(d_m) Y_b over nb = k NB matrices, d_m the slice-m field
// diagonal of item b % NB, s_m = -1 at m = L-1 (the corner's sign)
template <typename T>
__global__ void k_yacc(int N, int L, int NB, int nb, int m, const T *Y, const double *dv, T *Yh)
{
	const long long NN = (long long)N * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < NN * nb;
	     q += (long long)gridDim.x * blockDim.x) {
		const int b = (int)(q / NN) % NB, i = (int)((q % NN) % N);
		const double f = dv[((size_t)b * L + m) * N + i] * (m == L - 1 ? -1.0 : 1.0);
		Yh[q] = Yh[q] + Y[q] * f;
	}
}

// per-slice vectors rotated by s slices: dst[b][l] = src[b][(l + s) mod L]
__global__ void k_rotate_slices(int N, int L, int NB, int s, const double *src, double *dst)
{
	const long long tot = (long long)NB * L * N;
	for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
	     q += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(q % N);
		const long long bl = q / N;
		const int l = (int)(bl % L), b = (int)(bl / L);
		dst[q] = src[((size_t)b * L + (l + s) % L) * N + i];
	}
}

// The delayed update runs as one CTA per chain with G in global memory
// (k_update), or with G held in shared memory (k_update_cl, one CTA per
// chain and spin in clusters of two) where one spin's G and panels fit
// there.  Both do the same arithmetic in the same order.  The on-chip form
// cuts the latency of a slice but holds a whole SM per CTA and pays a
// cross-CTA exchange per accept.  Engines of real scalars with N >= 96 and
// at most 64 chains take it: the 12 x 12 lattice at L = 120 ran 15% faster
// from 1 to 64 chains (one chain 15.3 -> 17.7 chain-sweeps/s), 10 x 10 2%
// faster, while 128 chains of 12 x 12 ran 5% slower and 4 x 4 and 8 x 8
// 5-8% slower at every count.  DQMC_UPDATE=cluster or =global overrides
// the rule (read when an engine is created, or a seam called).
static bool update_cl_wanted(bool cplx, int N, int chains)
{
	const char *v = getenv("DQMC_UPDATE");
	if (v && *v) return strcmp(v, "cluster") == 0;
	return !cplx && N >= 96 && chains <= 64;
}

template <typename T>
static bool update_cl_fits(int N, int kd)
{
	return N <= 480 && update_cl_smem_bytes<T>(N, kd) <= 226 * 1024;
}

template <typename T>
static cudaError_t update_attr(int N, int kd, size_t bytes, bool cl)
{
	if (cl) return raise_smem(k_update_cl<T>, update_cl_smem_bytes<T>(N, kd));
	const cudaError_t e = raise_smem(k_update<T>, bytes);
	return e != cudaSuccess ? e : raise_smem(k_update_big<T>, bytes);
}

// the delayed update of a.nchain chains: on chip (cl), two CTAs of
// ceil(N/32) test warps and one look-ahead warp per chain; else one CTA of
// 2 ceil(N/32) warps of tests and one look-ahead warp per chain, in the
// launch form sized for that CTA
template <typename T>
static void launch_update(const UpdArgs<T> &a, size_t smem, cudaStream_t st, bool cl)
{
	if (cl) {
		const int threads = (a.N + 31) / 32 * 32 + 32;
		k_update_cl<T><<<2 * a.nchain, threads, update_cl_smem_bytes<T>(a.N, a.n_delay), st>>>(a);
		return;
	}
	const int threads = 2 * ((a.N + 31) / 32 * 32) + 32;
	if (threads <= 352) k_update<T><<<a.nchain, threads, smem, st>>>(a);
	else k_update_big<T><<<a.nchain, threads, smem, st>>>(a);
}

struct GroupBase {
	virtual ~GroupBase() {}
	virtual int set_chain(int c, const double *el, const double *del, const uint64_t *rng,
	                      const int *hs, int sweep) = 0;
	virtual int set_acc(int c, int eqn, const void *eq, int uen, const void *ue) = 0;
	// chains [c0, c0 + n) at once, host arrays contiguous over those chains
	virtual int set_chains(int c0, int n, const double *el, const double *del, const uint64_t *rng,
	                       const int *hs, int sweep) = 0;
	virtual int get_chains(int c0, int n, uint64_t *rng, int *hs, int *sweep, int *eqn, void *eq,
	                       int *uen, void *ue) = 0;
	virtual int init() = 0;
	// init without waiting for it on the host
	virtual int init_async() = 0;
	virtual int sweeps(int n, int sync) = 0;
	virtual int get_chain(int c, uint64_t *rng, int *hs, int *sweep) = 0;
	virtual int get_acc(int c, int *eqn, void *eq, int *uen, void *ue) = 0;
	virtual int get_g(int c, void *gu, void *gd, void *phase) = 0;
	virtual int accepts(int c, long long *n) = 0;
	virtual unsigned errors() = 0;
	virtual int sync() = 0;
	virtual cudaStream_t stream() = 0;
	virtual int launches(int meq, int mue) = 0;
	virtual int profile(int meq, int mue, double *out, int ncls) = 0;
	virtual int logdet_grad(double *logdet, void *S) = 0;
	virtual int obs_grad(double *obs, void *Z) = 0;
	// one gradient evaluation (0: logdet_grad, 1: obs_grad) with per-launch
	// events: class sums as profile(), and the kernels it launched
	virtual int profile_grad(int which, double *out, int ncls, int *launches) = 0;
	// whether the delayed update holds G on chip (k_update_cl)
	virtual bool update_on_chip() = 0;
	// the eight hopping matrices exp(-+dt K), exp(-+dt K / 2) of both spins
	virtual int set_hopping(const void *const *m) = 0;
	// G drift self-check: on / off (resets the counters when turned on), and
	// per chain c0 .. c0+n-1 the largest and the mean |G - G_wrapped| over
	// the checked recalculations and both spins
	virtual int set_check_g(int on) = 0;
	virtual int g_drift(int which, int c0, int n, double *mx, double *mean, int *count) = 0;
	// one sweep of a batch graph (dqmc_batch_sweeps): the kind of the next
	// sweep (bit 0 equal-time, bit 1 unequal-time measurements; -1 when the
	// run is complete), the pending re-initialisation queued outside any
	// capture, the sweep's kernels queued eagerly on the group's streams
	// (captured by the caller) and the sweep counter advanced, or the counter
	// advanced alone when a captured graph replays the sweep
	virtual int sweep_kind() = 0;
	virtual int prepare() = 0;
	virtual int enqueue_one() = 0;
	virtual void advance() = 0;
	// make stream s wait for the work queued so far on every stream of the
	// group, and every stream of the group wait for event ev
	virtual int join_into(cudaStream_t s) = 0;
	virtual int wait_on(cudaEvent_t ev) = 0;
};

template <typename T>
struct Group : GroupBase, ProfHook {
	dqmc_params p;
	int C;        // chains
	int NB;       // items = 2 C
	int N, L, F, nmul;
	int sweep = 0;
	int kd = 0, ldp = 0;   // delayed-update flush period and panel ld
	bool upd_cl = false;   // delayed update with G on chip (k_update_cl)
	int eq_size = 0, ue_size = 0;
	cudaStream_t st = nullptr;
	std::map<int, cudaGraphExec_t> graphs;
	std::map<int, int> graph_launches;
	int launch_count = 0;
	// DQMC_DEBUG_SYNC=1: eager launches, each polled to completion with a
	// deadline; a kernel that does not finish is named and the process exits
	bool debug_sync = getenv("DQMC_DEBUG_SYNC") != nullptr;
	int watchdog(const char *what)
	{
		if (!debug_sync) return 0;
		// wall time: a CPU-time clock would run fast while other host
		// threads (the gradient paths' lane threads) are busy
		const auto t0 = std::chrono::steady_clock::now();
		for (;;) {
			const cudaError_t e = cudaStreamQuery(st);
			if (e == cudaSuccess) return 0;
			if (e != cudaErrorNotReady) {
				fprintf(stderr, "dqmc_b200 watchdog: %s failed: %s\n", what, cudaGetErrorString(e));
				fflush(stderr);
				_exit(4);
			}
			if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10)) {
				fprintf(stderr, "dqmc_b200 watchdog: %s (sweep %d) did not finish in 10 s\n", what, sweep);
				fflush(stderr);
				_exit(3);
			}
		}
	}

	// parameters
	DevBuf<T> expK, iexpK, ehK, iehK, peu, ped;
	DevBuf<int> i_off, i_idx, ij_off, ij_idx, bb_off, bb_idx, bonds;
	// the measurement toggles' maps (inverses) and two-hop bond phases
	DevBuf<int> bs_off, bs_idx, bb2_off, bb2_idx, b2b_off, b2b_idx, b2b2_off, b2b2_idx;
	DevBuf<int> nem_off, nem_idx, plq_off, plq_idx, b_off, b_idx, b2_off, b2_idx, plaqs, bond2s;
	DevBuf<T> ppu, ppd, ppru, pprd, gs_eq, gs_ue;
	AccLayout lay;
	// chains
	DevBuf<double> el, del, dv, dvi;
	DevBuf<uint64_t> rng, rng_ckpt;
	DevBuf<int> hs, nacc, n_eq, n_ue, order;
	DevBuf<double> ubuf;
	bool need_draws = true;
	bool need_init = true;     // G must be recomputed from the fields before sweeping
	DevBuf<T> phase, G, Cl, Qm, Tm, Tm2, Rs, X, W, Gh, acc_eq, acc_ue, phi, qdet;
	DevBuf<T> Sg;                  // gradient sums, allocated by the first logdet_grad
	struct ObsWork {               // observable-gradient work, allocated by the first obs_grad
		DevBuf<T> O, Gr, Qh, Tw, Rw, Yh, Zb, dg;
		DevBuf<double> wb;
		void release()
		{
			DevBuf<T> *b[] = {&O, &Gr, &Qh, &Tw, &Rw, &Yh, &Zb, &dg};
			for (auto *x : b) x->release();
			wb.release();
		}
	} og;
	// checkpointed observable-gradient work (per item: row and column of
	// Gst, each N x NL, two rows and three columns), allocated by the first
	// checkpointed obs_grad; the unequal-time state ue is allocated with it
	// when the engine measures no unequal-time quantities
	struct ObsCkptWork {
		DevBuf<T> R, X, Y, Yh, Cl, dg;
		DevBuf<double> dv, dvi, w, ones;
		void release()
		{
			DevBuf<T> *b[] = {&R, &X, &Y, &Yh, &Cl, &dg};
			for (auto *x : b) x->release();
			DevBuf<double> *d[] = {&dv, &dvi, &w, &ones};
			for (auto *x : d) x->release();
		}
	} ok;
	DevBuf<T> Pr;                  // pair products C_{(m+1)%F} C_m, F >= 2
	DevBuf<double> dR, ldet;       // UDT scales; log |det(I + B...B)| per item
	DevBuf<int> pvt;
	DevBuf<unsigned> err;
	UneqState<T> ue;
	// G drift self-check (off unless enabled): at every recalculation the G
	// of the previous slice wrapped once more, against the recalculated G
	// (the reference's CHECK_G_WRP, dqmc.c:15-16, 277-287, 339-343)
	bool check_g = false;
	DevBuf<T> Gw;                      // wrapped G of the recalculation slice
	DevBuf<unsigned long long> dmax;   // [item] running max |G - G_wrapped| (bits)
	DevBuf<double> dsum;               // [item] running sum of mean |G - G_wrapped|
	DevBuf<int> dcount;                // recalculations checked
	// the accurate recalculation check (the reference's CHECK_G_ACC,
	// dqmc.c:18-19, 283-287, 345-349): at every recalculation G again from
	// the L single-slice factors with a QR after each, against the G of the
	// cluster chain; the third slot of dmax / dsum / dcount
	bool check_acc = false;
	DevBuf<T> Bacc, Gacc, phacc;       // [item][L] factors, [item] G and phase
	DevBuf<double> ldacc;              // [item] log |det| of that recalculation

	~Group() override
	{
		for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
		if (jev) cudaEventDestroy(jev);
		DevBuf<T> *tb[] = {&expK, &iexpK, &ehK, &iehK, &peu, &ped, &phase, &G, &Cl, &Qm, &Tm,
		                   &Tm2, &Rs, &X, &W, &Gh, &acc_eq, &acc_ue, &phi, &qdet, &Sg, &Pr,
		                   &ppu, &ppd, &ppru, &pprd, &gs_eq, &gs_ue};
		for (auto *b : tb) b->release();
		DevBuf<int> *ib[] = {&i_off, &i_idx, &ij_off, &ij_idx, &bb_off, &bb_idx, &bonds, &hs,
		                     &nacc, &n_eq, &n_ue, &pvt, &bs_off, &bs_idx, &bb2_off, &bb2_idx,
		                     &b2b_off, &b2b_idx, &b2b2_off, &b2b2_idx, &nem_off, &nem_idx,
		                     &plq_off, &plq_idx, &b_off, &b_idx, &b2_off, &b2_idx, &plaqs,
		                     &bond2s};
		for (auto *b : ib) b->release();
		og.release();
		ok.release();
		Gw.release(); dmax.release(); dsum.release(); dcount.release();
		Bacc.release(); Gacc.release(); phacc.release(); ldacc.release();
		el.release(); del.release(); dv.release(); dvi.release(); dR.release(); ldet.release();
		rng.release(); rng_ckpt.release(); order.release(); ubuf.release(); err.release();
		ue.release();
		if (st) cudaStreamDestroy(st);
	}

	// the maps and phases the measurement toggles read (struct params,
	// data.h:7-38), as inverse maps per class; refuses a toggle whose maps
	// are missing, and nematic correlators with complex hoppings (the
	// reference stops there, meas.c:1363-1369)
	template <typename U>
	int toggle_maps(U &upv)
	{
		std::vector<int> off, idx;
		const bool ue_on = p.period_uneqlt > 0;
		const long long nb = p.num_b, nb2 = p.num_b2;
		auto all = [](long long) { return true; };
		auto inv = [&](const int *map, long long n, int ncls, DevBuf<int> &o, DevBuf<int> &x,
		               auto keep) -> int {
			if (!map || ncls < 1) return DQMC_E_ARG;
			if (!invert_map_if(map, n, ncls, keep, off, idx)) return DQMC_E_ARG;
			if (upv(o, off) || upv(x, idx)) return DQMC_E_NOMEM;
			return 0;
		};
		auto up_num = [&](DevBuf<T> &dst, const void *src, long long n) -> int {
			if (!src || n < 1) return DQMC_E_ARG;
			if (dst.alloc((size_t)n)) return DQMC_E_NOMEM;
			cudaMemcpy(dst.p, src, sizeof(T) * n, cudaMemcpyHostToDevice);
			return 0;
		};
		int rc;
		if (ue_on && p.meas_nematic_corr && is_cplx<T>::value) {
			fprintf(stderr, "dqmc_b200: nematic correlators have no complex form\n");
			return DQMC_E_ARG;
		}
		if (p.meas_energy_corr &&
		    (rc = inv(p.map_bs, (long long)N * nb, p.num_bs, bs_off, bs_idx, all)) != 0)
			return rc;
		const bool two_hop = ue_on && (p.meas_thermal || p.meas_2bond_corr);
		if (two_hop || p.meas_local_JQ) {
			if (nb2 < 1 || !p.bond2s) return DQMC_E_ARG;
			std::vector<int> b2(p.bond2s, p.bond2s + 2 * nb2);
			if (upv(bond2s, b2)) return DQMC_E_NOMEM;
			if ((rc = up_num(ppu, p.pp_u, nb2)) || (rc = up_num(ppd, p.pp_d, nb2)) ||
			    (rc = up_num(ppru, p.ppr_u, nb2)) || (rc = up_num(pprd, p.ppr_d, nb2)))
				return rc;
		}
		if (two_hop) {
			if ((rc = inv(p.map_bb2, nb2 * nb, p.num_bb2, bb2_off, bb2_idx, all)) ||
			    (rc = inv(p.map_b2b, nb * nb2, p.num_b2b, b2b_off, b2b_idx, all)))
				return rc;
			if (p.meas_2bond_corr &&
			    (rc = inv(p.map_b2b2, nb2 * nb2, p.num_b2b2, b2b2_off, b2b2_idx, all)) != 0)
				return rc;
		}
		if (ue_on && p.meas_nematic_corr) {
			const long long nem = std::min<long long>(2LL * N, nb);   // NEM_BONDS N bonds
			if ((rc = inv(p.map_bb, nb * nb, p.num_bb, nem_off, nem_idx,
			              [&](long long e) { return e % nb < nem && e / nb < nem; })) != 0)
				return rc;
		}
		if (p.meas_chiral) {
			if (!p.plaqs || p.num_plaq < 1) return DQMC_E_ARG;
			std::vector<int> pq(p.plaqs, p.plaqs + 3 * (size_t)p.num_plaq);
			if (upv(plaqs, pq)) return DQMC_E_NOMEM;
			if ((rc = inv(p.map_plaq, p.num_plaq, p.num_plaq_accum, plq_off, plq_idx, all)) != 0)
				return rc;
		}
		if (p.meas_local_JQ &&
		    ((rc = inv(p.map_b, nb, p.num_b_accum, b_off, b_idx, all)) ||
		     (rc = inv(p.map_b2, nb2, p.num_b2_accum, b2_off, b2_idx, all))))
			return rc;
		if (p.meas_gen_suscept) {
			if (p.Nx < 1 || p.Ny < 1) return DQMC_E_ARG;
			if (gs_eq.alloc((size_t)C * 4 * p.num_ij)) return DQMC_E_NOMEM;
			if (ue_on && gs_ue.alloc((size_t)C * L * 4 * p.num_ij)) return DQMC_E_NOMEM;
		}
		return 0;
	}

	bool eq_toggles() const
	{
		return p.meas_gen_suscept || p.meas_chiral || p.meas_energy_corr || p.meas_local_JQ;
	}

	// nchain chains of an engine of engine_chains (the update form's rule)
	int create(const dqmc_params &pp, int nchain, int engine_chains)
	{
		p = pp;
		C = nchain;
		NB = 2 * C;
		N = p.N; L = p.L; F = p.F; nmul = p.n_matmul;
		if (N < 1 || L < 1 || F < 1 || nmul < 1 || L != F * nmul || N > max_dense_n<T>() ||
		    N > 480 || C < 1)
			return DQMC_E_ARG;
		if (p.period_uneqlt > 0 && !UneqState<T>::supported(N, F, L)) return DQMC_E_ARG;
		CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
		const size_t NN = (size_t)N * N;
		int rc = 0;
		rc |= expK.alloc(2 * NN); rc |= iexpK.alloc(2 * NN);
		rc |= ehK.alloc(2 * NN); rc |= iehK.alloc(2 * NN);
		rc |= peu.alloc(NN); rc |= ped.alloc(NN);
		rc |= el.alloc((size_t)C * 2 * N); rc |= del.alloc((size_t)C * 2 * N);
		rc |= dv.alloc((size_t)C * 2 * L * N); rc |= dvi.alloc((size_t)C * 2 * L * N);
		rc |= rng.alloc((size_t)C * 17); rc |= rng_ckpt.alloc((size_t)C * 17);
		rc |= order.alloc((size_t)C * 2 * N); rc |= ubuf.alloc((size_t)C * 2 * N);
		rc |= hs.alloc((size_t)C * L * N);
		rc |= nacc.alloc(C); rc |= n_eq.alloc(C); rc |= n_ue.alloc(C);
		rc |= phase.alloc(C); rc |= phi.alloc(NB); rc |= qdet.alloc(NB);
		rc |= G.alloc(NB * NN); rc |= Cl.alloc((size_t)NB * F * NN);
		rc |= Qm.alloc(NB * NN); rc |= Tm.alloc(NB * NN); rc |= Tm2.alloc(NB * NN);
		rc |= Rs.alloc(NB * NN); rc |= X.alloc(NB * NN); rc |= W.alloc(NB * NN);
		rc |= Gh.alloc(NB * NN); rc |= dR.alloc((size_t)NB * N); rc |= pvt.alloc((size_t)NB * N);
		rc |= ldet.alloc(NB);
		if (F >= 2) rc |= Pr.alloc((size_t)NB * F * NN);
		rc |= err.alloc(1);
		lay = acc_layout(p);
		eq_size = (int)lay.eq_size;
		ue_size = (int)lay.ue_size;
		rc |= acc_eq.alloc((size_t)C * eq_size);
		if (ue_size) rc |= acc_ue.alloc((size_t)C * ue_size);
		if (rc) return DQMC_E_NOMEM;
		if (p.period_uneqlt > 0 && ue.alloc(N, L, F, NB)) return DQMC_E_NOMEM;
		// parameter matrices, per spin
		auto up2 = [&](DevBuf<T> &dst, const void *u, const void *d) {
			cudaMemcpy(dst.p, u, sizeof(T) * NN, cudaMemcpyHostToDevice);
			cudaMemcpy(dst.p + NN, d, sizeof(T) * NN, cudaMemcpyHostToDevice);
		};
		up2(expK, p.exp_Ku, p.exp_Kd);
		up2(iexpK, p.inv_exp_Ku, p.inv_exp_Kd);
		up2(ehK, p.exp_halfKu, p.exp_halfKd);
		up2(iehK, p.inv_exp_halfKu, p.inv_exp_halfKd);
		if (p.peierlsu) cudaMemcpy(peu.p, p.peierlsu, sizeof(T) * NN, cudaMemcpyHostToDevice);
		if (p.peierlsd) cudaMemcpy(ped.p, p.peierlsd, sizeof(T) * NN, cudaMemcpyHostToDevice);
		std::vector<int> off, idx;
		auto upv = [&](DevBuf<int> &dst, const std::vector<int> &v) -> int {
			if (dst.alloc(v.size() ? v.size() : 1)) return DQMC_E_NOMEM;
			if (!v.empty()) cudaMemcpy(dst.p, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice);
			return 0;
		};
		invert_map(p.map_i, N, p.num_i, off, idx);
		if (upv(i_off, off) || upv(i_idx, idx)) return DQMC_E_NOMEM;
		invert_map(p.map_ij, N * N, p.num_ij, off, idx);
		if (upv(ij_off, off) || upv(ij_idx, idx)) return DQMC_E_NOMEM;
		const bool ue_on = p.period_uneqlt > 0;
		const bool need_bb = (ue_on && (p.meas_bond_corr || p.meas_pair_bb_only || p.meas_thermal ||
		                                p.meas_nematic_corr)) || p.meas_energy_corr;
		if ((need_bb || p.meas_local_JQ || (ue_on && p.meas_2bond_corr)) && p.num_b > 0) {
			std::vector<int> bv(p.bonds, p.bonds + 2 * p.num_b);
			if (upv(bonds, bv)) return DQMC_E_NOMEM;
		}
		if (need_bb && p.num_b > 0) {
			if (!invert_map_if(p.map_bb, (long long)p.num_b * p.num_b, p.num_bb,
			                   [](long long) { return true; }, off, idx))
				return DQMC_E_ARG;
			if (upv(bb_off, off) || upv(bb_idx, idx)) return DQMC_E_NOMEM;
		}
		if ((rc = toggle_maps(upv)) != 0) return rc;
		// delayed-update panels: the file's n_delay unless shared memory is short
		kd = p.n_delay < 1 ? 1 : p.n_delay;
		ldp = (N + 15) / 16 * 16 + 4;
		while (kd > 1 && update_smem_bytes<T>(N, kd, ldp) > 200 * 1024) kd /= 2;
		upd_cl = update_cl_wanted(is_cplx<T>::value, N, engine_chains) && update_cl_fits<T>(N, kd);
		CK(update_attr<T>(N, kd, update_smem_bytes<T>(N, kd, ldp), upd_cl));
		CK(cudaDeviceSynchronize());
		return 0;
	}

	int set_chain(int c, const double *e, const double *d, const uint64_t *r, const int *h,
	              int sw) override
	{
		if (c < 0 || c >= C) return DQMC_E_ARG;
		// the copies below run on the legacy default stream: queued sweeps
		// that still read these buffers must finish first
		CK(cudaStreamSynchronize(st));
		CK(cudaMemcpy(el.p + (size_t)c * 2 * N, e, sizeof(double) * 2 * N, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(del.p + (size_t)c * 2 * N, d, sizeof(double) * 2 * N, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(rng.p + (size_t)c * 17, r, sizeof(uint64_t) * 17, cudaMemcpyHostToDevice));
		// get_chain reports rng_ckpt: it must show the state just set
		CK(cudaMemcpy(rng_ckpt.p + (size_t)c * 17, r, sizeof(uint64_t) * 17, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(hs.p + (size_t)c * L * N, h, sizeof(int) * L * N, cudaMemcpyHostToDevice));
		sweep = sw;
		need_draws = true;
		need_init = true;
		return 0;
	}

	int set_chains(int c0, int n, const double *e, const double *d, const uint64_t *r, const int *h,
	               int sw) override
	{
		if (c0 < 0 || n < 0 || c0 + n > C) return DQMC_E_ARG;
		if (n == 0) return 0;
		// stream-ordered after the queued sweeps that read these buffers
		CK(cudaMemcpyAsync(el.p + (size_t)c0 * 2 * N, e, sizeof(double) * 2 * N * n, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(del.p + (size_t)c0 * 2 * N, d, sizeof(double) * 2 * N * n, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(rng.p + (size_t)c0 * 17, r, sizeof(uint64_t) * 17 * n, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(rng_ckpt.p + (size_t)c0 * 17, r, sizeof(uint64_t) * 17 * n, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(hs.p + (size_t)c0 * L * N, h, sizeof(int) * L * N * n, cudaMemcpyHostToDevice, st));
		CK(cudaStreamSynchronize(st));
		sweep = sw;
		need_draws = true;
		need_init = true;
		return 0;
	}

	int get_chains(int c0, int n, uint64_t *r, int *h, int *sw, int *eqn, void *eq, int *uen,
	               void *uea) override
	{
		if (c0 < 0 || n < 0 || c0 + n > C) return DQMC_E_ARG;
		if (sw) *sw = sweep;
		if (n == 0) return 0;
		// the state at the sweep boundary, before the look-ahead draws
		if (r) CK(cudaMemcpyAsync(r, rng_ckpt.p + (size_t)c0 * 17, sizeof(uint64_t) * 17 * n, cudaMemcpyDeviceToHost, st));
		if (h) CK(cudaMemcpyAsync(h, hs.p + (size_t)c0 * L * N, sizeof(int) * L * N * n, cudaMemcpyDeviceToHost, st));
		if (eqn) CK(cudaMemcpyAsync(eqn, n_eq.p + c0, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
		if (eq) CK(cudaMemcpyAsync(eq, acc_eq.p + (size_t)c0 * eq_size, sizeof(T) * eq_size * n, cudaMemcpyDeviceToHost, st));
		if (ue_size) {
			if (uen) CK(cudaMemcpyAsync(uen, n_ue.p + c0, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
			if (uea) CK(cudaMemcpyAsync(uea, acc_ue.p + (size_t)c0 * ue_size, sizeof(T) * ue_size * n, cudaMemcpyDeviceToHost, st));
		}
		CK(cudaStreamSynchronize(st));
		return 0;
	}

	int set_acc(int c, int eqn, const void *eq, int uen, const void *uea) override
	{
		CK(cudaStreamSynchronize(st));
		if (c < 0 || c >= C) return DQMC_E_ARG;
		CK(cudaMemcpy(n_eq.p + c, &eqn, sizeof(int), cudaMemcpyHostToDevice));
		if (eq) CK(cudaMemcpy(acc_eq.p + (size_t)c * eq_size, eq, sizeof(T) * eq_size, cudaMemcpyHostToDevice));
		if (ue_size) {
			CK(cudaMemcpy(n_ue.p + c, &uen, sizeof(int), cudaMemcpyHostToDevice));
			if (uea) CK(cudaMemcpy(acc_ue.p + (size_t)c * ue_size, uea, sizeof(T) * ue_size, cudaMemcpyHostToDevice));
		}
		return 0;
	}

	// on: 0 off; else the wrap and unequal-time checks, and with bit 1 the
	// accurate recalculation check too
	int set_check_g(int on) override
	{
		CK(cudaStreamSynchronize(st));
		const bool acc = on != 0 && (on & 2) != 0;
		if (on && !Gw.p) {
			CK(cudaDeviceSynchronize());   // the allocations' zeroing runs on the default stream
			int rc = Gw.alloc((size_t)NB * N * N);
			// [0, NB): wrap check, [NB, 2 NB): unequal-time, [2 NB, 3 NB): accurate
			rc |= dmax.alloc(3 * (size_t)NB);
			rc |= dsum.alloc(3 * (size_t)NB);
			rc |= dcount.alloc(3);
			CK(cudaDeviceSynchronize());
			if (rc) return rc;
		}
		if (acc && !Bacc.p) {
			CK(cudaDeviceSynchronize());
			int rc = Bacc.alloc((size_t)NB * L * N * N);
			rc |= Gacc.alloc((size_t)NB * N * N);
			rc |= phacc.alloc((size_t)NB);
			rc |= ldacc.alloc((size_t)NB);
			CK(cudaDeviceSynchronize());
			if (rc) {
				Bacc.release(); Gacc.release(); phacc.release(); ldacc.release();
				return DQMC_E_NOMEM;
			}
		}
		if (on) {
			CK(cudaMemsetAsync(dmax.p, 0, sizeof(unsigned long long) * 3 * NB, st));
			CK(cudaMemsetAsync(dsum.p, 0, sizeof(double) * 3 * NB, st));
			CK(cudaMemsetAsync(dcount.p, 0, 3 * sizeof(int), st));
		}
		if ((on != 0) != check_g || acc != check_acc) {
			// the captured sweeps follow the setting from the next sweep on
			for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
			graphs.clear();
			graph_launches.clear();
			check_g = on != 0;
			check_acc = acc;
		}
		CK(cudaStreamSynchronize(st));
		return 0;
	}

	// G at slice l0 from the L single-slice factors, a QR after each
	// (calc_eq_g(l0, N, L, 1, B, ...), dqmc.c:283-287), into Gacc; the
	// cluster chain's scratch is free again once its G is done
	int calc_eq_g_acc(int l0)
	{
		const size_t NN = (size_t)N * N;
		k_build_b_items<T><<<grid_for((long long)NB * L * NN), 256, 0, st>>>(N, L, NB, expK.p, dv.p,
		                                                                   Bacc.p);
		launch_count++;
		EqWork<T> w = eq_work();
		w.F = L;
		w.Cl = Bacc.p; w.cl_stride = (long long)L * NN;
		w.Pr = nullptr;
		w.G = Gacc.p; w.g_stride = (long long)NN;
		w.phi = phacc.p;
		w.logdet = ldacc.p;
		const int rc = run_calc_eq_g<T>(w, l0, st, &launch_count, nullptr, 1);
		watchdog("calc_eq_g (accurate check)");
		return rc;
	}

	int g_drift(int which, int c0, int n, double *mx, double *mean, int *count) override
	{
		if (c0 < 0 || n < 0 || c0 + n > C || which < 0 || which > 2) return DQMC_E_ARG;
		if (!check_g || !dmax.p || (which == 2 && !check_acc)) return DQMC_E_ARG;
		std::vector<unsigned long long> hm((size_t)2 * n);
		std::vector<double> hs((size_t)2 * n);
		int cnt = 0;
		const size_t o = (size_t)which * NB + (size_t)2 * c0;
		CK(cudaMemcpyAsync(hm.data(), dmax.p + o, sizeof(unsigned long long) * 2 * n,
		                   cudaMemcpyDeviceToHost, st));
		CK(cudaMemcpyAsync(hs.data(), dsum.p + o, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st));
		CK(cudaMemcpyAsync(&cnt, dcount.p + which, sizeof(int), cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		for (int q = 0; q < n; q++) {
			double a, b;
			memcpy(&a, &hm[2 * q], sizeof(double));
			memcpy(&b, &hm[2 * q + 1], sizeof(double));
			if (mx) mx[q] = (a != a || b != b) ? (a != a ? a : b) : fmax(a, b);
			if (mean) mean[q] = cnt > 0 ? (hs[2 * q] + hs[2 * q + 1]) / (2.0 * cnt) : 0.0;
		}
		if (count) *count = cnt;
		return 0;
	}

	// ------------------------------------------------------------ steps

	void gemm(const GemmArgs<T> &g)
	{
		prof_begin(0);
		eq_gemm<T>(g, st, &launch_count, nullptr, err.p);
		watchdog("k_gemm");
		double fl = 2.0 * g.M * g.N * g.K * g.batch * (is_cplx<T>::value ? 4.0 : 1.0);
		if (g.mode & GM_A_UPPER) fl *= 0.5;
		prof_end(0, fl, (double)sizeof(T) * ((double)g.M * g.K + (double)g.K * g.N + (double)g.M * g.N) * g.batch);
	}

	// --- optional per-launch timing (one eager sweep, see profile())
	bool profiling = false;
	std::vector<cudaEvent_t> pev;
	struct PRec { int cls; double flops, bytes; int e0, e1; };
	std::vector<PRec> precs;
	int cur_e0 = -1;
	cudaEvent_t new_event()
	{
		cudaEvent_t e;
		cudaEventCreate(&e);
		pev.push_back(e);
		return e;
	}
	void prof_begin(int)
	{
		if (!profiling) return;
		cudaEvent_t e = new_event();
		cudaEventRecord(e, st);
		cur_e0 = (int)pev.size() - 1;
	}
	void begin() override { prof_begin(0); }
	void end(int cls, double flops, double bytes) override { prof_end(cls, flops, bytes); }
	void prof_end(int cls, double flops, double bytes)
	{
		if (!profiling) return;
		cudaEvent_t e = new_event();
		cudaEventRecord(e, st);
		precs.push_back(PRec{cls, flops, bytes, cur_e0, (int)pev.size() - 1});
	}

	// cluster C_f = B_{f n + n - 1} ... B_{f n}
	void build_cluster(int f)
	{
		const size_t NN = (size_t)N * N;
		prof_begin(0);
		run_mul_seq<T>(N, nmul, NB, expK.p, per_spin(NN), dv.p + (size_t)f * nmul * N, (long long)L * N,
		               Cl.p + (size_t)f * NN, per_item((long long)F * NN), X.p, W.p, st, &launch_count,
		               err.p);
		watchdog("mul_seq");
		const double fl = 2.0 * N * NN * NB * (nmul - 1) * (is_cplx<T>::value ? 4.0 : 1.0);
		prof_end(0, fl, 3.0 * sizeof(T) * NN * NB * (nmul - 1));
	}

	// pair product m: C_{(m+1)%F} C_m of every item (the products that
	// calc_eq_g's two-cluster groups start from)
	void build_pair(int m)
	{
		const size_t NN = (size_t)N * N;
		const Addr aC = per_item((long long)F * NN);
		gemm(gargs<T>(N, N, N, NB, Cl.p + (size_t)((m + 1) % F) * NN, aC, N, Cl.p + (size_t)m * NN, aC, N,
		              Pr.p + (size_t)m * NN, aC, N));
	}

	EqWork<T> eq_work()
	{
		EqWork<T> w;
		memset(&w, 0, sizeof(w));
		w.N = N; w.F = F; w.NB = NB;
		w.Cl = Cl.p; w.cl_stride = (long long)F * N * N;
		w.Qm = Qm.p; w.Tm = Tm.p; w.Tm2 = Tm2.p; w.Rs = Rs.p; w.X = X.p; w.W = W.p;
		w.dR = dR.p; w.pvt = pvt.p; w.qdet = qdet.p;
		w.G = G.p; w.g_stride = (long long)N * N;
		w.phi = phi.p; w.err = err.p;
		w.logdet = ldet.p;
		w.Pr = Pr.p; w.pr_stride = (long long)F * N * N;
		return w;
	}

	// G = (I + C_{l0-1} ... C_{l0})^-1 (cyclic), then the chain phases
	int calc_eq_g(int l0)
	{
		// the only pair that calc_eq_g(l0) uses and whose clusters changed
		// since it was formed is the one ending at cluster l0 - 1, the last
		// rebuilt (its groups start at l0 (F even) or l0 + 1 (F odd) and
		// step by two, always through (l0 - 2) mod F)
		if (F >= 2) build_pair((l0 - 2 + F) % F);
		int rc = run_calc_eq_g<T>(eq_work(), l0, st, &launch_count, profiling ? this : nullptr);
		watchdog("calc_eq_g");
		if (rc) return rc;
		k_combine_phase<T><<<(C + 127) / 128, 128, 0, st>>>(C, phi.p, phase.p);
		launch_count++;
		return 0;
	}

	// the draws of slice l for every chain, from the working RNG state
	void draws(int l)
	{
		k_draws<<<(C + 63) / 64, 64, 0, st>>>(N, L, C, l, del.p, rng.p, rng_ckpt.p, hs.p, order.p,
		                                      ubuf.p);
		launch_count++;
	}

	void update(int l)
	{
		UpdArgs<T> a;
		a.N = N; a.L = L; a.n_delay = kd; a.nchain = C; a.slice = l; a.ldp = ldp;
		a.del = del.p; a.exp_lambda = el.p; a.rng = rng.p; a.hs = hs.p; a.G = G.p;
		a.phase = phase.p; a.dv = dv.p; a.dvi = dvi.p; a.n_accept = nacc.p; a.err = err.p;
		a.rng_ckpt = rng_ckpt.p; a.order = order.p; a.u = ubuf.p;
		// the look-ahead warp draws the next slice, except when that is this
		// slice again (L = 1), whose fields this kernel is still changing
		a.next_slice = (L == 1) ? -1 : (l + 1) % L;
		prof_begin(1);
		launch_update<T>(a, update_smem_bytes<T>(N, kd, ldp), st, upd_cl);
		prof_end(PC_UPDATE, 0.0, 0.0);
		launch_count++;
		watchdog("k_update");
		if (L == 1) draws(0);
	}

	// G <- B_l G B_l^-1 = exp_K (D G D^-1) inv_exp_K
	// dst = B_l G B_l^-1 (dst = G: the wrap of dqmc.c:293-296, 331-334)
	void wrap_into(int l, T *dst)
	{
		const size_t NN = (size_t)N * N;
		const Addr aI = per_item(NN);
		GemmArgs<T> g = gargs<T>(N, N, N, NB, G.p, aI, N, iexpK.p, per_spin(NN), N, W.p, aI, N,
		                         one<T>(), zero<T>(), GM_A_DD);
		g.d = dv.p + (size_t)l * N;
		g.dinv = dvi.p + (size_t)l * N;
		g.aD = per_item((long long)L * N);
		gemm(g);
		gemm(gargs<T>(N, N, N, NB, expK.p, per_spin(NN), N, W.p, aI, N, dst, aI, N));
	}
	void wrap(int l) { wrap_into(l, G.p); }

	// Gh = inv_exp_halfK (G exp_halfK)  (dqmc.c:366-380)
	void half_wrap(const T *src, Addr as, T *dst, Addr ad, int batch_items)
	{
		const size_t NN = (size_t)N * N;
		gemm(gargs<T>(N, N, N, batch_items, src, as, N, ehK.p, per_spin(NN), N, W.p, per_item(NN), N));
		gemm(gargs<T>(N, N, N, batch_items, iehK.p, per_spin(NN), N, W.p, per_item(NN), N, dst, ad, N));
	}

	MeasArgs<T> meas_args()
	{
		MeasArgs<T> m;
		memset(&m, 0, sizeof(m));
		m.N = N; m.L = L; m.nchain = C; m.num_i = p.num_i; m.num_ij = p.num_ij;
		m.num_b = p.num_b; m.num_bb = p.num_bb;
		m.degen_i = p.degen_i; m.degen_ij = p.degen_ij; m.degen_bb = p.degen_bb;
		m.phase = phase.p;
		m.i_off = i_off.p; m.i_idx = i_idx.p; m.ij_off = ij_off.p; m.ij_idx = ij_idx.p;
		m.bb_off = bb_off.p; m.bb_idx = bb_idx.p; m.bonds = bonds.p;
		m.peu = peu.p; m.ped = ped.p;
		m.energy = p.meas_energy_corr; m.thermal = p.meas_thermal; m.two_bond = p.meas_2bond_corr;
		m.nematic = p.meas_nematic_corr; m.chiral = p.meas_chiral; m.local_jq = p.meas_local_JQ;
		m.gen_suscept = p.meas_gen_suscept; m.pair_bb_only = p.meas_pair_bb_only;
		m.Nx = p.Nx; m.Ny = p.Ny; m.num_bs = p.num_bs; m.num_b2 = p.num_b2;
		m.num_b2b = p.num_b2b; m.num_bb2 = p.num_bb2; m.num_b2b2 = p.num_b2b2;
		m.num_plaq = p.num_plaq; m.num_plaq_accum = p.num_plaq_accum;
		m.num_b_accum = p.num_b_accum; m.num_b2_accum = p.num_b2_accum;
		m.degen_bs = p.degen_bs; m.degen_b2b = p.degen_b2b; m.degen_bb2 = p.degen_bb2;
		m.degen_b2b2 = p.degen_b2b2; m.degen_plaq = p.degen_plaq; m.degen_b = p.degen_b;
		m.degen_b2 = p.degen_b2;
		m.bs_off = bs_off.p; m.bs_idx = bs_idx.p; m.bb2_off = bb2_off.p; m.bb2_idx = bb2_idx.p;
		m.b2b_off = b2b_off.p; m.b2b_idx = b2b_idx.p; m.b2b2_off = b2b2_off.p; m.b2b2_idx = b2b2_idx.p;
		m.nem_off = nem_off.p; m.nem_idx = nem_idx.p; m.plaq_off = plq_off.p; m.plaq_idx = plq_idx.p;
		m.b_off = b_off.p; m.b_idx = b_idx.p; m.b2_off = b2_off.p; m.b2_idx = b2_idx.p;
		m.plaqs = plaqs.p; m.bond2s = bond2s.p;
		m.pp_u = ppu.p; m.pp_d = ppd.p; m.ppr_u = ppru.p; m.ppr_d = pprd.p;
		m.lay = lay;
		return m;
	}

	void meas_eqlt()
	{
		const size_t NN = (size_t)N * N;
		half_wrap(G.p, per_item(NN), Gh.p, per_item(NN), NB);
		MeasArgs<T> m = meas_args();
		m.G = Gh.p;
		m.acc = acc_eq.p; m.acc_stride = eq_size; m.n_sample = n_eq.p;
		prof_begin(4);
		// one warp per class: enough chunks of 8 warps for every class
		const int chunks = std::max(1, std::min(32, (std::max(p.num_i, p.num_ij) + 7) / 8));
		k_meas_eqlt<T><<<dim3(C, chunks), 256, 2 * N * sizeof(T) + 64, st>>>(m);
		launch_count++;
		if (eq_toggles()) {
			k_meas_eqlt_x<T><<<C, 256, 0, st>>>(m, gs_eq.p);
			launch_count++;
		}
		prof_end(PC_MEAS, 0.0, 0.0);
		watchdog("k_meas_eqlt");
	}

	// ------------------------------------------------ unequal-time G

	// stack[l][item] through a table of slice indices, one entry per group
	Addr slice_addr(int tab_off) const
	{
		const long long NN = (long long)N * N;
		return Addr{(long long)NB * NN, NN, NB, ue.dtab + tab_off};
	}

	int launch_hqr(const HqrArgs<T> &h)
	{
		constexpr int NBK = 8, NW = 16;
		const size_t sm = hqr_smem_bytes<T, NBK, NW>(h.M);
		auto go = [&](auto kern) -> int {
			CK(raise_smem(kern, sm));
			prof_begin(0);
			kern<<<h.batch, NW * 32, sm, st>>>(h);
			prof_end(PC_UNEQ, 0.0, 0.0);
			launch_count++;
			return 0;
		};
		if (h.M <= 64) return go(k_hqr<T, NBK, 2, NW>);
		if (h.M <= 128) return go(k_hqr<T, NBK, 4, NW>);
		if (h.M <= 224) return go(k_hqr<T, NBK, 7, NW>);
		if (h.M <= 320) return go(k_hqr<T, NBK, 10, NW>);
		return DQMC_E_ARG;
	}

	// bsofi (greens.c:266-337) of NB block-cyclic matrices of E x E blocks
	// of N x N: O (leading dimension NE = N E, item stride NE^2) is
	// overwritten by R and O^-1 goes to Gr.  Work: Qh NB x max(E-1,1) x 4N^2,
	// Tw NB x E x N^2, Rw NB x NE x 2N.
	int bsofi(int E, T *O, T *Gr, T *Qh, T *Tw, T *Rw)
	{
		const size_t NN = (size_t)N * N;
		const int NE = N * E;
		const long long NE2 = (long long)NE * NE, q4 = 4LL * (long long)NN;
		const long long qstride = (long long)std::max(E - 1, 1) * q4;
		// bsofi (greens.c:266-337): QR of the 2N x N panels, Q^H carried to
		// the block columns l+1 and E-1 in the same kernel
		for (int l = 0; l + 2 < E; l++) {
			HqrArgs<T> h;
			memset(&h, 0, sizeof(h));
			h.M = 2 * N; h.n = N; h.batch = NB;
			h.A = O + (size_t)l * N * (1 + NE); h.aA = per_item(NE2); h.lda = NE;
			h.nx1 = N;
			h.nx2 = N; h.X = O + (size_t)l * N + (size_t)(E - 1) * N * NE; h.aX = per_item(NE2);
			h.Qh = Qh + (size_t)l * q4; h.aQ = per_item(qstride);
			h.err = err.p;
			if (launch_hqr(h)) return DQMC_E_ARG;
		}
		const int lf = std::max(E - 2, 0), wf = (E >= 2) ? 2 * N : N;
		{
			HqrArgs<T> h;
			memset(&h, 0, sizeof(h));
			h.M = wf; h.n = wf; h.batch = NB;
			h.A = O + (size_t)lf * N * (1 + NE); h.aA = per_item(NE2); h.lda = NE;
			h.Qh = Qh + (size_t)lf * q4; h.aQ = per_item(qstride);
			h.err = err.p;
			if (launch_hqr(h)) return DQMC_E_ARG;
		}
		// R^-1: diagonal blocks, then the blocks d above the diagonal,
		// X(i, i+d) = -X(i, i) R(i, i+1..i+d) X(i+1..i+d, i+d)
		CK(cudaMemsetAsync(Gr, 0, sizeof(T) * NB * NE2, st));
		{
			TriArgs<T> t{N, NE, E, NB, O, Gr, err.p};
			const size_t sm = trtri_smem_bytes<T>(N);
			CK(raise_smem(k_trtri<T>, sm));
			prof_begin(0);
			k_trtri<T><<<NB * E, 256, sm, st>>>(t);
			launch_count++;
			prof_end(PC_UNEQ, 0.0, 0.0);
		}
		for (int d = 1; d < E; d++) {
			const int na = E - d;
			const Addr dg{NE2, (long long)N * (1 + NE), na};
			gemm(gargs<T>(N, N, d * N, NB * na, O + (size_t)N * NE, dg, NE,
			              Gr + N + (size_t)d * N * NE, dg, NE, Tw, per_item((long long)NN), N));
			gemm(gargs<T>(N, N, N, NB * na, Gr, dg, NE, Tw, per_item((long long)NN), N,
			              Gr + (size_t)d * N * NE, dg, NE, from_re<T>(-1.0), zero<T>()));
		}
		// O^-1 = R^-1 Q_{E-2}^H ... Q_0^H, each on its two block columns
		for (int l = lf; l >= 0; l--) {
			T *cols = Gr + (size_t)l * N * NE;
			prof_begin(0);
			k_copy2d<T><<<grid_for((long long)NB * NE * wf), 256, 0, st>>>(NE, wf, NB, cols, NE2, NE,
			        Rw, (long long)NE * wf, NE, one<T>());
			launch_count++;
			prof_end(PC_UNEQ, 0.0, 0.0);
			gemm(gargs<T>(NE, wf, wf, NB, Rw, per_item((long long)NE * wf), NE,
			              Qh + (size_t)l * q4, per_item(qstride), wf, cols, per_item(NE2), NE));
		}
		return 0;
	}

	// G(0,t), G(t,t), G(t,0) of every slice from this sweep's clusters
	// (calc_ue_g, greens.c:471-494, with N_MUL = 2 as dqmc.c:399 calls it)
	int calc_ue_g()
	{
		const size_t NN = (size_t)N * N;
		const int E = ue.E, NE = ue.NE;
		const long long NE2 = (long long)NE * NE, q4 = 4LL * (long long)NN;
		const long long qstride = (long long)std::max(E - 1, 1) * q4;
		prof_begin(0);
		k_build_bib<T><<<grid_for((long long)L * NB * NN), 256, 0, st>>>(N, L, NB, expK.p, iexpK.p,
		                                                               dv.p, dvi.p, ue.Bs.p, ue.iBs.p);
		launch_count++;
		prof_end(PC_UNEQ, 0.0, 0.0);
		// calc_o (greens.c:247-264): I on the diagonal, -C_{2e+1} C_{2e} at
		// (e+1, e), the remaining clusters' product at (0, E-1)
		CK(cudaMemsetAsync(ue.O.p, 0, sizeof(T) * NB * NE2, st));
		if (E > 1)
			gemm(gargs<T>(N, N, N, NB * (E - 1), Cl.p + NN, Addr{(long long)(F * NN), 2LL * (long long)NN, E - 1},
			              N, Cl.p, Addr{(long long)(F * NN), 2LL * (long long)NN, E - 1}, N, ue.O.p + N,
			              Addr{NE2, (long long)N * (1 + NE), E - 1}, NE, from_re<T>(-1.0), zero<T>()));
		T *corner = ue.O.p + (size_t)(E - 1) * N * NE;
		if (F - 2 * (E - 1) == 2)
			gemm(gargs<T>(N, N, N, NB, Cl.p + (size_t)(F - 1) * NN, per_item((long long)F * NN), N,
			              Cl.p + (size_t)(F - 2) * NN, per_item((long long)F * NN), N, corner,
			              per_item(NE2), NE));
		else {
			prof_begin(0);
			k_copy2d<T><<<grid_for((long long)NB * NN), 256, 0, st>>>(N, N, NB, Cl.p + (size_t)(F - 1) * NN,
			        (long long)F * NN, N, corner, NE2, NE, one<T>());
			launch_count++;
			prof_end(PC_UNEQ, 0.0, 0.0);
		}
		prof_begin(0);
		k_add_diag<T><<<grid_for((long long)NE * NB), 256, 0, st>>>(NE, NB, ue.O.p, NE2);
		launch_count++;
		prof_end(PC_UNEQ, 0.0, 0.0);
		{
			const int rc = bsofi(E, ue.O.p, ue.Gr.p, ue.Qh.p, ue.Tw.p, ue.Rw.p);
			if (rc) return rc;
		}
		// expand_g (greens.c:339-469)
		prof_begin(0);
		k_ue_seed<T><<<grid_for((long long)NB * E * NN), 256, 0, st>>>(N, E, NB, ue.plan.nme, ue.Gr.p,
		                                                              ue.G0t.p, ue.Gtt.p, ue.Gt0.p);
		launch_count++;
		prof_end(PC_UNEQ, 0.0, 0.0);
		const long long sl = (long long)NB * NN;     // one slice of a stack
		for (const UeOp &o : ue.plan.ops) {
			T *stk = (o.kind < 2) ? ue.G0t.p : (o.kind < 4) ? ue.Gtt.p : ue.Gt0.p;
			// operands per kind: A, B, C (and D, the second GEMM's A, for Gtt)
			T *opA, *opB, *opD = nullptr;
			switch (o.kind) {
			case 0: opA = stk; opB = ue.Bs.p; break;
			case 1: opA = stk; opB = ue.iBs.p; break;
			case 2: opA = stk; opB = ue.Bs.p; opD = ue.iBs.p; break;
			case 3: opA = stk; opB = ue.iBs.p; opD = ue.Bs.p; break;
			case 4: opA = ue.iBs.p; opB = stk; break;
			default: opA = ue.Bs.p; opB = stk; break;
			}
			if (!o.special) {
				const int bt = o.nact * NB;
				const Addr tA = slice_addr(o.tab), tB = slice_addr(o.tab + o.nact);
				const Addr tC = slice_addr(o.tab + 2 * o.nact), tD = slice_addr(o.tab + 3 * o.nact);
				if (opD) {
					gemm(gargs<T>(N, N, N, bt, opA, tA, N, opB, tB, N, ue.Cw.p, per_item((long long)NN), N));
					gemm(gargs<T>(N, N, N, bt, opD, tD, N, ue.Cw.p, per_item((long long)NN), N, stk, tC, N));
				} else {
					gemm(gargs<T>(N, N, N, bt, opA, tA, N, opB, tB, N, stk, tC, N));
				}
				continue;
			}
			const Addr ai = per_item((long long)NN);
			auto at = [&](T *base, int k) { return base + UePlan::slice_of(o.kind, k, o.m, o.next) * sl; };
			T *dst = at(stk, 2);
			if (o.prefill) {
				const T *src = (o.prefill == 1) ? ue.iBs.p + o.m * sl
				             : (o.prefill == 2) ? ue.iBs.p + o.next * sl : nullptr;
				prof_begin(0);
				k_copy2d<T><<<grid_for((long long)NB * NN), 256, 0, st>>>(N, N, NB, src, (long long)NN, N, dst,
				        (long long)NN, N, one<T>());
				launch_count++;
				prof_end(PC_UNEQ, 0.0, 0.0);
			}
			gemm(gargs<T>(N, N, N, NB, at(opA, 0), ai, N, at(opB, 1), ai, N, dst, ai, N,
			              from_re<T>(o.alpha), from_re<T>(o.beta)));
		}
		watchdog("calc_ue_g");
		return 0;
	}

	int meas_uneqlt()
	{
		const size_t NN = (size_t)N * N;
		int rc = calc_ue_g();
		if (rc) return rc;
		if (check_g) {
			// the equal-time G against the (0, 0) block of G(tau, tau)
			// (the reference's CHECK_G_UE, dqmc.c:21-22, 405-408); the
			// stacks are slice-major, so slice 0 of item b is block b
			k_gdrift<T><<<NB, 256, 0, st>>>(N, G.p, ue.Gtt.p, (long long)NN, dmax.p + NB,
			                                dsum.p + NB, dcount.p + 1);
			launch_count++;
		}
		// half wrap of all 3 L slices per item (dqmc.c:415-451); the B stack
		// is free again and holds the intermediate product
		T *stk[3] = {ue.G0t.p, ue.Gtt.p, ue.Gt0.p};
		for (int q = 0; q < 3; q++) {
			gemm(gargs<T>(N, N, N, L * NB, stk[q], per_item((long long)NN), N, ehK.p, per_spin((long long)NN), N,
			              ue.Bs.p, per_item((long long)NN), N));
			gemm(gargs<T>(N, N, N, L * NB, iehK.p, per_spin((long long)NN), N, ue.Bs.p, per_item((long long)NN),
			              N, stk[q], per_item((long long)NN), N));
		}
		MeasArgs<T> m = meas_args();
		m.G0t = ue.G0t.p; m.Gtt = ue.Gtt.p; m.Gt0 = ue.Gt0.p;
		m.acc = acc_ue.p; m.acc_stride = ue_size; m.n_sample = n_ue.p;
		m.bond = p.meas_bond_corr;
		prof_begin(4);
		k_meas_uneqlt<T><<<dim3(C, L), 256, 0, st>>>(m);
		launch_count++;
		if (p.meas_gen_suscept || p.meas_energy_corr) {
			k_meas_uneqlt_xs<T><<<dim3(C, L), 256, 0, st>>>(m, gs_ue.p);
			launch_count++;
		}
		if (p.meas_thermal) {
			k_meas_uneqlt_xb<T><<<dim3(C, L), 128, 0, st>>>(m);
			launch_count++;
		}
		if (p.meas_thermal || p.meas_2bond_corr) {
			k_meas_uneqlt_x2<T><<<dim3(C, L), 128, 0, st>>>(m);
			launch_count++;
		}
		if (p.meas_nematic_corr) {
			k_meas_uneqlt_xn<T><<<dim3(C, L), 128, 0, st>>>(m);
			launch_count++;
		}
		prof_end(PC_MEAS, 0.0, 0.0);
		watchdog("k_meas_uneqlt");
		return 0;
	}

	// G, clusters and draws from the current fields, queued on the group's
	// stream (the lanes of an engine queue theirs side by side)
	int enqueue_init()
	{
		const long long tot = (long long)C * 2 * L * N;
		k_diag_all<<<grid_for(tot), 256, 0, st>>>(N, L, C, el.p, hs.p, dv.p, dvi.p);
		for (int f = 0; f < F; f++) build_cluster(f);
		for (int m = 0; F >= 2 && m < F; m++) build_pair(m);
		int rc = calc_eq_g(0);
		if (rc) return rc;
		draws(0);
		need_draws = false;
		need_init = false;
		return 0;
	}
	int init() override
	{
		const int rc = enqueue_init();
		if (rc) return rc;
		CK(cudaStreamSynchronize(st));
		return 0;
	}
	int init_async() override { return enqueue_init(); }

	// queue one sweep of the given kind
	int enqueue_sweep(bool meq, bool mue)
	{
		for (int l = 0; l < L; l++) {
			update(l);
			const int f = l / nmul;
			const bool recalc = ((l + 1) % nmul) == 0;
			if (recalc) {
				if (check_g) wrap_into(l, Gw.p);
				build_cluster(f);
				int rc = calc_eq_g((f + 1) % F);
				if (rc) return rc;
				if (check_g) {
					k_gdrift<T><<<NB, 256, 0, st>>>(N, G.p, Gw.p, (long long)N * N, dmax.p, dsum.p,
					                                dcount.p);
					launch_count++;
				}
				if (check_acc) {
					rc = calc_eq_g_acc((l + 1) % L);
					if (rc) return rc;
					k_gdrift<T><<<NB, 256, 0, st>>>(N, G.p, Gacc.p, (long long)N * N, dmax.p + 2 * NB,
					                                dsum.p + 2 * NB, dcount.p + 2);
					launch_count++;
				}
			} else {
				wrap(l);
			}
			if (meq && p.period_eqlt > 0 && (l + 1) % p.period_eqlt == 0) meas_eqlt();
		}
		if (mue) {
			int rc = meas_uneqlt();
			if (rc) return rc;
		}
		return 0;
	}

	int sweep_kind() override
	{
		if (sweep >= p.n_sweep) return -1;
		const bool meq = sweep >= p.n_sweep_warm;
		const bool mue = meq && p.period_uneqlt > 0 && sweep % p.period_uneqlt == 0;
		return (meq ? 1 : 0) | (mue ? 2 : 0);
	}
	int prepare() override
	{
		if (need_init) {
			const int rc = enqueue_init();
			if (rc) return rc;
		}
		if (need_draws) {
			draws(0);
			need_draws = false;
		}
		return 0;
	}
	int enqueue_one() override
	{
		const int kind = sweep_kind();
		if (kind < 0) return 0;
		launch_count = 0;
		const int rc = enqueue_sweep((kind & 1) != 0, (kind & 2) != 0);
		if (rc) return rc;
		if (!graph_launches.count(kind)) graph_launches[kind] = launch_count;
		sweep++;
		return 0;
	}
	void advance() override
	{
		if (sweep < p.n_sweep) sweep++;
	}
	cudaEvent_t jev = nullptr;
	int join_into(cudaStream_t s) override
	{
		if (!jev) CK(cudaEventCreateWithFlags(&jev, cudaEventDisableTiming));
		CK(cudaEventRecord(jev, st));
		CK(cudaStreamWaitEvent(s, jev, 0));
		return 0;
	}
	int wait_on(cudaEvent_t ev) override
	{
		CK(cudaStreamWaitEvent(st, ev, 0));
		return 0;
	}

	int sweeps(int n, int sync_after) override
	{
		if (need_init) {
			// fields were replaced: G, clusters and draws follow them again
			const int rc = enqueue_init();
			if (rc) return rc;
		}
		if (need_draws) {
			draws(0);
			need_draws = false;
		}
		for (int k = 0; k < n; k++) {
			if (sweep >= p.n_sweep) break;
			const bool meq = sweep >= p.n_sweep_warm;
			const bool mue = meq && p.period_uneqlt > 0 && sweep % p.period_uneqlt == 0;
			const int kind = (meq ? 1 : 0) | (mue ? 2 : 0);
			if (debug_sync) {
				int rc = enqueue_sweep(meq, mue);
				if (rc) return rc;
				sweep++;
				continue;
			}
			auto it = graphs.find(kind);
			if (it == graphs.end()) {
				cudaGraph_t gr;
				CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
				launch_count = 0;
				int rc = enqueue_sweep(meq, mue);
				cudaError_t ce = cudaStreamEndCapture(st, &gr);
				if (rc) {
					if (ce == cudaSuccess) cudaGraphDestroy(gr);
					return rc;
				}
				if (ce != cudaSuccess) {
					fprintf(stderr, "dqmc_b200: graph capture failed: %s\n", cudaGetErrorString(ce));
					return DQMC_E_CUDA;
				}
				cudaGraphExec_t ex;
				const cudaError_t ie = cudaGraphInstantiate(&ex, gr, 0);
				cudaGraphDestroy(gr);
				CK(ie);
				graphs[kind] = ex;
				graph_launches[kind] = launch_count;
				it = graphs.find(kind);
			}
			CK(cudaGraphLaunch(it->second, st));
			sweep++;
		}
		if (sync_after) return sync();
		return 0;
	}

	// One eager (not graph) sweep of the given kind with CUDA events around
	// every launch.  out[cls*4 + {0,1,2,3}] = {total ms, launches, flops, bytes}
	// for classes 0 gemm, 1 update, 2 calc_eq_g (all its launches, gemms
	// included), 4 measurement.  Advances the chains by one sweep.
	int profile(int meq, int mue, double *out, int ncls) override
	{
		if (sweep >= p.n_sweep) return DQMC_E_ARG;
		if (need_init) {
			const int rc = init();
			if (rc) return rc;
		}
		if (need_draws) {
			draws(0);
			need_draws = false;
		}
		// the update's work follows from its accepts: count them around the sweep
		std::vector<int> acc0(C), acc1(C);
		CK(cudaMemcpyAsync(acc0.data(), nacc.p, sizeof(int) * C, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		profiling = true;
		precs.clear();
		int rc = enqueue_sweep(meq, mue);
		profiling = false;
		if (rc) return rc;
		CK(cudaMemcpyAsync(acc1.data(), nacc.p, sizeof(int) * C, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		sweep++;
		for (int i = 0; i < ncls * 4; i++) out[i] = 0.0;
		if (PC_UPDATE < ncls) {
			// per accept and spin: one rank-1 column of the flush G += A B^T
			// (2 N^2) and the two panel products of the new column (2 N k
			// each, k = 0 .. kd-1 within a panel: 2 N (kd - 1) on average);
			// G read and written once per slice, chain and spin
			double a = 0.0;
			for (int c = 0; c < C; c++) a += (double)(acc1[c] - acc0[c]);
			const double cx = is_cplx<T>::value ? 4.0 : 1.0;
			out[PC_UPDATE * 4 + 2] = 2.0 * cx * a * (2.0 * N * N + 2.0 * N * (kd - 1));
			out[PC_UPDATE * 4 + 3] = 2.0 * 2.0 * sizeof(T) * (double)N * N * C * L;
		}
		fold_records(out, ncls);
		return 0;
	}

	// add the recorded launches to the class sums out[4 c + k] (the
	// update's FLOPs and bytes are counted from its accepts instead) and
	// release the events
	void fold_records(double *out, int ncls)
	{
		for (size_t i = 0; i < precs.size(); i++) {
			const PRec &r = precs[i];
			float ms = 0.f;
			cudaEventElapsedTime(&ms, pev[r.e0], pev[r.e1]);
			if (r.cls < ncls) {
				out[r.cls * 4 + 0] += ms;
				out[r.cls * 4 + 1] += 1;
				if (r.cls != PC_UPDATE) {
					out[r.cls * 4 + 2] += r.flops;
					out[r.cls * 4 + 3] += r.bytes;
				}
			}
		}
		for (cudaEvent_t e : pev) cudaEventDestroy(e);
		pev.clear();
		precs.clear();
	}

	bool update_on_chip() override { return upd_cl; }

	int profile_grad(int which, double *out, int ncls, int *launches) override
	{
		if (need_init) {
			const int rc = init();
			if (rc) return rc;
		}
		CK(cudaStreamSynchronize(st));
		for (int i = 0; i < ncls * 4; i++) out[i] = 0.0;
		profiling = true;
		precs.clear();
		launch_count = 0;
		const int rc = which ? obs_grad(nullptr, nullptr) : logdet_grad(nullptr, nullptr);
		profiling = false;
		if (launches) *launches = launch_count;
		cudaStreamSynchronize(st);
		fold_records(out, ncls);
		return rc;
	}

	// log |det(I + B_{L-1} ... B_0)| of every item and the sums
	// S = sum_l diag(d_l) (I - G_l) diag(1/d_l) over the slices of one
	// update-free sweep, G_l the equal-time G before slice l: the gradient
	// d log |det| / d theta = sum_l tr[S_l D_theta] with D_theta =
	// exp(dt K) d exp(-dt K) / d theta.  Fields, RNG and sweep count stay.
	int logdet_grad(double *ld_out, void *S_out) override
	{
		const size_t NN = (size_t)N * N;
		if (need_init) {
			const int rc = init();
			if (rc) return rc;
		}
		if (!Sg.p) {
			if (Sg.alloc(NB * NN)) return DQMC_E_NOMEM;
			CK(cudaDeviceSynchronize());   // its zeroing ran on the default stream
		}
		CK(cudaMemsetAsync(Sg.p, 0, sizeof(T) * NB * NN, st));
		for (int l = 0; l < L; l++) {
			k_grad_acc<T><<<grid_for((long long)NB * NN), 256, 0, st>>>(N, NB, L, l, G.p, dv.p, dvi.p, Sg.p);
			launch_count++;
			if ((l + 1) % nmul == 0) {
				const int rc = calc_eq_g((l / nmul + 1) % F);
				if (rc) return rc;
			} else {
				wrap(l);
			}
		}
		CK(cudaStreamSynchronize(st));
		CK(cudaGetLastError());
		std::vector<double> ld(NB);
		CK(cudaMemcpy(ld.data(), ldet.p, sizeof(double) * NB, cudaMemcpyDeviceToHost));
		for (int c = 0; c < C; c++) if (ld_out) ld_out[c] = ld[2 * c] + ld[2 * c + 1];
		if (S_out) CK(cudaMemcpy(S_out, Sg.p, sizeof(T) * NB * NN, cudaMemcpyDeviceToHost));
		return sync();
	}

	// Density and double occupancy of the fixed fields, averaged over the L
	// slices, and for each the matrices Z (per spin) with d obs / d theta =
	// sum_spin tr[Z D_theta]: Z = sum_m s_m exp(V_m) Y_m exp(-dt K),
	// Y_m = sum_l Gst(m, l) W_l Gst(l, m+1), Gst = O^-1 the space-time Green's
	// function and W_l the observable's weights at slice l.
	// obs[chain][2], Z[chain][obs][spin][N*N].  The checkpointed form holds
	// one row and one column of Gst per item at a time (O(N^2 L) memory);
	// the dense form (DQMC_OBS_GRAD=dense, and the sizes the unequal-time
	// kernels do not take) inverts the whole N L x N L matrix.
	int obs_grad(double *obs_out, void *Z_out) override
	{
		if (need_init) {
			const int rc = init();
			if (rc) return rc;
		}
		const char *ev = getenv("DQMC_OBS_GRAD");
		if ((ev && !strcmp(ev, "dense")) || !UneqState<T>::supported(N, F, L))
			return obs_grad_dense(obs_out, Z_out);
		return obs_grad_ckpt(obs_out, Z_out);
	}

	// <n> and <docc> of every chain from the equal-time diagonals hd
	// [item][N L] of both spins; w (when given) receives the weights W_l of
	// observable o (0: n, 1: docc) as [item][N L]
	void obs_values(const std::vector<T> &hd, double *obs_out, int o, double *w) const
	{
		const size_t NL = (size_t)N * L;
		const double inv = 1.0 / (double)NL;
		if (obs_out)
			for (int c = 0; c < C; c++) {
				double n = 0.0, d2 = 0.0;
				for (size_t r = 0; r < NL; r++) {
					const double nu = 1.0 - re(hd[(2 * c) * NL + r]), nd = 1.0 - re(hd[(2 * c + 1) * NL + r]);
					n += nu + nd;
					d2 += nu * nd;
				}
				obs_out[2 * c] = n * inv;
				obs_out[2 * c + 1] = d2 * inv;
			}
		if (w)
			for (int b = 0; b < NB; b++)
				for (size_t r = 0; r < NL; r++)
					w[b * NL + r] = o == 0 ? -inv : -inv * (1.0 - re(hd[(b ^ 1) * NL + r]));
	}

	// Z[chain][obs][spin] from the device sums Zb[obs][item]
	int z_out(const T *Zb, void *Z_out)
	{
		const size_t NN = (size_t)N * N;
		std::vector<T> hz(2 * NB * NN);
		CK(cudaMemcpyAsync(hz.data(), Zb, sizeof(T) * 2 * NB * NN, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		if (Z_out)
			for (int c = 0; c < C; c++)
				for (int o = 0; o < 2; o++)
					for (int sp = 0; sp < 2; sp++)
						memcpy((T *)Z_out + ((size_t)(c * 2 + o) * 2 + sp) * NN,
						       hz.data() + ((size_t)o * NB + 2 * c + sp) * NN, sizeof(T) * NN);
		return 0;
	}

	// the checkpointed form: the stabilised unequal-time Green's functions
	// (calc_ue_g) of the chain rotated to each cluster boundary s = c n_matmul
	// give Gst(s, .) and Gst(., s); the rows and columns of the cluster's
	// other slices follow by one B_m or B_m^-1 product each.  W_l of <n> is
	// -1/(N L) I and of <docc> -1/(N L) diag(1 - n_{-sigma}), so both Y_m take
	// alpha = -1/(N L) and only the <docc> column is weighted.  Per item: two
	// rows and three columns of N x N L (the current and next column and the
	// next column weighted for <docc>), beside the unequal-time stacks.  The
	// engine's G, clusters and fields are left as they were.
	int obs_grad_ckpt(double *obs_out, void *Z_out)
	{
		const size_t NN = (size_t)N * N, NL = (size_t)N * L, RS = NN * L;
		const long long rs = (long long)RS, nn = (long long)NN;
		ObsCkptWork &k = ok;
		int rc = 0;
		if (!k.R.p) {
			const bool had_ue = ue.G0t.p != nullptr;
			rc |= k.R.alloc(2 * NB * RS); rc |= k.X.alloc(3 * NB * RS);
			rc |= k.Y.alloc(2 * NB * NN); rc |= k.Yh.alloc(2 * NB * NN);
			rc |= k.Cl.alloc((size_t)NB * F * NN); rc |= k.dg.alloc(NB * NL);
			rc |= k.dv.alloc((size_t)NB * L * N); rc |= k.dvi.alloc((size_t)NB * L * N);
			rc |= k.w.alloc(NB * NL); rc |= k.ones.alloc(NB * NL);
			if (!rc && !had_ue && ue.alloc(N, L, F, NB)) {
				ue.release();
				rc = DQMC_E_NOMEM;
			}
			if (rc) { k.release(); return DQMC_E_NOMEM; }
			std::vector<double> one1(NB * NL, 1.0);
			CK(cudaMemcpy(k.ones.p, one1.data(), sizeof(double) * one1.size(), cudaMemcpyHostToDevice));
			// zeroed on the legacy default stream, which the engine's
			// non-blocking stream does not wait for
			CK(cudaDeviceSynchronize());
		}
		// the chain as it is: the equal-time diagonals give the observables
		// and their weights
		rc = calc_ue_g();
		if (rc) return rc;
		k_stack_diag<T><<<grid_for((long long)NB * NL), 256, 0, st>>>(N, L, NB, ue.Gtt.p, k.dg.p);
		launch_count++;
		std::vector<T> hd(NB * NL);
		CK(cudaMemcpyAsync(hd.data(), k.dg.p, sizeof(T) * NB * NL, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		obs_values(hd, obs_out, 0, nullptr);
		// the <docc> weights without their -1/(N L): 1 - n of the other spin
		std::vector<double> w(NB * NL);
		for (int b = 0; b < NB; b++)
			for (size_t r = 0; r < NL; r++) w[b * NL + r] = 1.0 - re(hd[(b ^ 1) * NL + r]);
		CK(cudaMemcpyAsync(k.w.p, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, st));
		const T a_obs = from_re<T>(-1.0 / (double)NL);
		CK(cudaMemsetAsync(k.Yh.p, 0, sizeof(T) * 2 * NB * NN, st));
		T *R0 = k.R.p, *R1 = k.R.p + NB * RS;
		T *Xc = k.X.p, *Xu = k.X.p + NB * RS, *Xw = k.X.p + 2 * NB * RS;
		const size_t cl_pitch = sizeof(T) * F * NN;
		for (int c = 0; c < F; c++) {
			const int s = c * nmul;
			if (c > 0) {
				// the rotated chain: fields shifted by s slices, its clusters
				// the chain's shifted by c (the same products, so no rebuild)
				k_rotate_slices<<<grid_for((long long)NB * L * N), 256, 0, st>>>(N, L, NB, s, dv.p, k.dv.p);
				k_rotate_slices<<<grid_for((long long)NB * L * N), 256, 0, st>>>(N, L, NB, s, dvi.p, k.dvi.p);
				launch_count += 2;
				CK(cudaMemcpy2DAsync(k.Cl.p, cl_pitch, Cl.p + (size_t)c * NN, cl_pitch,
				                     sizeof(T) * (F - c) * NN, NB, cudaMemcpyDeviceToDevice, st));
				CK(cudaMemcpy2DAsync(k.Cl.p + (size_t)(F - c) * NN, cl_pitch, Cl.p, cl_pitch,
				                     sizeof(T) * c * NN, NB, cudaMemcpyDeviceToDevice, st));
				std::swap(dv.p, k.dv.p); std::swap(dvi.p, k.dvi.p); std::swap(Cl.p, k.Cl.p);
				rc = calc_ue_g();
				std::swap(dv.p, k.dv.p); std::swap(dvi.p, k.dvi.p); std::swap(Cl.p, k.Cl.p);
				if (rc) return rc;
			}
			k_seed_rowcol<T><<<grid_for((long long)NB * RS), 256, 0, st>>>(N, L, NB, s, ue.G0t.p, ue.Gt0.p,
			                                                              R0, Xc);
			launch_count++;
			for (int j = 0; j < nmul; j++) {
				const int m = s + j;
				// slice j of the rotated stacks is slice m
				const T *Bm = ue.Bs.p + (size_t)j * NB * NN, *iBm = ue.iBs.p + (size_t)j * NB * NN;
				const T sg = from_re<T>(m == L - 1 ? -1.0 : 1.0);
				// column m+1, plain and weighted for <docc>
				k_shift_diag<T><<<grid_for((long long)NB * N), 256, 0, st>>>(N, NB, Xc + (size_t)m * N, rs,
				                                                            (long long)NL + 1, -1.0);
				launch_count++;
				gemm(gargs<T>((int)NL, N, N, NB, Xc, per_item(rs), (int)NL, iBm, per_item(nn), N, Xu,
				              per_item(rs), (int)NL, sg));
				GemmArgs<T> gw = gargs<T>((int)NL, N, N, NB, Xc, per_item(rs), (int)NL, iBm, per_item(nn), N,
				                          Xw, per_item(rs), (int)NL, sg, zero<T>(), GM_A_DD);
				gw.d = k.w.p; gw.dinv = k.ones.p; gw.aD = per_item((long long)NL);
				gemm(gw);
				// Y_m = Gst(m, .) W Gst(., m+1) of both observables: items
				// [0, NB) take the plain column, [NB, 2 NB) the weighted one
				gemm(gargs<T>(N, N, (int)NL, 2 * NB, R0, Addr{0, rs, NB}, N, Xu, Addr{(long long)(Xw - Xu), rs, NB},
				              (int)NL, k.Y.p, per_item(nn), N, a_obs));
				k_yacc<T><<<grid_for(2LL * NB * nn), 256, 0, st>>>(N, L, NB, 2 * NB, m, k.Y.p, dv.p, k.Yh.p);
				launch_count++;
				// row m+1
				if (j + 1 < nmul) {
					gemm(gargs<T>(N, (int)NL, N, NB, Bm, per_item(nn), N, R0, per_item(rs), N, R1, per_item(rs), N));
					k_shift_diag<T><<<grid_for((long long)NB * N), 256, 0, st>>>(N, NB, R1 + (size_t)(m + 1) * NN,
					                                                            rs, (long long)N + 1, 1.0);
					launch_count++;
					std::swap(R0, R1);
				}
				std::swap(Xc, Xu);
			}
		}
		// Z = Yh exp(-dt K) of both observables
		gemm(gargs<T>(N, N, N, 2 * NB, k.Yh.p, per_item(nn), N, expK.p, per_spin(nn), N, k.Y.p, per_item(nn), N));
		rc = z_out(k.Y.p, Z_out);
		if (rc) return rc;
		CK(cudaGetLastError());
		watchdog("obs_grad");
		return sync();
	}

	// the dense form: Gst from bsofi with one slice per block
	int obs_grad_dense(double *obs_out, void *Z_out)
	{
		const size_t NN = (size_t)N * N, NL = (size_t)N * L, NL2 = NL * NL;
		// the work buffers are allocated by the first call and kept, so that
		// repeated evaluations (new hopping, same fields) allocate nothing
		DevBuf<T> &O = og.O, &Gr = og.Gr, &Qh = og.Qh, &Tw = og.Tw, &Rw = og.Rw, &Yh = og.Yh,
		          &Zb = og.Zb, &dg = og.dg;
		DevBuf<double> &wb = og.wb;
		int rc = 0;
		if (!O.p) {
			rc |= O.alloc(NB * NL2); rc |= Gr.alloc(NB * NL2);
			rc |= Qh.alloc((size_t)NB * std::max(L - 1, 1) * 4 * NN); rc |= Tw.alloc((size_t)NB * L * NN);
			rc |= Rw.alloc((size_t)NB * NL * 2 * N); rc |= Yh.alloc(NB * NN); rc |= Zb.alloc(2 * NB * NN);
			rc |= dg.alloc(NB * NL); rc |= wb.alloc(NB * NL);
			if (rc) { og.release(); return DQMC_E_NOMEM; }
			// zeroed on the legacy default stream, which the engine's
			// non-blocking stream does not wait for
			CK(cudaDeviceSynchronize());
		}
		CK(cudaMemsetAsync(O.p, 0, sizeof(T) * NB * NL2, st));
		k_add_diag<T><<<grid_for((long long)NL * NB), 256, 0, st>>>((int)NL, NB, O.p, (long long)NL2);
		k_build_o<T><<<grid_for((long long)NN * L * NB), 256, 0, st>>>(N, L, NB, expK.p, dv.p, O.p);
		launch_count += 2;
		rc = bsofi(L, O.p, Gr.p, Qh.p, Tw.p, Rw.p);
		if (rc) return rc;
		k_diag_of<T><<<grid_for((long long)NL * NB), 256, 0, st>>>((long long)NL, NB, Gr.p, dg.p);
		launch_count++;
		std::vector<T> hd(NB * NL);
		CK(cudaMemcpyAsync(hd.data(), dg.p, sizeof(T) * NB * NL, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		obs_values(hd, obs_out, 0, nullptr);
		std::vector<double> w(NB * NL);
		for (int o = 0; o < 2; o++) {
			obs_values(hd, nullptr, o, w.data());
			// stream-ordered after the previous observable's use of wb; a
			// copy from pageable memory returns once w has been staged
			CK(cudaMemcpyAsync(wb.p, w.data(), sizeof(double) * NB * NL, cudaMemcpyHostToDevice, st));
			k_rowscale<T><<<grid_for((long long)NL2 * NB), 256, 0, st>>>((long long)NL, NB, Gr.p, wb.p, O.p);
			launch_count++;
			// Y_m = Gst(m-row) (W Gst)((m+1)-column): m < L-1 at once, then m = L-1
			if (L > 1)
				gemm(gargs<T>(N, N, (int)NL, NB * (L - 1), Gr.p, Addr{(long long)NL2, (long long)N, L - 1},
				              (int)NL, O.p + N * NL, Addr{(long long)NL2, (long long)(N * NL), L - 1}, (int)NL,
				              Tw.p, Addr{(long long)(L * NN), (long long)NN, L - 1}, N));
			gemm(gargs<T>(N, N, (int)NL, NB, Gr.p + (size_t)(L - 1) * N, per_item((long long)NL2), (int)NL,
			              O.p, per_item((long long)NL2), (int)NL, Tw.p + (size_t)(L - 1) * NN,
			              per_item((long long)(L * NN)), N));
			k_yhat<T><<<grid_for((long long)NN * NB), 256, 0, st>>>(N, L, NB, Tw.p, dv.p, Yh.p);
			launch_count++;
			gemm(gargs<T>(N, N, N, NB, Yh.p, per_item((long long)NN), N, expK.p, per_spin((long long)NN), N,
			              Zb.p + (size_t)o * NB * NN, per_item((long long)NN), N));
		}
		rc = z_out(Zb.p, Z_out);
		if (rc) return rc;
		CK(cudaGetLastError());
		return sync();
	}

	// replace the hopping matrices in place (stream-ordered after queued
	// work); G and the clusters are recomputed before the next use
	int set_hopping(const void *const *m) override
	{
		const size_t NN = (size_t)N * N;
		DevBuf<T> *dst[4] = {&expK, &iexpK, &ehK, &iehK};
		for (int k = 0; k < 4; k++)
			for (int sp = 0; sp < 2; sp++) {
				if (!m[2 * k + sp]) return DQMC_E_ARG;
				CK(cudaMemcpyAsync(dst[k]->p + sp * NN, m[2 * k + sp], sizeof(T) * NN,
				                   cudaMemcpyHostToDevice, st));
			}
		CK(cudaStreamSynchronize(st));
		need_init = true;
		return 0;
	}

	int sync() override
	{
		CK(cudaStreamSynchronize(st));
		unsigned e = 0;
		CK(cudaMemcpy(&e, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
		return e ? DQMC_E_DEVICE : 0;
	}

	unsigned errors() override
	{
		unsigned e = 0;
		cudaStreamSynchronize(st);
		cudaMemcpy(&e, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost);
		return e;
	}

	int launches(int meq, int mue) override
	{
		const int kind = (meq ? 1 : 0) | (mue ? 2 : 0);
		auto it = graph_launches.find(kind);
		if (it != graph_launches.end()) return it->second;
		return -1;
	}

	cudaStream_t stream() override { return st; }

	int get_chain(int c, uint64_t *r, int *h, int *sw) override
	{
		if (c < 0 || c >= C) return DQMC_E_ARG;
		CK(cudaStreamSynchronize(st));
		// the state the chain has at the sweep boundary, before the look-ahead
		if (r) CK(cudaMemcpy(r, rng_ckpt.p + (size_t)c * 17, sizeof(uint64_t) * 17, cudaMemcpyDeviceToHost));
		if (h) CK(cudaMemcpy(h, hs.p + (size_t)c * L * N, sizeof(int) * L * N, cudaMemcpyDeviceToHost));
		if (sw) *sw = sweep;
		return 0;
	}

	int get_acc(int c, int *eqn, void *eq, int *uen, void *uea) override
	{
		if (c < 0 || c >= C) return DQMC_E_ARG;
		CK(cudaStreamSynchronize(st));
		if (eqn) CK(cudaMemcpy(eqn, n_eq.p + c, sizeof(int), cudaMemcpyDeviceToHost));
		if (eq) CK(cudaMemcpy(eq, acc_eq.p + (size_t)c * eq_size, sizeof(T) * eq_size, cudaMemcpyDeviceToHost));
		if (ue_size) {
			if (uen) CK(cudaMemcpy(uen, n_ue.p + c, sizeof(int), cudaMemcpyDeviceToHost));
			if (uea) CK(cudaMemcpy(uea, acc_ue.p + (size_t)c * ue_size, sizeof(T) * ue_size, cudaMemcpyDeviceToHost));
		}
		return 0;
	}

	int get_g(int c, void *gu, void *gd, void *ph) override
	{
		if (c < 0 || c >= C) return DQMC_E_ARG;
		CK(cudaStreamSynchronize(st));
		const size_t NN = (size_t)N * N;
		if (gu) CK(cudaMemcpy(gu, G.p + (size_t)(2 * c) * NN, sizeof(T) * NN, cudaMemcpyDeviceToHost));
		if (gd) CK(cudaMemcpy(gd, G.p + (size_t)(2 * c + 1) * NN, sizeof(T) * NN, cudaMemcpyDeviceToHost));
		if (ph) CK(cudaMemcpy(ph, phase.p + c, sizeof(T), cudaMemcpyDeviceToHost));
		return 0;
	}

	int accepts(int c, long long *n) override
	{
		if (c < 0 || c >= C) return DQMC_E_ARG;
		int v = 0;
		CK(cudaStreamSynchronize(st));
		CK(cudaMemcpy(&v, nacc.p + c, sizeof(int), cudaMemcpyDeviceToHost));
		*n = v;
		return 0;
	}
};

// An engine's chains split into lanes: contiguous sub-batches, each a Group
// with its own stream and sweep graphs.  A sweep forks from the engine's
// stream, queues every lane, and joins back, so that work placed on the
// engine's stream before or after a sweep (events, copies) is ordered
// around all lanes.  Kernels of different lanes then overlap on the SMs:
// the latency-bound QR, recombine and update launches of one lane run
// beside the tensor-bound GEMMs of another, and the partial last wave of
// one launch is filled by the next lane's.  Each chain's arithmetic is the
// same in any lane, so results do not depend on the split.
struct Lanes : GroupBase {
	std::vector<GroupBase *> g;
	std::vector<int> c0;          // first chain of each lane; c0.back() = chains
	std::vector<cudaEvent_t> ev;  // ev[0] fork, ev[1 + k] join of lane k
	cudaStream_t st = nullptr;
	size_t s_elems = 0;           // N * N entries of T per spin (gradient outputs)
	size_t elem = 0;              // sizeof(T)
	size_t n_site = 0, hs_len = 0;          // N and L N per chain
	size_t eq_bytes = 0, ue_bytes = 0;      // accumulator bytes per chain
	int c0s() const { return c0.back(); }

	~Lanes() override
	{
		for (GroupBase *x : g) delete x;
		for (cudaEvent_t e : ev) cudaEventDestroy(e);
		if (st) cudaStreamDestroy(st);
	}

	int create(const dqmc_params &p, int n_chain, int n_lane)
	{
		n_lane = std::max(1, std::min(n_lane, n_chain));
		s_elems = (size_t)p.N * p.N;
		elem = p.cplx ? sizeof(zd) : sizeof(double);
		n_site = (size_t)p.N;
		hs_len = (size_t)p.L * p.N;
		const AccLayout al = acc_layout(p);
		eq_bytes = elem * (size_t)al.eq_size;
		ue_bytes = elem * (size_t)al.ue_size;
		CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
		ev.assign(n_lane + 1, nullptr);
		for (auto &e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		c0.push_back(0);
		for (int k = 0; k < n_lane; k++) {
			const int n = n_chain / n_lane + (k < n_chain % n_lane ? 1 : 0);
			GroupBase *x;
			int rc;
			if (p.cplx) {
				auto *gg = new Group<zd>();
				rc = gg->create(p, n, n_chain);
				x = gg;
			} else {
				auto *gg = new Group<double>();
				rc = gg->create(p, n, n_chain);
				x = gg;
			}
			if (rc) {
				delete x;
				return rc;
			}
			g.push_back(x);
			c0.push_back(c0.back() + n);
		}
		return 0;
	}

	// lane of chain c (and c relative to it), or -1
	int lane(int &c) const
	{
		if (c < 0 || c >= c0.back()) return -1;
		int k = (int)(std::upper_bound(c0.begin(), c0.end(), c) - c0.begin()) - 1;
		c -= c0[k];
		return k;
	}

	int set_chain(int c, const double *el, const double *del, const uint64_t *rng, const int *hs,
	              int sweep) override
	{
		const int k = lane(c);
		return k < 0 ? DQMC_E_ARG : g[k]->set_chain(c, el, del, rng, hs, sweep);
	}
	int set_acc(int c, int eqn, const void *eq, int uen, const void *ue) override
	{
		const int k = lane(c);
		return k < 0 ? DQMC_E_ARG : g[k]->set_acc(c, eqn, eq, uen, ue);
	}
	// every chain at once (first = 0, n = all): each lane its contiguous slice
	int set_chains(int first, int n, const double *el, const double *del, const uint64_t *rng,
	               const int *hs, int sweep) override
	{
		if (first != 0 || n != c0s()) return DQMC_E_ARG;
		CK(cudaStreamSynchronize(st));
		for (size_t k = 0; k < g.size(); k++) {
			const size_t a = c0[k], m = c0[k + 1] - c0[k];
			const int rc = g[k]->set_chains(0, (int)m, el + a * 2 * n_site, del + a * 2 * n_site,
			                                rng + a * 17, hs + a * hs_len, sweep);
			if (rc) return rc;
		}
		return 0;
	}
	int get_chains(int first, int n, uint64_t *rng, int *hs, int *sweep, int *eqn, void *eq, int *uen,
	               void *ue) override
	{
		if (first != 0 || n != c0s()) return DQMC_E_ARG;
		CK(cudaStreamSynchronize(st));
		for (size_t k = 0; k < g.size(); k++) {
			const size_t a = c0[k], m = c0[k + 1] - c0[k];
			const int rc = g[k]->get_chains(
				0, (int)m, rng ? rng + a * 17 : nullptr, hs ? hs + a * hs_len : nullptr, sweep,
				eqn ? eqn + a : nullptr, eq ? (char *)eq + a * eq_bytes : nullptr, uen ? uen + a : nullptr,
				ue ? (char *)ue + a * ue_bytes : nullptr);
			if (rc) return rc;
		}
		return 0;
	}
	int get_chain(int c, uint64_t *rng, int *hs, int *sweep) override
	{
		const int k = lane(c);
		return k < 0 ? DQMC_E_ARG : g[k]->get_chain(c, rng, hs, sweep);
	}
	int get_acc(int c, int *eqn, void *eq, int *uen, void *ue) override
	{
		const int k = lane(c);
		return k < 0 ? DQMC_E_ARG : g[k]->get_acc(c, eqn, eq, uen, ue);
	}
	int get_g(int c, void *gu, void *gd, void *ph) override
	{
		const int k = lane(c);
		return k < 0 ? DQMC_E_ARG : g[k]->get_g(c, gu, gd, ph);
	}
	int accepts(int c, long long *n) override
	{
		const int k = lane(c);
		return k < 0 ? DQMC_E_ARG : g[k]->accepts(c, n);
	}

	int init() override
	{
		// after work the caller queued on the engine's stream; the lanes
		// recompute side by side, each on its own stream
		CK(cudaStreamSynchronize(st));
		for (GroupBase *x : g) {
			const int rc = x->init_async();
			if (rc) return rc;
		}
		for (GroupBase *x : g) CK(cudaStreamSynchronize(x->stream()));
		return 0;
	}
	int init_async() override { return init(); }

	int sweeps(int n, int sync_after) override
	{
		CK(cudaEventRecord(ev[0], st));
		for (size_t k = 0; k < g.size(); k++) {
			CK(cudaStreamWaitEvent(g[k]->stream(), ev[0], 0));
			const int rc = g[k]->sweeps(n, 0);
			// join even a lane that failed, so the engine's stream stays ordered
			CK(cudaEventRecord(ev[1 + k], g[k]->stream()));
			CK(cudaStreamWaitEvent(st, ev[1 + k], 0));
			if (rc) return rc;
		}
		return sync_after ? sync() : 0;
	}

	int sync() override
	{
		int out = 0;
		for (GroupBase *x : g) {
			const int rc = x->sync();
			if (rc && !out) out = rc;
		}
		CK(cudaStreamSynchronize(st));
		return out;
	}

	unsigned errors() override
	{
		unsigned e = 0;
		for (GroupBase *x : g) e |= x->errors();
		return e;
	}

	cudaStream_t stream() override { return st; }

	int launches(int meq, int mue) override
	{
		int n = 0;
		for (GroupBase *x : g) {
			const int v = x->launches(meq, mue);
			if (v < 0) return -1;
			n += v;
		}
		return n;
	}

	// class sums over the lanes, each profiled alone
	int profile(int meq, int mue, double *out, int ncls) override
	{
		CK(cudaStreamSynchronize(st));
		std::vector<double> part(ncls * 4);
		for (int i = 0; i < ncls * 4; i++) out[i] = 0.0;
		for (GroupBase *x : g) {
			const int rc = x->profile(meq, mue, part.data(), ncls);
			if (rc) return rc;
			for (int i = 0; i < ncls * 4; i++) out[i] += part[i];
		}
		return 0;
	}

	bool update_on_chip() override { return g[0]->update_on_chip(); }

	// class sums and launches over the lanes, each profiled alone
	int profile_grad(int which, double *out, int ncls, int *launches) override
	{
		CK(cudaStreamSynchronize(st));
		std::vector<double> part(ncls * 4);
		for (int i = 0; i < ncls * 4; i++) out[i] = 0.0;
		int total = 0;
		for (GroupBase *x : g) {
			int n = 0;
			const int rc = x->profile_grad(which, part.data(), ncls, &n);
			if (rc) return rc;
			for (int i = 0; i < ncls * 4; i++) out[i] += part[i];
			total += n;
		}
		if (launches) *launches = total;
		return 0;
	}

	// the gradient paths launch eagerly and wait on the host between steps:
	// two host threads, each taking every second lane, keep two lanes' work
	// concurrent (more threads ran slower: their allocations and device-wide
	// waits serialise them)
	template <typename F>
	int per_lane(F f)
	{
		CK(cudaStreamSynchronize(st));
		int dev = 0;
		CK(cudaGetDevice(&dev));
		std::vector<int> rc(g.size(), 0);
		std::vector<std::thread> th;
		const size_t nth = std::min<size_t>(2, g.size());
		for (size_t t = 0; t < nth; t++)
			th.emplace_back([&, t] {
				const bool ok = cudaSetDevice(dev) == cudaSuccess;
				for (size_t k = t; k < g.size(); k += nth) {
					rc[k] = ok ? f(k) : DQMC_E_CUDA;
					if (rc[k]) break;
				}
			});
		for (auto &t : th) t.join();
		for (int r : rc) if (r) return r;
		return 0;
	}

	int logdet_grad(double *logdet, void *S) override
	{
		return per_lane([&](size_t k) {
			const size_t c = c0[k];
			return g[k]->logdet_grad(logdet ? logdet + c : nullptr,
			                         S ? (char *)S + c * 2 * s_elems * elem : nullptr);
		});
	}

	int set_hopping(const void *const *m) override
	{
		CK(cudaStreamSynchronize(st));
		for (GroupBase *x : g) {
			const int rc = x->set_hopping(m);
			if (rc) return rc;
		}
		return 0;
	}

	int set_check_g(int on) override
	{
		CK(cudaStreamSynchronize(st));
		for (GroupBase *x : g) {
			const int rc = x->set_check_g(on);
			if (rc) return rc;
		}
		return 0;
	}

	int sweep_kind() override { return g[0]->sweep_kind(); }
	int prepare() override
	{
		// after work the caller queued on the engine's stream
		CK(cudaEventRecord(ev[0], st));
		for (GroupBase *x : g) {
			CK(cudaStreamWaitEvent(x->stream(), ev[0], 0));
			const int rc = x->prepare();
			if (rc) return rc;
		}
		return 0;
	}
	int enqueue_one() override
	{
		CK(cudaEventRecord(ev[0], st));
		for (size_t k = 0; k < g.size(); k++) {
			CK(cudaStreamWaitEvent(g[k]->stream(), ev[0], 0));
			const int rc = g[k]->enqueue_one();
			CK(cudaEventRecord(ev[1 + k], g[k]->stream()));
			CK(cudaStreamWaitEvent(st, ev[1 + k], 0));
			if (rc) return rc;
		}
		return 0;
	}
	void advance() override
	{
		for (GroupBase *x : g) x->advance();
	}
	int join_into(cudaStream_t s) override
	{
		for (GroupBase *x : g) {
			const int rc = x->join_into(s);
			if (rc) return rc;
		}
		CK(cudaEventRecord(ev[0], st));
		CK(cudaStreamWaitEvent(s, ev[0], 0));
		return 0;
	}
	int wait_on(cudaEvent_t e) override
	{
		CK(cudaStreamWaitEvent(st, e, 0));
		for (GroupBase *x : g) {
			const int rc = x->wait_on(e);
			if (rc) return rc;
		}
		return 0;
	}

	int g_drift(int which, int first, int n, double *mx, double *mean, int *count) override
	{
		if (first != 0 || n != c0s()) return DQMC_E_ARG;
		CK(cudaStreamSynchronize(st));
		for (size_t k = 0; k < g.size(); k++) {
			const size_t a = c0[k], m = c0[k + 1] - c0[k];
			const int rc = g[k]->g_drift(which, 0, (int)m, mx ? mx + a : nullptr,
			                             mean ? mean + a : nullptr, count);
			if (rc) return rc;
		}
		return 0;
	}

	int obs_grad(double *obs, void *Z) override
	{
		return per_lane([&](size_t k) {
			const size_t c = c0[k];
			return g[k]->obs_grad(obs ? obs + 2 * c : nullptr,
			                      Z ? (char *)Z + c * 4 * s_elems * elem : nullptr);
		});
	}
};

// lanes of an engine of n_chain chains: DQMC_LANES when set, else for real
// chains one lane per 32 from 256 chains up (at most 8) and one per 64 below
// (at most 4), for complex chains one per 32 (at most 4).  Measured: 256
// chains of 12 x 12 run 1235 / 1268 / 1288 / 1297 chain-sweeps/s in 2 / 4 /
// 6 / 8 lanes (end to end 1136 in 4, 1156 in 8); the real gradients of 128
// configurations of 8 x 8 run 719 evaluations/s in two lanes and 628 in
// four; 64 complex 10 x 10 chains 507 in two lanes and 518 in four.
static int lane_count(int n_chain, bool cplx)
{
	if (const char *v = getenv("DQMC_LANES")) {
		const int n = atoi(v);
		if (n >= 1) return std::min(n, n_chain);
	}
	if (cplx) return std::max(1, std::min(4, n_chain / 32));
	if (n_chain >= 256) return std::min(8, n_chain / 32);
	return std::max(1, std::min(4, n_chain / 64));
}

}  // namespace dq

using namespace dq;

struct dqmc_engine {
	GroupBase *g;
	int cplx;
};

// engines advanced together, one CUDA graph launch per sweep for all of them
struct dqmc_batch {
	std::vector<dqmc_engine *> es;
	cudaStream_t st = nullptr;
	cudaEvent_t fork = nullptr, done = nullptr;
	std::vector<cudaEvent_t> join;
	std::map<std::vector<int>, cudaGraphExec_t> graphs;   // by the engines' sweep kinds
	~dqmc_batch()
	{
		for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
		for (cudaEvent_t e : join) cudaEventDestroy(e);
		if (fork) cudaEventDestroy(fork);
		if (done) cudaEventDestroy(done);
		if (st) cudaStreamDestroy(st);
	}
};

// One sweep of every engine of b that has sweeps left, as one graph launch
// on b's stream: the graph for this combination of sweep kinds is captured
// on first use (a fork from b's stream into every engine and its lanes, each
// engine's sweep kernels queued eagerly there, and the joins back), and
// replayed afterwards.  Pending re-initialisations run first, outside the
// graph.  Returns 1 when no engine had a sweep left.
static int batch_sweep(dqmc_batch *b)
{
	std::vector<int> key(b->es.size());
	bool any = false;
	for (size_t i = 0; i < b->es.size(); i++) {
		key[i] = b->es[i]->g->sweep_kind();
		any |= key[i] >= 0;
	}
	if (!any) return 1;
	for (size_t i = 0; i < b->es.size(); i++) {
		if (key[i] < 0) continue;
		int rc = b->es[i]->g->prepare();
		if (!rc) rc = b->es[i]->g->join_into(b->st);
		if (rc) return rc;
	}
	auto it = b->graphs.find(key);
	if (it == b->graphs.end()) {
		cudaGraph_t gr;
		CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
		int rc = 0;
		cudaError_t ce = cudaEventRecord(b->fork, b->st);
		for (size_t i = 0; i < b->es.size() && !rc && ce == cudaSuccess; i++) {
			if (key[i] < 0) continue;
			GroupBase *x = b->es[i]->g;
			ce = cudaStreamWaitEvent(x->stream(), b->fork, 0);
			if (ce == cudaSuccess) rc = x->enqueue_one();
			if (ce == cudaSuccess) ce = cudaEventRecord(b->join[i], x->stream());
			if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->st, b->join[i], 0);
		}
		const cudaError_t ee = cudaStreamEndCapture(b->st, &gr);
		if (ee == cudaSuccess && (rc || ce != cudaSuccess)) cudaGraphDestroy(gr);
		if (rc) return rc;
		if (ce != cudaSuccess || ee != cudaSuccess) {
			fprintf(stderr, "dqmc_b200: batch graph capture failed: %s\n",
			        cudaGetErrorString(ce != cudaSuccess ? ce : ee));
			return DQMC_E_CUDA;
		}
		cudaGraphExec_t ex;
		const cudaError_t ie = cudaGraphInstantiate(&ex, gr, 0);
		cudaGraphDestroy(gr);
		CK(ie);
		it = b->graphs.emplace(key, ex).first;
	} else {
		for (size_t i = 0; i < b->es.size(); i++)
			if (key[i] >= 0) b->es[i]->g->advance();
	}
	CK(cudaGraphLaunch(it->second, b->st));
	CK(cudaEventRecord(b->done, b->st));
	for (dqmc_engine *e : b->es) {
		const int rc = e->g->wait_on(b->done);
		if (rc) return rc;
	}
	return 0;
}

extern "C" {

int dqmc_acc_sizes(const dqmc_params *p, int *eq_size, int *ue_size)
{
	if (!p) return DQMC_E_ARG;
	const AccLayout al = acc_layout(*p);
	if (eq_size) *eq_size = (int)al.eq_size;
	if (ue_size) *ue_size = (int)al.ue_size;
	return 0;
}

int dqmc_engine_create(const dqmc_params *p, int n_chain, int device, dqmc_engine **out)
{
	if (!p || !out || n_chain < 1) return DQMC_E_ARG;
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
		fprintf(stderr, "dqmc_b200: no CUDA device\n");
		return DQMC_E_CUDA;
	}
	if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return DQMC_E_CUDA;
	auto *g = new Lanes();
	const int rc = g->create(*p, n_chain, lane_count(n_chain, p->cplx != 0));
	if (rc) {
		delete g;
		return rc;
	}
	*out = new dqmc_engine{g, p->cplx};
	return 0;
}

void dqmc_engine_destroy(dqmc_engine *e)
{
	if (!e) return;
	delete e->g;
	delete e;
}

int dqmc_engine_set_chain(dqmc_engine *e, int chain, const double *exp_lambda, const double *del,
		const uint64_t *rng, const int *hs, int sweep)
{
	if (!e || !exp_lambda || !del || !rng || !hs) return DQMC_E_ARG;
	return e->g->set_chain(chain, exp_lambda, del, rng, hs, sweep);
}

int dqmc_engine_set_acc(dqmc_engine *e, int chain, int eq_n_sample, const void *eq_acc,
		int ue_n_sample, const void *ue_acc)
{
	if (!e) return DQMC_E_ARG;
	return e->g->set_acc(chain, eq_n_sample, eq_acc, ue_n_sample, ue_acc);
}

int dqmc_engine_set_chains(dqmc_engine *e, const double *exp_lambda, const double *del,
		const uint64_t *rng, const int *hs, int sweep)
{
	if (!e || !exp_lambda || !del || !rng || !hs) return DQMC_E_ARG;
	const int n = ((Lanes *)e->g)->c0s();
	return e->g->set_chains(0, n, exp_lambda, del, rng, hs, sweep);
}

int dqmc_engine_get_chains(dqmc_engine *e, uint64_t *rng, int *hs, int *sweep, int *eq_n_sample,
		void *eq_acc, int *ue_n_sample, void *ue_acc)
{
	if (!e) return DQMC_E_ARG;
	const int n = ((Lanes *)e->g)->c0s();
	return e->g->get_chains(0, n, rng, hs, sweep, eq_n_sample, eq_acc, ue_n_sample, ue_acc);
}

int dqmc_engine_init(dqmc_engine *e) { return e ? e->g->init() : DQMC_E_ARG; }

int dqmc_engine_sweeps(dqmc_engine *e, int n, int sync)
{
	return e ? e->g->sweeps(n, sync) : DQMC_E_ARG;
}

int dqmc_engine_sync(dqmc_engine *e) { return e ? e->g->sync() : DQMC_E_ARG; }

unsigned dqmc_engine_errors(dqmc_engine *e) { return e ? e->g->errors() : 0u; }

int dqmc_engine_get_chain(dqmc_engine *e, int chain, uint64_t *rng, int *hs, int *sweep)
{
	return e ? e->g->get_chain(chain, rng, hs, sweep) : DQMC_E_ARG;
}

int dqmc_engine_get_acc(dqmc_engine *e, int chain, int *eq_n_sample, void *eq_acc,
		int *ue_n_sample, void *ue_acc)
{
	return e ? e->g->get_acc(chain, eq_n_sample, eq_acc, ue_n_sample, ue_acc) : DQMC_E_ARG;
}

int dqmc_engine_get_g(dqmc_engine *e, int chain, void *gu, void *gd, void *phase)
{
	return e ? e->g->get_g(chain, gu, gd, phase) : DQMC_E_ARG;
}

int dqmc_engine_accepts(dqmc_engine *e, int chain, long long *n)
{
	return (e && n) ? e->g->accepts(chain, n) : DQMC_E_ARG;
}

void *dqmc_engine_stream(dqmc_engine *e) { return e ? (void *)e->g->stream() : nullptr; }

int dqmc_engine_lanes(dqmc_engine *e) { return e ? (int)((Lanes *)e->g)->g.size() : DQMC_E_ARG; }

int dqmc_engine_launches_per_sweep(dqmc_engine *e, int meas_eq, int meas_ue)
{
	return e ? e->g->launches(meas_eq, meas_ue) : DQMC_E_ARG;
}

int dqmc_engine_logdet_grad(dqmc_engine *e, double *logdet, void *S)
{
	return e ? e->g->logdet_grad(logdet, S) : DQMC_E_ARG;
}

int dqmc_engine_obs_grad(dqmc_engine *e, double *obs, void *Z)
{
	return e ? e->g->obs_grad(obs, Z) : DQMC_E_ARG;
}

int dqmc_engine_set_hopping(dqmc_engine *e, const void *exp_Ku, const void *exp_Kd,
		const void *inv_exp_Ku, const void *inv_exp_Kd, const void *exp_halfKu,
		const void *exp_halfKd, const void *inv_exp_halfKu, const void *inv_exp_halfKd)
{
	if (!e) return DQMC_E_ARG;
	const void *m[8] = {exp_Ku, exp_Kd, inv_exp_Ku, inv_exp_Kd, exp_halfKu, exp_halfKd,
	                    inv_exp_halfKu, inv_exp_halfKd};
	return e->g->set_hopping(m);
}

int dqmc_batch_create(dqmc_engine *const *engines, int n, dqmc_batch **out)
{
	if (!engines || n < 1 || !out) return DQMC_E_ARG;
	*out = nullptr;
	if (getenv("DQMC_DEBUG_SYNC")) return DQMC_E_ARG;   // its eager checks cannot be captured
	dqmc_batch *b = new (std::nothrow) dqmc_batch;
	if (!b) return DQMC_E_NOMEM;
	for (int i = 0; i < n; i++) {
		if (!engines[i]) {
			delete b;
			return DQMC_E_ARG;
		}
		b->es.push_back(engines[i]);
	}
	b->join.assign(n, nullptr);
	bool ok = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
	          cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
	          cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
	for (int i = 0; ok && i < n; i++)
		ok = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
	if (!ok) {
		delete b;
		return DQMC_E_CUDA;
	}
	*out = b;
	return 0;
}

int dqmc_batch_sweeps(dqmc_batch *b, int n_sweeps, int sync)
{
	if (!b || n_sweeps < 0) return DQMC_E_ARG;
	for (int k = 0; k < n_sweeps; k++) {
		const int rc = batch_sweep(b);
		if (rc == 1) break;
		if (rc) return rc;
	}
	if (sync) CK(cudaStreamSynchronize(b->st));
	return 0;
}

void *dqmc_batch_stream(dqmc_batch *b) { return b ? (void *)b->st : nullptr; }

void dqmc_batch_destroy(dqmc_batch *b)
{
	if (!b) return;
	cudaStreamSynchronize(b->st);
	delete b;
}

int dqmc_engine_check_g(dqmc_engine *e, int on)
{
	return e ? e->g->set_check_g(on) : DQMC_E_ARG;
}

int dqmc_engine_g_drift(dqmc_engine *e, double *max_abs, double *mean_abs, int *n_recalc)
{
	if (!e) return DQMC_E_ARG;
	const int n = ((Lanes *)e->g)->c0s();
	return e->g->g_drift(0, 0, n, max_abs, mean_abs, n_recalc);
}

int dqmc_engine_g_drift_ue(dqmc_engine *e, double *max_abs, double *mean_abs, int *n_meas)
{
	if (!e) return DQMC_E_ARG;
	const int n = ((Lanes *)e->g)->c0s();
	return e->g->g_drift(1, 0, n, max_abs, mean_abs, n_meas);
}

int dqmc_engine_g_drift_acc(dqmc_engine *e, double *max_abs, double *mean_abs, int *n_recalc)
{
	if (!e) return DQMC_E_ARG;
	const int n = ((Lanes *)e->g)->c0s();
	return e->g->g_drift(2, 0, n, max_abs, mean_abs, n_recalc);
}

int dqmc_engine_profile_sweep(dqmc_engine *e, int meas_eq, int meas_ue, double *out, int n_class)
{
	return (e && out && n_class > 0) ? e->g->profile(meas_eq, meas_ue, out, n_class) : DQMC_E_ARG;
}

int dqmc_engine_update_on_chip(dqmc_engine *e)
{
	return e ? (e->g->update_on_chip() ? 1 : 0) : DQMC_E_ARG;
}

int dqmc_engine_profile_grad(dqmc_engine *e, int which, double *out, int n_class, int *launches)
{
	if (!e || !out || n_class <= 0 || (which != 0 && which != 1)) return DQMC_E_ARG;
	return e->g->profile_grad(which, out, n_class, launches);
}


}  // extern "C"

// ------------------------------------------------------------ kernel seams

template <typename T>
struct Scratch {
	std::vector<void *> ptrs;
	~Scratch() { for (void *p : ptrs) cudaFree(p); }
	template <typename U>
	U *get(size_t n)
	{
		void *p = nullptr;
		if (cudaMalloc(&p, sizeof(U) * (n ? n : 1)) != cudaSuccess) return nullptr;
		ptrs.push_back(p);
		return (U *)p;
	}
};

template <typename T>
static int seam_calc_eq_g(int batch, int N, int F, int l, const void *C, void *G, void *phase,
		cudaStream_t st)
{
	if (batch < 1 || N < 1 || N > max_dense_n<T>() || F < 1 || l < 0 || l >= F || !C || !G || !phase)
		return DQMC_E_ARG;
	const size_t NN = (size_t)N * N;
	Scratch<T> sc;
	EqWork<T> w;
	memset(&w, 0, sizeof(w));
	w.N = N; w.F = F; w.NB = batch;
	w.Cl = (const T *)C; w.cl_stride = (long long)F * NN;
	w.Qm = sc.template get<T>(batch * NN); w.Tm = sc.template get<T>(batch * NN);
	w.Tm2 = sc.template get<T>(batch * NN); w.Rs = sc.template get<T>(batch * NN);
	w.X = sc.template get<T>(batch * NN); w.W = sc.template get<T>(batch * NN);
	w.dR = sc.template get<double>((size_t)batch * N); w.pvt = sc.template get<int>((size_t)batch * N);
	w.qdet = sc.template get<T>(batch);
	w.G = (T *)G; w.g_stride = NN;
	w.phi = (T *)phase;
	w.err = sc.template get<unsigned>(1);
	if (!w.Qm || !w.Tm || !w.Tm2 || !w.Rs || !w.X || !w.W || !w.dR || !w.pvt || !w.qdet || !w.err)
		return DQMC_E_NOMEM;
	CK(cudaMemsetAsync(w.err, 0, sizeof(unsigned), st));
	int rc = run_calc_eq_g<T>(w, l, st, nullptr);
	if (rc) return rc;
	unsigned e = 0;
	CK(cudaMemcpyAsync(&e, w.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	CK(cudaGetLastError());
	return e ? DQMC_E_DEVICE : 0;
}

template <typename T>
static int seam_update(int batch, int N, int n_delay, const double *del, uint64_t *rng, int *hs,
		void *G, void *phase, cudaStream_t st)
{
	if (batch < 1 || N < 1 || N > 480 || n_delay < 1 || !del || !rng || !hs || !G || !phase)
		return DQMC_E_ARG;
	int kd = n_delay;
	const int ldp = (N + 15) / 16 * 16 + 4;
	while (kd > 1 && update_smem_bytes<T>(N, kd, ldp) > 200 * 1024) kd /= 2;
	const bool cl = update_cl_wanted(is_cplx<T>::value, N, batch) && update_cl_fits<T>(N, kd);
	CK(update_attr<T>(N, kd, update_smem_bytes<T>(N, kd, ldp), cl));
	Scratch<T> sc;
	uint64_t *ck = sc.template get<uint64_t>((size_t)batch * 17);
	int *ord = sc.template get<int>((size_t)batch * 2 * N);
	double *uu = sc.template get<double>((size_t)batch * 2 * N);
	if (!ck || !ord || !uu) return DQMC_E_NOMEM;
	k_draws<<<(batch + 63) / 64, 64, 0, st>>>(N, 1, batch, 0, del, rng, ck, hs, ord, uu);
	UpdArgs<T> a;
	memset(&a, 0, sizeof(a));
	a.N = N; a.L = 1; a.n_delay = kd; a.nchain = batch; a.slice = 0; a.ldp = ldp;
	a.del = del; a.rng = rng; a.rng_ckpt = ck; a.hs = hs; a.G = (T *)G; a.phase = (T *)phase;
	a.order = ord; a.u = uu; a.next_slice = -1;
	launch_update<T>(a, update_smem_bytes<T>(N, kd, ldp), st, cl);
	CK(cudaGetLastError());
	CK(cudaStreamSynchronize(st));
	return 0;
}

template <typename T>
static int seam_mul_seq(int batch, int N, int n, int spin, const void *expK, const double *el,
		const int *hs, void *C, cudaStream_t st)
{
	if (batch < 1 || N < 1 || n < 1 || (spin != 0 && spin != 1) || !expK || !el || !hs || !C)
		return DQMC_E_ARG;
	const size_t NN = (size_t)N * N;
	Scratch<T> sc;
	double *dv = sc.template get<double>((size_t)batch * n * N);
	double *dvi = sc.template get<double>((size_t)batch * n * N);
	T *X = sc.template get<T>(batch * NN), *W = sc.template get<T>(batch * NN);
	if (!dv || !dvi || !X || !W) return DQMC_E_NOMEM;
	// the d_l of the requested spin only: k_diag_all writes both spins of
	// each chain, so run it with spin-major strides and keep spin `spin`
	double *dv2 = sc.template get<double>((size_t)batch * 2 * n * N);
	double *dvi2 = sc.template get<double>((size_t)batch * 2 * n * N);
	if (!dv2 || !dvi2) return DQMC_E_NOMEM;
	k_diag_all<<<grid_for((long long)batch * 2 * n * N), 256, 0, st>>>(N, n, batch, el, hs, dv2, dvi2);
	run_mul_seq<T>(N, n, batch, (const T *)expK, Addr{0, 0, 1}, dv2 + (size_t)spin * n * N,
	               2LL * n * N, (T *)C, Addr{(long long)NN, 0, 1}, X, W, st, nullptr);
	CK(cudaGetLastError());
	CK(cudaStreamSynchronize(st));
	return 0;
}

template <typename T>
static int seam_gemm(int batch, int M, int N, int K, const void *alpha, const void *A, int lda,
		long long sA, const void *B, int ldb, long long sB, const void *beta, void *C, int ldc,
		long long sC, cudaStream_t st)
{
	if (!A || !B || !C || !alpha || !beta || lda < M || ldb < K || ldc < M) return DQMC_E_ARG;
	GemmArgs<T> g = gargs<T>(M, N, K, batch, (const T *)A, Addr{sA, 0, 1}, lda, (const T *)B,
	                         Addr{sB, 0, 1}, ldb, (T *)C, Addr{sC, 0, 1}, ldc,
	                         *(const T *)alpha, *(const T *)beta, 0);
	const int rc = launch_gemm<T>(g, st);
	if (rc) return rc;
	CK(cudaGetLastError());
	return 0;
}

extern "C" {

int dqmc_gpu_gemm(int batch, int M, int N, int K, int cplx, const void *alpha, const void *A,
		int lda, long long stride_a, const void *B, int ldb, long long stride_b, const void *beta,
		void *C, int ldc, long long stride_c, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	return cplx ? seam_gemm<zd>(batch, M, N, K, alpha, A, lda, stride_a, B, ldb, stride_b, beta, C,
	                             ldc, stride_c, st)
	            : seam_gemm<double>(batch, M, N, K, alpha, A, lda, stride_a, B, ldb, stride_b, beta,
	                                C, ldc, stride_c, st);
}

int dqmc_gpu_calc_eq_g(int batch, int N, int F, int l, int cplx, const void *C, void *G,
		void *phase, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	return cplx ? seam_calc_eq_g<zd>(batch, N, F, l, C, G, phase, st)
	            : seam_calc_eq_g<double>(batch, N, F, l, C, G, phase, st);
}

int dqmc_gpu_update_delayed(int batch, int N, int n_delay, int cplx, const double *del,
		uint64_t *rng, int *hs, void *G, void *phase, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	return cplx ? seam_update<zd>(batch, N, n_delay, del, rng, hs, G, phase, st)
	            : seam_update<double>(batch, N, n_delay, del, rng, hs, G, phase, st);
}

int dqmc_gpu_mul_seq(int batch, int N, int n, int spin, int cplx, const void *exp_K,
		const double *exp_lambda, const int *hs, void *C, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	return cplx ? seam_mul_seq<zd>(batch, N, n, spin, exp_K, exp_lambda, hs, C, st)
	            : seam_mul_seq<double>(batch, N, n, spin, exp_K, exp_lambda, hs, C, st);
}

}  // extern "C"

// ------------------------------------------- calc_eq_g without allocation
//
// Scratch of dqmc_gpu_calc_eq_g_noalloc: one array per device, created when
// the library's module loads and held until the process exits.  Host code
// must not pass `noalloc_scratch` itself to a kernel -- on the host that name
// is a stand-in, not a device address; the device address comes from
// cudaGetSymbolAddress below, once per device.

static __device__ __align__(256) unsigned char noalloc_scratch[DQMC_NOALLOC_SCRATCH_BYTES];

static std::mutex noalloc_mu;
static void *noalloc_ptr[64];  // device address of the array, per device id

static size_t al256(size_t n) { return (n + 255) & ~(size_t)255; }

// bytes calc_eq_g needs for `batch` items of size N: six N x N work
// matrices per item, the column norms, the pivots, det(Q) and the error word
template <typename T>
static size_t noalloc_bytes(int batch, int N)
{
	const size_t NN = (size_t)N * N;
	return 6 * al256(sizeof(T) * batch * NN) + al256(sizeof(double) * batch * N) +
	       al256(sizeof(int) * batch * N) + al256(sizeof(T) * batch) + al256(sizeof(unsigned));
}

static int noalloc_base(unsigned char **base)
{
	int dev = 0;
	CK(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 64) return DQMC_E_ARG;
	std::lock_guard<std::mutex> lk(noalloc_mu);
	if (!noalloc_ptr[dev]) {
		void *p = nullptr;
		CK(cudaGetSymbolAddress(&p, noalloc_scratch));
		noalloc_ptr[dev] = p;
	}
	*base = (unsigned char *)noalloc_ptr[dev];
	return 0;
}

template <typename T>
static int noalloc_calc_eq_g(int batch, int N, int F, int l, const void *C, void *G, void *phase,
		cudaStream_t st)
{
	if (batch < 1 || N < 1 || N > max_dense_n<T>() || F < 1 || l < 0 || l >= F || !C || !G || !phase)
		return DQMC_E_ARG;
	const size_t need = noalloc_bytes<T>(batch, N);
	if (need > (size_t)DQMC_NOALLOC_SCRATCH_BYTES) {
		fprintf(stderr, "dqmc_gpu_calc_eq_g_noalloc: batch %d of N = %d needs %zu bytes of "
		        "scratch, more than the %d the library holds\n", batch, N, need,
		        (int)DQMC_NOALLOC_SCRATCH_BYTES);
		return DQMC_E_SCRATCH;
	}
	unsigned char *p = nullptr;
	const int rc0 = noalloc_base(&p);
	if (rc0) return rc0;
	const size_t NN = (size_t)N * N;
	auto take = [&](size_t bytes) { unsigned char *q = p; p += al256(bytes); return (void *)q; };
	EqWork<T> w;
	memset(&w, 0, sizeof(w));
	w.N = N; w.F = F; w.NB = batch;
	w.Cl = (const T *)C; w.cl_stride = (long long)F * NN;
	w.Qm = (T *)take(sizeof(T) * batch * NN); w.Tm = (T *)take(sizeof(T) * batch * NN);
	w.Tm2 = (T *)take(sizeof(T) * batch * NN); w.Rs = (T *)take(sizeof(T) * batch * NN);
	w.X = (T *)take(sizeof(T) * batch * NN); w.W = (T *)take(sizeof(T) * batch * NN);
	w.dR = (double *)take(sizeof(double) * batch * N);
	w.pvt = (int *)take(sizeof(int) * batch * N);
	w.qdet = (T *)take(sizeof(T) * batch);
	w.err = (unsigned *)take(sizeof(unsigned));
	w.G = (T *)G; w.g_stride = NN;
	w.phi = (T *)phase;
	// the error word keeps the previous call's value: clear it in stream order
	CK(cudaMemsetAsync(w.err, 0, sizeof(unsigned), st));
	const int rc = run_calc_eq_g<T>(w, l, st, nullptr);
	if (rc) return rc;
	unsigned e = 0;
	CK(cudaMemcpyAsync(&e, w.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	CK(cudaGetLastError());
	return e ? DQMC_E_DEVICE : 0;
}

extern "C" int dqmc_gpu_calc_eq_g_noalloc(int batch, int N, int F, int l, int cplx, const void *C,
		void *G, void *phase, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	return cplx ? noalloc_calc_eq_g<zd>(batch, N, F, l, C, G, phase, st)
	            : noalloc_calc_eq_g<double>(batch, N, F, l, C, G, phase, st);
}
