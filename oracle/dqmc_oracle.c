/*
 * CPU oracle: plain-C restatement of the reference DQMC hot path.
 * TEST INFRASTRUCTURE ONLY (see dqmc_oracle.h).  Each function cites the
 * reference file:line it follows.  Linear algebra goes through the same
 * BLAS/LAPACK routines the reference calls (scipy's OpenBLAS), so with the
 * same call order the results are bit-identical to the reference build.
 */
#include "dqmc_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_CPLX
typedef double complex num;
#define NABS(x) cabs(x)
#define NCONJ(x) conj(x)
#define NRE(x) creal(x)
#define NIM(x) cimag(x)
#define FLOP_MUL 4.0
#define X(name) scipy_z##name##_
#else
typedef double num;
#define NABS(x) fabs(x)
#define NCONJ(x) (x)
#define NRE(x) (x)
#define NIM(x) 0.0
#define FLOP_MUL 1.0
#define X(name) scipy_d##name##_
#endif

/* ---------------- BLAS/LAPACK (scipy OpenBLAS, Fortran ABI) --------------- */

void X(gemm)(const char *, const char *, const int *, const int *, const int *,
		const num *, const num *, const int *, const num *, const int *,
		const num *, num *, const int *, size_t, size_t);
void X(gemv)(const char *, const int *, const int *, const num *, const num *,
		const int *, const num *, const int *, const num *, num *, const int *, size_t);
void X(trmm)(const char *, const char *, const char *, const char *, const int *,
		const int *, const num *, const num *, const int *, num *, const int *,
		size_t, size_t, size_t, size_t);
void X(getrf)(const int *, const int *, num *, const int *, int *, int *);
void X(getrs)(const char *, const int *, const int *, const num *, const int *,
		const int *, num *, const int *, int *, size_t);
void X(getri)(const int *, num *, const int *, const int *, num *, const int *, int *);
void X(geqrf)(const int *, const int *, num *, const int *, num *, num *, const int *, int *);
void X(trtri)(const char *, const char *, const int *, num *, const int *, int *,
		size_t, size_t);
#ifdef ORACLE_CPLX
void scipy_zgeqp3_(const int *, const int *, num *, const int *, int *, num *, num *,
		const int *, double *, int *);
void scipy_zunmqr_(const char *, const char *, const int *, const int *, const int *,
		const num *, const int *, const num *, num *, const int *, num *,
		const int *, int *, size_t, size_t);
#else
void scipy_dgeqp3_(const int *, const int *, num *, const int *, int *, num *, num *,
		const int *, int *);
void scipy_dormqr_(const char *, const char *, const int *, const int *, const int *,
		const num *, const int *, const num *, num *, const int *, num *,
		const int *, int *, size_t, size_t);
#endif

static double g_flops = 0.0;
double orc_flops(void) { return g_flops; }
void orc_flops_reset(void) { g_flops = 0.0; }

static void gemm(char ta, char tb, int m, int n, int k, num alpha, const num *a,
		int lda, const num *b, int ldb, num beta, num *c, int ldc)
{
	if (m <= 0 || n <= 0) return;
	g_flops += FLOP_MUL * 2.0 * m * n * k;
	X(gemm)(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc, 1, 1);
}

static void gemv(int m, int n, num alpha, const num *a, int lda, const num *x,
		int incx, num beta, num *y, int incy)
{
	const char t = 'N';
	g_flops += FLOP_MUL * 2.0 * m * n;
	X(gemv)(&t, &m, &n, &alpha, a, &lda, x, &incx, &beta, y, &incy, 1);
}

static void trmm(char side, char uplo, int m, int n, num alpha, const num *a,
		int lda, num *b, int ldb)
{
	const char t = 'N', d = 'N';
	g_flops += FLOP_MUL * (side == 'L' ? (double)m * m * n : (double)m * n * n);
	X(trmm)(&side, &uplo, &t, &d, &m, &n, &alpha, a, &lda, b, &ldb, 1, 1, 1, 1);
}

static void getrf(int n, num *a, int lda, int *ipiv)
{
	int info;
	g_flops += FLOP_MUL * 2.0 / 3.0 * n * n * n;
	X(getrf)(&n, &n, a, &lda, ipiv, &info);
}

static void getrs(int n, int nrhs, const num *a, int lda, const int *ipiv, num *b, int ldb)
{
	const char t = 'N';
	int info;
	g_flops += FLOP_MUL * 2.0 * n * n * nrhs;
	X(getrs)(&t, &n, &nrhs, a, &lda, ipiv, b, &ldb, &info, 1);
}

static void getri(int n, num *a, int lda, const int *ipiv)
{
	int info, lw = -1;
	num q;
	X(getri)(&n, a, &lda, ipiv, &q, &lw, &info);
	lw = (int)NRE(q) > n * n ? (int)NRE(q) : n * n;
	num *w = malloc(sizeof(num) * lw);
	g_flops += FLOP_MUL * 4.0 / 3.0 * n * n * n;
	X(getri)(&n, a, &lda, ipiv, w, &lw, &info);
	free(w);
}

static void geqrf(int m, int n, num *a, int lda, num *tau)
{
	int info, lw = -1;
	num q;
	X(geqrf)(&m, &n, a, &lda, tau, &q, &lw, &info);
	lw = (int)NRE(q) > 1 ? (int)NRE(q) : 1;
	num *w = malloc(sizeof(num) * lw);
	g_flops += FLOP_MUL * 2.0 * n * n * (m - n / 3.0);
	X(geqrf)(&m, &n, a, &lda, tau, w, &lw, &info);
	free(w);
}

static void geqp3(int n, num *a, int lda, int *jpvt, num *tau)
{
	int info, lw = -1;
	num q;
#ifdef ORACLE_CPLX
	double *rw = malloc(sizeof(double) * 2 * n);
	scipy_zgeqp3_(&n, &n, a, &lda, jpvt, tau, &q, &lw, rw, &info);
#else
	scipy_dgeqp3_(&n, &n, a, &lda, jpvt, tau, &q, &lw, &info);
#endif
	lw = (int)NRE(q) > 1 ? (int)NRE(q) : 1;
	num *w = malloc(sizeof(num) * lw);
	g_flops += FLOP_MUL * 4.0 / 3.0 * n * n * n;
#ifdef ORACLE_CPLX
	scipy_zgeqp3_(&n, &n, a, &lda, jpvt, tau, w, &lw, rw, &info);
	free(rw);
#else
	scipy_dgeqp3_(&n, &n, a, &lda, jpvt, tau, w, &lw, &info);
#endif
	free(w);
}

/* C <- C op(Q) (side 'R') or op(Q) C (side 'L'); trans 'N' or 'C' */
static void unmqr(char side, char trans, int m, int n, int k, const num *a,
		int lda, const num *tau, num *c, int ldc)
{
	int info, lw = -1;
	num q;
#ifdef ORACLE_CPLX
	const char tr = trans;
	scipy_zunmqr_(&side, &tr, &m, &n, &k, a, &lda, tau, c, &ldc, &q, &lw, &info, 1, 1);
#else
	const char tr = (trans == 'C') ? 'T' : trans;
	scipy_dormqr_(&side, &tr, &m, &n, &k, a, &lda, tau, c, &ldc, &q, &lw, &info, 1, 1);
#endif
	lw = (int)NRE(q) > 1 ? (int)NRE(q) : 1;
	num *w = malloc(sizeof(num) * lw);
	g_flops += FLOP_MUL * (side == 'R' ? 4.0 * m * n * k - 2.0 * m * k * k
	                                   : 4.0 * m * n * k - 2.0 * n * k * k);
#ifdef ORACLE_CPLX
	scipy_zunmqr_(&side, &tr, &m, &n, &k, a, &lda, tau, c, &ldc, w, &lw, &info, 1, 1);
#else
	scipy_dormqr_(&side, &tr, &m, &n, &k, a, &lda, tau, c, &ldc, w, &lw, &info, 1, 1);
#endif
	free(w);
}

static void trtri(int n, num *a, int lda)
{
	const char u = 'U', d = 'N';
	int info;
	g_flops += FLOP_MUL * (double)n * n * n / 3.0;
	X(trtri)(&u, &d, &n, a, &lda, &info, 1, 1);
}

static void *zalloc(size_t bytes)
{
	void *p = calloc(1, bytes ? bytes : 1);
	return p;
}

/* ------------------------------- RNG ------------------------------------- */

/* xorshift1024* step, rand.h:6-14 (state words rng[0..15], index rng[16]) */
uint64_t orc_rand_uint(uint64_t *rng)
{
	const uint64_t a = rng[rng[16]];
	const int p = (int)((rng[16] + 1) & 15);
	rng[16] = (uint64_t)p;
	uint64_t b = rng[p];
	b ^= b << 31;
	rng[p] = b ^ a ^ (b >> 11) ^ (a >> 30);
	return rng[p] * UINT64_C(1181783497276652981);
}

/* [0,1) double from the top 52 bits, rand.h:16-22 */
double orc_rand_doub(uint64_t *rng)
{
	union { uint64_t i; double d; } u;
	u.i = (UINT64_C(0x3FF) << 52) | (orc_rand_uint(rng) >> 12);
	return u.d - 1.0;
}

/* inside-out Fisher-Yates, rand.h:25-31 */
void orc_shuffle(uint64_t *rng, int n, int *a)
{
	for (int i = 0; i < n; i++) {
		const int j = (int)((orc_rand_uint(rng) >> 3) % (uint64_t)(i + 1));
		if (i != j) a[i] = a[j];
		a[j] = i;
	}
}

/* splitmix64 seeding, util/gen_util_shared.py:12-21 */
void orc_seed_splitmix64(uint64_t x, uint64_t *rng)
{
	for (int i = 0; i < 16; i++) {
		x += UINT64_C(0x9E3779B97F4A7C15);
		uint64_t z = (x ^ (x >> 30)) * UINT64_C(0xBF58476D1CE4E5B9);
		z = (z ^ (z >> 27)) * UINT64_C(0x94D049BB133111EB);
		rng[i] = z ^ (z >> 31);
	}
	rng[16] = 0;
}

/* 2^512 jump, util/gen_util_shared.py:34-66 */
void orc_rand_jump(uint64_t *rng)
{
	static const uint64_t jmp[16] = {
		0x84242F96ECA9C41DULL, 0xA3C65B8776F96855ULL, 0x5B34A39F070B5837ULL,
		0x4489AFFCE4F31A1EULL, 0x2FFEEB0A48316F40ULL, 0xDC2D9891FE68C022ULL,
		0x3659132BB12FEA70ULL, 0xAAC17D8EFA43CAB8ULL, 0xC4CB815590989B13ULL,
		0x5EE975283D71C93BULL, 0x691548C86C1BD540ULL, 0x7910C41D10A1E6A5ULL,
		0x0B5FC64563B3E2A8ULL, 0x047F7684E9FC949DULL, 0xB99181F2D8F685CAULL,
		0x284600E3F30E38C3ULL};
	uint64_t t[16] = {0};
	for (int i = 0; i < 16; i++)
		for (int b = 0; b < 64; b++) {
			if (jmp[i] & (UINT64_C(1) << b))
				for (int j = 0; j < 16; j++) t[j] ^= rng[(j + rng[16]) & 15];
			orc_rand_uint(rng);
		}
	for (int j = 0; j < 16; j++) rng[(j + rng[16]) & 15] = t[j];
}

/* --------------------------- B matrices ---------------------------------- */

/* dqmc.c:29-43: column j of B_l is column j of exp_K times
 * exp_lambda[j + N*h], h = hs (up) or !hs (down) */
void orc_build_B(int N, int L, const void *exp_K_, const double *exp_lambda,
		const int *hs, int spin, void *B_)
{
	const num *exp_K = exp_K_;
	num *B = B_;
	for (int l = 0; l < L; l++)
		for (int j = 0; j < N; j++) {
			const int h = spin ? !hs[j + N * l] : hs[j + N * l];
			const double el = exp_lambda[j + N * h];
			for (int i = 0; i < N; i++)
				B[i + N * j + (size_t)N * N * l] = exp_K[i + N * j] * el;
		}
}

/* dqmc.c:45-59: row i of B_l^-1 is row i of inv_exp_K times
 * exp_lambda[i + N*!h] */
void orc_build_iB(int N, int L, const void *inv_exp_K_, const double *exp_lambda,
		const int *hs, int spin, void *iB_)
{
	const num *inv_exp_K = inv_exp_K_;
	num *iB = iB_;
	for (int l = 0; l < L; l++)
		for (int i = 0; i < N; i++) {
			const int h = spin ? !hs[i + N * l] : hs[i + N * l];
			const double el = exp_lambda[i + N * !h];
			for (int j = 0; j < N; j++)
				iB[i + N * j + (size_t)N * N * l] = el * inv_exp_K[i + N * j];
		}
}

/* ------------------------------ greens.c --------------------------------- */

/* Ordered product B_{maxp1-1} ... B_{min} (indices mod L), greens.c:8-41.
 * Products are formed pairwise in the same association as the reference. */
static void mul_seq(int N, int L, int min, int maxp1, num alpha, const num *B,
		num *A, int ldA, num *work)
{
	const size_t NN = (size_t)N * N;
	const int count = (min == maxp1) ? L : (L + maxp1 - min) % L;
	if (count == 1) {
		for (int j = 0; j < N; j++)
			for (int i = 0; i < N; i++)
				A[i + (size_t)ldA * j] = alpha * B[i + N * j + NN * min];
		return;
	}
	int l = min;
	if (count % 2 == 0) {
		gemm('N', 'N', N, N, N, alpha, B + NN * ((l + 1) % L), N, B + NN * l, N, 0.0, A, ldA);
		l = (l + 2) % L;
	} else {
		gemm('N', 'N', N, N, N, alpha, B + NN * ((l + 1) % L), N, B + NN * l, N, 0.0, work, N);
		gemm('N', 'N', N, N, N, 1.0, B + NN * ((l + 2) % L), N, work, N, 0.0, A, ldA);
		l = (l + 3) % L;
	}
	while (l != maxp1) {
		gemm('N', 'N', N, N, N, 1.0, B + NN * l, N, A, ldA, 0.0, work, N);
		gemm('N', 'N', N, N, N, 1.0, B + NN * ((l + 1) % L), N, work, N, 0.0, A, ldA);
		l = (l + 2) % L;
	}
}

void orc_mul_seq(int N, int L, int min, int maxp1, const void *alpha,
		const void *B, void *A, int ldA)
{
	num *work = zalloc(sizeof(num) * N * N);
	mul_seq(N, L, min, maxp1, *(const num *)alpha, B, A, ldA, work);
	free(work);
}

/* Stabilised equal-time Green's function from the L cluster matrices B
 * (greens.c:69-208): G = (I + B_{l-1} ... B_l)^-1 via a UDT chain with a
 * column-pivoted QR first (geqp3) and norm pre-pivoted QRs after, grouped
 * n_mul matrices at a time; the final (D_b^-1 Q^H + D_s T) solve follows
 * eq. 2.12 of 10.1016/j.laa.2010.06.023.  Returns 1/phase(det G). */
static num calc_eq_g(int l, int N, int L, int n_mul, const num *B, num *g)
{
	num *Q = zalloc(sizeof(num) * N * N), *T = zalloc(sizeof(num) * N * N);
	num *tau = zalloc(sizeof(num) * N), *d = zalloc(sizeof(num) * 2 * N);
	num *v = zalloc(sizeof(num) * N), *work = zalloc(sizeof(num) * N * N);
	int *pvt = zalloc(sizeof(int) * N);

	int m = (l + 1 + (L - 1) % n_mul) % L;
	mul_seq(N, L, l, m, 1.0, B, Q, N, work);
	for (int i = 0; i < N; i++) pvt[i] = 0;
	geqp3(N, Q, N, pvt, tau);
	for (int i = 0; i < N; i++) {
		d[i] = Q[i + i * N];
		if (d[i] == 0.0) d[i] = 1.0;
		v[i] = 1.0 / d[i];
	}
	for (int i = 0; i < N * N; i++) T[i] = 0.0;
	for (int j = 0; j < N; j++)
		for (int i = 0; i <= j; i++)
			T[i + (pvt[j] - 1) * N] = v[i] * Q[i + j * N];

	while (m != l) {
		const int next = (m + n_mul) % L;
		mul_seq(N, L, m, next, 1.0, B, g, N, work);
		m = next;
		unmqr('R', 'N', N, N, N, Q, N, tau, g, N);
		for (int j = 0; j < N; j++)
			for (int i = 0; i < N; i++) g[i + j * N] *= d[j];
		/* column norms and a stable descending insertion sort */
		for (int j = 0; j < N; j++) {
			double s = 0.0;
			for (int i = 0; i < N; i++)
				s += NRE(g[i + j * N] * NCONJ(g[i + j * N]));
			d[j] = s;
		}
		pvt[0] = 0;
		for (int i = 1; i < N; i++) {
			int j = i;
			while (j > 0 && NRE(d[pvt[j - 1]]) < NRE(d[i])) {
				pvt[j] = pvt[j - 1];
				j--;
			}
			pvt[j] = i;
		}
		for (int j = 0; j < N; j++)
			memcpy(Q + (size_t)j * N, g + (size_t)pvt[j] * N, sizeof(num) * N);
		geqrf(N, N, Q, N, tau);
		for (int i = 0; i < N; i++) {
			d[i] = Q[i + i * N];
			if (d[i] == 0.0) d[i] = 1.0;
			v[i] = 1.0 / d[i];
		}
		for (int j = 0; j < N; j++)
			for (int i = 0; i <= j; i++) Q[i + j * N] *= v[i];
		for (int j = 0; j < N; j++) {
			for (int i = 0; i < N; i++) v[i] = T[pvt[i] + j * N];
			memcpy(T + (size_t)j * N, v, sizeof(num) * N);
		}
		trmm('L', 'U', N, N, 1.0, Q, N, T, N);
	}

	for (int i = 0; i < N * N; i++) g[i] = 0.0;
	for (int i = 0; i < N; i++) {
		if (NABS(d[i]) > 1.0) {
			v[i] = 1.0 / d[i];
			d[i] = 1.0;
		} else {
			v[i] = 1.0;
		}
		g[i + i * N] = v[i];
	}
	unmqr('R', 'C', N, N, N, Q, N, tau, g, N);
	for (int j = 0; j < N; j++)
		for (int i = 0; i < N; i++) T[i + j * N] *= d[i];
	for (int i = 0; i < N * N; i++) T[i] += g[i];
	getrf(N, T, N, pvt);
	getrs(N, N, T, N, pvt, g, N);

	num phase = 1.0;
	for (int i = 0; i < N; i++) {
		const num c = v[i] / T[i + N * i];
		phase *= c / NABS(c);
		double vv = 1.0;
		for (int j = i + 1; j < N; j++)
			vv += NRE(Q[j + i * N]) * NRE(Q[j + i * N]) + NIM(Q[j + i * N]) * NIM(Q[j + i * N]);
		const num ref = 1.0 - tau[i] * vv;
		phase *= NABS(ref) / ref;
		if (pvt[i] != i + 1) phase *= -1.0;
	}
	free(Q); free(T); free(tau); free(d); free(v); free(work); free(pvt);
	return 1.0 / phase;
}

void orc_calc_eq_g(int l, int N, int L, int n_mul, const void *B, void *g, void *phase_out)
{
	const num ph = calc_eq_g(l, N, L, n_mul, B, g);
	if (phase_out) *(num *)phase_out = ph;
}

/* Block-cyclic O of the cluster products, greens.c:247-264 */
static void calc_o(int N, int L, int n_mul, const num *B, num *G, num *work)
{
	const int E = 1 + (L - 1) / n_mul, NE = N * E;
	for (size_t i = 0; i < (size_t)NE * NE; i++) G[i] = 0.0;
	for (int e = 0; e < E - 1; e++)
		mul_seq(N, L, e * n_mul, (e + 1) * n_mul, -1.0, B,
		        G + N * (e + 1) + (size_t)NE * N * e, NE, work);
	mul_seq(N, L, (E - 1) * n_mul, 0, 1.0, B, G + (size_t)NE * N * (E - 1), NE, work);
	for (int i = 0; i < NE; i++) G[i + (size_t)NE * i] += 1.0;
}

/* Block structured orthogonal factorisation and inversion, greens.c:266-337 */
static void bsofi(int N, int L, num *G, num *tau, num *Q)
{
	if (L == 1) {
		int *ipiv = zalloc(sizeof(int) * N);
		getrf(N, G, N, ipiv);
		getri(N, G, N, ipiv);
		free(ipiv);
		return;
	}
	const int NL = N * L, N2 = 2 * N;
#define BLK(i, j) (G + (size_t)N * (i) + (size_t)NL * N * (j))
	for (int l = 0; l < L - 2; l++) {
		geqrf(N2, N, BLK(l, l), NL, tau + N * l);
		unmqr('L', 'C', N2, N, N, BLK(l, l), NL, tau + N * l, BLK(l, l + 1), NL);
		unmqr('L', 'C', N2, N, N, BLK(l, l), NL, tau + N * l, BLK(l, L - 1), NL);
	}
	geqrf(N2, N2, BLK(L - 2, L - 2), NL, tau + N * (L - 2));
	if (L <= 2) {
		trtri(NL, G, NL);
	} else {
		trtri(3 * N, BLK(L - 3, L - 3), NL);
		if (L > 3) {
			trmm('R', 'U', N * (L - 3), N, 1.0, BLK(L - 1, L - 1), NL, BLK(0, L - 1), NL);
			for (int l = L - 4; l >= 0; l--) {
				trtri(N, BLK(l, l), NL);
				trmm('L', 'U', N, N, -1.0, BLK(l, l), NL, BLK(l, L - 1), NL);
				trmm('L', 'U', N, N, -1.0, BLK(l, l), NL, BLK(l, l + 1), NL);
				gemm('N', 'N', N, N * (L - l - 2), N, 1.0, BLK(l, l + 1), NL,
				     BLK(l + 1, l + 2), NL, 1.0, BLK(l, l + 2), NL);
				trmm('R', 'U', N, N, 1.0, BLK(l + 1, l + 1), NL, BLK(l, l + 1), NL);
			}
		}
	}
	for (int i = 0; i < 4 * N * N; i++) Q[i] = 0.0;
	for (int j = 0; j < N2; j++)
		for (int i = j + 1; i < N2; i++) {
			Q[i + N2 * j] = BLK(L - 2, L - 2)[i + (size_t)NL * j];
			BLK(L - 2, L - 2)[i + (size_t)NL * j] = 0.0;
		}
	unmqr('R', 'C', NL, N2, N2, Q, N2, tau + N * (L - 2), BLK(0, L - 2), NL);
	for (int l = L - 3; l >= 0; l--) {
		for (int j = 0; j < N; j++)
			for (int i = j + 1; i < N2; i++) {
				Q[i + N2 * j] = BLK(l, l)[i + (size_t)NL * j];
				BLK(l, l)[i + (size_t)NL * j] = 0.0;
			}
		unmqr('R', 'C', NL, N2, N, Q, N2, tau + N * l, BLK(0, l), NL);
	}
#undef BLK
}

/* Spread the reduced inverse to every slice, greens.c:339-469 */
static void expand_g(int N, int L, int E, int n_matmul, const num *B, const num *iB,
		const num *Gred, num *G0t, num *Gtt, num *Gt0)
{
	const size_t NN = (size_t)N * N, NE = (size_t)N * E;
	const int n_left = (n_matmul - 1) / 2, n_right = n_matmul / 2;
	const int n_up = n_left, n_down = n_right;
	const int rstop_last = ((E - 1) * n_matmul + L) / 2;
	const int lstop_first = (rstop_last + 1) % L;
	const int dstop_last = rstop_last, ustop_first = lstop_first;

	for (int f = 0; f < E; f++) {
		const int t = f * n_matmul;
		for (int j = 0; j < N; j++)
			for (int i = 0; i < N; i++)
				G0t[i + N * j + NN * t] = Gred[i + NE * (j + (size_t)N * f)];
	}
	for (int f = 0; f < E; f++) {
		const int l = f * n_matmul;
		const int lstop = (f == 0) ? lstop_first : l - n_left;
		const int rstop = (f == E - 1) ? rstop_last : l + n_right;
		for (int m = l; m != lstop;) {
			const int next = (m - 1 + L) % L;
			const num alpha = (m == 0) ? -1.0 : 1.0;
			gemm('N', 'N', N, N, N, alpha, G0t + NN * m, N, B + NN * next, N, 0.0,
			     G0t + NN * next, N);
			m = next;
		}
		for (int m = l; m != rstop;) {
			const int next = (m + 1) % L;
			const num alpha = (next == 0) ? -1.0 : 1.0;
			const num beta = (m == 0) ? -alpha : 0.0;
			if (m == 0) memcpy(G0t + NN * next, iB + NN * m, sizeof(num) * NN);
			gemm('N', 'N', N, N, N, alpha, G0t + NN * m, N, iB + NN * m, N, beta,
			     G0t + NN * next, N);
			m = next;
		}
	}

	for (int e = 0; e < E; e++) {
		const int k = e * n_matmul;
		for (int j = 0; j < N; j++)
			for (int i = 0; i < N; i++)
				Gtt[i + N * j + NN * k] = Gred[(i + (size_t)N * e) + NE * (j + (size_t)N * e)];
	}
	for (int e = 0; e < E; e++) {
		const int k = e * n_matmul;
		const int ustop = (e == 0) ? ustop_first : k - n_up;
		const int dstop = (e == E - 1) ? dstop_last : k + n_down;
		for (int m = k; m != ustop;) {
			const int next = (m - 1 + L) % L;
			gemm('N', 'N', N, N, N, 1.0, Gtt + NN * m, N, B + NN * next, N, 0.0, Gt0, N);
			gemm('N', 'N', N, N, N, 1.0, iB + NN * next, N, Gt0, N, 0.0, Gtt + NN * next, N);
			m = next;
		}
		for (int m = k; m != dstop;) {
			const int next = (m + 1) % L;
			gemm('N', 'N', N, N, N, 1.0, Gtt + NN * m, N, iB + NN * m, N, 0.0, Gt0, N);
			gemm('N', 'N', N, N, N, 1.0, B + NN * m, N, Gt0, N, 0.0, Gtt + NN * next, N);
			m = next;
		}
	}

	for (int e = 0; e < E; e++) {
		const int t = e * n_matmul;
		for (int j = 0; j < N; j++)
			for (int i = 0; i < N; i++)
				Gt0[i + N * j + NN * t] = Gred[(i + (size_t)N * e) + NE * j];
	}
	for (int e = 0; e < E; e++) {
		const int k = e * n_matmul;
		const int ustop = (e == 0) ? ustop_first : k - n_up;
		const int dstop = (e == E - 1) ? dstop_last : k + n_down;
		for (int m = k; m != ustop;) {
			const int next = (m - 1 + L) % L;
			const num alpha = (m == 0) ? -1.0 : 1.0;
			const num beta = (m == 0) ? -alpha : 0.0;
			if (m == 0) memcpy(Gt0 + NN * next, iB + NN * next, sizeof(num) * NN);
			gemm('N', 'N', N, N, N, alpha, iB + NN * next, N, Gt0 + NN * m, N, beta,
			     Gt0 + NN * next, N);
			m = next;
		}
		for (int m = k; m != dstop;) {
			const int next = (m + 1) % L;
			const num alpha = (next == 0) ? -1.0 : 1.0;
			gemm('N', 'N', N, N, N, alpha, B + NN * m, N, Gt0 + NN * m, N, 0.0,
			     Gt0 + NN * next, N);
			if (next == 0)
				for (int i = 0; i < N; i++) Gt0[i + N * i + NN * next] += 1.0;
			m = next;
		}
	}
}

void orc_calc_ue_g(int N, int L, int F, int n_mul, const void *B, const void *iB,
		const void *C, void *G0t, void *Gtt, void *Gt0)
{
	const int E = 1 + (F - 1) / n_mul;
	num *Gred = zalloc(sizeof(num) * (size_t)N * E * N * E);
	num *tau = zalloc(sizeof(num) * (size_t)N * E);
	num *Q = zalloc(sizeof(num) * 4 * (size_t)N * N);
	num *work = zalloc(sizeof(num) * (size_t)N * N);
	calc_o(N, F, n_mul, C, Gred, work);
	bsofi(N, E, Gred, tau, Q);
	expand_g(N, L, E, (L / F) * n_mul, B, iB, Gred, G0t, Gtt, Gt0);
	free(Gred); free(tau); free(Q); free(work);
}

/* ------------------------------ updates.c -------------------------------- */

/* Delayed rank-k Sherman-Morrison Metropolis sweep over one slice's sites,
 * updates.c:7-84.  Columns a_k (from G e_i) and b_k (from G^T e_i) are
 * collected in panels and flushed into G every n_delay accepts. */
static void update_delayed(int N, int n_delay, const double *del, const int *order,
		uint64_t *rng, int *hs, num *gu, num *gd, num *phase,
		num *au, num *bu, num *du, num *ad, num *bd, num *dd)
{
	int k = 0;
	for (int j = 0; j < N; j++) du[j] = gu[j + N * j];
	for (int j = 0; j < N; j++) dd[j] = gd[j + N * j];
	for (int ii = 0; ii < N; ii++) {
		const int i = order[ii];
		const double delu = del[i + N * hs[i]];
		const double deld = del[i + N * !hs[i]];
		if (delu == 0.0 && deld == 0.0) continue;
		const num ru = 1.0 + (1.0 - du[i]) * delu;
		const num rd = 1.0 + (1.0 - dd[i]) * deld;
		const num prob = ru * rd;
		const double absprob = NABS(prob);
		if (orc_rand_doub(rng) < absprob) {
			num *pa[2] = {au, ad}, *pb[2] = {bu, bd}, *pg[2] = {gu, gd}, *pd[2] = {du, dd};
			const num scale[2] = {delu / ru, deld / rd};
			for (int s = 0; s < 2; s++) {
				num *a = pa[s], *b = pb[s], *g = pg[s], *dg = pd[s];
				for (int j = 0; j < N; j++) a[j + N * k] = g[j + N * i];
				for (int j = 0; j < N; j++) b[j + N * k] = g[i + N * j];
				gemv(N, k, 1.0, a, N, b + i, N, 1.0, a + N * k, 1);
				gemv(N, k, 1.0, b, N, a + i, N, 1.0, b + N * k, 1);
				a[i + N * k] -= 1.0;
				for (int j = 0; j < N; j++) a[j + N * k] *= scale[s];
				for (int j = 0; j < N; j++) dg[j] += a[j + N * k] * b[j + N * k];
			}
			k++;
			hs[i] = !hs[i];
			*phase *= prob / absprob;
		}
		if (k == n_delay) {
			k = 0;
			gemm('N', 'T', N, N, n_delay, 1.0, au, N, bu, N, 1.0, gu, N);
			for (int j = 0; j < N; j++) du[j] = gu[j + N * j];
			gemm('N', 'T', N, N, n_delay, 1.0, ad, N, bd, N, 1.0, gd, N);
			for (int j = 0; j < N; j++) dd[j] = gd[j + N * j];
		}
	}
	gemm('N', 'T', N, N, k, 1.0, au, N, bu, N, 1.0, gu, N);
	gemm('N', 'T', N, N, k, 1.0, ad, N, bd, N, 1.0, gd, N);
}

void orc_update_delayed(int N, int n_delay, const double *del, const int *site_order,
		uint64_t *rng, int *hs, void *gu, void *gd, void *phase)
{
	num *au = zalloc(sizeof(num) * N * N), *bu = zalloc(sizeof(num) * N * N);
	num *ad = zalloc(sizeof(num) * N * N), *bd = zalloc(sizeof(num) * N * N);
	num *du = zalloc(sizeof(num) * N), *dd = zalloc(sizeof(num) * N);
	update_delayed(N, n_delay, del, site_order, rng, hs, gu, gd, phase,
	               au, bu, du, ad, bd, dd);
	free(au); free(bu); free(ad); free(bd); free(du); free(dd);
}

/* -------------------------------- meas.c --------------------------------- */

/* Equal-time always-on measurements, meas.c:66-120 */
void orc_measure_eqlt(struct orc_sim *s, const void *phase_, const void *gu_, const void *gd_)
{
	const num phase = *(const num *)phase_;
	const num *gu = gu_, *gd = gd_;
	const num *pu = s->peierlsu, *pd = s->peierlsd;
	num *sign = s->eq_sign, *density = s->density, *density_u = s->density_u;
	num *density_d = s->density_d, *double_occ = s->double_occ;
	num *g00 = s->g00, *g00_u = s->g00_u, *g00_d = s->g00_d;
	num *nn = s->eq_nn, *xx = s->eq_xx, *zz = s->eq_zz, *pair_sw = s->eq_pair_sw;
	const int N = s->N;
	(*s->eq_n_sample)++;
	*sign += phase;
	for (int i = 0; i < N; i++) {
		const int r = s->map_i[i];
		const num pre = phase / s->degen_i;
		const num guii = gu[i + i * N], gdii = gd[i + i * N];
		density[r] += pre * (2. - guii - gdii);
		density_u[r] += pre * (1. - guii);
		density_d[r] += pre * (1. - gdii);
		double_occ[r] += pre * (1. - guii) * (1. - gdii);
	}
	for (int j = 0; j < N; j++)
		for (int i = 0; i < N; i++) {
			const int delta = (i == j);
			const int r = s->map_ij[i + j * N];
			const num pre = phase / s->degen_ij;
			const num guii = gu[i + i * N], gdii = gd[i + i * N];
			const num guij = gu[i + j * N], gdij = gd[i + j * N];
			const num guji = gu[j + i * N], gdji = gd[j + i * N];
			const num gujj = gu[j + j * N], gdjj = gd[j + j * N];
#ifdef ORACLE_CPLX
			g00[r] += 0.5 * pre * (guij * pu[j + i * N] + gdij * pd[j + i * N]);
			g00_u[r] += pre * (guij * pu[j + i * N]);
			g00_d[r] += pre * (gdij * pd[j + i * N]);
#else
			(void)pu; (void)pd;
			g00[r] += 0.5 * pre * (guij + gdij);
			g00_u[r] += pre * guij;
			g00_d[r] += pre * gdij;
#endif
			const num x = delta * (guii + gdii) - (guji * guij + gdji * gdij);
			nn[r] += pre * ((2. - guii - gdii) * (2. - gujj - gdjj) + x);
			xx[r] += 0.25 * pre * (delta * (guii + gdii) - (guji * gdij + gdji * guij));
			zz[r] += 0.25 * pre * ((gdii - guii) * (gdjj - gujj) + x);
			pair_sw[r] += pre * guij * gdij;
		}
}

/* Unequal-time always-on measurements (meas.c:728-801) and the bond-bond
 * correlators of meas_bond_corr (meas.c:860-964) */
void orc_measure_uneqlt(struct orc_sim *s, const void *phase_,
		const void *Gu0t_, const void *Gutt_, const void *Gut0_,
		const void *Gd0t_, const void *Gdtt_, const void *Gdt0_)
{
	const num phase = *(const num *)phase_;
	const num *Gu0t = Gu0t_, *Gutt = Gutt_, *Gut0 = Gut0_;
	const num *Gd0t = Gd0t_, *Gdtt = Gdtt_, *Gdt0 = Gdt0_;
	const num *peu = s->peierlsu, *ped = s->peierlsd;
	const int N = s->N, L = s->L, num_ij = s->num_ij, num_b = s->num_b, num_bb = s->num_bb;
	const size_t NN = (size_t)N * N;
	num *gt0 = s->gt0, *gt0_u = s->gt0_u, *gt0_d = s->gt0_d;
	num *nn = s->ue_nn, *xx = s->ue_xx, *zz = s->ue_zz, *pair_sw = s->ue_pair_sw;
	(*s->ue_n_sample)++;
	*(num *)s->ue_sign += phase;
	const num *Gu00 = Gutt, *Gd00 = Gdtt;
	for (int t = 0; t < L; t++) {
		const int delta_t = (t == 0);
		const num *u0t = Gu0t + NN * t, *utt = Gutt + NN * t, *ut0 = Gut0 + NN * t;
		const num *d0t = Gd0t + NN * t, *dtt = Gdtt + NN * t, *dt0 = Gdt0 + NN * t;
		for (int j = 0; j < N; j++)
			for (int i = 0; i < N; i++) {
				const int r = s->map_ij[i + j * N] + num_ij * t;
				const int delta_tij = delta_t * (i == j);
				const num pre = phase / s->degen_ij;
				const num guii = utt[i + N * i], guij = ut0[i + N * j];
				const num guji = u0t[j + N * i], gujj = Gu00[j + N * j];
				const num gdii = dtt[i + N * i], gdij = dt0[i + N * j];
				const num gdji = d0t[j + N * i], gdjj = Gd00[j + N * j];
#ifdef ORACLE_CPLX
				gt0[r] += 0.5 * pre * (guij * peu[j + i * N] + gdij * ped[j + i * N]);
				gt0_u[r] += pre * (guij * peu[j + i * N]);
				gt0_d[r] += pre * (gdij * ped[j + i * N]);
#else
				(void)peu; (void)ped;
				gt0[r] += 0.5 * pre * (guij + gdij);
				gt0_u[r] += pre * guij;
				gt0_d[r] += pre * gdij;
#endif
				const num x = delta_tij * (guii + gdii) - (guji * guij + gdji * gdij);
				nn[r] += pre * ((2. - guii - gdii) * (2. - gujj - gdjj) + x);
				xx[r] += 0.25 * pre * (delta_tij * (guii + gdii) - (guji * gdij + gdji * guij));
				zz[r] += 0.25 * pre * ((gdii - guii) * (gdjj - gujj) + x);
				pair_sw[r] += pre * guij * gdij;
			}
	}
	if (!s->meas_bond_corr) return;
	num *pair_bb = s->pair_bb, *jj = s->jj, *jsjs = s->jsjs, *kk = s->kk, *ksks = s->ksks;
	for (int t = 0; t < L; t++) {
		const int delta_t = (t == 0);
		const num *u0t = Gu0t + NN * t, *utt = Gutt + NN * t, *ut0 = Gut0 + NN * t;
		const num *d0t = Gd0t + NN * t, *dtt = Gdtt + NN * t, *dt0 = Gdt0 + NN * t;
		for (int c = 0; c < num_b; c++) {
			const int j0 = s->bonds[c], j1 = s->bonds[c + num_b];
#ifdef ORACLE_CPLX
			const num puj0j1 = peu[j0 + N * j1], puj1j0 = peu[j1 + N * j0];
			const num pdj0j1 = ped[j0 + N * j1], pdj1j0 = ped[j1 + N * j0];
#else
			const num puj0j1 = 1, puj1j0 = 1, pdj0j1 = 1, pdj1j0 = 1;
#endif
			for (int b = 0; b < num_b; b++) {
				const int i0 = s->bonds[b], i1 = s->bonds[b + num_b];
#ifdef ORACLE_CPLX
				const num pui0i1 = peu[i0 + N * i1], pui1i0 = peu[i1 + N * i0];
				const num pdi0i1 = ped[i0 + N * i1], pdi1i0 = ped[i1 + N * i0];
#else
				const num pui0i1 = 1, pui1i0 = 1, pdi0i1 = 1, pdi1i0 = 1;
#endif
				const int bb = s->map_bb[b + c * num_b] + num_bb * t;
				const num pre = phase / s->degen_bb;
				const num gui1i0 = utt[i1 + i0 * N], gui0i1 = utt[i0 + i1 * N];
				const num gui0j0 = ut0[i0 + j0 * N], gui1j0 = ut0[i1 + j0 * N];
				const num gui0j1 = ut0[i0 + j1 * N], gui1j1 = ut0[i1 + j1 * N];
				const num guj0i0 = u0t[j0 + i0 * N], guj1i0 = u0t[j1 + i0 * N];
				const num guj0i1 = u0t[j0 + i1 * N], guj1i1 = u0t[j1 + i1 * N];
				const num guj1j0 = Gu00[j1 + j0 * N], guj0j1 = Gu00[j0 + j1 * N];
				const num gdi1i0 = dtt[i1 + i0 * N], gdi0i1 = dtt[i0 + i1 * N];
				const num gdi0j0 = dt0[i0 + j0 * N], gdi1j0 = dt0[i1 + j0 * N];
				const num gdi0j1 = dt0[i0 + j1 * N], gdi1j1 = dt0[i1 + j1 * N];
				const num gdj0i0 = d0t[j0 + i0 * N], gdj1i0 = d0t[j1 + i0 * N];
				const num gdj0i1 = d0t[j0 + i1 * N], gdj1i1 = d0t[j1 + i1 * N];
				const num gdj1j0 = Gd00[j1 + j0 * N], gdj0j1 = Gd00[j0 + j1 * N];
				const int d00 = delta_t * (i0 == j0), d10 = delta_t * (i1 == j0);
				const int d01 = delta_t * (i0 == j1), d11 = delta_t * (i1 == j1);
				const num arr[8] = {
					(d01 - gdj1i0) * gdi1j0, (d00 - gdj0i0) * gdi1j1,
					(d11 - gdj1i1) * gdi0j0, (d10 - gdj0i1) * gdi0j1,
					(d01 - guj1i0) * gui1j0, (d00 - guj0i0) * gui1j1,
					(d11 - guj1i1) * gui0j0, (d10 - guj0i1) * gui0j1,
				};
				const num ap[8] = {
					pdi0i1 * pdj0j1 * arr[0], pdi0i1 * pdj1j0 * arr[1],
					pdi1i0 * pdj0j1 * arr[2], pdi1i0 * pdj1j0 * arr[3],
					pui0i1 * puj0j1 * arr[4], pui0i1 * puj1j0 * arr[5],
					pui1i0 * puj0j1 * arr[6], pui1i0 * puj1j0 * arr[7],
				};
				pair_bb[bb] += 0.5 * pre * (gui0j0 * gdi1j1 + gui1j0 * gdi0j1 +
				                            gui0j1 * gdi1j0 + gui1j1 * gdi0j0);
				const num x = ap[0] + ap[3] + ap[4] + ap[7];
				const num y = ap[1] + ap[2] + ap[5] + ap[6];
				const num tt[8] = {
					pui1i0 * gui0i1, pui0i1 * gui1i0, pdi1i0 * gdi0i1, pdi0i1 * gdi1i0,
					puj1j0 * guj0j1, puj0j1 * guj1j0, pdj1j0 * gdj0j1, pdj0j1 * gdj1j0,
				};
				jj[bb] += pre * ((tt[0] - tt[1] + tt[2] - tt[3]) * (tt[4] - tt[5] + tt[6] - tt[7]) + x - y);
				jsjs[bb] += pre * ((tt[0] - tt[1] - tt[2] + tt[3]) * (tt[4] - tt[5] - tt[6] + tt[7]) + x - y);
				kk[bb] += pre * ((tt[0] + tt[1] + tt[2] + tt[3]) * (tt[4] + tt[5] + tt[6] + tt[7]) + x + y);
				ksks[bb] += pre * ((tt[0] + tt[1] - tt[2] - tt[3]) * (tt[4] + tt[5] - tt[6] - tt[7]) + x + y);
			}
		}
	}
}

/* ------------------------------- dense G --------------------------------- */

void orc_dense_g(int N, int L, int l, const void *B_, void *g_)
{
	const num *B = B_;
	num *g = g_;
	const size_t NN = (size_t)N * N;
	num *P = zalloc(sizeof(num) * NN), *tmp = zalloc(sizeof(num) * NN);
	int *ipiv = zalloc(sizeof(int) * N);
	for (int i = 0; i < N; i++) P[i + N * i] = 1.0;
	for (int k = 0; k < L; k++) {
		const int s = (l + k) % L;
		gemm('N', 'N', N, N, N, 1.0, B + NN * s, N, P, N, 0.0, tmp, N);
		memcpy(P, tmp, sizeof(num) * NN);
	}
	for (int i = 0; i < N; i++) P[i + N * i] += 1.0;
	getrf(N, P, N, ipiv);
	getri(N, P, N, ipiv);
	memcpy(g, P, sizeof(num) * NN);
	free(P); free(tmp); free(ipiv);
}

/* -------------------------------- dqmc.c --------------------------------- */

/* Sweep driver, dqmc.c:84-459 (no checkpoints, signals or profiling) */
int orc_dqmc(struct orc_sim *s, int stop_sweep, void *gu_out, void *gd_out, void *phase_out)
{
	const int N = s->N, L = s->L, n_matmul = s->n_matmul, F = s->F;
	const size_t NN = (size_t)N * N;
	const int uneq = s->period_uneqlt > 0;
	num *B[2], *iB[2], *C[2], *g[2], *t1[2], *t2[2];
	num *G0t[2] = {0}, *Gtt[2] = {0}, *Gt0[2] = {0};
	const num *eK[2] = {s->exp_Ku, s->exp_Kd}, *ieK[2] = {s->inv_exp_Ku, s->inv_exp_Kd};
	const num *ehK[2] = {s->exp_halfKu, s->exp_halfKd};
	const num *iehK[2] = {s->inv_exp_halfKu, s->inv_exp_halfKd};
	for (int sp = 0; sp < 2; sp++) {
		B[sp] = zalloc(sizeof(num) * NN * L);
		iB[sp] = zalloc(sizeof(num) * NN * L);
		C[sp] = zalloc(sizeof(num) * NN * F);
		g[sp] = zalloc(sizeof(num) * NN);
		t1[sp] = zalloc(sizeof(num) * NN);
		t2[sp] = zalloc(sizeof(num) * NN);
		if (uneq) {
			G0t[sp] = zalloc(sizeof(num) * NN * L);
			Gtt[sp] = zalloc(sizeof(num) * NN * L);
			Gt0[sp] = zalloc(sizeof(num) * NN * L);
		}
	}
	num *au = zalloc(sizeof(num) * NN), *bu = zalloc(sizeof(num) * NN);
	num *ad = zalloc(sizeof(num) * NN), *bd = zalloc(sizeof(num) * NN);
	num *du = zalloc(sizeof(num) * N), *dd = zalloc(sizeof(num) * N);
	int *order = zalloc(sizeof(int) * N);
	num phase, ph[2];

	for (int sp = 0; sp < 2; sp++) {
		orc_build_iB(N, L, ieK[sp], s->exp_lambda, s->hs, sp, iB[sp]);
		orc_build_B(N, L, eK[sp], s->exp_lambda, s->hs, sp, B[sp]);
		for (int f = 0; f < F; f++)
			mul_seq(N, L, f * n_matmul, ((f + 1) * n_matmul) % L, 1.0, B[sp],
			        C[sp] + NN * f, N, t1[sp]);
		ph[sp] = calc_eq_g(0, N, F, 2, C[sp], g[sp]);
	}
	phase = ph[0] * ph[1];

	for (; *s->sweep < stop_sweep; (*s->sweep)++) {
		for (int l = 0; l < L; l++) {
			orc_shuffle(s->rng, N, order);
			update_delayed(N, s->n_delay, s->del, order, s->rng, s->hs + N * l,
			               g[0], g[1], &phase, au, bu, du, ad, bd, dd);
			const int f = l / n_matmul;
			const int recalc = ((l + 1) % n_matmul == 0);
			for (int sp = 0; sp < 2; sp++) {
				num *Bl = B[sp] + NN * l, *iBl = iB[sp] + NN * l;
				orc_build_B(N, 1, eK[sp], s->exp_lambda, s->hs + N * l, sp, Bl);
				orc_build_iB(N, 1, ieK[sp], s->exp_lambda, s->hs + N * l, sp, iBl);
				if (recalc) {
					mul_seq(N, L, f * n_matmul, ((f + 1) * n_matmul) % L, 1.0, B[sp],
					        C[sp] + NN * f, N, t1[sp]);
					ph[sp] = calc_eq_g((f + 1) % F, N, F, 2, C[sp], g[sp]);
				} else {
					gemm('N', 'N', N, N, N, 1.0, g[sp], N, iBl, N, 0.0, t1[sp], N);
					gemm('N', 'N', N, N, N, 1.0, Bl, N, t1[sp], N, 0.0, g[sp], N);
				}
			}
			if (recalc) phase = ph[0] * ph[1];
			if (*s->sweep >= s->n_sweep_warm && s->period_eqlt > 0 &&
			    (l + 1) % s->period_eqlt == 0) {
				for (int sp = 0; sp < 2; sp++) {
					gemm('N', 'N', N, N, N, 1.0, g[sp], N, ehK[sp], N, 0.0, t1[sp], N);
					gemm('N', 'N', N, N, N, 1.0, iehK[sp], N, t1[sp], N, 0.0, t2[sp], N);
				}
				orc_measure_eqlt(s, &phase, t2[0], t2[1]);
			}
		}
		if (*s->sweep >= s->n_sweep_warm && uneq && *s->sweep % s->period_uneqlt == 0) {
			for (int sp = 0; sp < 2; sp++) {
				orc_calc_ue_g(N, L, F, 2, B[sp], iB[sp], C[sp], G0t[sp], Gtt[sp], Gt0[sp]);
				num *stacks[3] = {G0t[sp], Gtt[sp], Gt0[sp]};
				for (int q = 0; q < 3; q++)
					for (int l = 0; l < L; l++) {
						gemm('N', 'N', N, N, N, 1.0, stacks[q] + NN * l, N, ehK[sp], N,
						     0.0, t1[sp], N);
						gemm('N', 'N', N, N, N, 1.0, iehK[sp], N, t1[sp], N, 0.0,
						     stacks[q] + NN * l, N);
					}
			}
			orc_measure_uneqlt(s, &phase, G0t[0], Gtt[0], Gt0[0], G0t[1], Gtt[1], Gt0[1]);
		}
	}
	if (gu_out) memcpy(gu_out, g[0], sizeof(num) * NN);
	if (gd_out) memcpy(gd_out, g[1], sizeof(num) * NN);
	if (phase_out) *(num *)phase_out = phase;
	for (int sp = 0; sp < 2; sp++) {
		free(B[sp]); free(iB[sp]); free(C[sp]); free(g[sp]); free(t1[sp]); free(t2[sp]);
		free(G0t[sp]); free(Gtt[sp]); free(Gt0[sp]);
	}
	free(au); free(bu); free(ad); free(bd); free(du); free(dd); free(order);
	return 0;
}
