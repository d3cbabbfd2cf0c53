/*
 * Quad-precision equal-time Green's function, for judging FP64 results.
 * Test infrastructure only: nothing here is linked into the engine.
 *
 *   G = (I + B_{L-1} ... B_0)^-1,  B_l = exp_K diag(exp_lambda[i + N*(hs_l[i] ^ spin)])
 *
 * as the reference defines it (src/dqmc.c:29-59 for B_l, src/greens.c:69-208
 * for G), evaluated in __float128 (113-bit significand) by the plain
 * product and an LU solve with partial pivoting, from the FP64 exp_K and
 * exp_lambda taken as exact inputs.  The product's singular values span
 * about 1e-13 .. 1e13 at the benchmark configurations, so the plain product
 * keeps G to about 1e-20 in quad, far below the FP64 errors it is used to
 * measure.  Column-major in and out; complex (interleaved re, im pairs)
 * when built with -DEXACT_CPLX.
 *
 *   exact_g(N, L, exp_K, exp_lambda, hs, spin, G)      hs: L x N, hs[i + N*l]
 */
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>

#ifdef EXACT_CPLX
typedef __complex128 qnum;
typedef double dnum[2];
static qnum q_in(const double *p) { return (__float128)p[0] + (__float128)p[1] * 1.0Qi; }
static void q_out(qnum v, double *p) { p[0] = (double)crealq(v); p[1] = (double)cimagq(v); }
static __float128 q_abs(qnum v) { return cabsq(v); }
#define STRIDE 2
#else
typedef __float128 qnum;
static qnum q_in(const double *p) { return (__float128)p[0]; }
static void q_out(qnum v, double *p) { p[0] = (double)v; }
static __float128 q_abs(qnum v) { return fabsq(v); }
#define STRIDE 1
#endif

int exact_g(int N, int L, const double *expK, const double *el, const int *hs, int spin,
		double *G)
{
	const size_t NN = (size_t)N * N;
	qnum *K = malloc(sizeof(qnum) * NN), *P = malloc(sizeof(qnum) * NN);
	qnum *T = malloc(sizeof(qnum) * NN), *X = malloc(sizeof(qnum) * NN);
	int *piv = malloc(sizeof(int) * N);
	if (!K || !P || !T || !X || !piv) return -1;
	for (size_t q = 0; q < NN; q++) K[q] = q_in(expK + STRIDE * q);
	for (size_t q = 0; q < NN; q++) P[q] = 0;
	for (int i = 0; i < N; i++) P[i + (size_t)N * i] = 1;
	for (int l = 0; l < L; l++) {
		/* P <- exp_K diag(d_l) P */
		for (int i = 0; i < N; i++) {
			const __float128 d = el[i + N * (hs[i + (size_t)N * l] ^ spin)];
			for (int j = 0; j < N; j++) P[i + (size_t)N * j] *= d;
		}
		for (size_t q = 0; q < NN; q++) T[q] = 0;
		for (int j = 0; j < N; j++)
			for (int k = 0; k < N; k++) {
				const qnum b = P[k + (size_t)N * j];
				for (int i = 0; i < N; i++) T[i + (size_t)N * j] += K[i + (size_t)N * k] * b;
			}
		memcpy(P, T, sizeof(qnum) * NN);
	}
	/* LU of M = I + P with partial pivoting, in place in P */
	for (int i = 0; i < N; i++) P[i + (size_t)N * i] += 1;
	for (int k = 0; k < N; k++) {
		int p = k;
		__float128 best = q_abs(P[k + (size_t)N * k]);
		for (int i = k + 1; i < N; i++) {
			const __float128 a = q_abs(P[i + (size_t)N * k]);
			if (a > best) { best = a; p = i; }
		}
		piv[k] = p;
		if (best == 0) return -2;
		if (p != k)
			for (int j = 0; j < N; j++) {
				const qnum t = P[k + (size_t)N * j];
				P[k + (size_t)N * j] = P[p + (size_t)N * j];
				P[p + (size_t)N * j] = t;
			}
		const qnum inv = 1 / P[k + (size_t)N * k];
		for (int i = k + 1; i < N; i++) P[i + (size_t)N * k] *= inv;
		for (int j = k + 1; j < N; j++) {
			const qnum u = P[k + (size_t)N * j];
			for (int i = k + 1; i < N; i++) P[i + (size_t)N * j] -= P[i + (size_t)N * k] * u;
		}
	}
	/* X = M^-1: solve M X = I column by column */
	for (size_t q = 0; q < NN; q++) X[q] = 0;
	for (int i = 0; i < N; i++) X[i + (size_t)N * i] = 1;
	for (int k = 0; k < N; k++)
		if (piv[k] != k)
			for (int j = 0; j < N; j++) {
				const qnum t = X[k + (size_t)N * j];
				X[k + (size_t)N * j] = X[piv[k] + (size_t)N * j];
				X[piv[k] + (size_t)N * j] = t;
			}
	for (int j = 0; j < N; j++) {
		qnum *x = X + (size_t)N * j;
		for (int k = 0; k < N; k++)
			for (int i = k + 1; i < N; i++) x[i] -= P[i + (size_t)N * k] * x[k];
		for (int k = N - 1; k >= 0; k--) {
			x[k] /= P[k + (size_t)N * k];
			for (int i = 0; i < k; i++) x[i] -= P[i + (size_t)N * k] * x[k];
		}
	}
	for (size_t q = 0; q < NN; q++) q_out(X[q], G + STRIDE * q);
	free(K); free(P); free(T); free(X); free(piv);
	return 0;
}
