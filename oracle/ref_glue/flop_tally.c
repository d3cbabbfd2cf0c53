/*
 * FLOP tally of the reference build: wrappers around the BLAS and LAPACK
 * routines that src/linalg_generic.h calls, counting each call's
 * LAPACK-standard floating-point operations (the leading terms of the
 * LAPACK Working Note 41 counts; complex routines count four real
 * operations per complex multiply-add pair, as the engine's counters do)
 * before calling scipy's OpenBLAS.  Workspace queries (lwork = -1) count
 * nothing.  Compiled only into the tally variant of the reference build
 * (make tally, -DDQ_FLOP_TALLY); test-side glue, never part of the engine.
 * At exit the total goes to the file named by DQ_FLOP_TALLY_OUT.
 */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#include "cblas.h"
#include "lapacke.h"

static double tally_total = 0.0;

static void add(double f)
{
#pragma omp atomic
	tally_total += f;
}

__attribute__((destructor)) static void tally_report(void)
{
	const char *path = getenv("DQ_FLOP_TALLY_OUT");
	if (!path) return;
	FILE *f = fopen(path, "w");
	if (!f) return;
	fprintf(f, "%.17g\n", tally_total);
	fclose(f);
}

/* the OpenBLAS entry points behind the wrappers */
void scipy_cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, int, int,
		int, double, const double *, int, const double *, int, double, double *, int);
void scipy_cblas_dgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int, int, double, const double *,
		int, const double *, int, double, double *, int);
void scipy_cblas_dtrmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE,
		enum CBLAS_DIAG, int, int, double, const double *, int, double *, int);
void scipy_cblas_zgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, int, int,
		int, const void *, const void *, int, const void *, int, const void *, void *, int);
void scipy_cblas_zgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int, int, const void *,
		const void *, int, const void *, int, const void *, void *, int);
void scipy_cblas_ztrmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE,
		enum CBLAS_DIAG, int, int, const void *, const void *, int, void *, int);

/* LAWN 41 leading terms, real arithmetic */
static double f_gemm(double m, double n, double k) { return 2.0 * m * n * k; }
static double f_gemv(double m, double n) { return 2.0 * m * n; }
static double f_trmm(int side, double m, double n) { return side == CblasLeft ? m * m * n : m * n * n; }
static double f_geqrf(double m, double n)
{
	return m >= n ? 2.0 * n * n * (m - n / 3.0) : 2.0 * m * m * (n - m / 3.0);
}
static double f_ormqr(char side, double m, double n, double k)
{
	return (side == 'L' || side == 'l') ? 2.0 * n * k * (2.0 * m - k) : 2.0 * m * k * (2.0 * n - k);
}
static double f_getrf(double m, double n)
{
	return m >= n ? m * n * n - n * n * n / 3.0 : n * m * m - m * m * m / 3.0;
}
static double f_getri(double n) { return 4.0 / 3.0 * n * n * n; }
static double f_getrs(double n, double nrhs) { return 2.0 * n * n * nrhs; }
static double f_trtri(double n) { return n * n * n / 3.0; }

void dq_tally_dgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m,
		int n, int k, double alpha, const double *a, int lda, const double *b, int ldb, double beta,
		double *c, int ldc)
{
	add(f_gemm(m, n, k));
	scipy_cblas_dgemm(o, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void dq_tally_dgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int m, int n, double alpha,
		const double *a, int lda, const double *x, int incx, double beta, double *y, int incy)
{
	add(f_gemv(m, n));
	scipy_cblas_dgemv(o, t, m, n, alpha, a, lda, x, incx, beta, y, incy);
}

void dq_tally_dtrmm(enum CBLAS_ORDER o, enum CBLAS_SIDE s, enum CBLAS_UPLO u, enum CBLAS_TRANSPOSE t,
		enum CBLAS_DIAG d, int m, int n, double alpha, const double *a, int lda, double *b, int ldb)
{
	add(f_trmm(s, m, n));
	scipy_cblas_dtrmm(o, s, u, t, d, m, n, alpha, a, lda, b, ldb);
}

void dq_tally_zgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m,
		int n, int k, const void *alpha, const void *a, int lda, const void *b, int ldb,
		const void *beta, void *c, int ldc)
{
	add(4.0 * f_gemm(m, n, k));
	scipy_cblas_zgemm(o, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void dq_tally_zgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int m, int n, const void *alpha,
		const void *a, int lda, const void *x, int incx, const void *beta, void *y, int incy)
{
	add(4.0 * f_gemv(m, n));
	scipy_cblas_zgemv(o, t, m, n, alpha, a, lda, x, incx, beta, y, incy);
}

void dq_tally_ztrmm(enum CBLAS_ORDER o, enum CBLAS_SIDE s, enum CBLAS_UPLO u, enum CBLAS_TRANSPOSE t,
		enum CBLAS_DIAG d, int m, int n, const void *alpha, const void *a, int lda, void *b, int ldb)
{
	add(4.0 * f_trmm(s, m, n));
	scipy_cblas_ztrmm(o, s, u, t, d, m, n, alpha, a, lda, b, ldb);
}

void dq_tally_dgetrf(const int *m, const int *n, double *a, const int *lda, int *ipiv, int *info)
{
	add(f_getrf(*m, *n));
	scipy_dgetrf_(m, n, a, lda, ipiv, info);
}

void dq_tally_dgetri(const int *n, double *a, const int *lda, const int *ipiv, double *work,
		const int *lwork, int *info)
{
	if (*lwork != -1) add(f_getri(*n));
	scipy_dgetri_(n, a, lda, ipiv, work, lwork, info);
}

void dq_tally_dgetrs(const char *t, const int *n, const int *nrhs, const double *a, const int *lda,
		const int *ipiv, double *b, const int *ldb, int *info, size_t lt)
{
	add(f_getrs(*n, *nrhs));
	scipy_dgetrs_(t, n, nrhs, a, lda, ipiv, b, ldb, info, lt);
}

void dq_tally_dgeqp3(const int *m, const int *n, double *a, const int *lda, int *jpvt, double *tau,
		double *work, const int *lwork, int *info)
{
	if (*lwork != -1) add(f_geqrf(*m, *n));
	scipy_dgeqp3_(m, n, a, lda, jpvt, tau, work, lwork, info);
}

void dq_tally_dgeqrf(const int *m, const int *n, double *a, const int *lda, double *tau,
		double *work, const int *lwork, int *info)
{
	if (*lwork != -1) add(f_geqrf(*m, *n));
	scipy_dgeqrf_(m, n, a, lda, tau, work, lwork, info);
}

void dq_tally_dormqr(const char *side, const char *t, const int *m, const int *n, const int *k,
		const double *a, const int *lda, const double *tau, double *c, const int *ldc,
		double *work, const int *lwork, int *info, size_t ls, size_t lt)
{
	if (*lwork != -1) add(f_ormqr(*side, *m, *n, *k));
	scipy_dormqr_(side, t, m, n, k, a, lda, tau, c, ldc, work, lwork, info, ls, lt);
}

void dq_tally_dtrtri(const char *u, const char *d, const int *n, double *a, const int *lda, int *info,
		size_t lu, size_t ld)
{
	add(f_trtri(*n));
	scipy_dtrtri_(u, d, n, a, lda, info, lu, ld);
}

void dq_tally_zgetrf(const int *m, const int *n, void *a, const int *lda, int *ipiv, int *info)
{
	add(4.0 * f_getrf(*m, *n));
	scipy_zgetrf_(m, n, a, lda, ipiv, info);
}

void dq_tally_zgetri(const int *n, void *a, const int *lda, const int *ipiv, void *work,
		const int *lwork, int *info)
{
	if (*lwork != -1) add(4.0 * f_getri(*n));
	scipy_zgetri_(n, a, lda, ipiv, work, lwork, info);
}

void dq_tally_zgetrs(const char *t, const int *n, const int *nrhs, const void *a, const int *lda,
		const int *ipiv, void *b, const int *ldb, int *info, size_t lt)
{
	add(4.0 * f_getrs(*n, *nrhs));
	scipy_zgetrs_(t, n, nrhs, a, lda, ipiv, b, ldb, info, lt);
}

void dq_tally_zgeqp3(const int *m, const int *n, void *a, const int *lda, int *jpvt, void *tau,
		void *work, const int *lwork, double *rwork, int *info)
{
	if (*lwork != -1) add(4.0 * f_geqrf(*m, *n));
	scipy_zgeqp3_(m, n, a, lda, jpvt, tau, work, lwork, rwork, info);
}

void dq_tally_zgeqrf(const int *m, const int *n, void *a, const int *lda, void *tau, void *work,
		const int *lwork, int *info)
{
	if (*lwork != -1) add(4.0 * f_geqrf(*m, *n));
	scipy_zgeqrf_(m, n, a, lda, tau, work, lwork, info);
}

void dq_tally_zunmqr(const char *side, const char *t, const int *m, const int *n, const int *k,
		const void *a, const int *lda, const void *tau, void *c, const int *ldc, void *work,
		const int *lwork, int *info, size_t ls, size_t lt)
{
	if (*lwork != -1) add(4.0 * f_ormqr(*side, *m, *n, *k));
	scipy_zunmqr_(side, t, m, n, k, a, lda, tau, c, ldc, work, lwork, info, ls, lt);
}

void dq_tally_ztrtri(const char *u, const char *d, const int *n, void *a, const int *lda, int *info,
		size_t lu, size_t ld)
{
	add(4.0 * f_trtri(*n));
	scipy_ztrtri_(u, d, n, a, lda, info, lu, ld);
}
