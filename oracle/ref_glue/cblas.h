/*
 * cblas.h for building the reference C sources against the OpenBLAS that
 * ships inside scipy (its exports carry a "scipy_" prefix).  Only the
 * routines the reference's src/linalg_generic.h calls are declared.
 * Test-side build glue: never part of the engine.
 */
#pragma once

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };

#ifdef DQ_FLOP_TALLY
/* the tally variant: counting wrappers (flop_tally.c) in front of OpenBLAS */
#define cblas_dgemm dq_tally_dgemm
#define cblas_dgemv dq_tally_dgemv
#define cblas_dtrmm dq_tally_dtrmm
#define cblas_zgemm dq_tally_zgemm
#define cblas_zgemv dq_tally_zgemv
#define cblas_ztrmm dq_tally_ztrmm
#else
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dtrmm scipy_cblas_dtrmm
#define cblas_zgemm scipy_cblas_zgemm
#define cblas_zgemv scipy_cblas_zgemv
#define cblas_ztrmm scipy_cblas_ztrmm
#endif

void cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
		int m, int n, int k, double alpha, const double *a, int lda,
		const double *b, int ldb, double beta, double *c, int ldc);
void cblas_dgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int m, int n,
		double alpha, const double *a, int lda, const double *x, int incx,
		double beta, double *y, int incy);
void cblas_dtrmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO,
		enum CBLAS_TRANSPOSE, enum CBLAS_DIAG, int m, int n, double alpha,
		const double *a, int lda, double *b, int ldb);
void cblas_zgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
		int m, int n, int k, const void *alpha, const void *a, int lda,
		const void *b, int ldb, const void *beta, void *c, int ldc);
void cblas_zgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int m, int n,
		const void *alpha, const void *a, int lda, const void *x, int incx,
		const void *beta, void *y, int incy);
void cblas_ztrmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO,
		enum CBLAS_TRANSPOSE, enum CBLAS_DIAG, int m, int n, const void *alpha,
		const void *a, int lda, void *b, int ldb);
