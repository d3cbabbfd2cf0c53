/*
 * lapacke.h for building the reference C sources against scipy's OpenBLAS.
 * Maps the LAPACK_x macros that src/linalg_generic.h uses onto the Fortran
 * entry points (scipy_ prefix, LP64), passing the hidden character-length
 * arguments that gfortran-built LAPACK expects.  Test-side build glue.
 */
#pragma once
#include <stddef.h>

void scipy_dgetrf_(const int *, const int *, double *, const int *, int *, int *);
void scipy_dgetri_(const int *, double *, const int *, const int *, double *, const int *, int *);
void scipy_dgetrs_(const char *, const int *, const int *, const double *, const int *,
		const int *, double *, const int *, int *, size_t);
void scipy_dgeqp3_(const int *, const int *, double *, const int *, int *, double *,
		double *, const int *, int *);
void scipy_dgeqrf_(const int *, const int *, double *, const int *, double *, double *,
		const int *, int *);
void scipy_dormqr_(const char *, const char *, const int *, const int *, const int *,
		const double *, const int *, const double *, double *, const int *,
		double *, const int *, int *, size_t, size_t);
void scipy_dtrtri_(const char *, const char *, const int *, double *, const int *, int *,
		size_t, size_t);

void scipy_zgetrf_(const int *, const int *, void *, const int *, int *, int *);
void scipy_zgetri_(const int *, void *, const int *, const int *, void *, const int *, int *);
void scipy_zgetrs_(const char *, const int *, const int *, const void *, const int *,
		const int *, void *, const int *, int *, size_t);
void scipy_zgeqp3_(const int *, const int *, void *, const int *, int *, void *,
		void *, const int *, double *, int *);
void scipy_zgeqrf_(const int *, const int *, void *, const int *, void *, void *,
		const int *, int *);
void scipy_zunmqr_(const char *, const char *, const int *, const int *, const int *,
		const void *, const int *, const void *, void *, const int *,
		void *, const int *, int *, size_t, size_t);
void scipy_ztrtri_(const char *, const char *, const int *, void *, const int *, int *,
		size_t, size_t);

#ifdef DQ_FLOP_TALLY
void dq_tally_dgetrf(const int *, const int *, double *, const int *, int *, int *);
void dq_tally_dgetri(const int *, double *, const int *, const int *, double *, const int *, int *);
void dq_tally_dgetrs(const char *, const int *, const int *, const double *, const int *,
		const int *, double *, const int *, int *, size_t);
void dq_tally_dgeqp3(const int *, const int *, double *, const int *, int *, double *,
		double *, const int *, int *);
void dq_tally_dgeqrf(const int *, const int *, double *, const int *, double *, double *,
		const int *, int *);
void dq_tally_dormqr(const char *, const char *, const int *, const int *, const int *,
		const double *, const int *, const double *, double *, const int *,
		double *, const int *, int *, size_t, size_t);
void dq_tally_dtrtri(const char *, const char *, const int *, double *, const int *, int *,
		size_t, size_t);

void dq_tally_zgetrf(const int *, const int *, void *, const int *, int *, int *);
void dq_tally_zgetri(const int *, void *, const int *, const int *, void *, const int *, int *);
void dq_tally_zgetrs(const char *, const int *, const int *, const void *, const int *,
		const int *, void *, const int *, int *, size_t);
void dq_tally_zgeqp3(const int *, const int *, void *, const int *, int *, void *,
		void *, const int *, double *, int *);
void dq_tally_zgeqrf(const int *, const int *, void *, const int *, void *, void *,
		const int *, int *);
void dq_tally_zunmqr(const char *, const char *, const int *, const int *, const int *,
		const void *, const int *, const void *, void *, const int *,
		void *, const int *, int *, size_t, size_t);
void dq_tally_ztrtri(const char *, const char *, const int *, void *, const int *, int *,
		size_t, size_t);
#endif

#ifdef DQ_FLOP_TALLY
/* the tally variant: counting wrappers (flop_tally.c) in front of OpenBLAS */
#define LAPACK_dgetrf(...) dq_tally_dgetrf(__VA_ARGS__)
#define LAPACK_dgetri(...) dq_tally_dgetri(__VA_ARGS__)
#define LAPACK_dgetrs(...) dq_tally_dgetrs(__VA_ARGS__, 1)
#define LAPACK_dgeqp3(...) dq_tally_dgeqp3(__VA_ARGS__)
#define LAPACK_dgeqrf(...) dq_tally_dgeqrf(__VA_ARGS__)
#define LAPACK_dormqr(...) dq_tally_dormqr(__VA_ARGS__, 1, 1)
#define LAPACK_dtrtri(...) dq_tally_dtrtri(__VA_ARGS__, 1, 1)
#define LAPACK_zgetrf(...) dq_tally_zgetrf(__VA_ARGS__)
#define LAPACK_zgetri(...) dq_tally_zgetri(__VA_ARGS__)
#define LAPACK_zgetrs(...) dq_tally_zgetrs(__VA_ARGS__, 1)
#define LAPACK_zgeqp3(...) dq_tally_zgeqp3(__VA_ARGS__)
#define LAPACK_zgeqrf(...) dq_tally_zgeqrf(__VA_ARGS__)
#define LAPACK_zunmqr(...) dq_tally_zunmqr(__VA_ARGS__, 1, 1)
#define LAPACK_ztrtri(...) dq_tally_ztrtri(__VA_ARGS__, 1, 1)
#else
#define LAPACK_dgetrf(...) scipy_dgetrf_(__VA_ARGS__)
#define LAPACK_dgetri(...) scipy_dgetri_(__VA_ARGS__)
#define LAPACK_dgetrs(...) scipy_dgetrs_(__VA_ARGS__, 1)
#define LAPACK_dgeqp3(...) scipy_dgeqp3_(__VA_ARGS__)
#define LAPACK_dgeqrf(...) scipy_dgeqrf_(__VA_ARGS__)
#define LAPACK_dormqr(...) scipy_dormqr_(__VA_ARGS__, 1, 1)
#define LAPACK_dtrtri(...) scipy_dtrtri_(__VA_ARGS__, 1, 1)
#define LAPACK_zgetrf(...) scipy_zgetrf_(__VA_ARGS__)
#define LAPACK_zgetri(...) scipy_zgetri_(__VA_ARGS__)
#define LAPACK_zgetrs(...) scipy_zgetrs_(__VA_ARGS__, 1)
#define LAPACK_zgeqp3(...) scipy_zgeqp3_(__VA_ARGS__)
#define LAPACK_zgeqrf(...) scipy_zgeqrf_(__VA_ARGS__)
#define LAPACK_zunmqr(...) scipy_zunmqr_(__VA_ARGS__, 1, 1)
#define LAPACK_ztrtri(...) scipy_ztrtri_(__VA_ARGS__, 1, 1)
#endif
