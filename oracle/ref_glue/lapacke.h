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
