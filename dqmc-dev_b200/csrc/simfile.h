/*
 * C reader/writer for the DQSF sim-file container (layout documented in
 * dqmc_b200/simfile.py).  Plays the role of the HDF5 calls in the reference
 * data layer (src/data.c:18-30 my_read/my_write): lookups by dataset path,
 * integer datasets converted on read and write whatever their stored width
 * (as H5LTread_dataset_int does), in-place writes of existing datasets.
 */
#pragma once

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { DQSF_I32 = 1, DQSF_I64 = 2, DQSF_F64 = 3, DQSF_C128 = 4, DQSF_U64 = 5,
       DQSF_STR = 6, DQSF_LINK = 7 };

/* error codes, matching the reference data layer (src/data.c:10-13) */
enum { DQSF_OPEN_FAIL = -1, DQSF_CORRUPT_FAIL = -2, DQSF_RW_FAIL = -3,
       DQSF_CLOSE_FAIL = -4 };

typedef struct dqsf_file dqsf_file;

int dqsf_open(const char *path, int writable, dqsf_file **out);
int dqsf_close(dqsf_file *f);

/* 1 if the dataset exists (links followed), 0 otherwise */
int dqsf_has(dqsf_file *f, const char *name);
/* dtype and element count of a dataset; returns 0 or DQSF_RW_FAIL */
int dqsf_info(dqsf_file *f, const char *name, int *dtype, size_t *count);

/* typed reads; `count` must equal the stored element count */
int dqsf_read_int(dqsf_file *f, const char *name, int *dst, size_t count);
int dqsf_read_u64(dqsf_file *f, const char *name, uint64_t *dst, size_t count);
int dqsf_read_f64(dqsf_file *f, const char *name, double *dst, size_t count);
/* complex128 as interleaved (re, im) doubles: `count` complex elements */
int dqsf_read_c128(dqsf_file *f, const char *name, double *dst, size_t count);
/* reads a string dataset into buf (NUL-terminated, truncated to cap) */
int dqsf_read_str(dqsf_file *f, const char *name, char *buf, size_t cap);

/* in-place writes of existing datasets in this file (links are read-only) */
int dqsf_write_int(dqsf_file *f, const char *name, const int *src, size_t count);
int dqsf_write_u64(dqsf_file *f, const char *name, const uint64_t *src, size_t count);
int dqsf_write_f64(dqsf_file *f, const char *name, const double *src, size_t count);
int dqsf_write_c128(dqsf_file *f, const char *name, const double *src, size_t count);

#ifdef __cplusplus
}
#endif
