/*
 * DQSF container access in C.  See simfile.h and dqmc_b200/simfile.py.
 */
#include "simfile.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define DQSF_MAX_LINK_DEPTH 4

typedef struct {
	char name[80];
	uint32_t dtype;
	uint32_t ndim;
	uint64_t shape[3];
	uint64_t offset;
	uint64_t size;
} dqsf_entry;

struct dqsf_file {
	FILE *fp;
	char *dir;       /* directory of the file, for relative links */
	uint64_t n;
	dqsf_entry *tab;
	int depth;
	/* linked files opened on demand, one per link entry */
	dqsf_file **linked;
};

static size_t dt_size(uint32_t dt)
{
	switch (dt) {
	case DQSF_I32: return 4;
	case DQSF_I64: return 8;
	case DQSF_F64: return 8;
	case DQSF_C128: return 16;
	case DQSF_U64: return 8;
	default: return 1;
	}
}

static int open_depth(const char *path, int writable, int depth, dqsf_file **out)
{
	*out = NULL;
	if (depth > DQSF_MAX_LINK_DEPTH) return DQSF_OPEN_FAIL;
	FILE *fp = fopen(path, writable ? "r+b" : "rb");
	if (fp == NULL) return DQSF_OPEN_FAIL;
	char head[24];
	if (fread(head, 1, 24, fp) != 24 || memcmp(head, "DQSF0001", 8) != 0) {
		fclose(fp);
		return DQSF_CORRUPT_FAIL;
	}
	uint64_t n, toff;
	memcpy(&n, head + 8, 8);
	memcpy(&toff, head + 16, 8);
	if (n > (1u << 20)) { fclose(fp); return DQSF_CORRUPT_FAIL; }
	dqsf_file *f = calloc(1, sizeof(*f));
	f->fp = fp;
	f->n = n;
	f->depth = depth;
	f->tab = calloc(n ? n : 1, sizeof(dqsf_entry));
	f->linked = calloc(n ? n : 1, sizeof(dqsf_file *));
	if (fseek(fp, (long)toff, SEEK_SET) != 0 ||
	    fread(f->tab, sizeof(dqsf_entry), n, fp) != n) {
		dqsf_close(f);
		return DQSF_CORRUPT_FAIL;
	}
	for (uint64_t i = 0; i < n; i++) f->tab[i].name[79] = '\0';
	const char *slash = strrchr(path, '/');
	if (slash == NULL) {
		f->dir = strdup(".");
	} else {
		size_t len = (size_t)(slash - path);
		f->dir = malloc(len + 1);
		memcpy(f->dir, path, len);
		f->dir[len] = '\0';
	}
	*out = f;
	return 0;
}

int dqsf_open(const char *path, int writable, dqsf_file **out)
{
	return open_depth(path, writable, 0, out);
}

int dqsf_close(dqsf_file *f)
{
	if (f == NULL) return 0;
	int rc = 0;
	for (uint64_t i = 0; i < f->n; i++)
		if (f->linked[i]) dqsf_close(f->linked[i]);
	if (f->fp && fclose(f->fp) != 0) rc = DQSF_CLOSE_FAIL;
	free(f->linked);
	free(f->tab);
	free(f->dir);
	free(f);
	return rc;
}

static const char *strip(const char *name)
{
	while (*name == '/') name++;
	return name;
}

/* find `name` in f or in a linked file; returns the owning file and entry */
static int lookup(dqsf_file *f, const char *name, dqsf_file **owner, dqsf_entry **ent)
{
	name = strip(name);
	for (uint64_t i = 0; i < f->n; i++) {
		if (f->tab[i].dtype != DQSF_LINK && strcmp(f->tab[i].name, name) == 0) {
			*owner = f;
			*ent = &f->tab[i];
			return 0;
		}
	}
	for (uint64_t i = 0; i < f->n; i++) {
		dqsf_entry *e = &f->tab[i];
		size_t len = strlen(e->name);
		if (e->dtype != DQSF_LINK || strncmp(e->name, name, len) != 0 ||
		    (name[len] != '/' && name[len] != '\0'))
			continue;
		if (f->linked[i] == NULL) {
			char target[1024], full[2048];
			if (e->size >= sizeof(target)) return DQSF_RW_FAIL;
			if (fseek(f->fp, (long)e->offset, SEEK_SET) != 0 ||
			    fread(target, 1, e->size, f->fp) != e->size)
				return DQSF_RW_FAIL;
			target[e->size] = '\0';
			if (target[0] == '/')
				snprintf(full, sizeof(full), "%s", target);
			else
				snprintf(full, sizeof(full), "%s/%s", f->dir, target);
			if (open_depth(full, 0, f->depth + 1, &f->linked[i]) != 0)
				return DQSF_OPEN_FAIL;
		}
		return lookup(f->linked[i], name, owner, ent);
	}
	return DQSF_RW_FAIL;
}

int dqsf_has(dqsf_file *f, const char *name)
{
	dqsf_file *o;
	dqsf_entry *e;
	return lookup(f, name, &o, &e) == 0;
}

int dqsf_info(dqsf_file *f, const char *name, int *dtype, size_t *count)
{
	dqsf_file *o;
	dqsf_entry *e;
	if (lookup(f, name, &o, &e) != 0) return DQSF_RW_FAIL;
	*dtype = (int)e->dtype;
	*count = (size_t)(e->size / dt_size(e->dtype));
	return 0;
}

static int read_raw(dqsf_file *f, const char *name, dqsf_entry **ent, void **buf)
{
	dqsf_file *o;
	if (lookup(f, name, &o, ent) != 0) {
		fprintf(stderr, "dqsf: dataset %s not found\n", name);
		return DQSF_RW_FAIL;
	}
	*buf = malloc((*ent)->size ? (*ent)->size : 1);
	if (fseek(o->fp, (long)(*ent)->offset, SEEK_SET) != 0 ||
	    fread(*buf, 1, (*ent)->size, o->fp) != (*ent)->size) {
		free(*buf);
		return DQSF_RW_FAIL;
	}
	return 0;
}

int dqsf_read_int(dqsf_file *f, const char *name, int *dst, size_t count)
{
	dqsf_entry *e;
	void *buf;
	int rc = read_raw(f, name, &e, &buf);
	if (rc) return rc;
	size_t have = e->size / dt_size(e->dtype);
	if (have != count) rc = DQSF_RW_FAIL;
	else if (e->dtype == DQSF_I32) memcpy(dst, buf, count * 4);
	else if (e->dtype == DQSF_I64 || e->dtype == DQSF_U64)
		for (size_t i = 0; i < count; i++) dst[i] = (int)((int64_t *)buf)[i];
	else if (e->dtype == DQSF_F64)
		for (size_t i = 0; i < count; i++) dst[i] = (int)((double *)buf)[i];
	else rc = DQSF_RW_FAIL;
	if (rc) fprintf(stderr, "dqsf: cannot read %s as int[%zu]\n", name, count);
	free(buf);
	return rc;
}

int dqsf_read_u64(dqsf_file *f, const char *name, uint64_t *dst, size_t count)
{
	dqsf_entry *e;
	void *buf;
	int rc = read_raw(f, name, &e, &buf);
	if (rc) return rc;
	if ((e->dtype != DQSF_U64 && e->dtype != DQSF_I64) || e->size != count * 8)
		rc = DQSF_RW_FAIL;
	else memcpy(dst, buf, count * 8);
	free(buf);
	return rc;
}

int dqsf_read_f64(dqsf_file *f, const char *name, double *dst, size_t count)
{
	dqsf_entry *e;
	void *buf;
	int rc = read_raw(f, name, &e, &buf);
	if (rc) return rc;
	if (e->dtype == DQSF_F64 && e->size == count * 8) memcpy(dst, buf, count * 8);
	else if (e->dtype == DQSF_I64 && e->size == count * 8)
		for (size_t i = 0; i < count; i++) dst[i] = (double)((int64_t *)buf)[i];
	else if (e->dtype == DQSF_I32 && e->size == count * 4)
		for (size_t i = 0; i < count; i++) dst[i] = (double)((int32_t *)buf)[i];
	else rc = DQSF_RW_FAIL;
	if (rc) fprintf(stderr, "dqsf: cannot read %s as double[%zu]\n", name, count);
	free(buf);
	return rc;
}

int dqsf_read_c128(dqsf_file *f, const char *name, double *dst, size_t count)
{
	dqsf_entry *e;
	void *buf;
	int rc = read_raw(f, name, &e, &buf);
	if (rc) return rc;
	if (e->dtype == DQSF_C128 && e->size == count * 16) {
		memcpy(dst, buf, count * 16);
	} else if (e->dtype == DQSF_F64 && e->size == count * 8) {
		for (size_t i = 0; i < count; i++) {
			dst[2 * i] = ((double *)buf)[i];
			dst[2 * i + 1] = 0.0;
		}
	} else {
		rc = DQSF_RW_FAIL;
		fprintf(stderr, "dqsf: cannot read %s as complex[%zu]\n", name, count);
	}
	free(buf);
	return rc;
}

int dqsf_read_str(dqsf_file *f, const char *name, char *out, size_t cap)
{
	dqsf_entry *e;
	void *buf;
	int rc = read_raw(f, name, &e, &buf);
	if (rc) return rc;
	if (e->dtype != DQSF_STR || cap == 0) {
		free(buf);
		return DQSF_RW_FAIL;
	}
	size_t n = e->size < cap - 1 ? e->size : cap - 1;
	memcpy(out, buf, n);
	out[n] = '\0';
	free(buf);
	return 0;
}

static int write_raw(dqsf_file *f, const char *name, uint32_t want_dt,
		const void *src, size_t bytes)
{
	name = strip(name);
	for (uint64_t i = 0; i < f->n; i++) {
		dqsf_entry *e = &f->tab[i];
		if (e->dtype == DQSF_LINK || strcmp(e->name, name) != 0) continue;
		if (e->dtype != want_dt || e->size != bytes) return DQSF_RW_FAIL;
		if (fseek(f->fp, (long)e->offset, SEEK_SET) != 0 ||
		    fwrite(src, 1, bytes, f->fp) != bytes)
			return DQSF_RW_FAIL;
		return 0;
	}
	fprintf(stderr, "dqsf: dataset %s not writable here\n", name);
	return DQSF_RW_FAIL;
}

int dqsf_write_int(dqsf_file *f, const char *name, const int *src, size_t count)
{
	dqsf_file *o;
	dqsf_entry *e;
	if (lookup(f, name, &o, &e) != 0 || o != f) return DQSF_RW_FAIL;
	if (e->dtype == DQSF_I32) return write_raw(f, name, DQSF_I32, src, count * 4);
	if (e->dtype == DQSF_I64) {
		int64_t *tmp = malloc(count * 8 + 8);
		for (size_t i = 0; i < count; i++) tmp[i] = src[i];
		int rc = write_raw(f, name, DQSF_I64, tmp, count * 8);
		free(tmp);
		return rc;
	}
	return DQSF_RW_FAIL;
}

int dqsf_write_u64(dqsf_file *f, const char *name, const uint64_t *src, size_t count)
{
	return write_raw(f, name, DQSF_U64, src, count * 8);
}

int dqsf_write_f64(dqsf_file *f, const char *name, const double *src, size_t count)
{
	return write_raw(f, name, DQSF_F64, src, count * 8);
}

int dqsf_write_c128(dqsf_file *f, const char *name, const double *src, size_t count)
{
	return write_raw(f, name, DQSF_C128, src, count * 16);
}
