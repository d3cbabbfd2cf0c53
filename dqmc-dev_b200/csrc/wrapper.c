/*
 * Host lifecycle of a simulation: the drop-in dqmc_wrapper and its batched
 * form.  Follows the reference's src/dqmc.c:525-671 (dqmc_wrapper), with
 * the signal/time-limit handling of src/sig.c, the checkpoint cadence of
 * dqmc.c:233-244, the data layer of src/data.c:345-789 (read, save with the
 * partial_write guard) and a profile table in the spirit of src/prof.c.
 * The sweeps themselves run on the GPU through the engine (engine.cu).
 */
#define _GNU_SOURCE
#include <math.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "dqmc_b200.h"
#include "simfile.h"

#ifndef DQMC_GIT_ID
#define DQMC_GIT_ID "dqmc-b200"
#endif
#define DQMC_REPO "dqmc-b200"

#define WRAP_FAIL -1
#define WRAP_INCOMPLETE 1

/* ----------------------------------------------------------- time, signals */

static int64_t time_wall(void)
{
	struct timespec t;
	clock_gettime(CLOCK_MONOTONIC, &t);
	return (int64_t)t.tv_sec * 1000000000LL + t.tv_nsec;
}

/* sig.c:7-59: SIGUSR1/INT/TERM/HUP set a stop flag checked once per sweep */
static volatile sig_atomic_t stop_flag = 0;
static void on_stop(int signum) { stop_flag = signum; }

static void sig_init(void)
{
	static int called = 0;
	if (called) return;
	called = 1;
	struct sigaction sa;
	memset(&sa, 0, sizeof(sa));
	sa.sa_handler = on_stop;
	sigaction(SIGUSR1, &sa, NULL);
	sigaction(SIGINT, &sa, NULL);
	sigaction(SIGTERM, &sa, NULL);
	sigaction(SIGHUP, &sa, NULL);
}

struct stopper {
	FILE *log;
	int64_t wall_start, max_time, t_first;
	int first;
};

/* sig.c:70-127: -1 when max_time (nanoseconds after the call began, as the
 * reference's time_wall ticks) is reached, the signal number on a signal */
static int check_stop(struct stopper *s, int sweep, int n_sweep_warm, int n_sweep)
{
	const int64_t now = time_wall();
	if (s->max_time > 0 && now >= s->wall_start + s->max_time) stop_flag = -1;
	if (s->t_first == 0) {
		s->first = sweep;
		s->t_first = now;
	}
	if (stop_flag) {
		const double el = (now - s->wall_start) * 1e-9;
		const double done = (now - s->t_first) * 1e-9;
		const int sd = sweep - s->first;
		const double left = sd > 0 ? done / sd * (n_sweep - sweep) : 0.0;
		fprintf(s->log, "%d/%d sweeps completed (%s)\n", sweep, n_sweep,
		        sweep >= n_sweep_warm ? "measuring" : "warming up");
		fprintf(s->log, "\telapsed: %.3f%c\n", el < 3600 ? el : el / 3600, el < 3600 ? 's' : 'h');
		fprintf(s->log, "\tremaining%s: %.3f%c\n",
		        (s->first < n_sweep_warm) ? " (ignoring measurement cost)" : "",
		        left < 3600 ? left : left / 3600, left < 3600 ? 's' : 'h');
		fprintf(s->log, "stop_flag = %d, stopping\n", (int)stop_flag);
		fflush(s->log);
	}
	if (sweep == n_sweep_warm) {
		s->first = sweep;
		s->t_first = now;
	}
	return stop_flag;
}

/* ------------------------------------------------------------- profiling */

enum { PR_WALL, PR_READ, PR_INIT, PR_SWEEPS, PR_CHECKPOINT, PR_SAVE, PR_N };
static const char *pr_name[PR_N] = {"wall", "read", "init_g", "sweeps", "checkpoint", "save"};
struct prof {
	int64_t t[PR_N];
	int n[PR_N];
};

static void prof_print(FILE *log, const struct prof *p)
{
	fprintf(log, "region___________|_%% of all_|___total (s)_|___us per call_|___# calls\n");
	for (int i = 0; i < PR_N; i++) {
		if (!p->n[i]) continue;
		fprintf(log, "%16s |%9.3f |%12.3f |%14.3f |%10d\n", pr_name[i],
		        100.0 * p->t[i] / (p->t[PR_WALL] ? p->t[PR_WALL] : 1), p->t[i] * 1e-9,
		        1e-3 * p->t[i] / p->n[i], p->n[i]);
	}
	fprintf(log, "---------------------------------------------------------------------\n");
}

/* ------------------------------------------------------------- sim data */

struct sim {
	const char *file;
	dqmc_params p;
	int cplx, n_sweep_meas, checkpoint_every, num_b_alloc;
	int *map_i, *map_ij, *bonds, *map_bb;
	double *peierlsu, *peierlsd;
	double *mats[8];
	double *exp_lambda, *del;
	uint64_t rng[17];
	int sweep;
	int *hs;
	int eq_n, ue_n;
	double *eq_acc, *ue_acc;      /* num arrays in the engine's layout */
	int eq_size, ue_size;
	int *tmap[9];                 /* the measurement toggles' maps, tmap_names order */
	double *pp[4];                /* two-hop phases pp_u, pp_d, ppr_u, ppr_d (num) */
};

/* the measurement toggles and sizes appended to dqmc_params, with their
 * dataset names (params/...) */
static const char *toggle_int_names[] = {
	"meas_energy_corr", "meas_thermal", "meas_2bond_corr", "meas_nematic_corr",
	"meas_chiral", "meas_local_JQ", "meas_gen_suscept", "meas_pair_bb_only", "Nx", "Ny",
	"num_plaq", "num_plaq_accum", "num_b_accum", "num_b2_accum", "num_bs", "num_b2",
	"num_b2b", "num_bb2", "num_b2b2", "degen_plaq", "degen_b", "degen_b2", "degen_bs",
	"degen_b2b", "degen_bb2", "degen_b2b2"};
#define N_TOGGLE_INTS (int)(sizeof(toggle_int_names) / sizeof(toggle_int_names[0]))
static const char *tmap_names[9] = {"plaqs", "map_plaq", "map_b", "map_bs", "bond2s", "map_b2",
                                    "map_bb2", "map_b2b", "map_b2b2"};
static const char *pp_names[4] = {"pp_u", "pp_d", "ppr_u", "ppr_d"};

/* the accumulated datasets after `sign`, in the engine's accumulator order
 * (csrc/meas.cuh), with the reference's names and sizes (data.c:441-522) */
struct dset { const char *name; size_t n; };
#define MAX_DSETS 48

static int acc_sets(const dqmc_params *p, int uneqlt, struct dset *d)
{
	const size_t L = p->L, ni = p->num_i, nij = p->num_ij, nbb = p->num_bb, nbs = p->num_bs;
	int k = 0;
#define D(nm, cnt) d[k++] = (struct dset){nm, (cnt)}
	if (!uneqlt) {
		D("density", ni); D("density_u", ni); D("density_d", ni); D("double_occ", ni);
		D("g00", nij); D("g00_u", nij); D("g00_d", nij); D("nn", nij); D("xx", nij);
		D("zz", nij); D("pair_sw", nij);
		if (p->meas_gen_suscept) {
			D("uuuu", nij * nij); D("dddd", nij * nij); D("dduu", nij * nij); D("uudd", nij * nij);
		}
		if (p->meas_chiral) D("chi", (size_t)p->num_plaq_accum);
		if (p->meas_energy_corr) { D("kk", nbb); D("kv", nbs); D("kn", nbs); D("vv", nij); D("vn", nij); }
		if (p->meas_local_JQ) {
			D("j", (size_t)p->num_b_accum); D("jn", (size_t)p->num_b_accum);
			D("j2", (size_t)p->num_b2_accum);
		}
		return k;
	}
	D("gt0", nij * L); D("gt0_u", nij * L); D("gt0_d", nij * L); D("nn", nij * L);
	D("xx", nij * L); D("zz", nij * L); D("pair_sw", nij * L);
	if (p->meas_gen_suscept) {
		D("uuuu", nij * nij * L); D("dddd", nij * nij * L);
		D("dduu", nij * nij * L); D("uudd", nij * nij * L);
	}
	if (p->meas_bond_corr || p->meas_pair_bb_only) D("pair_bb", nbb * L);
	if (p->meas_bond_corr) { D("jj", nbb * L); D("jsjs", nbb * L); D("kk", nbb * L); D("ksks", nbb * L); }
	if (p->meas_thermal) {
		D("j2jn", (size_t)p->num_b2b * L); D("jnj2", (size_t)p->num_bb2 * L);
		D("jnjn", nbb * L); D("jnj", nbb * L); D("jjn", nbb * L);
	}
	if (p->meas_2bond_corr) {
		const size_t n4 = (size_t)p->num_b2b2 * L;
		D("pair_b2b2", n4); D("j2j2", n4); D("j2j", (size_t)p->num_b2b * L);
		D("jj2", (size_t)p->num_bb2 * L); D("js2js2", n4); D("k2k2", n4); D("ks2ks2", n4);
	}
	if (p->meas_energy_corr) { D("kv", nbs * L); D("kn", nbs * L); D("vv", nij * L); D("vn", nij * L); }
	if (p->meas_nematic_corr) { D("nem_nnnn", nbb * L); D("nem_ssss", nbb * L); }
#undef D
	return k;
}

static const char *mat_names[8] = {
	"params/exp_Ku", "params/exp_Kd", "params/inv_exp_Ku", "params/inv_exp_Kd",
	"params/exp_halfKu", "params/exp_halfKd", "params/inv_exp_halfKu", "params/inv_exp_halfKd"};


static void sim_free(struct sim *s)
{
	free(s->map_i); free(s->map_ij); free(s->bonds); free(s->map_bb);
	free(s->peierlsu); free(s->peierlsd);
	for (int i = 0; i < 8; i++) free(s->mats[i]);
	free(s->exp_lambda); free(s->del); free(s->hs);
	free(s->eq_acc); free(s->ue_acc);
	for (int i = 0; i < 9; i++) free(s->tmap[i]);
	for (int i = 0; i < 4; i++) free(s->pp[i]);
	memset(s, 0, sizeof(*s));
}

static int rd_num(dqsf_file *f, const char *name, double *dst, size_t n, int cplx)
{
	return cplx ? dqsf_read_c128(f, name, dst, n) : dqsf_read_f64(f, name, dst, n);
}

static int wr_num(dqsf_file *f, const char *name, const double *src, size_t n, int cplx)
{
	return cplx ? dqsf_write_c128(f, name, src, n) : dqsf_write_f64(f, name, src, n);
}

#define TRY(x) do { int rc_ = (x); if (rc_) { dqsf_close(f); sim_free(s); return rc_ < 0 ? rc_ : DQSF_RW_FAIL; } } while (0)

/* data.c:345-658 for the datasets this engine carries */
static int sim_read(struct sim *s)
{
	dqsf_file *f;
	int rc = dqsf_open(s->file, 0, &f);
	if (rc) return rc;
	int pw = 0;
	TRY(dqsf_read_int(f, "state/partial_write", &pw, 1));
	if (pw) {
		fprintf(stderr, "Last checkpoint in %s contained partial write\n", s->file);
		dqsf_close(f);
		return DQSF_CORRUPT_FAIL;
	}
	dqmc_params *p = &s->p;
	struct { const char *n; int *d; } sc[] = {
		{"params/N", &p->N}, {"params/L", &p->L}, {"params/n_matmul", &p->n_matmul},
		{"params/n_delay", &p->n_delay}, {"params/F", &p->F},
		{"params/n_sweep_warm", &p->n_sweep_warm}, {"params/n_sweep", &p->n_sweep},
		{"params/n_sweep_meas", &s->n_sweep_meas},
		{"params/period_eqlt", &p->period_eqlt}, {"params/period_uneqlt", &p->period_uneqlt},
		{"params/meas_bond_corr", &p->meas_bond_corr}, {"params/num_i", &p->num_i},
		{"params/num_ij", &p->num_ij}, {"params/num_b", &p->num_b}, {"params/num_bb", &p->num_bb},
		{"params/degen_i", &p->degen_i}, {"params/degen_ij", &p->degen_ij},
		{"params/degen_bb", &p->degen_bb}, {"params/checkpoint_every", &s->checkpoint_every},
		{"state/sweep", &s->sweep},
	};
	for (size_t i = 0; i < sizeof(sc) / sizeof(sc[0]); i++) TRY(dqsf_read_int(f, sc[i].n, sc[i].d, 1));
	/* the measurement toggles and the sizes of their maps (absent: 0) */
	int *tf[N_TOGGLE_INTS] = {&p->meas_energy_corr, &p->meas_thermal, &p->meas_2bond_corr,
		&p->meas_nematic_corr, &p->meas_chiral, &p->meas_local_JQ, &p->meas_gen_suscept,
		&p->meas_pair_bb_only, &p->Nx, &p->Ny, &p->num_plaq, &p->num_plaq_accum,
		&p->num_b_accum, &p->num_b2_accum, &p->num_bs, &p->num_b2, &p->num_b2b, &p->num_bb2,
		&p->num_b2b2, &p->degen_plaq, &p->degen_b, &p->degen_b2, &p->degen_bs, &p->degen_b2b,
		&p->degen_bb2, &p->degen_b2b2};
	for (int i = 0; i < N_TOGGLE_INTS; i++) {
		char nm[64];
		snprintf(nm, sizeof(nm), "params/%s", toggle_int_names[i]);
		*tf[i] = 0;
		if (dqsf_has(f, nm)) TRY(dqsf_read_int(f, nm, tf[i], 1));
	}
	/* files written without the two-hop bond family run with num_b2 = 0 */
	if (!dqsf_has(f, "params/bond2s") || !dqsf_has(f, "params/map_b2b2")) p->num_b2 = 0;
	int dt;
	size_t cnt;
	TRY(dqsf_info(f, "params/exp_Ku", &dt, &cnt));
	s->cplx = p->cplx = (dt == DQSF_C128);
	const size_t N = p->N, L = p->L, NN = N * N, w = s->cplx ? 2 : 1;
	s->map_i = calloc(N, sizeof(int));
	s->map_ij = calloc(NN, sizeof(int));
	TRY(dqsf_read_int(f, "params/map_i", s->map_i, N));
	TRY(dqsf_read_int(f, "params/map_ij", s->map_ij, NN));
	s->num_b_alloc = p->num_b > 0 ? p->num_b : 1;
	s->bonds = calloc(2 * (size_t)s->num_b_alloc, sizeof(int));
	s->map_bb = calloc((size_t)s->num_b_alloc * s->num_b_alloc, sizeof(int));
	/* the bonds and bond-pair map feed the bond correlators and most
	 * toggles: read them whenever the file has them */
	if (p->num_b > 0 && dqsf_has(f, "params/bonds"))
		TRY(dqsf_read_int(f, "params/bonds", s->bonds, 2 * (size_t)p->num_b));
	if (p->num_b > 0 && dqsf_has(f, "params/map_bb"))
		TRY(dqsf_read_int(f, "params/map_bb", s->map_bb, (size_t)p->num_b * p->num_b));
	s->peierlsu = calloc(NN * w, sizeof(double));
	s->peierlsd = calloc(NN * w, sizeof(double));
	TRY(rd_num(f, "params/peierlsu", s->peierlsu, NN, s->cplx));
	TRY(rd_num(f, "params/peierlsd", s->peierlsd, NN, s->cplx));
	for (int i = 0; i < 8; i++) {
		s->mats[i] = calloc(NN * w, sizeof(double));
		TRY(rd_num(f, mat_names[i], s->mats[i], NN, s->cplx));
	}
	s->exp_lambda = calloc(2 * N, sizeof(double));
	s->del = calloc(2 * N, sizeof(double));
	TRY(dqsf_read_f64(f, "params/exp_lambda", s->exp_lambda, 2 * N));
	TRY(dqsf_read_f64(f, "params/del", s->del, 2 * N));
	TRY(dqsf_read_u64(f, "state/rng", s->rng, 17));
	s->hs = calloc(N * L, sizeof(int));
	TRY(dqsf_read_int(f, "state/hs", s->hs, N * L));
	p->map_i = s->map_i; p->map_ij = s->map_ij; p->bonds = s->bonds; p->map_bb = s->map_bb;
	p->peierlsu = s->peierlsu; p->peierlsd = s->peierlsd;
	p->exp_Ku = s->mats[0]; p->exp_Kd = s->mats[1]; p->inv_exp_Ku = s->mats[2];
	p->inv_exp_Kd = s->mats[3]; p->exp_halfKu = s->mats[4]; p->exp_halfKd = s->mats[5];
	p->inv_exp_halfKu = s->mats[6]; p->inv_exp_halfKd = s->mats[7];
	/* the measurement toggles' maps and two-hop phases, where present */
	const size_t nb = p->num_b, nb2 = p->num_b2, npl = p->num_plaq;
	const size_t tmap_n[9] = {3 * npl, npl, nb, N * nb, 2 * nb2, nb2, nb * nb2, nb2 * nb, nb2 * nb2};
	for (int i = 0; i < 9; i++) {
		char nm[64];
		snprintf(nm, sizeof(nm), "params/%s", tmap_names[i]);
		if (tmap_n[i] == 0 || !dqsf_has(f, nm)) continue;
		s->tmap[i] = calloc(tmap_n[i], sizeof(int));
		TRY(dqsf_read_int(f, nm, s->tmap[i], tmap_n[i]));
	}
	for (int i = 0; i < 4; i++) {
		char nm[64];
		snprintf(nm, sizeof(nm), "params/%s", pp_names[i]);
		if (nb2 == 0 || !dqsf_has(f, nm)) continue;
		s->pp[i] = calloc(nb2 * w, sizeof(double));
		TRY(rd_num(f, nm, s->pp[i], nb2, s->cplx));
	}
	p->plaqs = s->tmap[0]; p->map_plaq = s->tmap[1]; p->map_b = s->tmap[2];
	p->map_bs = s->tmap[3]; p->bond2s = s->tmap[4]; p->map_b2 = s->tmap[5];
	p->map_bb2 = s->tmap[6]; p->map_b2b = s->tmap[7]; p->map_b2b2 = s->tmap[8];
	p->pp_u = s->pp[0]; p->pp_d = s->pp[1]; p->ppr_u = s->pp[2]; p->ppr_d = s->pp[3];
	dqmc_acc_sizes(p, &s->eq_size, &s->ue_size);
	s->eq_acc = calloc((size_t)s->eq_size * w, sizeof(double));
	s->ue_acc = calloc((size_t)(s->ue_size ? s->ue_size : 1) * w, sizeof(double));
	char name[128];
	struct dset ds[MAX_DSETS];
	TRY(dqsf_read_int(f, "meas_eqlt/n_sample", &s->eq_n, 1));
	TRY(rd_num(f, "meas_eqlt/sign", s->eq_acc, 1, s->cplx));
	size_t o = 1;
	for (int k = 0, n = acc_sets(p, 0, ds); k < n; o += ds[k].n, k++) {
		snprintf(name, sizeof(name), "meas_eqlt/%s", ds[k].name);
		TRY(rd_num(f, name, s->eq_acc + w * o, ds[k].n, s->cplx));
	}
	if (p->period_uneqlt > 0) {
		TRY(dqsf_read_int(f, "meas_uneqlt/n_sample", &s->ue_n, 1));
		TRY(rd_num(f, "meas_uneqlt/sign", s->ue_acc, 1, s->cplx));
		o = 1;
		for (int k = 0, n = acc_sets(p, 1, ds); k < n; o += ds[k].n, k++) {
			snprintf(name, sizeof(name), "meas_uneqlt/%s", ds[k].name);
			TRY(rd_num(f, name, s->ue_acc + w * o, ds[k].n, s->cplx));
		}
	}
	return dqsf_close(f);
}

#undef TRY
#define TRYW(x) do { if ((x) != 0) { dqsf_close(f); return DQSF_RW_FAIL; } } while (0)

/* data.c:667-789: partial_write set, state and accumulators, partial_write clear */
static int sim_save(const struct sim *s)
{
	dqsf_file *f;
	int rc = dqsf_open(s->file, 1, &f);
	if (rc) return rc;
	int pw = 0;
	TRYW(dqsf_read_int(f, "state/partial_write", &pw, 1));
	if (pw) {
		dqsf_close(f);
		return DQSF_CORRUPT_FAIL;
	}
	pw = 1;
	TRYW(dqsf_write_int(f, "state/partial_write", &pw, 1));
	fflush(NULL);
	const dqmc_params *p = &s->p;
	const size_t L = p->L, w = s->cplx ? 2 : 1;
	char name[128];
	struct dset ds[MAX_DSETS];
	TRYW(dqsf_write_u64(f, "state/rng", s->rng, 17));
	TRYW(dqsf_write_int(f, "state/sweep", &s->sweep, 1));
	TRYW(dqsf_write_int(f, "state/hs", s->hs, (size_t)p->N * L));
	TRYW(dqsf_write_int(f, "meas_eqlt/n_sample", &s->eq_n, 1));
	TRYW(wr_num(f, "meas_eqlt/sign", s->eq_acc, 1, s->cplx));
	size_t o = 1;
	for (int k = 0, n = acc_sets(p, 0, ds); k < n; o += ds[k].n, k++) {
		snprintf(name, sizeof(name), "meas_eqlt/%s", ds[k].name);
		TRYW(wr_num(f, name, s->eq_acc + w * o, ds[k].n, s->cplx));
	}
	if (p->period_uneqlt > 0) {
		TRYW(dqsf_write_int(f, "meas_uneqlt/n_sample", &s->ue_n, 1));
		TRYW(wr_num(f, "meas_uneqlt/sign", s->ue_acc, 1, s->cplx));
		o = 1;
		for (int k = 0, n = acc_sets(p, 1, ds); k < n; o += ds[k].n, k++) {
			snprintf(name, sizeof(name), "meas_uneqlt/%s", ds[k].name);
			TRYW(wr_num(f, name, s->ue_acc + w * o, ds[k].n, s->cplx));
		}
	}
	fflush(NULL);
	pw = 0;
	TRYW(dqsf_write_int(f, "state/partial_write", &pw, 1));
	return dqsf_close(f);
}

#undef TRYW

/* data.c:69-99 */
static int consistency_check(const char *file, FILE *log)
{
	dqsf_file *f;
	if (dqsf_open(file, 0, &f) != 0) return DQSF_OPEN_FAIL;
	char commit[256] = "";
	int rc = dqsf_read_str(f, "metadata/commit", commit, sizeof(commit));
	dqsf_close(f);
	if (rc) return rc;
	fprintf(log, "hdf5 generation script commit id %s\n", commit);
	return strcmp(commit, DQMC_GIT_ID);
}

/* estimate of the device memory one chain of this file needs */
static long long memory_req(const char *file)
{
	dqsf_file *f;
	if (dqsf_open(file, 0, &f) != 0) return DQSF_OPEN_FAIL;
	int N = 0, L = 0, F = 0, pu = 0, dt = 0;
	size_t cnt;
	if (dqsf_read_int(f, "params/N", &N, 1) || dqsf_read_int(f, "params/L", &L, 1) ||
	    dqsf_read_int(f, "params/F", &F, 1) || dqsf_read_int(f, "params/period_uneqlt", &pu, 1) ||
	    dqsf_info(f, "params/exp_Ku", &dt, &cnt)) {
		dqsf_close(f);
		return DQSF_RW_FAIL;
	}
	dqsf_close(f);
	const long long sz = dt == DQSF_C128 ? 16 : 8, NN = (long long)N * N;
	long long mats = 2 * (F + 9) * NN + 8 * NN;
	if (pu > 0) mats += 6 * (long long)L * NN + 4 * (long long)(F + 2) * (F + 2) * NN;
	return sz * mats + 4LL * L * N * 5;
}

/* ---------------------------------------------------------------- engine */

static int engine_from(struct sim **sims, int n, dqmc_engine **out)
{
	int rc = dqmc_engine_create(&sims[0]->p, n, 0, out);
	if (rc) return rc;
	/* the runtime forms of the reference's CHECK_G_WRP and CHECK_G_UE
	 * (dqmc.c:15-22), and with DQMC_CHECK_G=acc also CHECK_G_ACC */
	if (getenv("DQMC_CHECK_G")) {
		rc = dqmc_engine_check_g(*out, strcmp(getenv("DQMC_CHECK_G"), "acc") == 0 ? 3 : 1);
		if (rc) return rc;
	}
	for (int c = 0; c < n; c++) {
		struct sim *s = sims[c];
		rc = dqmc_engine_set_chain(*out, c, s->exp_lambda, s->del, s->rng, s->hs, s->sweep);
		if (!rc) rc = dqmc_engine_set_acc(*out, c, s->eq_n, s->eq_acc, s->ue_n, s->ue_acc);
		if (rc) return rc;
	}
	return dqmc_engine_init(*out);
}

/* the G drift of the check (DQMC_CHECK_G), per chain, in the wording of the
 * reference's matdiff lines (dqmc.c:61-71) */
static void log_drift(FILE *log, dqmc_engine *e, int n)
{
	if (!getenv("DQMC_CHECK_G") || n < 1) return;
	double *mx = malloc(sizeof(double) * 2 * (size_t)n);
	if (!mx) return;
	int cnt = 0;
	if (dqmc_engine_g_drift(e, mx, mx + n, &cnt) == 0)
		for (int c = 0; c < n; c++)
			fprintf(log, "chain %d: g - gwrp over %d recalculations:\tmax %.3e\tavg %.3e\n", c, cnt,
			        mx[c], mx[n + c]);
	if (dqmc_engine_g_drift_ue(e, mx, mx + n, &cnt) == 0 && cnt > 0)
		for (int c = 0; c < n; c++)
			fprintf(log, "chain %d: g - Gtt over %d unequal-time measurements:\tmax %.3e\tavg %.3e\n",
			        c, cnt, mx[c], mx[n + c]);
	if (dqmc_engine_g_drift_acc(e, mx, mx + n, &cnt) == 0)
		for (int c = 0; c < n; c++)
			fprintf(log, "chain %d: g - gacc over %d recalculations:\tmax %.3e\tavg %.3e\n", c, cnt,
			        mx[c], mx[n + c]);
	free(mx);
}

static int engine_pull(dqmc_engine *e, struct sim **sims, int n)
{
	for (int c = 0; c < n; c++) {
		struct sim *s = sims[c];
		int rc = dqmc_engine_get_chain(e, c, s->rng, s->hs, &s->sweep);
		if (!rc) rc = dqmc_engine_get_acc(e, c, &s->eq_n, s->eq_acc, &s->ue_n, s->ue_acc);
		if (rc) return rc;
	}
	return 0;
}

/* dqmc.c:222-244: per sweep, stop check then checkpoint then the sweep.
 * Returns 0 (done), 5 (interrupted) or 6 (checkpoint failed), or < 0. */
static int run_group(dqmc_engine *e, struct sim **sims, int n, struct stopper *stp,
		struct prof *pr)
{
	const dqmc_params *p = &sims[0]->p;
	int sweep = sims[0]->sweep;
	while (sweep < p->n_sweep) {
		if (check_stop(stp, sweep, p->n_sweep_warm, p->n_sweep)) return 5;
		const int ce = sims[0]->checkpoint_every;
		if (ce > 0 && sweep % ce == 0) {
			const int64_t t0 = time_wall();
			int rc = engine_pull(e, sims, n);
			for (int c = 0; rc == 0 && c < n; c++) rc = sim_save(sims[c]);
			pr->t[PR_CHECKPOINT] += time_wall() - t0;
			pr->n[PR_CHECKPOINT]++;
			if (rc) return 6;
		}
		const int64_t t0 = time_wall();
		int rc = dqmc_engine_sweeps(e, 1, 1);
		pr->t[PR_SWEEPS] += time_wall() - t0;
		pr->n[PR_SWEEPS]++;
		if (rc) return rc;
		sweep++;
	}
	return engine_pull(e, sims, n);
}

static FILE *open_log(const char *log_file)
{
	return log_file ? fopen(log_file, "a") : stdout;
}

static void log_header(FILE *log, const char *sim_file)
{
	fprintf(log, "executable commit id %s from repo %s\n", DQMC_GIT_ID, DQMC_REPO);
	fprintf(log, "compiled on %s %s\n", __DATE__, __TIME__);
	fprintf(log, "hdf5 and executable versions consistent? %s\n",
	        consistency_check(sim_file, log) ? "No" : "Yes");
	fprintf(log, "integer size on this system: %zu bytes\n", sizeof(int));
	fprintf(log, "measurements on the GPU (sm_100a engine)\n");
	const long long mem = memory_req(sim_file);
	if (mem < 0) fprintf(log, "minimum RAM check failed: %lld\n", mem);
	else fprintf(log, "minimum device memory requirement: %.2f MB\n", mem * 1e-6);
}

int dqmc_wrapper(const char *sim_file, const char *log_file, const int64_t max_time,
		const bool dry, const bool bench)
{
	const int64_t wall_start = time_wall();
	struct prof pr;
	memset(&pr, 0, sizeof(pr));
	FILE *log = open_log(log_file);
	if (log == NULL) {
		fprintf(stderr, "fopen() failed to open: %s\n", log_file);
		return WRAP_FAIL;
	}
	log_header(log, sim_file);
	if (dry) {
		fprintf(log, "toggled dry run for mem check only\n");
		fprintf(log, "Not performing: read sim file, alloc mem, run core DQMC logic, or save data\n");
		if (log != stdout) fclose(log); else fflush(log);
		return 0;
	}
	sig_init();
	struct stopper stp = {log, wall_start, max_time, 0, 0};
	int ret = 0;
	struct sim s;
	memset(&s, 0, sizeof(s));
	s.file = sim_file;
	fprintf(log, "opening %s\n", sim_file);
	struct stat info;
	if (stat(sim_file, &info) == 0)
		fprintf(log, "size of this hdf5 file: %.2f MB\n", ((double)info.st_size) * 1e-6);
	fflush(log);
	int64_t t0 = time_wall();
	const int rs = sim_read(&s);
	pr.t[PR_READ] += time_wall() - t0;
	pr.n[PR_READ]++;
	dqmc_engine *e = NULL;
	if (rs) {
		fprintf(log, "sim_data_read_alloc() failed: %d\n", rs);
		ret = WRAP_FAIL;
		goto cleanup;
	}
	if (s.checkpoint_every) fprintf(log, "checkpointing every %d sweeps\n", s.checkpoint_every);
	else fprintf(log, "warning: running with no checkpoints\n");
	fprintf(log, "%d/%d sweeps completed\n", s.sweep, s.p.n_sweep);
	if (s.sweep >= s.p.n_sweep) {
		fprintf(log, "already finished so don't do anything\n");
		goto cleanup;
	}
	time_t now;
	time(&now);
	fprintf(log, "[%.24s] starting dqmc\n", ctime(&now));
	fflush(log);
	t0 = time_wall();
	struct sim *one[1] = {&s};
	int rc = engine_from(one, 1, &e);
	pr.t[PR_INIT] += time_wall() - t0;
	pr.n[PR_INIT]++;
	if (rc) {
		fprintf(log, "engine setup failed: %d\n", rc);
		ret = WRAP_FAIL;
		goto cleanup;
	}
	rc = run_group(e, one, 1, &stp, &pr);
	log_drift(log, e, 1);
	if (rc == 5) {
		fprintf(log, "dqmc() interrupted\n");
		ret = WRAP_INCOMPLETE;
		goto cleanup;
	} else if (rc == 6) {
		fprintf(log, "dqmc() checkpoint failed\n");
		ret = WRAP_FAIL;
		goto cleanup;
	} else if (rc) {
		fprintf(log, "dqmc() failed on the device: %d (errors 0x%x)\n", rc, dqmc_engine_errors(e));
		ret = WRAP_FAIL;
		goto cleanup;
	}
	time(&now);
	fprintf(log, "[%.24s] %d/%d sweeps completed\n", ctime(&now), s.sweep, s.p.n_sweep);
	if (bench) {
		fprintf(log, "benchmark mode enabled; not saving data to disk\n");
		goto cleanup;
	}
	fprintf(log, "saving data to disk\n");
	t0 = time_wall();
	rc = sim_save(&s);
	pr.t[PR_SAVE] += time_wall() - t0;
	pr.n[PR_SAVE]++;
	if (rc < 0) {
		fprintf(log, "sim_data_save() failed: %d\n", rc);
		ret = WRAP_FAIL;
		goto cleanup;
	}
	fprintf(log, "sim_data_save() succeeded\n");
cleanup:
	dqmc_engine_destroy(e);
	sim_free(&s);
	pr.t[PR_WALL] = time_wall() - wall_start;
	pr.n[PR_WALL] = 1;
	fprintf(log, "wall time: %.3f\n", pr.t[PR_WALL] * 1e-9);
	prof_print(log, &pr);
	if (log != stdout) fclose(log); else fflush(log);
	return ret;
}

/* files whose parameter sets are byte-identical and whose sweep counters
 * agree can share an engine */
static int same_group(const struct sim *a, const struct sim *b)
{
	const dqmc_params *p = &a->p, *q = &b->p;
	if (memcmp(&p->N, &q->N, sizeof(int) * 18) != 0 ||
	    memcmp(&p->meas_energy_corr, &q->meas_energy_corr, sizeof(int) * N_TOGGLE_INTS) != 0 ||
	    a->sweep != b->sweep ||
	    a->checkpoint_every != b->checkpoint_every)
		return 0;
	const size_t NN = (size_t)p->N * p->N, w = a->cplx ? 2 : 1;
	for (int i = 0; i < 8; i++)
		if (memcmp(a->mats[i], b->mats[i], NN * w * sizeof(double))) return 0;
	if (memcmp(a->map_ij, b->map_ij, NN * sizeof(int)) || memcmp(a->map_i, b->map_i, p->N * sizeof(int)))
		return 0;
	if (memcmp(a->peierlsu, b->peierlsu, NN * w * sizeof(double))) return 0;
	return 1;
}

int dqmc_wrapper_batch(int n_files, const char *const *sim_files, const char *log_file,
		const int64_t max_time, const bool bench, int *status)
{
	if (n_files < 1 || !sim_files || !status) return WRAP_FAIL;
	const int64_t wall_start = time_wall();
	struct prof pr;
	memset(&pr, 0, sizeof(pr));
	FILE *log = open_log(log_file);
	if (!log) return WRAP_FAIL;
	sig_init();
	struct stopper stp = {log, wall_start, max_time, 0, 0};
	struct sim *sims = calloc(n_files, sizeof(struct sim));
	int *group = calloc(n_files, sizeof(int));
	int worst = 0;
	for (int i = 0; i < n_files; i++) {
		sims[i].file = sim_files[i];
		status[i] = 0;
		group[i] = -1;
		const int rc = sim_read(&sims[i]);
		if (rc) {
			fprintf(log, "%s: read failed: %d\n", sim_files[i], rc);
			status[i] = WRAP_FAIL;
		}
	}
	/* group the readable, unfinished files */
	int ng = 0;
	for (int i = 0; i < n_files; i++) {
		if (status[i] || group[i] >= 0) continue;
		if (sims[i].sweep >= sims[i].p.n_sweep) continue;
		group[i] = ng;
		for (int j = i + 1; j < n_files; j++)
			if (!status[j] && group[j] < 0 && same_group(&sims[i], &sims[j])) group[j] = ng;
		ng++;
	}
	fprintf(log, "%d files in %d parameter groups\n", n_files, ng);
	/* one engine (and CUDA stream) per group; each round queues one sweep
	 * of every unfinished group on its own stream, so that groups of
	 * different lattices, L or n_delay run concurrently, then waits for all */
	struct grp {
		dqmc_engine *e;
		struct sim **m;
		int *idx;
		int n, rc, done, queued;
	};
	struct grp *gs = calloc(ng > 0 ? ng : 1, sizeof(struct grp));
	for (int gi = 0; gi < ng; gi++) {
		struct grp *g = &gs[gi];
		for (int i = 0; i < n_files; i++) g->n += group[i] == gi;
		g->m = calloc(g->n, sizeof(struct sim *));
		g->idx = calloc(g->n, sizeof(int));
		int n = 0;
		for (int i = 0; i < n_files; i++)
			if (group[i] == gi) { g->idx[n] = i; g->m[n++] = &sims[i]; }
		const int64_t t0 = time_wall();
		g->rc = engine_from(g->m, g->n, &g->e);
		pr.t[PR_INIT] += time_wall() - t0;
		pr.n[PR_INIT]++;
	}
	/* every round of all groups as one CUDA graph launch (dqmc_batch) while
	 * every unfinished group sweeps; per-group launches otherwise */
	dqmc_batch *batch = NULL;
	{
		int ok = ng > 0;
		dqmc_engine **es = calloc(ng > 0 ? ng : 1, sizeof(dqmc_engine *));
		for (int gi = 0; ok && gi < ng; gi++) {
			if (gs[gi].rc || !gs[gi].e) ok = 0;
			else es[gi] = gs[gi].e;
		}
		if (ok && es && dqmc_batch_create(es, ng, &batch) != 0) batch = NULL;
		free(es);
	}
	for (;;) {
		int active = 0;
		const int64_t t0 = time_wall();
		for (int gi = 0; gi < ng; gi++) {
			struct grp *g = &gs[gi];
			g->queued = 0;
			if (g->done || g->rc) continue;
			const dqmc_params *p = &g->m[0]->p;
			const int sweep = g->m[0]->sweep;
			if (sweep >= p->n_sweep) { g->done = 1; continue; }
			if (check_stop(&stp, sweep, p->n_sweep_warm, p->n_sweep)) { g->rc = 5; continue; }
			const int ce = g->m[0]->checkpoint_every;
			if (ce > 0 && sweep % ce == 0) {
				const int64_t tc = time_wall();
				int rc = engine_pull(g->e, g->m, g->n);
				for (int c = 0; rc == 0 && c < g->n; c++) rc = sim_save(g->m[c]);
				pr.t[PR_CHECKPOINT] += time_wall() - tc;
				pr.n[PR_CHECKPOINT]++;
				if (rc) { g->rc = 6; continue; }
			}
			g->queued = 1;
			active = 1;
		}
		if (!active) break;
		int whole = batch != NULL;
		for (int gi = 0; gi < ng; gi++)
			if (!gs[gi].queued && !gs[gi].done) whole = 0;   /* stopped or failed */
		if (whole) {
			const int rc = dqmc_batch_sweeps(batch, 1, 1);
			for (int gi = 0; rc && gi < ng; gi++)
				if (gs[gi].queued) gs[gi].rc = rc;
		} else {
			for (int gi = 0; gi < ng; gi++)
				if (gs[gi].queued) gs[gi].rc = dqmc_engine_sweeps(gs[gi].e, 1, 0);
		}
		for (int gi = 0; gi < ng; gi++) {
			struct grp *g = &gs[gi];
			if (!g->queued || g->rc) continue;
			if (!whole) g->rc = dqmc_engine_sync(g->e);
			if (g->rc) continue;
			for (int c = 0; c < g->n; c++) g->m[c]->sweep++;
		}
		pr.t[PR_SWEEPS] += time_wall() - t0;
		pr.n[PR_SWEEPS]++;
	}
	dqmc_batch_destroy(batch);   /* before its engines */
	for (int gi = 0; gi < ng; gi++) {
		struct grp *g = &gs[gi];
		int rc = g->rc;
		if (!rc && g->e) rc = engine_pull(g->e, g->m, g->n);
		int st = 0;
		if (rc == 5) st = WRAP_INCOMPLETE;
		else if (rc) st = WRAP_FAIL;
		if (st == 0 && !bench)
			for (int k = 0; k < g->n; k++)
				if (sim_save(g->m[k]) < 0) status[g->idx[k]] = WRAP_FAIL;
		for (int k = 0; k < g->n; k++)
			if (!status[g->idx[k]]) status[g->idx[k]] = st;
		fprintf(log, "group %d: %d chains, status %d\n", gi, g->n, st);
		if (g->e) dqmc_engine_destroy(g->e);
		free(g->m);
		free(g->idx);
	}
	free(gs);
	for (int i = 0; i < n_files; i++) {
		if (status[i] == WRAP_FAIL) worst = WRAP_FAIL;
		else if (status[i] == WRAP_INCOMPLETE && worst == 0) worst = WRAP_INCOMPLETE;
		sim_free(&sims[i]);
	}
	free(sims);
	free(group);
	pr.t[PR_WALL] = time_wall() - wall_start;
	pr.n[PR_WALL] = 1;
	fprintf(log, "wall time: %.3f\n", pr.t[PR_WALL] * 1e-9);
	prof_print(log, &pr);
	if (log != stdout) fclose(log); else fflush(log);
	return worst;
}
