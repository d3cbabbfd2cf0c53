/*
 * Replacement for the reference's src/data.c (the only reference file that
 * needs libhdf5), implementing the same data.h interface over the DQSF
 * container.  It reads and writes the dataset list of data.c:345-789, keeps
 * the partial_write protocol (data.c:353-357, 676-686, 781-783) and the
 * error codes (data.c:10-13).  Test-side build glue for the reference
 * checker in oracle/_ref; the engine has its own host layer.
 */
#include <stdio.h>
#include <string.h>
#include <complex.h>

#include "data.h"
#include "simfile.h"

#ifdef USE_CPLX
#define read_num(f, name, dst, n) dqsf_read_c128((f), (name), (double *)(dst), (n))
#define write_num(f, name, src, n) dqsf_write_c128((f), (name), (const double *)(src), (n))
#else
#define read_num(f, name, dst, n) dqsf_read_f64((f), (name), (dst), (n))
#define write_num(f, name, src, n) dqsf_write_f64((f), (name), (src), (n))
#endif

#define RD(expr) do { if ((expr) != 0) { dqsf_close(fp); return DQSF_RW_FAIL; } } while (0)

int set_num_h5t(void) { return 0; }

int consistency_check(const char *file, FILE *log)
{
	dqsf_file *fp;
	if (dqsf_open(file, 0, &fp) != 0) return DQSF_OPEN_FAIL;
	char commit[256] = "";
	RD(dqsf_read_str(fp, "metadata/commit", commit, sizeof(commit)));
	fprintf(log, "hdf5 generation script commit id %s\n", commit);
	dqsf_close(fp);
	return strcmp(commit, GIT_ID);
}

int get_memory_req(const char *file)
{
	dqsf_file *fp;
	if (dqsf_open(file, 0, &fp) != 0) return DQSF_OPEN_FAIL;
	int N, L, F, num_ij;
	RD(dqsf_read_int(fp, "params/N", &N, 1));
	RD(dqsf_read_int(fp, "params/L", &L, 1));
	RD(dqsf_read_int(fp, "params/F", &F, 1));
	RD(dqsf_read_int(fp, "params/num_ij", &num_ij, 1));
	dqsf_close(fp);
	/* dominant terms of data.c:112-335: B, iB for both spins, C, G */
	const size_t bytes = sizeof(num) * ((size_t)N * N * (4 * (size_t)L + 2 * (size_t)F + 16)
	                                    + (size_t)num_ij * 16);
	return (int)bytes;
}

struct ientry { const char *name; int *dst; size_t n; };
struct nentry { const char *name; num *dst; size_t n; };

/* Every array measurement dataset of data.c:441-522 with the toggle that
 * enables it: the one list that allocation, read, save and free walk (the
 * scalar n_sample and sign are handled beside it). */
#define MEAS_MAX 64
struct mentry { const char *name; num **dst; size_t n; int on; };

static int meas_table(struct sim_data *sim, struct mentry *m)
{
	const struct params *p = &sim->p;
	struct meas_eqlt *e = &sim->m_eq;
	struct meas_uneqlt *u = &sim->m_ue;
	const size_t L = p->L, ni = p->num_i, nij = p->num_ij, nbb = p->num_bb, nbs = p->num_bs;
	const size_t nba = p->num_b_accum, nb2a = p->num_b2_accum, npa = p->num_plaq_accum;
	const size_t nb2b = p->num_b2b, nbb2 = p->num_bb2, nb2b2 = p->num_b2b2;
	const int ue = p->period_uneqlt > 0;
	int k = 0;
#define M(nm, ptr, cnt, cond) m[k++] = (struct mentry){nm, &(ptr), (cnt), (cond)}
	M("meas_eqlt/density", e->density, ni, 1);
	M("meas_eqlt/density_u", e->density_u, ni, 1);
	M("meas_eqlt/density_d", e->density_d, ni, 1);
	M("meas_eqlt/double_occ", e->double_occ, ni, 1);
	M("meas_eqlt/g00", e->g00, nij, 1);
	M("meas_eqlt/g00_u", e->g00_u, nij, 1);
	M("meas_eqlt/g00_d", e->g00_d, nij, 1);
	M("meas_eqlt/nn", e->nn, nij, 1);
	M("meas_eqlt/xx", e->xx, nij, 1);
	M("meas_eqlt/zz", e->zz, nij, 1);
	M("meas_eqlt/pair_sw", e->pair_sw, nij, 1);
	M("meas_eqlt/uuuu", e->uuuu, nij * nij, p->meas_gen_suscept);
	M("meas_eqlt/dddd", e->dddd, nij * nij, p->meas_gen_suscept);
	M("meas_eqlt/dduu", e->dduu, nij * nij, p->meas_gen_suscept);
	M("meas_eqlt/uudd", e->uudd, nij * nij, p->meas_gen_suscept);
	M("meas_eqlt/chi", e->chi, npa, p->meas_chiral);
	M("meas_eqlt/kk", e->kk, nbb, p->meas_energy_corr);
	M("meas_eqlt/kv", e->kv, nbs, p->meas_energy_corr);
	M("meas_eqlt/kn", e->kn, nbs, p->meas_energy_corr);
	M("meas_eqlt/vv", e->vv, nij, p->meas_energy_corr);
	M("meas_eqlt/vn", e->vn, nij, p->meas_energy_corr);
	M("meas_eqlt/j", e->j, nba, p->meas_local_JQ);
	M("meas_eqlt/jn", e->jn, nba, p->meas_local_JQ);
	M("meas_eqlt/j2", e->j2, nb2a, p->meas_local_JQ);
	M("meas_uneqlt/gt0", u->gt0, nij * L, ue);
	M("meas_uneqlt/gt0_u", u->gt0_u, nij * L, ue);
	M("meas_uneqlt/gt0_d", u->gt0_d, nij * L, ue);
	M("meas_uneqlt/nn", u->nn, nij * L, ue);
	M("meas_uneqlt/xx", u->xx, nij * L, ue);
	M("meas_uneqlt/zz", u->zz, nij * L, ue);
	M("meas_uneqlt/pair_sw", u->pair_sw, nij * L, ue);
	M("meas_uneqlt/uuuu", u->uuuu, nij * nij * L, ue && p->meas_gen_suscept);
	M("meas_uneqlt/dddd", u->dddd, nij * nij * L, ue && p->meas_gen_suscept);
	M("meas_uneqlt/dduu", u->dduu, nij * nij * L, ue && p->meas_gen_suscept);
	M("meas_uneqlt/uudd", u->uudd, nij * nij * L, ue && p->meas_gen_suscept);
	M("meas_uneqlt/pair_bb", u->pair_bb, nbb * L, ue && (p->meas_bond_corr || p->meas_pair_bb_only));
	M("meas_uneqlt/jj", u->jj, nbb * L, ue && p->meas_bond_corr);
	M("meas_uneqlt/jsjs", u->jsjs, nbb * L, ue && p->meas_bond_corr);
	M("meas_uneqlt/kk", u->kk, nbb * L, ue && p->meas_bond_corr);
	M("meas_uneqlt/ksks", u->ksks, nbb * L, ue && p->meas_bond_corr);
	M("meas_uneqlt/j2jn", u->j2jn, nb2b * L, ue && p->meas_thermal);
	M("meas_uneqlt/jnj2", u->jnj2, nbb2 * L, ue && p->meas_thermal);
	M("meas_uneqlt/jnjn", u->jnjn, nbb * L, ue && p->meas_thermal);
	M("meas_uneqlt/jnj", u->jnj, nbb * L, ue && p->meas_thermal);
	M("meas_uneqlt/jjn", u->jjn, nbb * L, ue && p->meas_thermal);
	M("meas_uneqlt/pair_b2b2", u->pair_b2b2, nb2b2 * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/j2j2", u->j2j2, nb2b2 * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/j2j", u->j2j, nb2b * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/jj2", u->jj2, nbb2 * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/js2js2", u->js2js2, nb2b2 * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/k2k2", u->k2k2, nb2b2 * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/ks2ks2", u->ks2ks2, nb2b2 * L, ue && p->meas_2bond_corr);
	M("meas_uneqlt/kv", u->kv, nbs * L, ue && p->meas_energy_corr);
	M("meas_uneqlt/kn", u->kn, nbs * L, ue && p->meas_energy_corr);
	M("meas_uneqlt/vv", u->vv, nij * L, ue && p->meas_energy_corr);
	M("meas_uneqlt/vn", u->vn, nij * L, ue && p->meas_energy_corr);
	M("meas_uneqlt/nem_nnnn", u->nem_nnnn, nbb * L, ue && p->meas_nematic_corr);
	M("meas_uneqlt/nem_ssss", u->nem_ssss, nbb * L, ue && p->meas_nematic_corr);
#undef M
	return k;
}

int sim_data_read_alloc(struct sim_data *sim)
{
	dqsf_file *fp;
	const int orc = dqsf_open(sim->file, 0, &fp);
	if (orc != 0) return orc;
	int partial_write = 0;
	RD(dqsf_read_int(fp, "state/partial_write", &partial_write, 1));
	if (partial_write) {
		fprintf(stderr, "Last checkpoint in %s contained partial write\n", sim->file);
		dqsf_close(fp);
		return DQSF_CORRUPT_FAIL;
	}
	struct params *p = &sim->p;
	const struct ientry scalars[] = {
		{"params/N", &p->N, 1}, {"params/L", &p->L, 1}, {"params/Nx", &p->Nx, 1},
		{"params/Ny", &p->Ny, 1}, {"params/num_i", &p->num_i, 1},
		{"params/num_ij", &p->num_ij, 1}, {"params/num_plaq_accum", &p->num_plaq_accum, 1},
		{"params/num_b_accum", &p->num_b_accum, 1}, {"params/num_b2_accum", &p->num_b2_accum, 1},
		{"params/num_plaq", &p->num_plaq, 1}, {"params/num_b", &p->num_b, 1},
		{"params/num_b2", &p->num_b2, 1}, {"params/num_bs", &p->num_bs, 1},
		{"params/num_bb", &p->num_bb, 1}, {"params/num_b2b", &p->num_b2b, 1},
		{"params/num_bb2", &p->num_bb2, 1}, {"params/num_b2b2", &p->num_b2b2, 1},
		{"params/degen_i", &p->degen_i, 1}, {"params/degen_ij", &p->degen_ij, 1},
		{"params/degen_plaq", &p->degen_plaq, 1}, {"params/degen_b", &p->degen_b, 1},
		{"params/degen_b2", &p->degen_b2, 1}, {"params/degen_bs", &p->degen_bs, 1},
		{"params/degen_bb", &p->degen_bb, 1}, {"params/degen_b2b", &p->degen_b2b, 1},
		{"params/degen_bb2", &p->degen_bb2, 1}, {"params/degen_b2b2", &p->degen_b2b2, 1},
		{"params/period_uneqlt", &p->period_uneqlt, 1},
		{"params/meas_bond_corr", &p->meas_bond_corr, 1},
		{"params/meas_thermal", &p->meas_thermal, 1},
		{"params/meas_2bond_corr", &p->meas_2bond_corr, 1},
		{"params/meas_local_JQ", &p->meas_local_JQ, 1},
		{"params/meas_gen_suscept", &p->meas_gen_suscept, 1},
		{"params/meas_energy_corr", &p->meas_energy_corr, 1},
		{"params/meas_nematic_corr", &p->meas_nematic_corr, 1},
		{"params/meas_pair_bb_only", &p->meas_pair_bb_only, 1},
		{"params/meas_chiral", &p->meas_chiral, 1},
		{"params/checkpoint_every", &p->checkpoint_every, 1},
		{"params/n_matmul", &p->n_matmul, 1}, {"params/n_delay", &p->n_delay, 1},
		{"params/n_sweep_warm", &p->n_sweep_warm, 1},
		{"params/n_sweep_meas", &p->n_sweep_meas, 1},
		{"params/period_eqlt", &p->period_eqlt, 1}, {"params/F", &p->F, 1},
		{"params/n_sweep", &p->n_sweep, 1}, {"state/sweep", &sim->s.sweep, 1},
	};
	for (size_t i = 0; i < sizeof(scalars) / sizeof(scalars[0]); i++)
		RD(dqsf_read_int(fp, scalars[i].name, scalars[i].dst, 1));

	/* the two-bond family (bond2s, map_b2*, pp_*) feeds only the thermal and
	 * two-bond correlators; files written without it run with num_b2 = 0 */
	if (!dqsf_has(fp, "params/bond2s") || !dqsf_has(fp, "params/map_b2b2")) p->num_b2 = 0;
	const size_t N = p->N, L = p->L;
	const size_t num_b = p->num_b, num_b2 = p->num_b2, num_plaq = p->num_plaq;
	p->map_i = my_calloc(N * sizeof(int));
	p->map_ij = my_calloc(N * N * sizeof(int));
	p->bonds = my_calloc(num_b * 2 * sizeof(int));
	p->map_bb = my_calloc(num_b * num_b * sizeof(int));
	p->bond2s = my_calloc(num_b2 * 2 * sizeof(int));
	p->plaqs = my_calloc(num_plaq * 3 * sizeof(int));
	p->map_plaq = my_calloc(num_plaq * sizeof(int));
	p->map_b = my_calloc(num_b * sizeof(int));
	p->map_b2 = my_calloc(num_b2 * sizeof(int));
	p->map_bs = my_calloc(num_b * N * sizeof(int));
	p->map_b2b2 = my_calloc(num_b2 * num_b2 * sizeof(int));
	p->map_b2b = my_calloc(num_b2 * num_b * sizeof(int));
	p->map_bb2 = my_calloc(num_b * num_b2 * sizeof(int));
	p->pp_u = my_calloc(num_b2 * sizeof(num));
	p->pp_d = my_calloc(num_b2 * sizeof(num));
	p->ppr_u = my_calloc(num_b2 * sizeof(num));
	p->ppr_d = my_calloc(num_b2 * sizeof(num));
	p->peierlsu = my_calloc(N * N * sizeof(num));
	p->peierlsd = my_calloc(N * N * sizeof(num));
	p->exp_Ku = my_calloc(N * N * sizeof(num));
	p->exp_Kd = my_calloc(N * N * sizeof(num));
	p->inv_exp_Ku = my_calloc(N * N * sizeof(num));
	p->inv_exp_Kd = my_calloc(N * N * sizeof(num));
	p->exp_halfKu = my_calloc(N * N * sizeof(num));
	p->exp_halfKd = my_calloc(N * N * sizeof(num));
	p->inv_exp_halfKu = my_calloc(N * N * sizeof(num));
	p->inv_exp_halfKd = my_calloc(N * N * sizeof(num));
	p->exp_lambda = my_calloc(N * 2 * sizeof(double));
	p->del = my_calloc(N * 2 * sizeof(double));
	sim->s.hs = my_calloc(N * L * sizeof(int));
	struct mentry m[MEAS_MAX];
	const int nm = meas_table(sim, m);
	for (int i = 0; i < nm; i++)
		if (m[i].on) *m[i].dst = my_calloc(m[i].n * sizeof(num));
	const struct ientry iarrays[] = {
		{"params/map_i", p->map_i, N}, {"params/map_ij", p->map_ij, N * N},
		{"params/bonds", p->bonds, num_b * 2}, {"params/map_bb", p->map_bb, num_b * num_b},
		{"params/bond2s", p->bond2s, num_b2 * 2}, {"params/plaqs", p->plaqs, num_plaq * 3},
		{"params/map_plaq", p->map_plaq, num_plaq}, {"params/map_b", p->map_b, num_b},
		{"params/map_b2", p->map_b2, num_b2}, {"params/map_bs", p->map_bs, num_b * N},
		{"params/map_b2b2", p->map_b2b2, num_b2 * num_b2},
		{"params/map_b2b", p->map_b2b, num_b2 * num_b},
		{"params/map_bb2", p->map_bb2, num_b * num_b2},
		{"state/hs", sim->s.hs, N * L},
	};
	for (size_t i = 0; i < sizeof(iarrays) / sizeof(iarrays[0]); i++)
		if (iarrays[i].n > 0 && dqsf_has(fp, iarrays[i].name))
			RD(dqsf_read_int(fp, iarrays[i].name, iarrays[i].dst, iarrays[i].n));
	const struct nentry narrays[] = {
		{"params/peierlsu", p->peierlsu, N * N}, {"params/peierlsd", p->peierlsd, N * N},
		{"params/exp_Ku", p->exp_Ku, N * N}, {"params/exp_Kd", p->exp_Kd, N * N},
		{"params/inv_exp_Ku", p->inv_exp_Ku, N * N}, {"params/inv_exp_Kd", p->inv_exp_Kd, N * N},
		{"params/exp_halfKu", p->exp_halfKu, N * N}, {"params/exp_halfKd", p->exp_halfKd, N * N},
		{"params/inv_exp_halfKu", p->inv_exp_halfKu, N * N},
		{"params/inv_exp_halfKd", p->inv_exp_halfKd, N * N},
		{"params/pp_u", p->pp_u, num_b2}, {"params/pp_d", p->pp_d, num_b2},
		{"params/ppr_u", p->ppr_u, num_b2}, {"params/ppr_d", p->ppr_d, num_b2},
	};
	for (size_t i = 0; i < sizeof(narrays) / sizeof(narrays[0]); i++)
		if (narrays[i].n > 0)
			RD(read_num(fp, narrays[i].name, narrays[i].dst, narrays[i].n));
	RD(dqsf_read_f64(fp, "params/exp_lambda", p->exp_lambda, N * 2));
	RD(dqsf_read_f64(fp, "params/del", p->del, N * 2));
	RD(dqsf_read_u64(fp, "state/rng", sim->s.rng, 17));
	RD(dqsf_read_int(fp, "meas_eqlt/n_sample", &sim->m_eq.n_sample, 1));
	RD(read_num(fp, "meas_eqlt/sign", &sim->m_eq.sign, 1));
	if (p->period_uneqlt > 0) {
		RD(dqsf_read_int(fp, "meas_uneqlt/n_sample", &sim->m_ue.n_sample, 1));
		RD(read_num(fp, "meas_uneqlt/sign", &sim->m_ue.sign, 1));
	}
	for (int i = 0; i < nm; i++)
		if (m[i].on) RD(read_num(fp, m[i].name, *m[i].dst, m[i].n));
	return dqsf_close(fp);
}

#define WR(expr) do { if ((expr) != 0) { dqsf_close(fp); return DQSF_RW_FAIL; } } while (0)

int sim_data_save(const struct sim_data *sim)
{
	dqsf_file *fp;
	const int orc = dqsf_open(sim->file, 1, &fp);
	if (orc != 0) return orc;
	int partial_write = 0;
	WR(dqsf_read_int(fp, "state/partial_write", &partial_write, 1));
	if (partial_write) {
		dqsf_close(fp);
		return DQSF_CORRUPT_FAIL;
	}
	partial_write = 1;
	WR(dqsf_write_int(fp, "state/partial_write", &partial_write, 1));
	fflush(NULL);
	const struct params *p = &sim->p;
	WR(dqsf_write_u64(fp, "state/rng", sim->s.rng, 17));
	WR(dqsf_write_int(fp, "state/sweep", &sim->s.sweep, 1));
	WR(dqsf_write_int(fp, "state/hs", sim->s.hs, (size_t)p->N * p->L));
	WR(dqsf_write_int(fp, "meas_eqlt/n_sample", &sim->m_eq.n_sample, 1));
	WR(write_num(fp, "meas_eqlt/sign", (num *)&sim->m_eq.sign, 1));
	if (p->period_uneqlt > 0) {
		WR(dqsf_write_int(fp, "meas_uneqlt/n_sample", &sim->m_ue.n_sample, 1));
		WR(write_num(fp, "meas_uneqlt/sign", (num *)&sim->m_ue.sign, 1));
	}
	struct mentry m[MEAS_MAX];
	const int nm = meas_table((struct sim_data *)sim, m);
	for (int i = 0; i < nm; i++)
		if (m[i].on) WR(write_num(fp, m[i].name, *m[i].dst, m[i].n));
	fflush(NULL);
	partial_write = 0;
	WR(dqsf_write_int(fp, "state/partial_write", &partial_write, 1));
	return dqsf_close(fp);
}

void sim_data_free(const struct sim_data *sim)
{
	const struct params *p = &sim->p;
	struct mentry m[MEAS_MAX];
	const int nm = meas_table((struct sim_data *)sim, m);
	for (int i = 0; i < nm; i++)
		if (m[i].on) my_free(*m[i].dst);
	my_free(sim->s.hs); my_free(p->del); my_free(p->exp_lambda);
	my_free(p->inv_exp_halfKd); my_free(p->inv_exp_halfKu); my_free(p->exp_halfKd);
	my_free(p->exp_halfKu); my_free(p->inv_exp_Kd); my_free(p->inv_exp_Ku);
	my_free(p->exp_Kd); my_free(p->exp_Ku); my_free(p->peierlsd); my_free(p->peierlsu);
	my_free(p->pp_u); my_free(p->pp_d); my_free(p->ppr_u); my_free(p->ppr_d);
	my_free(p->map_bb2); my_free(p->map_b2b); my_free(p->map_b2b2); my_free(p->map_bs);
	my_free(p->map_b2); my_free(p->map_b); my_free(p->map_plaq);
	my_free(p->plaqs); my_free(p->bond2s); my_free(p->map_bb); my_free(p->bonds);
	my_free(p->map_ij); my_free(p->map_i);
}
