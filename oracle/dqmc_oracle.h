/*
 * CPU oracle for the DQMC sweep: a plain-C restatement of the reference's
 * hot path (katherineding/dqmc-dev src/{rand.h,updates.c,greens.c,meas.c,
 * dqmc.c}).  TEST INFRASTRUCTURE ONLY: tests, the smoke check and the
 * benchmark's CPU baseline call it as the checker; the engine never links it.
 *
 * The same source builds a real library (liboracle_r.so, num = double) and a
 * complex one (liboracle_c.so, num = double complex, -DORACLE_CPLX), as the
 * reference builds dqmc_*_r and dqmc_*_c.  Matrices are column-major with
 * leading dimension N unless stated; `num` arrays are passed as void*.
 */
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* rand.h:6-31 and util/gen_util_shared.py:12-66 */
uint64_t orc_rand_uint(uint64_t *rng);
double orc_rand_doub(uint64_t *rng);
void orc_shuffle(uint64_t *rng, int n, int *a);
void orc_seed_splitmix64(uint64_t seed, uint64_t *rng);
void orc_rand_jump(uint64_t *rng);

/* In-memory simulation: parameters, state and accumulators, mirroring
 * struct params / state / meas_eqlt / meas_uneqlt (data.h:7-105) for the
 * always-on measurements plus the bond correlators. */
struct orc_sim {
	int N, L, n_matmul, n_delay, F, n_sweep_warm, n_sweep;
	int period_eqlt, period_uneqlt, meas_bond_corr;
	int num_i, num_ij, num_b, num_bb, degen_i, degen_ij, degen_bb;
	const int *map_i, *map_ij, *bonds, *map_bb;
	const void *peierlsu, *peierlsd;
	const void *exp_Ku, *exp_Kd, *inv_exp_Ku, *inv_exp_Kd;
	const void *exp_halfKu, *exp_halfKd, *inv_exp_halfKu, *inv_exp_halfKd;
	const double *exp_lambda, *del;
	/* state */
	uint64_t *rng;
	int *sweep;
	int *hs;            /* [L][N] */
	/* equal-time accumulators */
	int *eq_n_sample;
	void *eq_sign, *density, *density_u, *density_d, *double_occ;
	void *g00, *g00_u, *g00_d, *eq_nn, *eq_xx, *eq_zz, *eq_pair_sw;
	/* unequal-time accumulators ([L][num_ij] or [L][num_bb]) */
	int *ue_n_sample;
	void *ue_sign, *gt0, *gt0_u, *gt0_d, *ue_nn, *ue_xx, *ue_zz, *ue_pair_sw;
	void *pair_bb, *jj, *jsjs, *kk, *ksks;
};

/* dqmc.c:84-511 without I/O: run sweeps until *sweep == stop_sweep.
 * If phase_out is non-NULL it receives the phase after the last slice. */
int orc_dqmc(struct orc_sim *sim, int stop_sweep, void *gu_out, void *gd_out,
		void *phase_out);

/* dqmc.c:29-59: B_l = exp_K diag(exp_lambda[hs]) and its inverse for all
 * slices of one spin (spin 0 = up uses hs, spin 1 = down uses !hs). */
void orc_build_B(int N, int L, const void *exp_K, const double *exp_lambda,
		const int *hs, int spin, void *B);
void orc_build_iB(int N, int L, const void *inv_exp_K, const double *exp_lambda,
		const int *hs, int spin, void *iB);

/* greens.c:8-41 */
void orc_mul_seq(int N, int L, int min, int maxp1, const void *alpha,
		const void *B, void *A, int ldA);
/* greens.c:69-208: returns the phase through phase_out */
void orc_calc_eq_g(int l, int N, int L, int n_mul, const void *B, void *g,
		void *phase_out);
/* greens.c:471-494 (with calc_o, bsofi, expand_g) */
void orc_calc_ue_g(int N, int L, int F, int n_mul, const void *B, const void *iB,
		const void *C, void *G0t, void *Gtt, void *Gt0);
/* updates.c:7-84 */
void orc_update_delayed(int N, int n_delay, const double *del, const int *site_order,
		uint64_t *rng, int *hs, void *gu, void *gd, void *phase);
/* meas.c:66-120 (always-on part) */
void orc_measure_eqlt(struct orc_sim *sim, const void *phase, const void *gu,
		const void *gd);
/* meas.c:728-801 and 860-964 (meas_bond_corr) */
void orc_measure_uneqlt(struct orc_sim *sim, const void *phase,
		const void *Gu0t, const void *Gutt, const void *Gut0,
		const void *Gd0t, const void *Gdtt, const void *Gdt0);

/* Dense reference: G = (I + B_{l-1} ... B_0 B_{L-1} ... B_l)^{-1} from a plain
 * product and LU inverse (no stabilisation; for well-conditioned cases). */
void orc_dense_g(int N, int L, int l, const void *B, void *g);

/* FLOPs the oracle counted in BLAS/LAPACK calls since the last reset */
double orc_flops(void);
void orc_flops_reset(void);

#ifdef __cplusplus
}
#endif
