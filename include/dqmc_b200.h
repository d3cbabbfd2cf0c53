/*
 * dqmc_b200: B200-native DQMC sweep engine -- C ABI.
 *
 * Drop-in for the sweep of katherineding/dqmc-dev.  Plain pointers, sizes and
 * int status codes; no CUDA, C++ or torch types in any signature.  Matrices
 * are column-major (element (i, j) at [i + N*j]) exactly as the reference
 * stores them; `num` arrays are double, or interleaved (re, im) double pairs
 * when the parameter set is complex (cplx = 1), like C99 double complex.
 *
 * Status codes: 0 success, negative on failure (DQMC_E_*).
 */
#ifndef DQMC_B200_H
#define DQMC_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
	DQMC_OK = 0,
	DQMC_E_ARG = -10,      /* invalid argument or unsupported size */
	DQMC_E_CUDA = -11,     /* CUDA runtime error (no device, launch failure) */
	DQMC_E_NOMEM = -12,    /* device allocation failed */
	DQMC_E_DEVICE = -13,   /* a kernel reported an error (see dqmc_engine_errors) */
	DQMC_E_SCRATCH = -14,  /* the problem does not fit the library's fixed scratch */
};

/* ---------------------------------------------------------------------------
 * Drop-in entry point.  Replaces
 *   int dqmc_wrapper(const char *sim_file, const char *log_file,
 *                    const int64_t max_time, const bool dry, const bool bench);
 * of the reference (src/dqmc.h:9-10, body src/dqmc.c:525-671): same
 * arguments, same log lines, same return codes (-1 failure, 0 complete,
 * 1 partial: stopped by signal or max_time), same checkpoint and
 * partial_write protocol.  max_time is in nanoseconds after the call
 * starts (0: no limit), the unit of the reference's time_wall ticks
 * (src/sig.c:76, src/time_.h:6); the dqmc_1 and dqmc_stack CLIs convert
 * their -t seconds.  The sim file is the DQSF container written by the
 * generator (dqmc_b200/gen.py or the reference generator under the DQSF
 * h5py stand-in).
 * ------------------------------------------------------------------------ */
int dqmc_wrapper(const char *sim_file, const char *log_file,
		const int64_t max_time, const bool dry, const bool bench);

/* Batched drop-in: runs every file of a list as chains of one engine (files
 * with equal parameters share kernel launches).  status[i] receives what
 * dqmc_wrapper would have returned for file i.  Returns the worst status.
 * No reference counterpart; the reference runs such lists one file per
 * process through its stack job board (src/main_stack.c:399-479).
 * max_time in nanoseconds, as for dqmc_wrapper. */
int dqmc_wrapper_batch(int n_files, const char *const *sim_files,
		const char *log_file, const int64_t max_time, const bool bench,
		int *status);

/* ---------------------------------------------------------------------------
 * Engine: a group of chains sharing one parameter set (struct params,
 * src/data.h:7-38) advanced together on one GPU.
 * ------------------------------------------------------------------------ */
typedef struct dqmc_engine dqmc_engine;

typedef struct {
	int N, L, n_matmul, n_delay, F;
	int n_sweep_warm, n_sweep, period_eqlt, period_uneqlt, meas_bond_corr;
	int num_i, num_ij, num_b, num_bb, degen_i, degen_ij, degen_bb;
	int cplx;                         /* 0 real, 1 complex */
	const int *map_i, *map_ij;        /* [N], [N*N] */
	const int *bonds, *map_bb;        /* [2*num_b], [num_b*num_b] */
	const void *peierlsu, *peierlsd;  /* num[N*N] */
	const void *exp_Ku, *exp_Kd, *inv_exp_Ku, *inv_exp_Kd;
	const void *exp_halfKu, *exp_halfKd, *inv_exp_halfKu, *inv_exp_halfKd;
	/* The measurement toggles beyond meas_bond_corr (struct params,
	 * src/data.h:21-26; 0 = off) and the maps they read, as the sim file's
	 * params group holds them.  All zero / NULL when no toggle is on. */
	int meas_energy_corr, meas_thermal, meas_2bond_corr, meas_nematic_corr;
	int meas_chiral, meas_local_JQ, meas_gen_suscept, meas_pair_bb_only;
	int Nx, Ny;
	int num_plaq, num_plaq_accum, num_b_accum, num_b2_accum;
	int num_bs, num_b2, num_b2b, num_bb2, num_b2b2;
	int degen_plaq, degen_b, degen_b2, degen_bs, degen_b2b, degen_bb2, degen_b2b2;
	const int *plaqs, *map_plaq;             /* [3*num_plaq], [num_plaq] */
	const int *map_b, *map_bs;               /* [num_b], [N*num_b] */
	const int *bond2s, *map_b2;              /* [2*num_b2], [num_b2] */
	const int *map_bb2, *map_b2b, *map_b2b2; /* [num_b*num_b2] x 2, [num_b2^2] */
	const void *pp_u, *pp_d, *ppr_u, *ppr_d; /* num[num_b2] */
} dqmc_params;

/* Accumulator sizes in num elements per chain (layout documented in
 * dqmc-dev_b200/csrc/meas.cuh: sign, the always-on datasets, then those of
 * each enabled toggle). */
int dqmc_acc_sizes(const dqmc_params *p, int *eq_size, int *ue_size);

/* An engine advances n_chain chains of one parameter set (the batched form
 * of the reference's one chain per process, main_1.c:27-60 and dqmc.c).
 * It splits them into lanes, contiguous sub-batches with their own streams
 * whose kernels overlap on the GPU: one lane per 32 real chains from 256
 * chains up (at most 8), one per 64 real chains below (at most 4), one per
 * 32 complex chains (at most 4), or
 * the value of the environment variable DQMC_LANES at creation.  Results do
 * not depend on the split. */
int dqmc_engine_create(const dqmc_params *p, int n_chain, int device,
		dqmc_engine **out);
void dqmc_engine_destroy(dqmc_engine *e);
/* number of lanes the engine's chains are split into (no counterpart in the
 * reference, which runs one chain per process) */
int dqmc_engine_lanes(dqmc_engine *e);

/* Per-chain state (host arrays, copied): exp_lambda[2N], del[2N] as in the
 * sim file, rng[17], hs[L*N] (hs[i + N*l]), and the sweep counter (equal
 * for every chain of an engine).  The equal-time G of every chain is
 * recomputed from the fields before the next sweep (as the reference does
 * when it starts from a file, dqmc.c:188-220). */
int dqmc_engine_set_chain(dqmc_engine *e, int chain, const double *exp_lambda,
		const double *del, const uint64_t *rng, const int *hs, int sweep);
int dqmc_engine_set_acc(dqmc_engine *e, int chain, int eq_n_sample,
		const void *eq_acc, int ue_n_sample, const void *ue_acc);

/* Every chain's state at once (no counterpart in the reference, whose
 * process holds one chain): the arrays of dqmc_engine_set_chain for all
 * n_chain chains, contiguous in chain order: exp_lambda[n_chain][2N],
 * del[n_chain][2N], rng[n_chain][17], hs[n_chain][L*N].  One copy per array
 * and lane instead of one call per chain.  G is recomputed before the next
 * sweep, as after dqmc_engine_set_chain. */
int dqmc_engine_set_chains(dqmc_engine *e, const double *exp_lambda,
		const double *del, const uint64_t *rng, const int *hs, int sweep);
/* Every chain's state and accumulators at once, the counterpart of
 * dqmc_engine_get_chain plus dqmc_engine_get_acc for all chains: rng[n][17],
 * hs[n][L*N], eq_n_sample[n], eq_acc[n][eq_size], ue_n_sample[n],
 * ue_acc[n][ue_size] (the last two only with unequal-time measurements);
 * any pointer may be NULL. */
int dqmc_engine_get_chains(dqmc_engine *e, uint64_t *rng, int *hs, int *sweep,
		int *eq_n_sample, void *eq_acc, int *ue_n_sample, void *ue_acc);

/* Computes the initial G of every chain (dqmc.c:188-220). */
int dqmc_engine_init(dqmc_engine *e);

/* Advances every chain by n sweeps (dqmc.c:222-459), measuring as the
 * parameters and the sweep counter say.  Stream-ordered; returns after the
 * work is queued unless sync != 0. */
int dqmc_engine_sweeps(dqmc_engine *e, int n, int sync);
int dqmc_engine_sync(dqmc_engine *e);
/* OR of the device error words since creation (0 = none) */
unsigned dqmc_engine_errors(dqmc_engine *e);

int dqmc_engine_get_chain(dqmc_engine *e, int chain, uint64_t *rng, int *hs,
		int *sweep);
int dqmc_engine_get_acc(dqmc_engine *e, int chain, int *eq_n_sample, void *eq_acc,
		int *ue_n_sample, void *ue_acc);
/* G of both spins (column-major) and the chain's phase */
int dqmc_engine_get_g(dqmc_engine *e, int chain, void *gu, void *gd, void *phase);
/* total Metropolis accepts of a chain since creation */
int dqmc_engine_accepts(dqmc_engine *e, int chain, long long *n);
/* CUDA stream the engine queues on, as an opaque handle (cudaStream_t):
 * every sweep forks from it to the lanes' streams and joins back to it */
void *dqmc_engine_stream(dqmc_engine *e);
/* 1 when the engine's delayed update holds G on chip (k_update_cl: a
 * cluster of two CTAs per chain, one per spin), 0 when G stays in device
 * memory (k_update); both give bit-identical results.  Chosen at creation:
 * DQMC_UPDATE=cluster or =global when set, else on chip for real scalars
 * with N >= 96 and at most 64 chains; on chip only where one spin's G and
 * panels fit in shared memory.  dqmc_gpu_update_delayed applies the same
 * rule to its batch. */
int dqmc_engine_update_on_chip(dqmc_engine *e);
/* number of kernels one sweep of the given kind launches */
int dqmc_engine_launches_per_sweep(dqmc_engine *e, int meas_eq, int meas_ue);
/* Runs one sweep eagerly with CUDA events around every launch (it advances
 * the chains like dqmc_engine_sweeps(e, 1, 1)).  out[4*c + k], c < n_class:
 * k = 0 total ms, 1 launches, 2 algorithmic FLOPs, 3 operand bytes, for the
 * launch classes c = 0 batched GEMM (calc_eq_g's included), 1 delayed
 * update, 2 column-pivoted QR, 3 unequal-time G (its GEMMs under 0),
 * 4 measurements, 5 pre-sorted QR, 6 recombine (LU solve of G).  The
 * update's FLOPs are counted from the sweep's accepts: per accept and spin
 * 2 N^2 (its column of the flush) + 2 N (n_delay - 1) (the panel products,
 * on average), times 4 for complex; its bytes are one read and one write
 * of G per slice, chain and spin. */
int dqmc_engine_profile_sweep(dqmc_engine *e, int meas_eq, int meas_ue, double *out,
		int n_class);
/* One gradient evaluation, its results discarded (which = 0:
 * dqmc_engine_logdet_grad, 1: dqmc_engine_obs_grad), with CUDA events around
 * the engine's recorded launches; out as for dqmc_engine_profile_sweep
 * (the gradient paths' GEMMs under class 0, calc_eq_g's QRs and recombine
 * under 2, 5 and 6, the unequal-time kernels under 3), lanes profiled one
 * after another.  *launches (may be null) receives the number of kernels
 * the evaluation launched. */
int dqmc_engine_profile_grad(dqmc_engine *e, int which, double *out, int n_class,
		int *launches);

/* Fixed-field log-determinant and its gradient sums (no counterpart in the
 * reference, whose sweep only samples).  For every chain: logdet[chain] =
 * log |det(I + B_{L-1} ... B_0)| summed over both spins, and
 * S[chain][spin] (N x N, column-major num) = sum_l exp(V_l) (I - G_l)
 * exp(-V_l) over one sweep without updates, G_l the equal-time Green's
 * function before slice l.  Then for any parameter theta of the hopping
 * matrix K_spin, d logdet / d theta = sum_spin tr[S_spin D_theta,spin] with
 * D_theta = exp(dt K) d exp(-dt K) / d theta.  The chains' fields, RNG
 * states and sweep counts do not change. */
int dqmc_engine_logdet_grad(dqmc_engine *e, double *logdet, void *S);

/* Fixed-field density and double occupancy (no counterpart in the
 * reference), each averaged over the L slices of the chain's own fields:
 * obs[chain][0] = <n> = sum_spin sum_l sum_i (1 - G_l,ii) / (N L),
 * obs[chain][1] = <docc> = sum_l sum_i (1 - Gup_l,ii)(1 - Gdn_l,ii) / (N L),
 * and Z[chain][obs][spin] (N x N, column-major num) with
 * d obs / d theta = sum_spin tr[Z_spin D_theta], D_theta as for
 * dqmc_engine_logdet_grad.  Z comes from the space-time Green's function
 * O^-1 (src/greens.c:247-264 with one slice per block): Z = sum_m s_m
 * exp(V_m) Y_m exp(-dt K), Y_m = sum_l O^-1(m, l) W_l O^-1(l, m+1),
 * s_m = -1 for the corner block m = L-1 and +1 otherwise.  O^-1 is never
 * formed: at each cluster boundary s = c n_matmul the stabilised
 * unequal-time Green's functions of the chain rotated by s slices
 * (src/greens.c:247-494) give row and column s of O^-1, and one B_m or
 * B_m^-1 product per slice gives the rows and columns in between.  Device
 * work per chain and spin: 10 N^2 L nums (the unequal-time stacks and the
 * rows and columns), kept for the next call.  DQMC_OBS_GRAD=dense, and the
 * sizes the unequal-time kernels do not take (N above 160 real / 112
 * complex), invert the whole N L x N L matrix instead: 2 (N L)^2 nums. */
int dqmc_engine_obs_grad(dqmc_engine *e, double *obs, void *Z);

/* Engines advanced together (the ragged batch: one engine per parameter
 * group, any lattice, L or hopping): every dqmc_batch_sweeps sweep of all
 * engines that have sweeps left is ONE CUDA graph launch on the batch's own
 * stream.  The graph of a combination of the engines' sweep kinds (warm-up,
 * equal-time, unequal-time) is captured on first use: it forks from the
 * batch stream into every engine and each of its lanes, holds each engine's
 * sweep kernels, and joins back.  Fields replaced through
 * dqmc_engine_set_chain(s) are taken up (G recomputed) before the launch,
 * outside the graph.  Work queued afterwards on an engine (its calls, its
 * stream) is ordered after the batch's sweeps.  The engines must belong to
 * one device and stay alive for the batch's lifetime; dqmc_batch_create
 * refuses while DQMC_DEBUG_SYNC is set (its per-launch host checks cannot be
 * captured).  No counterpart in the reference, which runs one chain per
 * process; the sweep of each engine is that of src/dqmc.c:247-386. */
typedef struct dqmc_batch dqmc_batch;
int dqmc_batch_create(dqmc_engine *const *engines, int n, dqmc_batch **out);
/* n_sweeps sweeps (fewer when every engine completes); sync: wait for them */
int dqmc_batch_sweeps(dqmc_batch *b, int n_sweeps, int sync);
/* the batch's cudaStream_t, as void* */
void *dqmc_batch_stream(dqmc_batch *b);
void dqmc_batch_destroy(dqmc_batch *b);

/* G drift self-check, the runtime form of the reference's compile-time
 * CHECK_G_WRP (src/dqmc.c:15-16, 277-287, 339-343): with it on, at every
 * recalculation of G the engine also wraps the previous slice's G once more
 * (B_l G B_l^-1, as at the other slices) and compares it with the
 * recalculated G, entry by entry as the reference's matdiff (dqmc.c:61-71).
 * dqmc_engine_check_g turns it on (and clears the counters) or off; it costs
 * one wrap and one N x N comparison per recalculation and N x N nums of
 * device memory per chain and spin.  The results leave the sweep unchanged.
 * With bit 1 of `on` set (on = 3) the accurate recalculation check runs
 * too (dqmc_engine_g_drift_acc).
 * dqmc_engine_g_drift gives per chain (arrays of n_chain) the largest
 * |G - G_wrapped| over the checked recalculations and both spins, and its
 * mean over the entries averaged over the recalculations and spins, and the
 * number of recalculations checked; DQMC_E_ARG while the check is off.
 * dqmc_wrapper turns it on when the environment variable DQMC_CHECK_G is
 * set and writes the drift to its log. */
int dqmc_engine_check_g(dqmc_engine *e, int on);
int dqmc_engine_g_drift(dqmc_engine *e, double *max_abs, double *mean_abs, int *n_recalc);
/* The same check also compares, at every unequal-time measurement, the
 * equal-time G with the (0, 0) block of G(tau, tau) that the unequal-time
 * path computed (the reference's CHECK_G_UE, dqmc.c:21-22, 405-408), before
 * the half wrap; per chain as above, over the measurements checked. */
int dqmc_engine_g_drift_ue(dqmc_engine *e, double *max_abs, double *mean_abs, int *n_meas);
/* The accurate recalculation check, the runtime form of the reference's
 * compile-time CHECK_G_ACC (src/dqmc.c:18-19, 283-287, 345-349): at every
 * recalculation G is computed again from the L single-slice factors B_l
 * with a QR after each one (calc_eq_g(l, N, L, 1, B, ...)) and compared
 * with the G of the cluster chain.  It costs a calc_eq_g of L factors per
 * recalculation and L N x N nums of device memory per chain and spin, and
 * leaves the sweep unchanged; per chain as above, over the recalculations
 * checked, DQMC_E_ARG unless the check was turned on with bit 1. */
int dqmc_engine_g_drift_acc(dqmc_engine *e, double *max_abs, double *mean_abs, int *n_recalc);

/* Replaces the hopping matrices of every chain (the eight exp(-+dt K) and
 * exp(-+dt K / 2) of dqmc_params, both spins) in place, without any device
 * allocation; G and the cluster products are recomputed from the chains'
 * fields before their next use.  No counterpart in the reference, which
 * fixes the hopping per sim file: it serves the fixed-field gradient
 * evaluations, which visit many hoppings for the same fields. */
int dqmc_engine_set_hopping(dqmc_engine *e, const void *exp_Ku, const void *exp_Kd,
		const void *inv_exp_Ku, const void *inv_exp_Kd, const void *exp_halfKu,
		const void *exp_halfKd, const void *inv_exp_halfKu, const void *inv_exp_halfKd);

/* ---------------------------------------------------------------------------
 * Kernel-level seams on device pointers, batched over `batch` independent
 * problems laid out back to back.  Each mirrors one reference function.
 * stream: a cudaStream_t passed as void* (NULL = default stream).
 * ------------------------------------------------------------------------ */

/* xgemm("N", "N", ...) (src/linalg_generic.h:23-40) for `batch` column-major
 * problems: C_b = alpha A_b B_b + beta C_b with A_b = A + b*stride_a (M x K,
 * leading dimension lda) and likewise B (K x N), C (M x N).
 * alpha, beta: host pointers to one num.  Asynchronous on `stream`. */
int dqmc_gpu_gemm(int batch, int M, int N, int K, int cplx, const void *alpha,
		const void *A, int lda, long long stride_a, const void *B, int ldb,
		long long stride_b, const void *beta, void *C, int ldc, long long stride_c,
		void *stream);

/* calc_eq_g (src/greens.c:69-208, called as calc_eq_g(l, N, F, 2, C, g, ...)
 * by dqmc.c:202, 288): G = (I + C_{l-1} ... C_{l})^-1 from F cluster
 * matrices per problem (C: batch x F x N*N), writing G (batch x N*N) and
 * phase[batch] = 1/phase(det G). */
int dqmc_gpu_calc_eq_g(int batch, int N, int F, int l, int cplx, const void *C,
		void *G, void *phase, void *stream);

/* update_delayed (src/updates.c:7-84) preceded by shuffle (src/rand.h:25-31)
 * as dqmc.c:249-253 calls them, for `batch` chains: del[batch][2N],
 * rng[batch][17], hs[batch][N] (this slice's fields), G[batch][2][N*N]
 * (up, down), phase[batch]; n_delay as in the sim file. */
int dqmc_gpu_update_delayed(int batch, int N, int n_delay, int cplx,
		const double *del, uint64_t *rng, int *hs, void *G, void *phase,
		void *stream);

/* mul_seq (src/greens.c:8-41) for B_l = exp_K diag(exp_lambda[hs_l]):
 * C = B_{l0+n-1} ... B_{l0} for one spin (spin 0 uses hs, 1 uses !hs) of
 * `batch` chains: exp_K[N*N] shared, exp_lambda[batch][2N],
 * hs[batch][n][N] (the n slices), C[batch][N*N]. */
int dqmc_gpu_mul_seq(int batch, int N, int n, int spin, int cplx,
		const void *exp_K, const double *exp_lambda, const int *hs, void *C,
		void *stream);

/* Size of the fixed device scratch of dqmc_gpu_calc_eq_g_noalloc (16 MiB).
 * A call needs six parts of batch*N*N*sizeof(num) bytes, one of batch*N*8,
 * one of batch*N*4, one of batch*sizeof(num) and 256 for the error word,
 * each part rounded up to a multiple of 256.  That admits at most 84
 * problems of N = 64 or 16 of N = 144 (real), and 17 of N = 100 or 13 of
 * N = 112 (complex). */
#define DQMC_NOALLOC_SCRATCH_BYTES (16 << 20)

/* dqmc_gpu_calc_eq_g without any device allocation; no counterpart in the
 * reference.  Same arguments, results and status codes as
 * dqmc_gpu_calc_eq_g, which allocates its work matrices with cudaMalloc on
 * every call.  Some callers cannot allow that: a process whose free device
 * memory is already reserved by another allocator (a framework's caching
 * allocator that holds the HBM, so cudaMalloc fails), or a driver that keeps
 * sweeps queued on other streams and cannot take the device-wide
 * synchronisation that cudaFree implies.  This variant works in one static
 * device array of DQMC_NOALLOC_SCRATCH_BYTES that the library holds on every
 * device it loads on until the process exits, and returns DQMC_E_SCRATCH
 * (with a message on stderr) when batch x N does not fit it.
 * - The first call on a device looks up the array's device address (no
 *   allocation); make that first call before any stream capture on it.
 * - Every call on a device shares the one array and it keeps the previous
 *   call's contents (the error word is cleared at the start of each call):
 *   calls that overlap on the GPU -- from several threads, or on several
 *   streams -- race and give wrong results.  Serialise them.
 * Like dqmc_gpu_calc_eq_g it synchronises `stream` before it returns. */
int dqmc_gpu_calc_eq_g_noalloc(int batch, int N, int F, int l, int cplx,
		const void *C, void *G, void *phase, void *stream);

#ifdef __cplusplus
}
#endif

#endif
