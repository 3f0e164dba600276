/*
 * glac_b200 -- C ABI of the B200 (sm_100a) implementation of GLAC's pure-gauge
 * SU(3) hot path: Wilson-action Metropolis, Luscher RK3 gradient flow with SU(3)
 * exponentials, and plaquette / clover energy density / topological charge.
 *
 * Plain C: pointers and sizes only.  Every entry point returns a glac_status;
 * on failure glac_last_error() gives the message.  A context owns one lattice,
 * its device buffers and one CUDA stream; calls on one context are not
 * re-entrant.
 *
 * Host field layout (every *_links argument): 4 blocks (mu = 0..3) of V SU(3)
 * matrices, each 18 doubles (re, im; row-major), sites in lexicographic order
 * x + Nx(y + Ny(z + Nz t)) -- exactly the memory of the reference's
 * Lattice<SU3>[4] (GLAC/math/lattice.h:23-180, GLAC/parallelization/index.h:32-35).
 *
 * Observable vectors (every *obs argument): [plaq, topc, energy, topct[0..Nt-1]],
 * the normalisation of MasterSamplerTopcXYZ::getObservablesVector
 * (GLAC/observables/mastersamplertopcxyz.cpp:223-234).
 */
#ifndef GLAC_B200_H
#define GLAC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GLAC_OK = 0,
    GLAC_ERR_ARG = 1,       /* invalid argument (sizes, parities, options) */
    GLAC_ERR_CUDA = 2,      /* CUDA runtime error or no usable device */
    GLAC_ERR_TIMEOUT = 3,   /* a bounded device wait ran out */
    GLAC_ERR_NONFINITE = 4, /* non-finite value in a field or result */
    GLAC_ERR_IO = 5,        /* file missing, short or of the wrong size */
    GLAC_ERR_STATE = 6      /* call out of order (e.g. no field set yet) */
} glac_status;

typedef enum { GLAC_FP64 = 0, GLAC_FP32 = 1 } glac_precision;

/* Reference expFunc names "morningstar", "luscher", "taylor2", "taylor4"
 * (GLAC/flow/flow.cpp:75-93). */
typedef enum { GLAC_EXP_MORNINGSTAR = 0, GLAC_EXP_LUSCHER = 1, GLAC_EXP_TAYLOR2 = 2, GLAC_EXP_TAYLOR4 = 3 } glac_exp;

typedef struct {
    int dims[4];            /* Nx, Ny, Nz, Nt; each even and >= 4 (NSpatial/NTemporal) */
    double beta;            /* "beta" */
    int precision;          /* glac_precision */
    int n_updates;          /* "NUpdates": Metropolis hits per link */
    double su3_eps;         /* "SU3Eps": proposal spread */
    double flow_eps;        /* "flowEpsilon" */
    int exp_func;           /* glac_exp ("expFunc") */
    uint64_t seed;          /* Philox key ("metropolisSeed") */
    uint32_t stream_id;     /* Philox stream (independent chains share a seed) */
    int reunit_interval;    /* FP32: reunitarise every k sweeps / flow steps (0 = never) */
    int device;             /* CUDA device ordinal */
} glac_desc;

typedef struct glac_ctx glac_ctx;

/* ---- lifetime ---------------------------------------------------------- */
/* Replaces System::latticeSetup's allocation (GLAC/system.cpp:148-177, 193-231).
 * Every extent even and >= 4 (checkerboard), Nt <= 1024, and a volume whose
 * fields fit 32-bit element offsets: V < 1.19e8 sites in FP64, < 2.68e8 in FP32
 * (beyond what two fields and the force of one lattice leave room for in
 * 180 GB anyway).  Errors: GLAC_ERR_ARG, message in glac_global_error(). */
glac_status glac_create(const glac_desc *desc, glac_ctx **out);
void glac_destroy(glac_ctx *ctx);
const char *glac_last_error(const glac_ctx *ctx);
/* Message of the last failure of a call that had no context (create, exp_batch ...). */
const char *glac_global_error(void);
/* The context's CUDA stream (cudaStream_t), for callers that time or order work. */
void *glac_stream(glac_ctx *ctx);
glac_status glac_sync(glac_ctx *ctx);
/* Number of kernels this context has launched so far. */
uint64_t glac_launch_count(const glac_ctx *ctx);
/* Switches by name; unknown keys give GLAC_ERR_ARG.
 *   "su2_sign_flips" (default 1): 1 draws the SU(2) factors of each proposal as
 *   the reference does, x0 = sign(u0) sqrt(1 - eps^2)
 *   (su3matrixgenerator.h:202-243); 0 keeps x0 = +sqrt(1 - eps^2), every factor
 *   near the identity (a symmetric proposal as well; no reference counterpart).
 *   Applies to glac_metropolis and glac_esj_data.
 *   "fused_measure": 1 or 2 (default 2 in FP32, 1 in FP64): glac_flow
 *   measures the field before each step inside that step's first RK3 stage,
 *   from the staple pieces the stage computes anyway (two extra 3x3 products
 *   per plane instead of the ten of a separate clover pass), and the last one
 *   in a pass of its own; 1 uses the stage kernel's own register allocation, 2
 *   a 128-register variant, and in FP32 3 a thread per site and 4 a
 *   96-register variant; 0 measures every field in a pass of its own.  The
 *   results are the same to rounding.
 *   "fused_combine" (default 1): with fused_measure on, the measurement's
 *   per-site combination and block reduction run inside the step's second
 *   stage where each half time slice is a whole number of 128-site blocks
 *   (Nx Ny Nz / 2 divisible by 128), else in a pass of their own; 0: always a
 *   pass of their own. */
glac_status glac_set_option(glac_ctx *ctx, const char *key, long value);

/* ---- field --------------------------------------------------------------- */
/* Cold start (all links 1) -- System::latticeSetup cold branch (GLAC/system.cpp:216-223). */
glac_status glac_cold_start(glac_ctx *ctx);
/* Seeded Haar-random start (replaces the hot start, GLAC/system.cpp:200-214). */
glac_status glac_hot_start(glac_ctx *ctx, uint64_t seed);
/* Every link a random RST matrix near unity with spread su3_eps (the
 * reference's RSTHotStart, GLAC/system.cpp:205-210). */
glac_status glac_rst_start(glac_ctx *ctx, uint64_t seed);
/* Host <-> device in the reference layout; FP32 contexts convert. */
glac_status glac_set_links(glac_ctx *ctx, const double *host_links);
glac_status glac_get_links(glac_ctx *ctx, double *host_links);
/* Same, from / to device memory in the host layout (no host copy). */
glac_status glac_set_links_device(glac_ctx *ctx, const double *dev_links);
glac_status glac_get_links_device(glac_ctx *ctx, double *dev_links);
/* Device copy of src's field into dst (same dims and precision); the flow
 * lattice copy of System::copyToFlowLattice (GLAC/system.cpp:179-188). */
glac_status glac_copy_field(glac_ctx *dst, glac_ctx *src);
/* FP64 Gram-Schmidt projection of every link back onto SU(3). */
glac_status glac_reunitarize(glac_ctx *ctx);
/* max over links and entries of |U U^+ - 1|. */
glac_status glac_unitarity_violation(glac_ctx *ctx, double *out);

/* ---- hot path ------------------------------------------------------------- */
/* n_sweeps checkerboard Metropolis sweeps (replaces System::update,
 * GLAC/system.cpp:333-361, with WilsonGaugeAction::computeStaple / getDeltaAction,
 * GLAC/actions/wilsongaugeaction.cpp:24-53).  *acceptance (may be NULL) receives
 * the mean acceptance per sweep (accepted / (4 NUpdates V), system.cpp:359). */
glac_status glac_metropolis(glac_ctx *ctx, int n_sweeps, double *acceptance);
/* n_steps Luscher RK3 steps of the field in place (replaces Flow::flowField,
 * GLAC/flow/flow.cpp:43-73).  obs (may be NULL) receives (n_steps + 1)
 * observable vectors: before the first step and after each, as
 * System::flowConfiguration measures them (GLAC/system.cpp:471-517). */
glac_status glac_flow(glac_ctx *ctx, int n_steps, double *obs);
/* Observables of the current field (replaces MasterSamplerTopcXYZ::calculate,
 * GLAC/observables/mastersamplertopcxyz.cpp:236-384). */
glac_status glac_measure(glac_ctx *ctx, double *obs);
/* As glac_measure, plus the per-site densities of LatticeActionChargeDensity
 * (GLAC/observables/latticeactionchargedensity.cpp:169-306), V doubles each in
 * the host site order: q_density[n] = -(1/(16^2 pi^2)) sum_nu ReTr(C_0nu C_rhosigma)
 * (sums to topc) and e_density[n] = sum ReTr(C C) (unnormalised; energy =
 * sum / V).  obs may be NULL.  Host pointers; synchronous. */
glac_status glac_measure_density(glac_ctx *ctx, double *obs, double *q_density, double *e_density);
/* SuperSampler::calculate (GLAC/observables/supersampler.cpp:298-496), the
 * sampler the observable list "weinberg" selects: obs = [plaq, topc, energy,
 * weinberg, topct[Nt], weinbergt[Nt]] (4 + 2 Nt doubles, host). */
glac_status glac_measure_weinberg(glac_ctx *ctx, double *obs);
/* The Philox sweep counter of this context (advanced by every Metropolis sweep):
 * saved beside a stored configuration, it lets a loaded chain continue its
 * random stream where it stopped.  No counterpart in the reference. */
glac_status glac_get_sweep(glac_ctx *ctx, uint32_t *sweep);
glac_status glac_set_sweep(glac_ctx *ctx, uint32_t sweep);
/* One load-and-flow pass from host memory: set the field from host_links, then
 * glac_flow(n_steps, obs) (System::flowConfigurations, GLAC/system.cpp:570-602). */
glac_status glac_flow_configuration(glac_ctx *ctx, const double *host_links, int n_steps, double *obs);

/* Mean device time in seconds of each of the three RK3 stage launches over
 * n_steps flow steps of the current field (CUDA events on the context's
 * stream); advances the field by n_steps. */
glac_status glac_flow_stage_times(glac_ctx *ctx, int n_steps, double *seconds3);
/* The same for flow steps that measure the field before each step inside
 * stage 0 ("fused_measure" on): seconds4 = [stage 0 with the clover parts,
 * the measurement's per-site combination and reduction, stage 1, stage 2].
 * GLAC_ERR_STATE where the measurement is not fused for this context. */
glac_status glac_flow_stage_times_measured(glac_ctx *ctx, int n_steps, double *seconds4);

/* Launch-variant autotuner (no reference counterpart): times each launch
 * variant (register cap / resident blocks per SM) of the flow-stage,
 * Metropolis and observable kernels on this lattice, reps calls each, keeps the
 * fastest, and restores the field and random stream.  report (may be NULL)
 * receives 3 x 4 seconds-per-call entries [family][variant], 0 where unused. */
glac_status glac_autotune(glac_ctx *ctx, int reps, double *report);
/* The chosen variant per family (flow, metropolis, observables), and a setter
 * for a previously tuned choice. */
glac_status glac_get_tuning(glac_ctx *ctx, int *variants3);
glac_status glac_set_tuning(glac_ctx *ctx, const int *variants3);

/* ---- test exports (parity checks against the reference) ------------------ */
/* Staples of every link of the current field, host layout (computeStaple). */
glac_status glac_staples(glac_ctx *ctx, double *host_out);
/* Flow force Z_mu(n) of every link as full matrices (getActionDerivative,
 * GLAC/actions/wilsongaugeaction.cpp:55-86). */
glac_status glac_force(glac_ctx *ctx, double *host_out);
/* exp of n traceless anti-Hermitian matrices on the device (SU3Exp::exp,
 * GLAC/math/exponentiation/su3exp.cpp:16-79, or the alternates). */
glac_status glac_exp_batch(int precision, int exp_func, const double *host_in, long n, double *host_out);
/* dS = -(beta/3) ReTr[(U' - U) A] for n independent triples
 * (WilsonGaugeAction::getDeltaAction, GLAC/actions/wilsongaugeaction.cpp:24-27). */
glac_status glac_delta_s_batch(int precision, double beta, long n, const double *host_U, const double *host_Uprime,
                               const double *host_A, double *host_out);
/* Metropolis accept step fed with given proposals X[k][h] and uniforms r[k][h]
 * for independent links k with staple A[k] (GLAC/system.cpp:340-352);
 * U is updated in place, accept[k][h] receives the decisions. */
glac_status glac_accept_fed(int precision, double beta, long n_links, int n_hits, double *host_U,
                            const double *host_A, const double *host_X, const double *host_r,
                            unsigned char *host_accept);

/* ---- allocation-free measurement ------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc --
 * code under a host framework that owns all device memory through its own pool
 * and forbids library allocations, latency-critical phases where a driver
 * allocation would synchronise the device, deployments whose device memory is
 * fixed at load time -- this entry point measures [plaq, topc, energy,
 * topct[Nt]] of a field without allocating anything: dev_links is a device
 * pointer to the field in the host layout above (FP64, 16-byte aligned),
 * dev_obs a device pointer to 3 + Nt doubles (8-byte aligned), stream a
 * cudaStream_t (NULL: default stream); the call is asynchronous on that stream.
 * A misaligned pointer, an extent below 2 or V above 2^31 gives GLAC_ERR_ARG.
 * Its only working memory is a fixed
 * 96 KiB device array inside this library (4096 partial-sum slots), held by
 * every GPU that loads the library until the process exits; Nt above 4096 is
 * rejected with GLAC_ERR_ARG.  Every call outside stream capture resolves that
 * array's address in the current context (cudaGetSymbolAddress); a call made
 * while its stream is capturing reuses the address of the device's last
 * uncaptured call, so make the first call on each device outside any stream
 * capture (otherwise GLAC_ERR_STATE).  All calls share the array and every call overwrites the
 * slots it reads, so nothing needs clearing between calls -- but calls that
 * overlap on the GPU (different streams, or different host threads, at the same
 * time) race on it and must be serialised by the caller.  Errors:
 * glac_noalloc_error(). */
glac_status glac_measure_noalloc(const int dims[4], const double *dev_links, double *dev_obs, void *stream);
const char *glac_noalloc_error(void);

/* ---- learned proposal spread (no counterpart in the reference) ---------- */
/* The reference draws every proposal with the run-config's SU3Eps
 * (su3matrixgenerator.cpp:16-35).  Here a small network may choose the spread
 * of each link's proposals from eight gauge-invariant features of its staple;
 * the staple does not change when its own link is updated, so the proposal
 * stays symmetric and the accept step (system.cpp:333-361) stays exact.
 * Network: 8 -> 32 -> 32 -> 1, leaky ReLU (slope 1/16), eps = eps_min +
 * (eps_max - eps_min) sigmoid(z); BF16 operands, FP32 accumulation.
 * Parameters, GLAC_MLP_NPARAMS floats, flat: W1[8][32], b1[32], W2[32][32],
 * b2[32], W3[32], b3 (x W1 + b1, row-vector convention). */
#define GLAC_MLP_NPARAMS 1377

/* Use the network for this context's Metropolis proposals from now on
 * (params = NULL: back to the fixed spread su3_eps).  0 < eps_min < eps_max <= 1. */
glac_status glac_set_proposal_net(glac_ctx *ctx, const float *params, double eps_min,
                                  double eps_max);

/* Expected-squared-jump training data from the current field.  Samples the
 * links s = o + i*stride (i < V/2/stride, o = snapshot*7919 mod stride) of each
 * (mu, parity) plane: rows = 8 * (V/2 / stride), written to *n_rows.  Per row:
 * dev_features[row*8 .. +8] = the staple's features; for each of the n_eps
 * spreads, dev_esj[row*n_eps + k] = mean over `trials` of ||U' - U||^2 after
 * n_updates Metropolis hits of that link with spread eps_grid[k] (its own
 * Philox stream, so the chain's draws are untouched; the field is not
 * modified); dev_link_ids[row] = mu*V + site (may be NULL).  n_eps = 0 gives
 * the features alone.  Device pointers; capacity = rows the buffers hold.
 * Synchronous. */
glac_status glac_esj_data(glac_ctx *ctx, int n_eps, const double *eps_grid, int trials, int stride,
                          uint32_t snapshot, float *dev_features, float *dev_esj, uint32_t *dev_link_ids,
                          long long capacity, long long *n_rows);

/* Trainer: FP32 master parameters with Adam state on one device; forward and
 * backward passes on the tensor cores.  Device-pointer inputs must be ready
 * (their producers synchronised) before each call; every call is synchronous. */
typedef struct glac_mlp glac_mlp;
glac_status glac_mlp_create(int device, glac_mlp **out);
void glac_mlp_destroy(glac_mlp *mlp);
const char *glac_mlp_last_error(const glac_mlp *mlp);
/* Set / read the GLAC_MLP_NPARAMS parameters (setting resets Adam). */
glac_status glac_mlp_set_params(glac_mlp *mlp, const float *host_params);
glac_status glac_mlp_get_params(glac_mlp *mlp, float *host_params);
/* He-normal initialisation from seed with the output bias at spread eps0. */
glac_status glac_mlp_init(glac_mlp *mlp, uint64_t seed, double eps_min, double eps_max, double eps0);
/* dev_eps[i] = spread for dev_features[i*8 .. +8], i < n.  Mode 0 (default):
 * the warp-level tensor-core routine the sampler itself runs (mma.m16n8k16 from
 * registers); mode 1: 128-row tiles on the 5th-generation tensor cores (tcgen05
 * MMA into tensor memory; GLAC_ERR_TIMEOUT if a completion wait runs out).
 * Both round at the same points; at this network size mode 0 is the faster
 * (36.7 vs 84.2 us per 2M rows on B200). */
glac_status glac_mlp_set_forward_mode(glac_mlp *mlp, int mode);
/* Test export for the failure path of mode 1.  wait_ns (1 ns .. 10 s, default
 * 1 s) bounds each completion wait of the tcgen05 kernel by the GPU's global
 * timer; issue_mma = 0 makes the kernel issue no MMA, so its first wait runs
 * out with nothing in flight: glac_mlp_forward then returns GLAC_ERR_TIMEOUT
 * and the next call (issue_mma = 1) works normally.  If a wait runs out while
 * an issued MMA is still in flight and a second wait of the same length does
 * not see it drain, the call returns GLAC_ERR_TIMEOUT and every later mode-1
 * call on this trainer returns GLAC_ERR_STATE.  No reference counterpart. */
glac_status glac_mlp_test_tc_wait(glac_mlp *mlp, unsigned long long wait_ns, int issue_mma);
glac_status glac_mlp_forward(glac_mlp *mlp, const float *dev_features, long long n, double eps_min, double eps_max,
                             float *dev_eps);
/* Loss L = -(1/n) sum_i J_i(eps_i), J_i linear between the n_eps grid points
 * (eps_min, eps_max = the grid's ends) over rows dev_esj[i*n_eps ..], and its
 * gradient (host_grad may be NULL).  Deterministic for a given n. */
glac_status glac_mlp_loss_grad(glac_mlp *mlp, const float *dev_features, const float *dev_esj, long long n,
                               int n_eps, const double *eps_grid, double *loss, float *host_grad);
/* `steps` Adam steps (learning rate lr) on consecutive batches of `batch` rows,
 * cycling over the n rows in order; host_losses[steps] (may be NULL) receives
 * the loss of each step's batch before its update. */
glac_status glac_mlp_train(glac_mlp *mlp, const float *dev_features, const float *dev_esj, long long n, int n_eps,
                           const double *eps_grid, int steps, long long batch, double lr, double *host_losses);

/* ---- batched ensemble (no counterpart in the reference) ----------------- */
/* Many independent lattices of uneven sizes and couplings driven together: each
 * Metropolis sub-sweep, flow stage and observable pass is one launch over all
 * of them, and glac_ensemble_run replays the whole schedule as one CUDA graph.
 * Lattice i is dims[4i .. 4i+3] at coupling betas[i]; `common` supplies the
 * precision, n_updates, su3_eps, flow_eps, exp_func (Morningstar only), the
 * Philox key `seed`, the first stream id (lattice i uses stream_id + i, so it
 * draws exactly what a single context with that stream id draws) and the device;
 * common->dims and beta are ignored. */
typedef struct glac_ensemble glac_ensemble;
glac_status glac_ensemble_create(int n, const int *dims, const double *betas, const glac_desc *common,
                                 glac_ensemble **out);
void glac_ensemble_destroy(glac_ensemble *ens);
const char *glac_ensemble_last_error(const glac_ensemble *ens);
/* Message of the last failed glac_ensemble_create on this thread. */
const char *glac_ensemble_global_error(void);
uint64_t glac_ensemble_launch_count(const glac_ensemble *ens);
/* "su2_sign_flips" 0/1 as for glac_set_option; "fused_measure" 1 (default):
 * each flow measurement inside the next step's first stage, 0: every
 * measurement in a pass of its own (as glac_set_option). */
glac_status glac_ensemble_set_option(glac_ensemble *ens, const char *key, long value);
/* Seeded Haar start of every lattice (as glac_hot_start with the lattice's stream). */
glac_status glac_ensemble_hot_start(glac_ensemble *ens, uint64_t seed);
/* Lattice i's Markov-chain field in the host layout of glac_set_links. */
glac_status glac_ensemble_set_links(glac_ensemble *ens, int i, const double *host_links);
glac_status glac_ensemble_get_links(glac_ensemble *ens, int i, double *host_links);
/* n checkerboard sweeps of every lattice; acceptance[i] (may be NULL) per lattice. */
glac_status glac_ensemble_metropolis(glac_ensemble *ens, int n_sweeps, double *acceptance);
/* Doubles of the measurement output for n_steps flow steps: lattice i holds
 * (n_steps + 1) rows of 3 + Nt_i (plaq, topc, energy, topct), lattices in order. */
long long glac_ensemble_obs_count(const glac_ensemble *ens, int n_steps);
/* Flow copies of every chain field (System::flowConfiguration, GLAC/system.cpp:
 * 471-517): measurement at t = 0 and after each of n_steps RK3 steps; the
 * chains are not modified.  obs (may be NULL): glac_ensemble_obs_count doubles. */
glac_status glac_ensemble_flow(glac_ensemble *ens, int n_steps, double *obs);
/* n_sweeps sweeps then the flow of glac_ensemble_flow, as one CUDA graph launch
 * (captured on the first call for this (n_sweeps, n_steps), replayed after);
 * gpu_seconds (may be NULL) = device time of the graph. */
glac_status glac_ensemble_run(glac_ensemble *ens, int n_sweeps, int n_steps, double *acceptance, double *obs,
                              double *gpu_seconds);
/* The same schedule as one persistent cooperative launch (FP32 ensembles with
 * fused_measure on): every co-resident block walks each phase's blocks in turn,
 * with a grid-wide barrier between phases whose waits are bounded by the GPU's
 * global timer (option "persistent_wait_ms", default 5000); a wait that runs
 * out gives GLAC_ERR_TIMEOUT and leaves the fields undefined.  Same results as
 * glac_ensemble_run.  "persistent_test_stall" = 1 (tests only) keeps one block
 * from arriving, so the others' waits run out.  No reference counterpart. */
glac_status glac_ensemble_run_persistent(glac_ensemble *ens, int n_sweeps, int n_steps, double *acceptance,
                                         double *obs, double *gpu_seconds);
/* Launch-variant autotuner over the whole ensemble (flow site-block shapes and
 * register caps, Metropolis and observable register caps); report[4 f + v] =
 * seconds per flow step (f = 0) / per sweep (f = 1) / per measurement (f = 2)
 * of variant v.  Leaves the chains as they were (a measurement row written
 * while timing is overwritten by the next run). */
glac_status glac_ensemble_autotune(glac_ensemble *ens, int reps, double *report);
glac_status glac_ensemble_get_tuning(const glac_ensemble *ens, int *variants3);
glac_status glac_ensemble_set_tuning(glac_ensemble *ens, const int *variants3);

/* ---- gauge-field files (GLAC/io/fieldio.cpp) ----------------------------- */
/* Read a GLAC .bin configuration (per site 4 links x 18 doubles, x fastest;
 * fieldio.cpp:195-257) or, with chroma != 0, its byte-swapped Chroma variant
 * (fieldio.cpp:259-330) into the host layout. */
glac_status glac_read_field(const char *path, const int dims[4], int chroma, double *host_links);
/* Write host-layout links as a GLAC .bin configuration (fieldio.cpp:61-135). */
glac_status glac_write_field(const char *path, const int dims[4], const double *host_links);
/* Message of the last failed glac_read_field / glac_write_field on this thread. */
const char *glac_io_error(void);

#ifdef __cplusplus
}
#endif
#endif
