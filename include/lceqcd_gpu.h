/*
 * lceqcd_gpu.h -- C ABI of the B200 (sm_100a) Monte Carlo hot path for the
 * 3D SU(2) + adjoint Higgs (A0) lattice code derek-teaney/lceqcd.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns an int status (LCE_OK = 0, negative = error; see lce_strerror).
 * A Fortran driver binds these with ISO_C_BINDING; the C++ driver
 * (lceqcd_b200/driver/lce_main.cpp) and the Python mirror
 * (lceqcd_b200/lattice.py) call them directly.
 *
 * The reference exposes no plugin API: the boundary replaced here is the set
 * of Fortran subroutines that f/main.f:21-78 calls inside its sweep loop, and
 * the COMMON blocks they share (f/INCLUDE/gaugefield.inc:35-36,
 * f/INCLUDE/measurement.inc:30-35).  Each declaration below names the
 * reference routine it replaces.
 *
 * Host field layout ("reference order"), matching the COMMON arrays
 * COMPLEX u(2, maxarray, 0:1, 3) and REAL a(3, maxarray, 0:1):
 *   u[((mu*2 + eo)*ld + site)*4 + c], c = (Re a, Im a, Re b, Im b) of the first
 *       row (a, b) of U = {{a, b}, {-b*, a*}};  mu = 0..2, eo = 0..1
 *   a[(eo*ld + site)*3 + k],  A = a_k sigma_k
 * with site in the half-row order of f/adresses.f and ld >= L1*L2*L3/2 the
 * leading site dimension (maxarray for the Fortran COMMON blocks).
 *
 * Threading: one host thread per context.  All work of a context is queued
 * on its CUDA stream; calls that return values to host memory synchronise
 * that stream.
 */
#ifndef LCEQCD_GPU_H
#define LCEQCD_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define LCE_ABI_VERSION 2

/* status codes */
#define LCE_OK 0
#define LCE_ERR_INVALID (-1)        /* bad argument or lattice shape */
#define LCE_ERR_CUDA (-2)           /* CUDA runtime error (lce_last_error) */
#define LCE_ERR_GF_NOT_CONVERGED (-3)  /* gauge fixing hit max_iters */
#define LCE_ERR_STREAM (-4)         /* validation uniform stream exhausted */
#define LCE_ERR_NAN (-5)            /* non-finite value in a reduction */
#define LCE_ERR_NOMEM (-6)          /* device allocation failed */
#define LCE_ERR_UNSUPPORTED (-7)    /* call not valid for this context */

/* precision of the device fields */
#define LCE_PREC_F32 0  /* FP32 fields; FP64 reunitarisation, sums, theta */
#define LCE_PREC_F64 1  /* FP64 everywhere (validation / plain path) */

/* uniform sources */
#define LCE_RNG_PHILOX 0  /* counter-based Philox4x32-10, per (seed, pass, site) */
#define LCE_RNG_STREAM 1  /* host-supplied uniforms in the reference's order */

/* gauge-fixing angle evaluation.  The reference takes theta = acos(Re Omega),
 * which cannot resolve rotations below ~sqrt(eps) (~3e-4 rad in FP32, ~1e-8 in
 * FP64), so the iteration stalls near theta ~ 1e-7 (FP32) or 1e-14 (FP64).
 * ATAN2 takes the same angle as atan2(|vector part|, scalar part) of w, which
 * is accurate for small angles; it is the default. */
#define LCE_GF_ACOS 0
#define LCE_GF_ATAN2 1

/* execution form of lce_sweep(s): one kernel per parity pass chained in a
 * CUDA graph (one site per thread, or two sites per thread), or one
 * cooperative persistent kernel per sweep that loops over the (chain, tile)
 * work list of every pass with a grid barrier in between.  AUTO times the
 * forms -- and, for FP32 contexts, the tile shapes of the per-pass forms
 * (128, 256, 448 or 512 threads per block, see lce_params.tile_threads) -- on the
 * first sweeps and keeps the fastest (lce_get_sweep_mode, lce_get_tile_shape). */
#define LCE_SWEEP_AUTO 0
#define LCE_SWEEP_PASSES 1
#define LCE_SWEEP_PERSISTENT 2
#define LCE_SWEEP_PASSES2 3
#define LCE_SWEEP_DIRECT 4   /* the per-pass kernels launched on the stream
                                without a graph (one site per thread) */

/* field selectors for upload/download */
#define LCE_FIELDS 0        /* u, a        (COMMON /linkvar/ u, a) */
#define LCE_FIELDS_FIXED 1  /* u_f, a_f    (COMMON /linkvar/ u_f, a_f) */

typedef struct lce_ctx lce_ctx;

/* Input parameters: the hot-path subset of the reference's inputfile
 * (f/paraminit.f:82-101) plus build-only knobs. */
typedef struct lce_params {
  int L[3];              /* global lattice extents (even)            inputfile line 1 */
  double beta, x, y;     /* couplings                                  lines 8-10 */
  double lambda;         /* gauge-fixing overrelaxation parameter      line 11 */
  double alpha;          /* z-link weight of the gauge functional      line 12 */
  double limit_or;       /* stopping value of theta                    line 13 */
  int imode;             /* Higgs heatbath mode 0/1                    line 20 */
  int precision;         /* LCE_PREC_F32 | LCE_PREC_F64 */
  int rng;               /* LCE_RNG_PHILOX | LCE_RNG_STREAM */
  unsigned long long seed;  /* Philox key */
  int device;            /* CUDA device ordinal */
  int n_link_or;         /* link overrelaxation hits per lce_sweep (0: reference composition) */
  int n_higgs_metro;     /* ahiggs1 calls per lce_sweep (0: reference composition); the calls of
                            one sweep share the step in force at its start, and the step is
                            adapted after each call's acceptance, in order, at the sweep's end */
  double delta0;         /* initial ahiggs1 step */
  int gf_angle;          /* gauge-fixing rotation angle: LCE_GF_ACOS (the
                            reference, f/or_gauge_fixing1.f:174) or LCE_GF_ATAN2 */
  int sweep_mode;        /* LCE_SWEEP_AUTO (time the forms on the first sweeps
                            and keep the fastest), LCE_SWEEP_PASSES,
                            LCE_SWEEP_PASSES2, LCE_SWEEP_PERSISTENT or
                            LCE_SWEEP_DIRECT */
  int agauge_hits;       /* link update of lce_sweep: 1 = f/agauge.f (default;
                            0 is read as 1), 3 = f/agauge1.f (three heatbath +
                            Metropolis hits per link) -- the reference selects
                            one of the two files at build time */
  int tile_threads;      /* threads per block of the per-pass update kernels:
                            0 (default) = tuned with LCE_SWEEP_AUTO, else 256;
                            or 128, 256, 448, 512 (448: one site per thread
                            only).  FP32 only: the FP64 validation
                            path and z-slabs use 256.  Results do not depend on
                            it (per-site work and random numbers are the same;
                            FP64 sums are grouped per tile). */
  int tile_registers;    /* per-thread register cap of those kernels: 0
                            (default: 64 in FP32), or 56 with tile_threads =
                            128 (nine blocks per SM; FP32 only) */
} lce_params;

/* Measured quantities: /aver_loc/ (plaq0, a0kin, a02, a04, a0f) and the
 * acceptances of f/INCLUDE/measurement.inc, in FP64. */
typedef struct lce_meas {
  double plaq;        /* agauge plaquette against the pre-update staple, /(12V) */
  double akin;        /* sum a.F / (6V) of the last Higgs update */
  double a2;          /* <A^2> of the last Higgs update */
  double a4;          /* <A^4> of the last Higgs update */
  double acc_gauge;   /* agauge accept (KP rate x Metropolis rate / 4) */
  double acc_hb;      /* ahiggs2 accept */
  double acc_or;      /* ahiggs3 accept */
  double acc_metro;   /* ahiggs1 accept */
  double acc_link_or; /* link overrelaxation accept */
  double delta;       /* current ahiggs1 step */
  double af[3];       /* meas2a: average of A_f */
} lce_meas;

/* ---- library ---- */
const char* lce_version(void);
const char* lce_strerror(int status);
/* last CUDA/validation error message of a context (or of the last failed create) */
const char* lce_last_error(lce_ctx* ctx);
void lce_default_params(lce_params* p);
/* f/paraminit.f:150-153: beta_a, beta_2, beta_4 from beta, x, y (FP64) */
int lce_couplings(const lce_params* p, double out[3]);
/* f/adresses.f:91-337 neighbour tables (single rank, periodic), 0-based:
 * t[(eo*3 + mu)*nh + site]; computed by the same index arithmetic the kernels use */
int lce_geometry_tables(int L1, int L2, int L3, int* siteup, int* sitedn);

/* ---- context (replaces f/initialize.f:23-53 state set-up for the hot path) ---- */
lce_ctx* lce_create(const lce_params* p);
/* many independent chains (uneven volumes and couplings) in one context;
 * every update call advances all chains together */
lce_ctx* lce_create_batch(const lce_params* p, int nchains);
void lce_destroy(lce_ctx* ctx);
int lce_nchains(lce_ctx* ctx);
/* lattice extents of a chain */
int lce_get_extents(lce_ctx* ctx, int chain, int L[3]);
int lce_set_stream(lce_ctx* ctx, void* cuda_stream); /* NULL: the context's own stream */
int lce_synchronize(lce_ctx* ctx);

/* ---- fields (COMMON /linkvar/ mirrors; f/confget.f / f/confsave.f boundary) ---- */
int lce_upload(lce_ctx* ctx, int chain, int which, const float* u, const float* a, long ld);
int lce_upload_f64(lce_ctx* ctx, int chain, int which, const double* u, const double* a, long ld);
/* lce_upload without waiting, FP32 contexts.  lce_upload_stage queues the
 * host-to-device copy on a copy stream of the context, into one of two
 * staging slots; lce_upload_apply makes the update calls queued after it see
 * the oldest staged upload (a device copy on the context stream, after the
 * staged copy).  At most two uploads are staged and not yet applied.  The host
 * buffers must stay unchanged until the next call that synchronises the
 * context stream after the apply (lce_synchronize, lce_get_meas, lce_sweep
 * with an lce_meas, lce_download).  Pinned buffers let the copy overlap the
 * work queued before it: a streaming client stages step k+2's input while
 * step k sweeps and step k+1's is applied behind it.
 * lce_upload_async = lce_upload_stage + lce_upload_apply (nothing staged). */
int lce_upload_stage(lce_ctx* ctx, int chain, int which, const float* u, const float* a, long ld);
int lce_upload_apply(lce_ctx* ctx);
int lce_upload_async(lce_ctx* ctx, int chain, int which, const float* u, const float* a, long ld);
int lce_download(lce_ctx* ctx, int chain, int which, float* u, float* a, long ld);
int lce_download_f64(lce_ctx* ctx, int chain, int which, double* u, double* a, long ld);
/* f/confget.f unitconf (:295-307): U = 1, A = (0, 0, a3) on every chain */
int lce_init_unit(lce_ctx* ctx, double a3);
/* hot start: Haar links (normalised 4-Gaussians), A components ~ N(0,1) */
int lce_init_hot(lce_ctx* ctx, unsigned long long seed);

/* ---- configuration files (f/confsave.f:18-258, f/confget.f oldconf :318-526) ----
 * Direct-access unformatted records, single precision: links one record per
 * (mu, eo, z), Higgs one per (eo, z), each one global xy slice in half-row
 * order, record lengths u_rl = 16*2*L1*L2/2 and a_rl = 8*3*L1*L2/2 bytes as the
 * reference declares them (payload first, zero padding).  lce_confsave also
 * writes "<u_path>.rng" (Philox pass counter); lce_confget restores it when
 * present, so a resumed chain continues its random stream. */
int lce_confsave(lce_ctx* ctx, int chain, const char* u_path, const char* a_path);
int lce_confget(lce_ctx* ctx, int chain, const char* u_path, const char* a_path);
/* f/measinit.f file names: "<prefix>_sLL_beBBBBB_xXXXXX_yYYYYY_uNNNNNN" with
 * BBBBB = nint(1000 beta), XXXXX = nint(10000 x), YYYYY = nint(10000 y); the
 * reference's lower-case "_be" / "_u" form is used for saving too */
int lce_conf_filename(char* buf, size_t n, const char* prefix, int L3, double beta, double x, double y,
                      int number);

/* ---- random numbers ---- */
/* validation mode (LCE_RNG_STREAM, single chain): uniforms consumed in the
 * reference's order, 29*V per reference sweep (f/heat_kpi.f, f/gauss.f,
 * f/agauge.f, f/ahiggs2.f, f/ahiggs3.f draw order) */
int lce_set_rng_stream(lce_ctx* ctx, const double* uniforms, size_t n);
int lce_get_rng_position(lce_ctx* ctx, unsigned long long* pass_ctr, unsigned long long* stream_pos);
int lce_set_rng_position(lce_ctx* ctx, unsigned long long pass_ctr, unsigned long long stream_pos);

/* ---- Monte Carlo updates (accept may be NULL: no synchronisation) ---- */
/* f/ahiggs1.f:7-127 Metropolis; *delta is adapted as the reference does */
int lce_ahiggs1(lce_ctx* ctx, float* delta, int measflag, float* accept);
/* f/ahiggs2.f:7-152 heatbath (with f/a_force.f, f/gauss.f) */
int lce_ahiggs2(lce_ctx* ctx, int measflag, float* accept);
/* f/ahiggs3.f:7-148 overrelaxation */
int lce_ahiggs3(lce_ctx* ctx, int measflag, float* accept);
/* f/agauge.f:7-205 with f/staples.f, f/heat_kpi.f */
int lce_agauge(lce_ctx* ctx, int measflag, float* accept);
/* f/agauge1.f:7-237: the 3-hit link update (staple once per (parity, mu),
 * then three heatbath + Metropolis hits of 7 uniforms per site each; the
 * acceptance divides the Metropolis count by the hits, :227-232) */
int lce_agauge1(lce_ctx* ctx, int measflag, float* accept);
/* link overrelaxation with the agauge Metropolis test (no reference counterpart) */
int lce_link_or(lce_ctx* ctx, int measflag, float* accept);
/* f/renorm.f:6-37 */
int lce_renorm(lce_ctx* ctx);
/* f/main.f:38-41: ahiggs2, ahiggs3, [ahiggs1 x n_higgs_metro], agauge,
 * [link OR x n_link_or], reunitarisation fused into the link writers; one
 * CUDA graph per measflag.  m (chain 0) may be NULL: no synchronisation. */
int lce_sweep(lce_ctx* ctx, int measflag, lce_meas* m);
/* nsweeps sweeps as graph replays without synchronisation (graphs of 8 sweeps
 * while nsweeps allows, whose sweeps chain by programmatic launch, then
 * one-sweep graphs; with LCE_SWEEP_AUTO the first sweeps of a context rotate
 * through the forms and tile shapes under CUDA events -- every one of them a
 * real sweep -- and the fastest is kept) */
int lce_sweeps(lce_ctx* ctx, int nsweeps, int measflag);
/* the form lce_sweeps uses now (LCE_SWEEP_AUTO while still undecided) */
int lce_get_sweep_mode(lce_ctx* ctx);
/* the tile shape of the update kernels in use: threads per block, sites per
 * thread and the per-thread register cap they are compiled for (a tuned
 * choice once lce_get_sweep_mode is no longer AUTO); any output may be NULL */
int lce_get_tile_shape(lce_ctx* ctx, int* threads, int* sites_per_thread, int* register_cap);
/* f/meas1.f inputs: the last measured quantities of a chain */
int lce_get_meas(lce_ctx* ctx, int chain, lce_meas* m);
int lce_get_meas_batch(lce_ctx* ctx, lce_meas* m /* [nchains] */);

/* ---- gauge fixing (f/landau_gauge.f:6-63, f/or_gauge_fixing1.f) ---- */
/* copy U,A -> U_f,A_f, iterate overrelaxed gauge fixing until theta <= limit_or.
 * max_iters <= 0 means no cap (the reference has none).  Returns
 * LCE_ERR_GF_NOT_CONVERGED when the cap ends the loop. */
int lce_landau_gauge(lce_ctx* ctx, int chain, double* theta, int* iters, int max_iters);
/* iterate on the current U_f,A_f without the copy (warm starts, continuation) */
int lce_gauge_fix_continue(lce_ctx* ctx, int chain, double* theta, int* iters, int max_iters);
/* Gauge fixing that also tracks the accumulated transform G, with
 * U_f(x,mu) = G(x) U(x,mu) G(x+mu)^+ and A_f = G A G^+ throughout (no
 * reference counterpart: the reference keeps no transform).  start:
 *   LCE_GF_START_IDENTITY   G = 1 (the reference's start, f/landau_gauge.f:33-49)
 *   LCE_GF_START_TRANSFORM  start from the context's current G (warm start:
 *                           the previous measurement's converged transform,
 *                           a transform set by lce_set_transform)
 * theta_start (may be NULL) receives theta of the starting U_f. */
#define LCE_GF_START_IDENTITY 0
#define LCE_GF_START_TRANSFORM 1
int lce_landau_gauge_from(lce_ctx* ctx, int chain, int start, double* theta_start, double* theta, int* iters,
                          int max_iters);
/* Fourier-accelerated Landau gauge fixing (no reference counterpart; Davies
 * et al., Phys. Rev. D 37 (1988) 1581).  Each step rotates every site by
 * g = exp(-i omega.sigma), omega = step * F^-1[F[Delta]/p^2], Delta the
 * divergence of the gauge field (the vector part whose square is theta) and
 * p^2 the lattice Laplacian with the functional's weights (1, 1, alpha), so
 * that long wavelengths relax as fast as short ones.  From `start` (as in
 * lce_landau_gauge_from; G is tracked) it iterates until theta <=
 * theta_switch (<= 0: limit_or); if that is above limit_or the plain
 * overrelaxed iteration continues to theta <= limit_or -- the stopping
 * criterion of lce_landau_gauge either way.  step <= 0 selects 1 (a Newton
 * step near the Landau gauge); a step that doubles theta is shortened by 0.7
 * on the device.  Extents must be powers of two up to 1024, else
 * LCE_ERR_UNSUPPORTED.  max_iters caps both phases together. */
int lce_landau_gauge_fourier(lce_ctx* ctx, int chain, int start, double step, double theta_switch, double* theta,
                             int* iters_fourier, int* iters_plain, int max_iters);
/* The same fixing by nonlinear conjugate gradients with the same Fourier
 * preconditioner (after Hudspith, Comput. Phys. Commun. 187 (2015) 115):
 * direction s = F^-1[F[Delta]/p^2] + beta s_prev, beta = max(0,
 * Polak-Ribiere), and the step along s that maximises the second-order
 * expansion of the gauge functional (its derivatives exact per link, summed
 * in FP64), bounded by a trust region on the rotation angle.
 * No reference counterpart; arguments and stopping criterion as
 * lce_landau_gauge_fourier (no step argument). */
int lce_landau_gauge_fourier_cg(lce_ctx* ctx, int chain, int start, double theta_switch, double* theta,
                                int* iters_fourier, int* iters_plain, int max_iters);
/* The reference's iterative gauge fixing, f/it_gauge_fixing.f:5-206
 * (compiled into the reference, never called by it).  One iteration, parity
 * by parity: g = antihermitian part of sum_mu [U_f(x,mu) - U_f(x-mu,mu)]
 * in first-row form, Omega = exp(step g) = cos|step g| + step g
 * sin|step g|/|step g|, U_f and A_f transformed as in the overrelaxed
 * iteration; *da1 = mean |g|^2 over the second parity, before its step
 * (f/it_gauge_fixing.f:116-120).  step <= 0 takes the context's alpha, the
 * reference's step.  flags:
 *   LCE_ITGF_FIX_COMPONENT  second component g1(2) - g2(2); the reference
 *                           writes g1(1) - g2(2) (f/it_gauge_fixing.f:110),
 *                           with which the iteration does not converge
 *   LCE_ITGF_ASCEND         Omega = exp(-step g): raises the Landau
 *                           functional (the reference's sign lowers it and
 *                           ends at the Z2 mirror, U_f -> -U_f on one
 *                           parity's transform, physically equivalent)
 *   LCE_ITGF_TRACK          also G(x) -> Omega(x) G(x)
 * The single iteration does not reunitarise (the reference's subroutine
 * does not).  Steepest descent is stable only for steps below ~1/3. */
#define LCE_ITGF_FIX_COMPONENT 1
#define LCE_ITGF_ASCEND 2
#define LCE_ITGF_TRACK 4
int lce_it_gauge_fixing(lce_ctx* ctx, int chain, double step, int flags, double* da1);
/* f/landau_gauge.f:28-59 with it_gauge_fixing in place of
 * or_gauge_fixing: copy U,A -> U_f,A_f (and G = 1 with LCE_ITGF_TRACK),
 * then iterate + reunitarise U_f until da1 <= limit_or, on the device in
 * captured batches like lce_landau_gauge.  max_iters <= 0: 10^6 cap;
 * LCE_ERR_GF_NOT_CONVERGED when the cap ends the loop. */
int lce_it_landau_gauge(lce_ctx* ctx, int chain, double step, int flags, double* da1, int* iters, int max_iters);
/* one preconditioned direction omega [2][V/2][3] (components a3, Re b, Im b
 * of the vector part, parity-split order) from the current U_f; nothing is
 * updated (test hook for the FFT path) */
int lce_debug_fourier_step(lce_ctx* ctx, int chain, double step, double* omega);
/* U_f, A_f := (U, A) transformed by the current G */
int lce_apply_transform(lce_ctx* ctx, int chain);
/* the transform field G: g[(eo*ld + site)*4 + c], SU(2) first rows like the links */
int lce_set_transform(lce_ctx* ctx, int chain, const float* g, long ld);
int lce_get_transform(lce_ctx* ctx, int chain, float* g, long ld);
/* gauge functional (1/((2+alpha)V)) sum_x,mu c_mu Re a of U_f */
int lce_gauge_functional(lce_ctx* ctx, int chain, double* value);
/* theta of the current U_f (odd sites, FP64), without updating */
int lce_theta(lce_ctx* ctx, int chain, double* theta);

/* ---- measurements ---- */
/* f/correlator.f:11-186 (z-slice correlators of A_f and U_f, all z) and
 * f/meas2a.f:39-49 (average of A_f); any output may be NULL */
int lce_correlator(lce_ctx* ctx, int chain, double* corr_a, double* corr_u, double* corr_3,
                   double af[3]);
/* f/polyakov.f:10-123: slice means of cos(4|A|), their correlator, mean^2 */
int lce_polyakov(lce_ctx* ctx, int chain, double* slice, double* corr, double* mean2);
/* f/scalarcorr.f:10-119: slice means of |A|^2, their correlator, mean */
int lce_scalarcorr(lce_ctx* ctx, int chain, double* slice, double* corr, double* mean);
/* average plaquette 1/2 Re Tr of the current U (all 3V plaquettes) */
int lce_plaquette(lce_ctx* ctx, int chain, double* plaq);

/* ---- validation entry points (FP64 outputs) ---- */
/* staple V(x) of f/staples.f for (eo, mu): out[site*4 + c] */
int lce_debug_staple(lce_ctx* ctx, int eo, int mu, double* out);
/* Higgs force F(x) of f/a_force.f for parity eo: out[site*3 + k] */
int lce_debug_force(lce_ctx* ctx, int eo, double* out);

/* ---- timing ---- */
/* write a device buffer larger than L2 (126 MB) on the context stream */
int lce_flush_l2(lce_ctx* ctx);
/* one sweep (per-pass form, the tile shape in use) as a CUDA graph with a
 * timing event at its start and after every kernel, each on a side stream
 * forked from the context stream, so the passes keep their
 * programmatic-dependent-launch overlap and every difference carries the
 * same fork latency: ms[i] = completion of pass i minus completion of pass
 * i-1 (pass 0: minus the graph's start; 10 passes for the reference
 * composition), ms[npasses] = the finalize kernel's (when max_passes >
 * npasses); returns the pass count */
int lce_profile_sweep(lce_ctx* ctx, int measflag, float* ms, int max_passes);
/* events on the context stream */
int lce_timer_start(lce_ctx* ctx);
int lce_timer_stop(lce_ctx* ctx, float* ms);


/* ---- z-slab decomposition (f/topology.f with dimproc = (1, 1, n): the
 * reference's MPI domain decomposition and the halo exchange of
 * f/staples.f / f/a_force.f), for lattices larger than one GPU's memory.
 * The lattice of *p is split along z into nslabs slabs of L3/nslabs planes
 * (an even number >= 2); slab k lives on devices[k] (a device may hold
 * several).  A slab keeps one halo plane on each side; after every pass the
 * written field's boundary planes are copied to the neighbouring slabs
 * (peer copies between devices, ordered by events).  The Philox counters use
 * whole-lattice site indices, so the fields after a sweep are bit for bit
 * those of an undecomposed context with the same seed; measurements are the
 * whole lattice's (sums over slabs, in another order), and the ahiggs1 step
 * adapts to the whole lattice's acceptance.  Philox uniforms, or in FP64 the
 * validation stream (lce_slabs_set_rng_stream); the sweep composition of
 * lce_sweep.  Gauge fixing (the overrelaxed method of lce_landau_gauge) and
 * the z-slice measurements also run on the slabs. */
typedef struct lce_slabs lce_slabs;
lce_slabs* lce_slabs_create(const lce_params* p, int nslabs, const int* devices);  /* NULL: lce_last_error(NULL) */
void lce_slabs_destroy(lce_slabs* s);
/* the whole lattice in the reference order of lce_upload / lce_download */
int lce_slabs_upload(lce_slabs* s, const float* u, const float* a, long ld);
int lce_slabs_upload_f64(lce_slabs* s, const double* u, const double* a, long ld);
int lce_slabs_download(lce_slabs* s, float* u, float* a, long ld);
int lce_slabs_download_f64(lce_slabs* s, double* u, double* a, long ld);
/* one sweep of f/main.f:38-41 over all slabs; m (may be NULL) receives the
 * whole lattice's measurements when measflag = 1 */
int lce_slabs_sweep(lce_slabs* s, int measflag, lce_meas* m);
/* validation mode (slabs created with LCE_RNG_STREAM, LCE_PREC_F64): the
 * whole lattice's uniform stream, in the reference's consumption order
 * (lce_set_rng_stream), copied to every slab; each slab draws the slots of
 * its own sites, so a slab sweep consumes the stream exactly as the
 * undecomposed lattice (and the reference at one rank) does */
int lce_slabs_set_rng_stream(lce_slabs* s, const double* u, size_t n);
/* u_f, a_f (LCE_FIELDS_FIXED of lce_download) of the whole lattice */
int lce_slabs_download_fixed(lce_slabs* s, float* u, float* a, long ld);
int lce_slabs_download_fixed_f64(lce_slabs* s, double* u, double* a, long ld);
/* lce_landau_gauge (f/landau_gauge.f:33-49, f/or_gauge_fixing1.f) on the
 * slabs: a half-step's update of the U_z links below a slab's first plane
 * goes back to the slab below, theta is the whole lattice's; same iterations
 * and (up to the order of the theta sum) the same u_f, a_f as undecomposed */
int lce_slabs_landau_gauge(lce_slabs* s, double* theta, int* iters, int max_iters);
/* the same fixing tracking the gauge transform G (lce_landau_gauge_from on
 * the slabs), from G = 1 (LCE_GF_START_IDENTITY) or from the transform of
 * the slabs' last tracked fixing applied to the current fields
 * (LCE_GF_START_TRANSFORM, the previous measurement's warm start); same
 * iterations and u_f, a_f as undecomposed */
int lce_slabs_landau_gauge_from(lce_slabs* s, int start, double* theta, int* iters, int max_iters);
/* lce_landau_gauge_fourier on the slabs (G tracked; start IDENTITY or
 * TRANSFORM): the divergence, g and its application run on every slab's
 * planes, the x transforms of a slab's lines too; the whole lattice's two
 * transformed fields (16 bytes per site) live on the first slab's device,
 * where the y and z transforms run.  Same iterations and u_f, a_f as
 * undecomposed.  Extents: powers of two up to 1024. */
int lce_slabs_landau_gauge_fourier(lce_slabs* s, int start, double step, double theta_switch, double* theta,
                                   int* iters_fourier, int* iters_plain, int max_iters);
/* lce_landau_gauge_fourier_cg on the slabs: the stages of
 * lce_slabs_landau_gauge_fourier with the conjugate-gradient direction (its
 * halo plane exchanged), the momentum-space sums on the first slab's device
 * and the line search summed per slab.  The step's sums are grouped per slab,
 * so the run takes steps equal to the undecomposed run's but for the last
 * bits: the same iterations, u_f, a_f equal within what the stopping theta
 * leaves free (~1e-8 at theta < 1e-10 in FP64), not bit for bit. */
int lce_slabs_landau_gauge_fourier_cg(lce_slabs* s, int start, double theta_switch, double* theta,
                                      int* iters_fourier, int* iters_plain, int max_iters);
/* lce_it_landau_gauge (f/it_gauge_fixing.f under f/landau_gauge.f) on the
 * slabs: the same halo traffic as lce_slabs_landau_gauge; same iterations
 * and u_f, a_f as undecomposed */
int lce_slabs_it_landau_gauge(lce_slabs* s, double step, int flags, double* da1, int* iters, int max_iters);
/* lce_correlator / lce_polyakov / lce_scalarcorr of the whole lattice
 * (f/correlator.f, f/polyakov.f, f/scalarcorr.f): slice sums per slab,
 * correlated on the first slab's device */
int lce_slabs_correlator(lce_slabs* s, double* corr_a, double* corr_u, double* corr_3, double af[3]);
int lce_slabs_polyakov(lce_slabs* s, double* slice, double* corr, double* mean2);
int lce_slabs_scalarcorr(lce_slabs* s, double* slice, double* corr, double* mean);

/* ---- allocation-free measurement ----
 * No counterpart in the reference.  For callers that cannot let this library
 * allocate device memory -- a driver whose GPU memory belongs to another
 * allocator (a caching allocator or a CUDA Fortran pool) or a fixed budget,
 * or code between asynchronous launches where cudaMalloc/cudaFree could
 * synchronise the device.  Average plaquette (1/2 Re Tr, all 3V plaquettes)
 * of a caller-owned FP32 link field u (device memory, reference order, leading
 * dimension ld >= V/2, 16-byte aligned), written to *plaq (device memory) on
 * `stream` (a cudaStream_t; NULL = default stream).  No host synchronisation.
 * Allocates nothing: the per-block scratch is a fixed 512 KiB __device__
 * array held by every GPU that loads the library; lattices larger than
 * 16,777,216 sites (256^3) are rejected with LCE_ERR_INVALID.  The first call
 * on a device looks up the array's address (make it before any stream
 * capture) and keeps it for the life of the process: do not call it across a
 * cudaDeviceReset, which reloads the module elsewhere.  All calls share the
 * array: calls whose kernels overlap on the GPU race and must be serialised
 * by the caller. */
int lce_plaquette_noalloc(const float* u, long ld, int L1, int L2, int L3, double* plaq, void* stream);

/* ---- learned warm start for Landau gauge fixing (no reference counterpart;
 * the reference always starts f/landau_gauge.f from G = 1).
 * A 4-layer, 16-channel, 3x3x3 periodic convolutional network (BF16 weights
 * and activations, FP32 accumulation on the tensor cores) maps the
 * configuration in the gauge of the previous converged transform G_prev
 * (12 link components of U_f and 3 of A_f per site) to a unit quaternion
 * Omega(x); the warm start is G = Omega G_prev.  The network is trained on
 * the device from pairs recorded by lce_landau_gauge_warm (target: the
 * converged G_new G_prev^+; loss 1 - Omega . target per site, Adam).
 * Nothing about the gauge-fixed result depends on the network: the plain
 * overrelaxed iteration runs to the same theta <= limit_or from whichever
 * start is taken.  A network object is not thread-safe. */
typedef struct lce_net lce_net;
lce_net* lce_net_create(int device, unsigned long long seed);  /* untrained: Omega = 1 */
void lce_net_destroy(lce_net* net);
int lce_net_num_params(lce_net* net);
/* parameters, FP32 master copy: per layer [27][16 out][16 in] weights then 16 biases */
int lce_net_get_params(lce_net* net, float* w);
int lce_net_set_params(lce_net* net, const float* w);
int lce_net_save(lce_net* net, const char* path);
int lce_net_load(lce_net* net, const char* path);
/* forward + loss + gradient on caller data, no update: feat [2][V/2][16]
 * (parity-split site order, rounded to BF16), target [2][V/2][4]; out
 * [2][V/2][4] (raw network output) and grad [nparam] may be NULL */
int lce_net_eval(lce_net* net, int L1, int L2, int L3, const float* feat, const float* target, float* out,
                 float* grad, double* loss);
int lce_net_num_pairs(lce_net* net);
int lce_net_clear_pairs(lce_net* net);
/* `epochs` Adam passes over the recorded pairs; *mean_loss = last epoch's */
int lce_net_train(lce_net* net, int epochs, double lr, double* mean_loss);

/* Tracked gauge fixing of `chain` from a warm start.  Candidates: the
 * identity (0), the previous transform G_prev held by the context (1), and,
 * with LCE_WARM_NET, the network's Omega G_prev (2).  With LCE_WARM_JUDGE
 * every candidate's gauge functional is evaluated (functional[0..2], NaN for
 * one not evaluated) and the start with the largest is taken -- the fallback
 * to the plain start when the prediction is worse; otherwise the network's
 * start (LCE_WARM_NET) or G_prev.  LCE_WARM_RECORD stores the pair
 * (configuration in G_prev gauge, G_new G_prev^+) for lce_net_train after
 * convergence.  LCE_WARM_FOURIER iterates from the chosen start with the
 * Fourier-accelerated step of lce_landau_gauge_fourier instead of the plain
 * overrelaxation (power-of-two extents); with LCE_WARM_CG as well, the
 * conjugate-gradient form of lce_landau_gauge_fourier_cg.  net may be NULL
 * when neither NET nor RECORD is set. */
#define LCE_WARM_NET 1
#define LCE_WARM_JUDGE 2
#define LCE_WARM_RECORD 4
#define LCE_WARM_FOURIER 8
#define LCE_WARM_CG 16
#define LCE_GF_START_NET 2
int lce_landau_gauge_warm(lce_ctx* ctx, int chain, lce_net* net, int flags, int* start_used, double functional[3],
                          double* theta, int* iters, int max_iters);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* LCEQCD_GPU_H */
