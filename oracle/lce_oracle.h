/*
 * lce_oracle.h -- CPU restatement of the lceqcd Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle for the
 * CUDA path in lceqcd_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * path never calls it.
 *
 * It restates, in the reference's site order and random-number consumption
 * order, the single-rank (nproc = 1) semantics of:
 *   couplings        f/paraminit.f:150-153 (sigma at :47 of the original, 290 here)
 *   geometry         f/adresses.f:91-337 (dimproc = 1 periodic branch)
 *   SU(2) products   f/matmul.f:1-194
 *   staples          f/staples.f:65-221
 *   KP heatbath      f/heat_kpi.f:9-101
 *   link update      f/agauge.f:7-205
 *   Higgs force      f/a_force.f:7-115
 *   gauss            f/gauss.f:10-31
 *   Higgs updates    f/ahiggs1.f, f/ahiggs2.f, f/ahiggs3.f
 *   reunitarisation  f/renorm.f, f/u_f_renorm.f
 *   gauge fixing     f/landau_gauge.f, f/or_gauge_fixing1.f, f/it_gauge_fixing.f
 *   measurements     f/correlator.f, f/polyakov.f, f/scalarcorr.f,
 *                    f/meas1.f, f/meas2a.f
 *   RANLUX           f/luxury.f (pinned to the expected output in f/luxtst.f:88-162)
 *   configurations   f/confget.f unitconf/randomconf/testconf
 *
 * Parity status: RANLUX is pinned to the reference's own known-answer block.
 * The Monte Carlo routines are "parity unpinned": the reference ships no
 * golden vectors for them and cannot be compiled here (Fortran + MPI, no
 * Fortran compiler in the image), so the restatement is checked only by
 * derived known answers (unit configuration, gauge invariance/covariance,
 * testconf closed forms, stream-consumption counts) in tests/.
 *
 * Build: FP64 (default) or FP32 (-DLCE_ORACLE_F32).  Measurement sums are
 * accumulated in double in both modes.
 */
#ifndef LCE_ORACLE_H
#define LCE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef LCE_ORACLE_F32
typedef float lco_real;
#else
typedef double lco_real;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* uniform sources */
enum { LCO_SRC_STREAM = 0, LCO_SRC_RANLUX = 1, LCO_SRC_PHILOX = 2 };

typedef struct lco_ctx lco_ctx;

typedef struct lco_meas {
  double plaq, akin, a2, a4;          /* /aver_loc/ after the last update */
  double acc_gauge, acc_hb, acc_or, acc_metro;
  double af[3];                       /* meas2a average of A_f */
} lco_meas;

/* ---- RANLUX (f/luxury.f) ---- */
void lco_ranlux_default(void);                 /* reset to "never initialised" */
void lco_rluxgo(int lux, int ins, int k1, int k2);
void lco_ranlux(float *rvec, int lenv);
void lco_rluxut(int32_t isdext[25]);
void lco_rluxin(const int32_t isdext[25]);
void lco_rluxat(int *lout, int *inout, int *k1, int *k2);

/* ---- Philox4x32-10 (Salmon et al., SC'11) ---- */
void lco_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double lco_u01(uint32_t x);

/* ---- context ---- */
lco_ctx *lco_create(int L1, int L2, int L3, double beta, double x, double y,
                    double lambda, double alpha, double limit_or, int imode);
void lco_destroy(lco_ctx *c);
int  lco_nh(const lco_ctx *c);
void lco_set_threads(lco_ctx *c, int n);
void lco_couplings(const lco_ctx *c, double out[3]);     /* beta_a, beta_2, beta_4 */

/* uniform source selection */
void lco_set_stream(lco_ctx *c, const double *u, size_t n);  /* LCO_SRC_STREAM */
size_t lco_stream_pos(const lco_ctx *c);
void lco_set_ranlux_source(lco_ctx *c);                       /* LCO_SRC_RANLUX */
void lco_set_philox(lco_ctx *c, uint64_t seed, uint64_t pass_ctr); /* LCO_SRC_PHILOX */
uint64_t lco_pass_ctr(const lco_ctx *c);
/* gauge-fixing rotation angle: 0 = acos(Re Omega) as f/or_gauge_fixing1.f:174
 * (default), 1 = atan2(|vector part|, scalar part), accurate for small angles */
void lco_set_gf_angle(lco_ctx *c, int mode);

/* field access in the reference's COMPLEX u(2,site,eo,mu) / REAL a(3,site,eo)
 * order with ld = nh:  u[((mu*2+eo)*nh+site)*4 + {re a, im a, re b, im b}],
 * a[(eo*nh+site)*3 + k]. which: 0 = u/a, 1 = u_f/a_f. */
void lco_set_fields(lco_ctx *c, int which, const lco_real *u, const lco_real *a);
void lco_get_fields(const lco_ctx *c, int which, lco_real *u, lco_real *a);
void lco_get_staple(const lco_ctx *c, lco_real *v);
void lco_get_force(const lco_ctx *c, lco_real *f);    /* last a_force: [site][3] */

/* geometry tables, 0-based: t[(eo*3+mu)*nh + site] */
void lco_tables(const lco_ctx *c, int *siteup, int *sitedn);

/* configurations (f/confget.f) */
void lco_unitconf(lco_ctx *c, double a3);
int  lco_randomconf(lco_ctx *c);     /* consumes 3*3V + 2V sequential uniforms */
void lco_testconf(lco_ctx *c);

/* hot path (return 0 or negative on exhausted stream) */
int  lco_staples(lco_ctx *c, int eo, int mu);   /* fills v(:,:,eo,mu) */
int  lco_a_force(lco_ctx *c, int eo);
int  lco_ahiggs1(lco_ctx *c, lco_real *delta, int measflag, lco_real *accept);
int  lco_ahiggs2(lco_ctx *c, int measflag, lco_real *accept);
int  lco_ahiggs3(lco_ctx *c, int measflag, lco_real *accept);
int  lco_agauge(lco_ctx *c, int measflag, lco_real *accept);
/* f/agauge1.f: the 3-hit form (staple once per pass, three heatbath +
 * Metropolis hits of 7 uniforms per site each) */
int  lco_agauge1(lco_ctx *c, int measflag, lco_real *accept);
int  lco_link_or(lco_ctx *c, int measflag, lco_real *accept);
void lco_renorm(lco_ctx *c);
int  lco_sweep(lco_ctx *c, int measflag, lco_meas *m);   /* main.f:38-41 order */

/* gauge fixing and measurements */
void lco_landau_copy(lco_ctx *c);
double lco_or_gauge_fixing(lco_ctx *c);          /* one iteration, returns da1 */
void lco_u_f_renorm(lco_ctx *c);
int  lco_landau_gauge(lco_ctx *c, int max_iters, double *da1);  /* returns iterations */
/* f/it_gauge_fixing.f: one iteration (returns da1); flags 1 = second
 * component from g1(2), 2 = rotate by exp(-step g) */
double lco_it_gauge_fixing(lco_ctx *c, double step, int flags);
int  lco_it_landau_gauge(lco_ctx *c, double step, int flags, int max_iters, double *da1);
double lco_gauge_functional(const lco_ctx *c);   /* (1/3V) sum Re Tr_2/2 U_f */
double lco_theta_direct(const lco_ctx *c);       /* mean over odd sites, fresh */
void lco_correlator(const lco_ctx *c, double *corr_a, double *corr_u, double *corr_3);
void lco_polyakov(const lco_ctx *c, double *slice, double *corr, double *mean2);
void lco_scalarcorr(const lco_ctx *c, double *slice, double *corr, double *mean);
void lco_meas2(const lco_ctx *c, double af[3]);
double lco_plaquette(const lco_ctx *c);          /* fresh average plaquette */
void lco_get_meas(const lco_ctx *c, lco_meas *m);

#ifdef __cplusplus
}
#endif
#endif
