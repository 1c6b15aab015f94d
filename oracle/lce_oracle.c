/*
 * lce_oracle.c -- CPU restatement of the lceqcd Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the correctness oracle and the timed CPU
 * baseline ("port") for the CUDA path.  See lce_oracle.h for the list of
 * reference routines restated here; each function below cites the
 * reference lines it follows.
 *
 * Semantics are single-rank (nproc = 1, dimproc = 1): the MPI halo exchanges
 * of the reference are no-ops and the neighbour tables wrap periodically
 * (f/adresses.f dimproc == 1 branches).
 *
 * Random numbers.  The reference draws uniforms one at a time inside its site
 * loops.  Here every update pass first materialises the uniforms it needs in
 * the reference's consumption order (see draw_pass), then runs its site loops
 * (OpenMP-parallel) indexing that buffer.  The sources are:
 *   STREAM  a host-supplied array, consumed sequentially (validation mode);
 *   RANLUX  the f/luxury.f generator, consumed sequentially;
 *   PHILOX  counter-based: slot k of site s in a pass is word k&3 of
 *           Philox4x32-10(key = seed, ctr = {s, k>>2, pass_lo, pass_hi}),
 *           with the pass counter advanced once per pass -- the same stream
 *           the CUDA production kernels draw.
 */
#include "lce_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef lco_real real;

/* complex in the Fortran sense (default COMPLEX of the build's real type) */
typedef struct { real re, im; } cplx;
/* SU(2) element stored as its first row (a, b): {{a, b}, {-b*, a*}},
 * f/INCLUDE/gaugefield.inc:39-51 */
typedef struct { cplx a, b; } su2;

static inline cplx cmul(cplx x, cplx y) {
  cplx r = {x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re};
  return r;
}
static inline cplx cconj(cplx x) { cplx r = {x.re, -x.im}; return r; }
static inline cplx cadd(cplx x, cplx y) { cplx r = {x.re + y.re, x.im + y.im}; return r; }
static inline cplx csub(cplx x, cplx y) { cplx r = {x.re - y.re, x.im - y.im}; return r; }
static inline cplx cneg(cplx x) { cplx r = {-x.re, -x.im}; return r; }
static inline cplx cmk(real re, real im) { cplx r = {re, im}; return r; }

/* f/matmul.f MULTALLNN:22-23  U1*U2 */
static inline su2 mul_nn(su2 u1, su2 u2) {
  su2 h;
  h.a = csub(cmul(u1.a, u2.a), cmul(u1.b, cconj(u2.b)));
  h.b = cadd(cmul(u1.a, u2.b), cmul(u1.b, cconj(u2.a)));
  return h;
}
/* MULTALLDN:52-56  U1^+ * U2 */
static inline su2 mul_dn(su2 u1, su2 u2) {
  su2 h;
  h.a = cadd(cmul(cconj(u1.a), u2.a), cmul(u1.b, cconj(u2.b)));
  h.b = csub(cmul(cconj(u1.a), u2.b), cmul(u1.b, cconj(u2.a)));
  return h;
}
/* MULTALLND:85-89  U1 * U2^+ */
static inline su2 mul_nd(su2 u1, su2 u2) {
  su2 h;
  h.a = cadd(cmul(u1.a, cconj(u2.a)), cmul(u1.b, cconj(u2.b)));
  h.b = cadd(cneg(cmul(u1.a, u2.b)), cmul(u1.b, u2.a));
  return h;
}
/* MULTALLDD:118-122  U1^+ * U2^+ */
static inline su2 mul_dd(su2 u1, su2 u2) {
  su2 h;
  h.a = csub(cmul(cconj(u1.a), cconj(u2.a)), cmul(u1.b, cconj(u2.b)));
  h.b = csub(cneg(cmul(cconj(u1.a), u2.b)), cmul(u1.b, u2.a));
  return h;
}
/* MULTALLAD:150-154  (iA) * U^+ with iA first row (i a3, a2 + i a1) */
static inline su2 mul_ad(const real *A, su2 u) {
  cplx x = cmk(0, A[2]), y = cmk(A[1], A[0]);
  su2 h;
  h.a = cadd(cmul(x, cconj(u.a)), cmul(y, cconj(u.b)));
  h.b = cadd(cneg(cmul(x, u.b)), cmul(y, u.a));
  return h;
}
/* MULTALLAN:183-187  (iA) * U */
static inline su2 mul_an(const real *A, su2 u) {
  cplx x = cmk(0, A[2]), y = cmk(A[1], A[0]);
  su2 h;
  h.a = csub(cmul(x, u.a), cmul(y, cconj(u.b)));
  h.b = cadd(cmul(x, u.b), cmul(y, cconj(u.a)));
  return h;
}

struct lco_ctx {
  int L[3], hx, nxy, nh, vol;
  real *u, *a, *uf, *af, *v;   /* u[((mu*2+eo)*nh+s)*4], a[(eo*nh+s)*3] */
  real *force;                 /* force[s*3+k] */
  int *up, *dn;                /* [(eo*3+mu)*nh + s] */
  real beta, x, y, lambda, alpha, limit_or;
  real beta_a, beta_2, beta_4;
  int imode;
  int src;
  const double *stream;
  size_t stream_n, stream_pos;
  uint32_t key[2];
  uint64_t pass_ctr;
  real *unif;                  /* per-pass uniform buffer */
  size_t unif_cap;
  /* /aver_loc/ and acceptance results */
  double plaq0, a0kin, a02, a04, a0f[3];
  double acc_gauge, acc_hb, acc_or, acc_metro;
  int nthreads;
  int gf_angle;                /* 0: acos (reference), 1: atan2 */
};

static inline su2 ld_su2(const real *p) {
  su2 r = {{p[0], p[1]}, {p[2], p[3]}};
  return r;
}
static inline void st_su2(real *p, su2 x) {
  p[0] = x.a.re; p[1] = x.a.im; p[2] = x.b.re; p[3] = x.b.im;
}
#define UIDX(c, mu, eo, s) ((((size_t)(mu) * 2 + (eo)) * (c)->nh + (s)) * 4)
#define AIDX(c, eo, s) (((size_t)(eo) * (c)->nh + (s)) * 3)
#define UP(c, eo, mu, s) ((c)->up[((size_t)(eo) * 3 + (mu)) * (c)->nh + (s)])
#define DN(c, eo, mu, s) ((c)->dn[((size_t)(eo) * 3 + (mu)) * (c)->nh + (s)])

/* ------------------------------------------------------------------ */
/* Philox4x32-10: two 32x32->64 multiplies per round, Weyl key bumps.   */
/* ------------------------------------------------------------------ */
void lco_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* (2k+1)/2^24 with k the top 23 bits: strictly inside (0,1), exact in float */
double lco_u01(uint32_t x) { return (double)((x >> 9) * 2u + 1u) * (1.0 / 16777216.0); }

/* ------------------------------------------------------------------ */
/* uniform materialisation                                             */
/* ------------------------------------------------------------------ */
/* Layout of a pass's uniforms in the reference's consumption order:
 *   PLANAR:  slot k of site s at k*nh + s (one site loop per slot);
 *   TRIPLE:  slots 0..2 interleaved per site (3s + k), later slots planar.
 * TRIPLE is f/heat_kpi.f:33-40 (a1,a2,a3 per site) followed by :54-56,
 * :76-78, :91-93 and the agauge accept loop f/agauge.f:167-168; it is also
 * f/ahiggs1.f:51-56 (3 per site) followed by :82-83. */
enum { LAY_PLANAR = 0, LAY_TRIPLE = 1 };

static inline size_t slot_off(int layout, int nh, int k, int s) {
  if (layout == LAY_TRIPLE && k < 3) return (size_t)3 * s + k;
  return (size_t)k * nh + s;
}

static int draw_pass(lco_ctx *c, int nslots, int layout) {
  size_t n = (size_t)nslots * c->nh;
  if (n > c->unif_cap) {
    free(c->unif);
    c->unif = (real *)malloc(n * sizeof(real));
    c->unif_cap = n;
  }
  if (c->src == LCO_SRC_STREAM) {
    if (c->stream_pos + n > c->stream_n) return -1;
    for (size_t i = 0; i < n; ++i) c->unif[i] = (real)c->stream[c->stream_pos + i];
    c->stream_pos += n;
  } else if (c->src == LCO_SRC_RANLUX) {
    float buf[256];
    size_t i = 0;
    while (i < n) {
      int m = (int)((n - i) < 256 ? (n - i) : 256);
      lco_ranlux(buf, m);
      for (int j = 0; j < m; ++j) c->unif[i + j] = (real)buf[j];
      i += (size_t)m;
    }
  } else {
    const int nh = c->nh;
    const uint32_t plo = (uint32_t)c->pass_ctr, phi = (uint32_t)(c->pass_ctr >> 32);
    const int ncalls = (nslots + 3) / 4;
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      for (int q = 0; q < ncalls; ++q) {
        uint32_t ctr[4] = {(uint32_t)s, (uint32_t)q, plo, phi}, out[4];
        lco_philox4x32(ctr, c->key, out);
        for (int w = 0; w < 4 && 4 * q + w < nslots; ++w)
          c->unif[slot_off(layout, nh, 4 * q + w, s)] = (real)lco_u01(out[w]);
      }
    }
    c->pass_ctr += 1;
  }
  return 0;
}
#define UNI(c, layout, k, s) ((c)->unif[slot_off((layout), (c)->nh, (k), (s))])

/* sequential draws, for the initial-configuration routines */
static int draw_seq(lco_ctx *c, real *out, size_t n) {
  if (c->src == LCO_SRC_STREAM) {
    if (c->stream_pos + n > c->stream_n) return -1;
    for (size_t i = 0; i < n; ++i) out[i] = (real)c->stream[c->stream_pos + i];
    c->stream_pos += n;
    return 0;
  }
  if (c->src == LCO_SRC_RANLUX) {
    for (size_t i = 0; i < n; ++i) {
      float f;
      lco_ranlux(&f, 1);
      out[i] = (real)f;
    }
    return 0;
  }
  for (size_t i = 0; i < n; ++i) {
    uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), (uint32_t)c->pass_ctr,
                       (uint32_t)(c->pass_ctr >> 32) | 0x80000000u}, o[4];
    lco_philox4x32(ctr, c->key, o);
    out[i] = (real)lco_u01(o[0]);
  }
  c->pass_ctr += 1;
  return 0;
}

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
/* f/adresses.f:91-337, dimproc == 1 branches, converted to 0-based */
static void build_tables(lco_ctx *c) {
  const int hx = c->hx, nxy = c->nxy, nh = c->nh;
  const int L2 = c->L[1], L3 = c->L[2];
  int i0 = 0, i1 = 0;
  for (int z = 1; z <= c->L[2]; ++z)
    for (int y = 1; y <= c->L[1]; ++y)
      for (int x = 1; x <= c->L[0]; ++x) {
        int eo, i;
        if ((x + y + z) % 2 == 1) {
          eo = 0; i = ++i0;
        } else {
          eo = 1; i = ++i1;
        }
        int up1, dn1;
        int rowstart = ((i - 1) / hx) * hx;
        int xflag = (eo == 0) ? ((y + z) % 2 == 1) : ((y + z) % 2 == 0);
        if (xflag) {
          up1 = (i % hx) + 1 + rowstart;
          dn1 = i;
        } else {
          up1 = i;
          dn1 = ((i + hx - 2) % hx) + 1 + rowstart;
        }
        int pl = ((i - 1) / nxy) * nxy;
        int up2 = ((i - 1 + hx) % nxy) + 1 + pl;
        int dn2 = ((i - 1 + hx * (L2 - 1)) % nxy) + 1 + pl;
        int vl = ((i - 1) / nh) * nh;
        int up3 = ((i - 1 + nxy) % nh) + 1 + vl;
        int dn3 = ((i - 1 + nxy * (L3 - 1)) % nh) + 1 + vl;
        UP(c, eo, 0, i - 1) = up1 - 1; DN(c, eo, 0, i - 1) = dn1 - 1;
        UP(c, eo, 1, i - 1) = up2 - 1; DN(c, eo, 1, i - 1) = dn2 - 1;
        UP(c, eo, 2, i - 1) = up3 - 1; DN(c, eo, 2, i - 1) = dn3 - 1;
      }
}

lco_ctx *lco_create(int L1, int L2, int L3, double beta, double x, double y,
                    double lambda, double alpha, double limit_or, int imode) {
  if (L1 <= 0 || L2 <= 0 || L3 <= 0 || (L1 & 1) || (L2 & 1) || (L3 & 1)) return NULL;
  lco_ctx *c = (lco_ctx *)calloc(1, sizeof(lco_ctx));
  c->L[0] = L1; c->L[1] = L2; c->L[2] = L3;
  c->hx = L1 / 2; c->nxy = L1 * L2 / 2; c->vol = L1 * L2 * L3; c->nh = c->vol / 2;
  size_t nu = (size_t)3 * 2 * c->nh * 4, na = (size_t)2 * c->nh * 3;
  c->u = (real *)calloc(nu, sizeof(real));
  c->uf = (real *)calloc(nu, sizeof(real));
  c->v = (real *)calloc(nu, sizeof(real));
  c->a = (real *)calloc(na, sizeof(real));
  c->af = (real *)calloc(na, sizeof(real));
  c->force = (real *)calloc((size_t)c->nh * 3, sizeof(real));
  c->up = (int *)calloc((size_t)6 * c->nh, sizeof(int));
  c->dn = (int *)calloc((size_t)6 * c->nh, sizeof(int));
  build_tables(c);
  c->beta = (real)beta; c->x = (real)x; c->y = (real)y;
  c->lambda = (real)lambda; c->alpha = (real)alpha; c->limit_or = (real)limit_or;
  c->imode = imode;
  /* f/paraminit.f:44-47 constants and :150-153 couplings, in the build's precision */
  const real pi = (real)2.0 * (real)acos((real)0.0);
  const real sigma = (real)3.1759114;
  const real b = c->beta, xx = c->x, yy = c->y;
  c->beta_a = b;
  c->beta_2 = c->beta_a * ((real)3 + (real)8 * yy / (b * b) - sigma * ((real)4 + (real)5 * xx) / ((real)2 * pi * b) -
                           (((real)20 * xx - (real)10 * (xx * xx)) * ((real)log((real)1.5 * b) + (real)0.09) +
                            (real)8.7 + (real)11.6 * xx) / (((real)2 * (pi * pi)) * (b * b)));
  c->beta_4 = xx * b;
  c->src = LCO_SRC_PHILOX;
  c->key[0] = 12345u; c->key[1] = 0u;
  c->nthreads = 1;
  return c;
}

void lco_destroy(lco_ctx *c) {
  if (!c) return;
  free(c->u); free(c->uf); free(c->v); free(c->a); free(c->af);
  free(c->force); free(c->up); free(c->dn); free(c->unif);
  free(c);
}

int lco_nh(const lco_ctx *c) { return c->nh; }
void lco_set_threads(lco_ctx *c, int n) { c->nthreads = n > 0 ? n : 1; }
void lco_couplings(const lco_ctx *c, double out[3]) {
  out[0] = c->beta_a; out[1] = c->beta_2; out[2] = c->beta_4;
}

void lco_set_stream(lco_ctx *c, const double *u, size_t n) {
  c->src = LCO_SRC_STREAM; c->stream = u; c->stream_n = n; c->stream_pos = 0;
}
size_t lco_stream_pos(const lco_ctx *c) { return c->stream_pos; }
void lco_set_ranlux_source(lco_ctx *c) { c->src = LCO_SRC_RANLUX; }
void lco_set_philox(lco_ctx *c, uint64_t seed, uint64_t pass_ctr) {
  c->src = LCO_SRC_PHILOX;
  c->key[0] = (uint32_t)seed; c->key[1] = (uint32_t)(seed >> 32);
  c->pass_ctr = pass_ctr;
}
uint64_t lco_pass_ctr(const lco_ctx *c) { return c->pass_ctr; }
void lco_set_gf_angle(lco_ctx *c, int mode) { c->gf_angle = mode; }

void lco_set_fields(lco_ctx *c, int which, const lco_real *u, const lco_real *a) {
  size_t nu = (size_t)3 * 2 * c->nh * 4, na = (size_t)2 * c->nh * 3;
  if (u) memcpy(which ? c->uf : c->u, u, nu * sizeof(real));
  if (a) memcpy(which ? c->af : c->a, a, na * sizeof(real));
}
void lco_get_fields(const lco_ctx *c, int which, lco_real *u, lco_real *a) {
  size_t nu = (size_t)3 * 2 * c->nh * 4, na = (size_t)2 * c->nh * 3;
  if (u) memcpy(u, which ? c->uf : c->u, nu * sizeof(real));
  if (a) memcpy(a, which ? c->af : c->a, na * sizeof(real));
}
void lco_get_staple(const lco_ctx *c, lco_real *v) {
  memcpy(v, c->v, (size_t)3 * 2 * c->nh * 4 * sizeof(real));
}
void lco_get_force(const lco_ctx *c, lco_real *f) {
  memcpy(f, c->force, (size_t)c->nh * 3 * sizeof(real));
}
void lco_tables(const lco_ctx *c, int *siteup, int *sitedn) {
  memcpy(siteup, c->up, (size_t)6 * c->nh * sizeof(int));
  memcpy(sitedn, c->dn, (size_t)6 * c->nh * sizeof(int));
}

/* ------------------------------------------------------------------ */
/* configurations, f/confget.f                                          */
/* ------------------------------------------------------------------ */
/* unitconf f/confget.f:295-307 uses A = (0,0,1); a3 selects that or 0 */
void lco_unitconf(lco_ctx *c, double a3) {
  for (int mu = 0; mu < 3; ++mu)
    for (int eo = 0; eo < 2; ++eo)
      for (int s = 0; s < c->nh; ++s) {
        real *p = c->u + UIDX(c, mu, eo, s);
        p[0] = 1; p[1] = 0; p[2] = 0; p[3] = 0;
      }
  for (int eo = 0; eo < 2; ++eo)
    for (int s = 0; s < c->nh; ++s) {
      real *p = c->a + AIDX(c, eo, s);
      p[0] = 0; p[1] = 0; p[2] = (real)a3;
    }
}

/* randomconf f/confget.f:115-149, including its use of the stale s3 from the
 * link loop in a(2) (:147) */
int lco_randomconf(lco_ctx *c) {
  const real twopi = (real)2.0 * ((real)2.0 * (real)acos((real)0.0));
  real r[3], s3 = 0;
  for (int mu = 0; mu < 3; ++mu)
    for (int eo = 0; eo < 2; ++eo)
      for (int s = 0; s < c->nh; ++s) {
        if (draw_seq(c, r, 3)) return -1;
        real x1 = (real)2.0 * r[0] - (real)1.0;
        real s1 = (real)sqrt((real)1.0 - x1 * x1);
        real s2 = (real)2.0 * r[1] - (real)1.0;
        real x2 = s1 * s2;
        s3 = (real)sqrt((real)1.0 - s2 * s2);
        real s4 = s1 * s3;
        real s5 = twopi * r[2];
        real x4 = s4 * (real)cos(s5);
        real x3 = s4 * (real)sin(s5);
        real *p = c->u + UIDX(c, mu, eo, s);
        p[0] = x1; p[1] = x2; p[2] = x3; p[3] = x4;
      }
  for (int s = 0; s < c->nh; ++s)
    for (int eo = 0; eo < 2; ++eo) {
      if (draw_seq(c, r, 2)) return -1;
      real *p = c->a + AIDX(c, eo, s);
      p[2] = (real)2.0 * r[0] - (real)1.0;
      real s1 = (real)sqrt((real)1.0 - p[2] * p[2]);
      real s2 = twopi * r[1];
      p[0] = s1 * (real)cos(s2);
      p[1] = s1 * (real)sin(s3);
    }
  return 0;
}

/* testconf f/confget.f:528-575 (single rank: z-column rank 0).  The
 * reference's slice loop runs one slice past the end into the halo tail;
 * only the owned slices are stored here. */
void lco_testconf(lco_ctx *c) {
  for (int mu = 0; mu < 3; ++mu)
    for (int eo = 0; eo < 2; ++eo)
      for (int s = 0; s < c->nh; ++s) {
        int z = s / c->nxy;
        real *p = c->u + UIDX(c, mu, eo, s);
        p[0] = 0; p[1] = (real)(mu + 1) * (real)z;
        p[2] = 0; p[3] = (real)(mu + 1) * (real)z;
      }
  const real r3 = (real)1.0 / (real)sqrt((real)3.0);
  for (int eo = 0; eo < 2; ++eo)
    for (int s = 0; s < c->nh; ++s) {
      real *p = c->a + AIDX(c, eo, s);
      p[0] = r3; p[1] = r3; p[2] = r3;
    }
}

/* ------------------------------------------------------------------ */
/* staples  f/staples.f:65-221                                          */
/* ------------------------------------------------------------------ */
int lco_staples(lco_ctx *c, int eo, int mu) {
  const int oe = 1 - eo, nh = c->nh;
  int nus[2], k = 0;
  for (int n = 0; n < 3; ++n)
    if (n != mu) nus[k++] = n;
  su2 *bt1 = (su2 *)malloc(sizeof(su2) * nh);
  su2 *bt2 = (su2 *)malloc(sizeof(su2) * nh);
  su2 *up1 = (su2 *)malloc(sizeof(su2) * nh);
  su2 *up2 = (su2 *)malloc(sizeof(su2) * nh);
  real *V = c->v;
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
  for (int s = 0; s < nh; ++s) {
    real *p = V + UIDX(c, mu, eo, s);
    p[0] = p[1] = p[2] = p[3] = 0;
  }
  for (int in = 0; in < 2; ++in) {
    const int nu = nus[in];
    /* 1b) helpbt1 = U_mu(oe)^+ U_nu(oe)   (:293-295) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s)
      bt1[s] = mul_dn(ld_su2(c->u + UIDX(c, mu, oe, s)), ld_su2(c->u + UIDX(c, nu, oe, s)));
    /* 2b) helpup1 = U_mu(oe)(siteup(eo,nu))^+ U_nu(eo)^+   (:324-326) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s)
      up1[s] = mul_dd(ld_su2(c->u + UIDX(c, mu, oe, UP(c, eo, nu, s))), ld_su2(c->u + UIDX(c, nu, eo, s)));
    /* 3b) helpbt2 = U_nu(eo)(siteup(oe,mu))^+ helpbt1   (:356-358) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s)
      bt2[s] = mul_dn(ld_su2(c->u + UIDX(c, nu, eo, UP(c, oe, mu, s))), bt1[s]);
    /* 4b) helpup2 = U_nu(oe)(siteup(eo,mu)) helpup1   (:388-390) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s)
      up2[s] = mul_nn(ld_su2(c->u + UIDX(c, nu, oe, UP(c, eo, mu, s))), up1[s]);
    /* 5) v = v + helpup2 + helpbt2(sitedn(eo,nu))   (:404-410) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      real *p = V + UIDX(c, mu, eo, s);
      su2 b2 = bt2[DN(c, eo, nu, s)];
      p[0] = p[0] + up2[s].a.re + b2.a.re;
      p[1] = p[1] + up2[s].a.im + b2.a.im;
      p[2] = p[2] + up2[s].b.re + b2.b.re;
      p[3] = p[3] + up2[s].b.im + b2.b.im;
    }
  }
  free(bt1); free(bt2); free(up1); free(up2);
  return 0;
}

/* ------------------------------------------------------------------ */
/* link update  f/agauge.f:49-200 with f/heat_kpi.f:9-101; nhit = 3 is  */
/* f/agauge1.f:58-231 (staple once per pass, then three heatbath +      */
/* Metropolis hits, each drawing its own 7 uniforms per site)           */
/* ------------------------------------------------------------------ */
static int agauge_hits(lco_ctx *c, int measflag, int nhit, lco_real *accept_out) {
  const int nh = c->nh;
  const real tpi = (real)2.0 * (real)acos((real)-1.0);
  double kp_acc = 0, acc1 = 0, plaq = 0;
  c->plaq0 = 0;
  for (int eo = 0; eo < 2; ++eo) {
    const int oe = 1 - eo;
    for (int mu = 0; mu < 3; ++mu) {
      lco_staples(c, eo, mu);
      double pass_kp = 0, pass_acc = 0, pass_plaq = 0;
      for (int hit = 0; hit < nhit; ++hit) {
        if (draw_pass(c, 7, LAY_TRIPLE)) return -1;
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : pass_kp, pass_acc)
        for (int s = 0; s < nh; ++s) {
          /* 2) normalise the staple (f/agauge.f:71-84, f/agauge1.f:80-91) */
          const real *vp = c->v + UIDX(c, mu, eo, s);
          su2 vv = ld_su2(vp);
          real t1 = vv.a.re * vv.a.re + vv.a.im * vv.a.im + vv.b.re * vv.b.re + vv.b.im * vv.b.im;
          t1 = (real)1.0 / (real)sqrt(t1);
          su2 vh = {{t1 * vv.a.re, t1 * vv.a.im}, {t1 * vv.b.re, t1 * vv.b.im}};
          t1 = t1 / c->beta;
          /* the current link: updated by an earlier hit (f/agauge1.f:101-108) */
          su2 uo = ld_su2(c->u + UIDX(c, mu, eo, s));
          real t2 = csub(cmul(uo.a, vh.a), cmul(uo.b, cconj(vh.b))).re;
          /* 3) heat_kpi (f/heat_kpi.f:33-98) */
          real a1 = UNI(c, LAY_TRIPLE, 0, s), a2 = UNI(c, LAY_TRIPLE, 1, s), a3 = UNI(c, LAY_TRIPLE, 2, s);
          if (a1 == (real)0.0) a1 = (real)0.0000033;
          if (a2 == (real)0.0) a2 = (real)0.0000066;
          real cc = (real)cos(tpi * a3);
          real a0 = -((real)log(a1) + (real)log(a2) * (cc * cc)) * t1;
          real r4 = UNI(c, LAY_TRIPLE, 3, s);
          int lacc = (r4 * r4 <= ((real)1.0 - (real)0.5 * a0));
          if (lacc) a0 = (real)1.0 - a0;
          else a0 = t2;
          pass_kp += lacc;
          real b1 = (real)1.0 - a0 * a0;
          b1 = (b1 >= (real)0.0) ? (real)sqrt(b1) : (real)0.0;
          real b2 = (real)2.0 * (UNI(c, LAY_TRIPLE, 4, s) - (real)0.5);
          real b3 = b1 * b2;
          su2 X;
          X.a = cmk(a0, b3);
          real q0 = (real)1.0 - b2 * b2;
          q0 = (q0 >= (real)0.0) ? b1 * (real)sqrt(q0) : (real)0.0;
          real ph = tpi * UNI(c, LAY_TRIPLE, 5, s);
          real q1 = q0 * (real)cos(ph);
          real q2 = q0 * (real)sin(ph);
          X.b = cmk(q2, q1);
          /* 4) proposal h = X * Vhat^+ (f/agauge.f:98-104) */
          su2 hn = mul_nd(X, vh);
          /* hopping term, old and new (:126-159) */
          const real *ax = c->a + AIDX(c, eo, s);
          const real *axm = c->a + AIDX(c, oe, UP(c, eo, mu, s));
          su2 o1 = mul_an(ax, uo), n1 = mul_an(ax, hn);
          su2 o3 = mul_ad(axm, uo), n3 = mul_ad(axm, hn);
          real sa_old = c->beta_a * mul_nn(o1, o3).a.re;
          real sa_new = c->beta_a * mul_nn(n1, n3).a.re;
          /* accept (:167-174) */
          real rx = UNI(c, LAY_TRIPLE, 6, s);
          if ((real)exp(sa_old - sa_new) >= rx) {
            st_su2(c->u + UIDX(c, mu, eo, s), hn);
            pass_acc += 1.0;
          }
        }
      }
      /* plaquette against the staple, after the hits (f/agauge.f:179-185, f/agauge1.f:205-211) */
      if (measflag == 1) {
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : pass_plaq)
        for (int s = 0; s < nh; ++s)
          pass_plaq += mul_nn(ld_su2(c->u + UIDX(c, mu, eo, s)), ld_su2(c->v + UIDX(c, mu, eo, s))).a.re;
      }
      kp_acc += pass_kp;
      acc1 += pass_acc;
      plaq += pass_plaq;
    }
  }
  double accept = kp_acc;
  if (measflag == 1) {
    /* f/agauge.f:195-200; f/agauge1.f:227-232 divides acc1 by nhit too */
    c->plaq0 = plaq / (12.0 * c->vol);
    accept = accept / (3.0 * c->vol);
    acc1 = acc1 / (12.0 * c->vol) / nhit;
    accept = accept * acc1;
  }
  c->acc_gauge = accept;
  if (accept_out) *accept_out = (real)accept;
  return 0;
}

int lco_agauge(lco_ctx *c, int measflag, lco_real *accept_out) { return agauge_hits(c, measflag, 1, accept_out); }

int lco_agauge1(lco_ctx *c, int measflag, lco_real *accept_out) { return agauge_hits(c, measflag, 3, accept_out); }

/* Link overrelaxation (no reference counterpart; the reference has no link
 * OR).  Proposal U' = Vhat^+ U^+ Vhat^+ keeps Re Tr(U V) fixed; the hopping
 * term breaks that invariance so it is accepted with the agauge Metropolis
 * test (f/agauge.f:126-174).  One uniform per site (planar). */
int lco_link_or(lco_ctx *c, int measflag, lco_real *accept_out) {
  const int nh = c->nh;
  double acc = 0;
  for (int eo = 0; eo < 2; ++eo) {
    const int oe = 1 - eo;
    for (int mu = 0; mu < 3; ++mu) {
      lco_staples(c, eo, mu);
      if (draw_pass(c, 1, LAY_PLANAR)) return -1;
      double pass_acc = 0;
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : pass_acc)
      for (int s = 0; s < nh; ++s) {
        su2 vv = ld_su2(c->v + UIDX(c, mu, eo, s));
        real t1 = vv.a.re * vv.a.re + vv.a.im * vv.a.im + vv.b.re * vv.b.re + vv.b.im * vv.b.im;
        t1 = (real)1.0 / (real)sqrt(t1);
        su2 vh = {{t1 * vv.a.re, t1 * vv.a.im}, {t1 * vv.b.re, t1 * vv.b.im}};
        su2 uo = ld_su2(c->u + UIDX(c, mu, eo, s));
        /* W = Vhat^+ U^+ Vhat^+ = (Vhat U Vhat)^+ */
        su2 w = mul_nn(mul_nn(vh, uo), vh);
        su2 hn = {cconj(w.a), cneg(w.b)};
        const real *ax = c->a + AIDX(c, eo, s);
        const real *axm = c->a + AIDX(c, oe, UP(c, eo, mu, s));
        real sa_old = c->beta_a * mul_nn(mul_an(ax, uo), mul_ad(axm, uo)).a.re;
        real sa_new = c->beta_a * mul_nn(mul_an(ax, hn), mul_ad(axm, hn)).a.re;
        real rx = c->unif[s];
        if ((real)exp(sa_old - sa_new) >= rx) {
          st_su2(c->u + UIDX(c, mu, eo, s), hn);
          pass_acc += 1.0;
        }
      }
      acc += pass_acc;
    }
  }
  (void)measflag;
  c->acc_metro = acc / (3.0 * c->vol);
  if (accept_out) *accept_out = (real)(acc / (3.0 * c->vol));
  return 0;
}

/* ------------------------------------------------------------------ */
/* Higgs force  f/a_force.f:50-110                                      */
/* ------------------------------------------------------------------ */
int lco_a_force(lco_ctx *c, int eo) {
  const int oe = 1 - eo, nh = c->nh;
  su2 *t2 = (su2 *)malloc(sizeof(su2) * nh);
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
  for (int s = 0; s < nh * 3; ++s) c->force[s] = 0;
  for (int mu = 0; mu < 3; ++mu) {
    /* 2)+3) u_tmp2(y) = U(y)^+ (iA(y)) U(y) on oe sites (:64-68) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      su2 uy = ld_su2(c->u + UIDX(c, mu, oe, s));
      t2[s] = mul_dn(uy, mul_an(c->a + AIDX(c, oe, s), uy));
    }
    /* 6)+7)+9) (:85-108) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      su2 ux = ld_su2(c->u + UIDX(c, mu, eo, s));
      su2 t3 = mul_ad(c->a + AIDX(c, oe, UP(c, eo, mu, s)), ux);
      su2 t1 = mul_nn(ux, t3);
      su2 tb = t2[DN(c, eo, mu, s)];
      real *f = c->force + (size_t)s * 3;
      f[2] = f[2] + (t1.a.im + tb.a.im);
      f[1] = f[1] + (t1.b.re + tb.b.re);
      f[0] = f[0] + (t1.b.im + tb.b.im);
    }
  }
  free(t2);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Higgs updates                                                        */
/* ------------------------------------------------------------------ */
/* width/cxval/alph of f/ahiggs2.f:52-77 (identical in f/ahiggs3.f:61-87) */
static inline void hb_params(const lco_ctx *c, const real *f, real *alph, real *width, real *cxval) {
  if (c->imode == 1) {
    real conf2 = 0;
    for (int i = 0; i < 3; ++i) conf2 = conf2 + c->beta_a * (f[i] * f[i]);
    /* alph = beta_4*conf2 / (2*(beta_2+beta_4*conf2)**2) */
    real q = c->beta_2 + c->beta_4 * conf2;
    real al = (c->beta_4 * conf2) / ((real)2 * (q * q));
    *alph = al;
    *width = c->beta_2 + al;
    *cxval = (real)1 / (real)2.0 / *width;
  } else {
    *alph = 0;
    *width = c->beta_2;
    *cxval = (real)1 / c->beta_2 / (real)2;
  }
}

/* common accept + measurement tail, f/ahiggs2.f:105-147 */
static void higgs_finish(lco_ctx *c, int eo, real *an_all, int acc_slot, int layout,
                         const real *alph_all, double *acc, double *s2, double *s4, double *skin, int measflag) {
  const int nh = c->nh;
  double lacc = 0, l2 = 0, l4 = 0, lk = 0;
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : lacc, l2, l4, lk)
  for (int s = 0; s < nh; ++s) {
    real *ao = c->a + AIDX(c, eo, s);
    real *an = an_all + (size_t)s * 3;
    real rho_o = 0, rho_n = 0;
    for (int i = 0; i < 3; ++i) {
      rho_o = rho_o + ao[i] * ao[i];
      rho_n = rho_n + an[i] * an[i];
    }
    real boltz = (real)exp(-alph_all[s] * (rho_o - rho_n) + c->beta_4 * (rho_o * rho_o - rho_n * rho_n));
    real rx = UNI(c, layout, acc_slot, s);
    if (boltz >= rx) {
      ao[0] = an[0]; ao[1] = an[1]; ao[2] = an[2];
      rho_o = rho_n;
      lacc += 1;
    }
    if (measflag == 1) {
      l2 += rho_o;
      l4 += (double)rho_o * rho_o;
      const real *f = c->force + (size_t)s * 3;
      lk += (double)ao[0] * f[0] + (double)ao[1] * f[1] + (double)ao[2] * f[2];
    }
  }
  *acc += lacc; *s2 += l2; *s4 += l4; *skin += lk;
}

/* f/ahiggs2.f:7-152 heatbath; gauss per f/gauss.f:10-31 */
int lco_ahiggs2(lco_ctx *c, int measflag, lco_real *accept) {
  const int nh = c->nh;
  const real tpi = (real)2.0 * (real)acos((real)-1.);
  double acc = 0, s2 = 0, s4 = 0, sk = 0;
  real *an = (real *)malloc(sizeof(real) * 3 * nh);
  real *alph = (real *)malloc(sizeof(real) * nh);
  for (int eo = 0; eo < 2; ++eo) {
    lco_a_force(c, eo);
    if (draw_pass(c, 7, LAY_PLANAR)) { free(an); free(alph); return -1; }
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      const real *f = c->force + (size_t)s * 3;
      real al, width, cxval;
      hb_params(c, f, &al, &width, &cxval);
      alph[s] = al;
      real rr = (real)1.0 / width;
      for (int i = 0; i < 3; ++i) {
        real w1 = -(real)1.0 * rr * (real)log(UNI(c, LAY_PLANAR, 2 * i, s));
        real g = (real)sqrt(w1) * (real)cos(tpi * UNI(c, LAY_PLANAR, 2 * i + 1, s));
        an[(size_t)s * 3 + i] = g + c->beta_a * f[i] * cxval;
      }
    }
    higgs_finish(c, eo, an, 6, LAY_PLANAR, alph, &acc, &s2, &s4, &sk, measflag);
  }
  free(an); free(alph);
  double a = acc;
  if (measflag == 1) {
    c->a02 = s2 / c->vol; c->a04 = s4 / c->vol; c->a0kin = sk / (6.0 * c->vol);
    a = acc / c->vol;
  }
  c->acc_hb = a;
  if (accept) *accept = (real)a;
  return 0;
}

/* f/ahiggs3.f:7-148 overrelaxation */
int lco_ahiggs3(lco_ctx *c, int measflag, lco_real *accept) {
  const int nh = c->nh;
  double acc = 0, s2 = 0, s4 = 0, sk = 0;
  real *an = (real *)malloc(sizeof(real) * 3 * nh);
  real *alph = (real *)malloc(sizeof(real) * nh);
  for (int eo = 0; eo < 2; ++eo) {
    lco_a_force(c, eo);
    if (draw_pass(c, 1, LAY_PLANAR)) { free(an); free(alph); return -1; }
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      const real *f = c->force + (size_t)s * 3;
      const real *ao = c->a + AIDX(c, eo, s);
      real al, width, cxval;
      hb_params(c, f, &al, &width, &cxval);
      alph[s] = al;
      for (int i = 0; i < 3; ++i)
        an[(size_t)s * 3 + i] = -ao[i] + (real)2.0 * c->beta_a * f[i] * cxval;
    }
    higgs_finish(c, eo, an, 0, LAY_PLANAR, alph, &acc, &s2, &s4, &sk, measflag);
  }
  free(an); free(alph);
  double a = acc;
  if (measflag == 1) {
    c->a02 = s2 / c->vol; c->a04 = s4 / c->vol; c->a0kin = sk / (6.0 * c->vol);
    a = acc / c->vol;
  }
  c->acc_or = a;
  if (accept) *accept = (real)a;
  return 0;
}

/* f/ahiggs1.f:7-127 Metropolis with adaptive step */
int lco_ahiggs1(lco_ctx *c, lco_real *delta, int measflag, lco_real *accept) {
  const int nh = c->nh;
  double acc = 0, s2 = 0, s4 = 0, sk = 0;
  const real d = *delta;
  for (int eo = 0; eo < 2; ++eo) {
    lco_a_force(c, eo);
    if (draw_pass(c, 4, LAY_TRIPLE)) return -1;
    double lacc = 0, l2 = 0, l4 = 0, lk = 0;
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : lacc, l2, l4, lk)
    for (int s = 0; s < nh; ++s) {
      real *ao = c->a + AIDX(c, eo, s);
      const real *f = c->force + (size_t)s * 3;
      real an[3];
      for (int i = 0; i < 3; ++i) an[i] = ao[i] + (UNI(c, LAY_TRIPLE, i, s) - (real)0.5) * d;
      real sf_o = 0, sf_n = 0, rho_o = 0, rho_n = 0;
      for (int i = 0; i < 3; ++i) {
        sf_o = sf_o + ao[i] * f[i];
        sf_n = sf_n + an[i] * f[i];
        rho_o = rho_o + ao[i] * ao[i];
        rho_n = rho_n + an[i] * an[i];
      }
      real boltz = (real)exp(-c->beta_a * (sf_o - sf_n) + c->beta_2 * (rho_o - rho_n) +
                             c->beta_4 * (rho_o * rho_o - rho_n * rho_n));
      if (boltz >= UNI(c, LAY_TRIPLE, 3, s)) {
        ao[0] = an[0]; ao[1] = an[1]; ao[2] = an[2];
        rho_o = rho_n; sf_o = sf_n;
        lacc += 1;
      }
      if (measflag == 1) {
        l2 += rho_o; l4 += (double)rho_o * rho_o; lk += sf_o;
      }
    }
    acc += lacc; s2 += l2; s4 += l4; sk += lk;
  }
  if (measflag == 1) {
    c->a02 = s2 / c->vol; c->a04 = s4 / c->vol; c->a0kin = sk / (6.0 * c->vol);
  }
  real a = (real)(acc / c->vol);
  c->acc_metro = a;
  if (accept) *accept = a;
  /* f/ahiggs1.f:117-123 */
  if ((real)fabs(a - (real)0.5) > (real)0.1) {
    if (a > (real)0.5) *delta = (real)1.1131241 * *delta;
    else *delta = (real)0.8989669 * *delta;
  }
  return 0;
}

/* f/renorm.f:24-34 */
void lco_renorm(lco_ctx *c) {
  const size_t n = (size_t)3 * 2 * c->nh;
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
  for (size_t i = 0; i < n; ++i) {
    real *p = c->u + i * 4;
    real t = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
    t = (real)1.0 / (real)sqrt(t);
    p[0] = t * p[0]; p[1] = t * p[1]; p[2] = t * p[2]; p[3] = t * p[3];
  }
}

/* one sweep in the order of f/main.f:38-41 */
int lco_sweep(lco_ctx *c, int measflag, lco_meas *m) {
  real a2, a3, a1;
  if (lco_ahiggs2(c, measflag, &a2)) return -1;
  if (lco_ahiggs3(c, measflag, &a3)) return -1;
  if (lco_agauge(c, measflag, &a1)) return -1;
  lco_renorm(c);
  if (m) lco_get_meas(c, m);
  return 0;
}

/* ------------------------------------------------------------------ */
/* gauge fixing  f/landau_gauge.f, f/or_gauge_fixing1.f, u_f_renorm   */
/* ------------------------------------------------------------------ */
void lco_landau_copy(lco_ctx *c) {
  memcpy(c->uf, c->u, (size_t)3 * 2 * c->nh * 4 * sizeof(real));
  memcpy(c->af, c->a, (size_t)2 * c->nh * 3 * sizeof(real));
}

/* f/u_f_renorm.f:24-34 */
void lco_u_f_renorm(lco_ctx *c) {
  const size_t n = (size_t)3 * 2 * c->nh;
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
  for (size_t i = 0; i < n; ++i) {
    real *p = c->uf + i * 4;
    real t = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
    t = (real)1.0 / (real)sqrt(t);
    p[0] = t * p[0]; p[1] = t * p[1]; p[2] = t * p[2]; p[3] = t * p[3];
  }
}

/* f/or_gauge_fixing1.f:52-337 for one iteration (both parities).  The
 * reference accumulates da1 in single precision; here the per-site terms
 * are in the build's precision and the sum in double. */
double lco_or_gauge_fixing(lco_ctx *c) {
  const int nh = c->nh;
  double da1 = 0;
  su2 *om = (su2 *)malloc(sizeof(su2) * nh);
  for (int eo = 0; eo < 2; ++eo) {
    const int oe = 1 - eo;
    double dsum = 0;
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : dsum)
    for (int s = 0; s < nh; ++s) {
      /* 2) sum_mu c_mu U_mu(x)  (:97-107) */
      cplx t1a = cmk(0, 0), t1b = cmk(0, 0), t2a = cmk(0, 0), t2b = cmk(0, 0);
      for (int mu = 0; mu < 2; ++mu) {
        su2 u = ld_su2(c->uf + UIDX(c, mu, eo, s));
        t1a = cadd(t1a, u.a); t1b = cadd(t1b, u.b);
      }
      {
        su2 u = ld_su2(c->uf + UIDX(c, 2, eo, s));
        t1a = cadd(t1a, cmk(c->alpha * u.a.re, c->alpha * u.a.im));
        t1b = cadd(t1b, cmk(c->alpha * u.b.re, c->alpha * u.b.im));
      }
      /* 4)-6) sum_mu c_mu U_mu(x-mu)  (:116-142) */
      for (int mu = 0; mu < 2; ++mu) {
        su2 u = ld_su2(c->uf + UIDX(c, mu, oe, DN(c, eo, mu, s)));
        t2a = cadd(t2a, u.a); t2b = cadd(t2b, u.b);
      }
      {
        su2 u = ld_su2(c->uf + UIDX(c, 2, oe, DN(c, eo, 2, s)));
        t2a = cadd(t2a, cmk(c->alpha * u.a.re, c->alpha * u.a.im));
        t2b = cadd(t2b, cmk(c->alpha * u.b.re, c->alpha * u.b.im));
      }
      /* 7) (:145-146) */
      cplx w1 = cadd(t1a, cconj(t2a));
      cplx w2 = csub(t1b, t2b);
      /* theta (:153-158) */
      if (eo == 1) {
        real d = (t1a.im - t2a.im);
        dsum += (double)(d * d + (w2.re * w2.re + w2.im * w2.im));
      }
      /* k, Omega, OR (:162-184) */
      real k = w1.re * w1.re + w1.im * w1.im + w2.re * w2.re + w2.im * w2.im;
      real sk = (real)sqrt(k);
      su2 o = {{w1.re / sk, w1.im / sk}, {w2.re / sk, w2.im / sk}};
      if (c->gf_angle == 0) {
        /* Re Omega can round to just above 1 near convergence, where the
         * reference's acos would return NaN; clamp to the domain. */
        real ca = o.a.re > (real)1 ? (real)1 : (o.a.re < (real)-1 ? (real)-1 : o.a.re);
        real th = (real)acos(ca);
        if (th != (real)0) {
          real tho = c->lambda * th;
          real q1 = (real)cos(tho);
          real q2 = (real)sin(tho) / (real)sin(th) * o.a.im;
          real f = -(real)sin(tho) / (real)sin(th);
          o.a = cmk(q1, -q2);
          o.b = cmk(f * o.b.re, f * o.b.im);
        }
      } else {
        /* Same rotation with the angle from atan2(|vector part|, scalar part),
         * accurate for small angles where acos(Re Omega) loses all digits
         * (the acos form cannot resolve angles below ~sqrt(eps)). */
        real sv = (real)sqrt(w1.im * w1.im + w2.re * w2.re + w2.im * w2.im);
        if (sv != (real)0) {
          real th = (real)atan2(sv, w1.re);
          real tho = c->lambda * th;
          real f = (real)sin(tho) / sv;
          o.a = cmk((real)cos(tho), -f * w1.im);
          o.b = cmk(-f * w2.re, -f * w2.im);
        }
      }
      om[s] = o;
    }
    if (eo == 1) da1 = dsum / nh;
    /* 2) A_f -> Omega (iA) Omega^+ on eo sites (:243-252) */
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      real *af = c->af + AIDX(c, eo, s);
      su2 t1 = mul_ad(af, om[s]);
      su2 t2 = mul_nn(om[s], t1);
      af[0] = t2.b.im;
      af[1] = t2.b.re;
      af[2] = t2.a.im;
    }
    /* 3)-5) U_mu(x) -> Omega(x) U_mu(x) on eo, U_mu(y) -> U_mu(y) Omega(y+mu)^+ on oe */
    for (int mu = 0; mu < 3; ++mu) {
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
      for (int s = 0; s < nh; ++s) {
        real *p = c->uf + UIDX(c, mu, eo, s);
        st_su2(p, mul_nn(om[s], ld_su2(p)));
      }
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
      for (int s = 0; s < nh; ++s) {
        real *p = c->uf + UIDX(c, mu, oe, s);
        st_su2(p, mul_nd(ld_su2(p), om[UP(c, oe, mu, s)]));
      }
    }
  }
  free(om);
  return da1;
}

/* f/it_gauge_fixing.f:5-206, one iteration of the reference's iterative
 * (steepest-descent) gauge fixing, parity by parity (the transform of a
 * parity is applied before the next parity's g is formed, :94-99):
 *   g1 = sum_mu (i Im a, b) of U_f(x,mu), g2 the same of U_f(x-mu,mu)
 *   (:62-84: the antihermitian part in first-row form);
 *   g(1) = g1(1) - g2(1); g(2) = g1(1) - g2(2) as written at :110
 *   (flag 1: g1(2) - g2(2), the antihermitian part of sum [U - U(x-mu)]);
 *   on the second parity da1 = mean |g|^2 (:116-120), before the step;
 *   Omega = cos|h| + h sin|h|/|h|, h = step g (:122-141; flag 2: h = -step g,
 *   the direction that raises the Landau functional; as written the step
 *   lowers it);
 *   U_mu(x) -> Omega(x) U_mu(x), U_mu(y) -> U_mu(y) Omega(y+mu)^+ and
 *   A_f -> Omega (iA_f) Omega^+ (:143-210).
 * g, |g|^2 and Omega are formed in double in both builds (the device does
 * the same); the transform is applied in the build's precision.  Where
 * |h| = 0 the reference divides 0 by 0; the limit sin(t)/t = 1 is used. */
double lco_it_gauge_fixing(lco_ctx *c, double step, int flags) {
  const int nh = c->nh;
  double da1 = 0;
  su2 *om = (su2 *)malloc(sizeof(su2) * nh);
  const double st = (flags & 2) ? -step : step;
  for (int eo = 0; eo < 2; ++eo) {
    const int oe = 1 - eo;
    double dsum = 0;
#pragma omp parallel for num_threads(c->nthreads) schedule(static) reduction(+ : dsum)
    for (int s = 0; s < nh; ++s) {
      double g1a = 0, g1br = 0, g1bi = 0, g2a = 0, g2br = 0, g2bi = 0;
      for (int mu = 0; mu < 3; ++mu) {
        su2 u = ld_su2(c->uf + UIDX(c, mu, eo, s));
        g1a += u.a.im; g1br += u.b.re; g1bi += u.b.im;
      }
      for (int mu = 0; mu < 3; ++mu) {
        su2 u = ld_su2(c->uf + UIDX(c, mu, oe, DN(c, eo, mu, s)));
        g2a += u.a.im; g2br += u.b.re; g2bi += u.b.im;
      }
      const double ga = g1a - g2a;
      const double gbr = (flags & 1) ? g1br - g2br : -g2br;
      const double gbi = (flags & 1) ? g1bi - g2bi : g1a - g2bi;
      if (eo == 1) dsum += ga * ga + (gbr * gbr + gbi * gbi);
      const double ha = st * ga, hbr = st * gbr, hbi = st * gbi;
      const double t1 = sqrt(ha * ha + hbr * hbr + hbi * hbi);
      const double t2 = t1 > 0 ? sin(t1) / t1 : 1.0;
      su2 o = {{(real)cos(t1), (real)(ha * t2)}, {(real)(hbr * t2), (real)(hbi * t2)}};
      om[s] = o;
    }
    if (eo == 1) da1 = dsum / nh;
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int s = 0; s < nh; ++s) {
      real *af = c->af + AIDX(c, eo, s);
      su2 t2 = mul_nn(om[s], mul_ad(af, om[s]));
      af[0] = t2.b.im;
      af[1] = t2.b.re;
      af[2] = t2.a.im;
    }
    for (int mu = 0; mu < 3; ++mu) {
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
      for (int s = 0; s < nh; ++s) {
        real *p = c->uf + UIDX(c, mu, eo, s);
        st_su2(p, mul_nn(om[s], ld_su2(p)));
      }
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
      for (int s = 0; s < nh; ++s) {
        real *p = c->uf + UIDX(c, mu, oe, s);
        st_su2(p, mul_nd(ld_su2(p), om[UP(c, oe, mu, s)]));
      }
    }
  }
  free(om);
  return da1;
}

/* f/landau_gauge.f:28-59 with it_gauge_fixing in place of
 * or_gauge_fixing: copy, then iterate + u_f_renorm while da1 > limit_or */
int lco_it_landau_gauge(lco_ctx *c, double step, int flags, int max_iters, double *da1_out) {
  double da1 = 10000.0;
  int it = 0;
  lco_landau_copy(c);
  while (da1 > (double)c->limit_or) {
    if (max_iters > 0 && it >= max_iters) break;
    it++;
    da1 = lco_it_gauge_fixing(c, step, flags);
    lco_u_f_renorm(c);
  }
  if (da1_out) *da1_out = da1;
  return it;
}

/* f/landau_gauge.f:28-59; max_iters <= 0 means no cap (as the reference) */
int lco_landau_gauge(lco_ctx *c, int max_iters, double *da1_out) {
  double da1 = 10000.0;
  int it = 0;
  lco_landau_copy(c);
  while (da1 > (double)c->limit_or) {
    if (max_iters > 0 && it >= max_iters) break;
    it++;
    da1 = lco_or_gauge_fixing(c);
    lco_u_f_renorm(c);
  }
  if (da1_out) *da1_out = da1;
  return it;
}

/* Landau functional F = (1/3V) sum_{x,mu} c_mu Re a_mu(x), with the
 * alpha weight on mu = 3 (f/or_gauge_fixing1.f:104-107) normalised by
 * (2 + alpha). */
double lco_gauge_functional(const lco_ctx *c) {
  double s = 0;
  for (int mu = 0; mu < 3; ++mu) {
    double w = (mu == 2) ? (double)c->alpha : 1.0, t = 0;
    for (int eo = 0; eo < 2; ++eo)
      for (int i = 0; i < c->nh; ++i) t += c->uf[UIDX(c, mu, eo, i)];
    s += w * t;
  }
  return s / ((2.0 + (double)c->alpha) * c->vol);
}

/* theta evaluated on the current U_f without updating (the testmax-style
 * independent check, f/testmax.f:45-97): mean over odd sites */
double lco_theta_direct(const lco_ctx *c) {
  double dsum = 0;
  const int eo = 1, oe = 0;
  for (int s = 0; s < c->nh; ++s) {
    cplx t1a = cmk(0, 0), t1b = cmk(0, 0), t2a = cmk(0, 0), t2b = cmk(0, 0);
    for (int mu = 0; mu < 3; ++mu) {
      real w = (mu == 2) ? c->alpha : (real)1;
      su2 u = ld_su2(c->uf + UIDX(c, mu, eo, s));
      su2 d = ld_su2(c->uf + UIDX(c, mu, oe, DN(c, eo, mu, s)));
      t1a = cadd(t1a, cmk(w * u.a.re, w * u.a.im)); t1b = cadd(t1b, cmk(w * u.b.re, w * u.b.im));
      t2a = cadd(t2a, cmk(w * d.a.re, w * d.a.im)); t2b = cadd(t2b, cmk(w * d.b.re, w * d.b.im));
    }
    cplx w2 = csub(t1b, t2b);
    double d = (double)t1a.im - (double)t2a.im;
    dsum += d * d + (double)w2.re * w2.re + (double)w2.im * w2.im;
  }
  return dsum / c->nh;
}

/* f/correlator.f:45-164 (single rank); sums in double */
void lco_correlator(const lco_ctx *c, double *corr_a, double *corr_u, double *corr_3) {
  const int L3 = c->L[2], nxy = c->nxy;
  double *as = (double *)calloc((size_t)3 * L3, sizeof(double));
  double *us = (double *)calloc((size_t)3 * 3 * L3, sizeof(double)); /* [mu][z][s1, s2re, s2im] */
  for (int eo = 0; eo < 2; ++eo)
    for (int z = 0; z < L3; ++z)
      for (int i = 0; i < nxy; ++i) {
        int s = z * nxy + i;
        const real *af = c->af + AIDX(c, eo, s);
        for (int k = 0; k < 3; ++k) as[z * 3 + k] += af[k];
        for (int mu = 0; mu < 3; ++mu) {
          const real *u = c->uf + UIDX(c, mu, eo, s);
          double *q = us + ((size_t)mu * L3 + z) * 3;
          q[0] += u[1];          /* aimag(a) */
          q[1] += u[3];          /* -i*b: re = im b */
          q[2] += -u[2];         /*       im = -re b */
        }
      }
  const double norm = (double)c->L[0] * c->L[1];
  for (int i = 0; i < 3 * L3; ++i) as[i] /= norm;
  for (int i = 0; i < 9 * L3; ++i) us[i] /= norm;
  for (int z = 0; z < L3; ++z) {
    double ca = 0, cu = 0, c3 = 0;
    for (int x0 = 0; x0 < L3; ++x0) {
      int x1 = (x0 + z) % L3;
      ca += as[x0 * 3] * as[x1 * 3] + as[x0 * 3 + 1] * as[x1 * 3 + 1] + as[x0 * 3 + 2] * as[x1 * 3 + 2];
      for (int mu = 0; mu < 3; ++mu) {
        const double *p = us + ((size_t)mu * L3 + x0) * 3, *q = us + ((size_t)mu * L3 + x1) * 3;
        /* Re[s1 s1' + s2 conj(s2')] */
        double t = p[0] * q[0] + (p[1] * q[1] + p[2] * q[2]);
        if (mu < 2) cu += t; else c3 += t;
      }
    }
    corr_a[z] = ca / L3;
    corr_u[z] = cu / (L3 * 2.0);
    corr_3[z] = c3 / L3;
  }
  free(as); free(us);
}

/* f/polyakov.f:47-108 on the un-fixed A */
void lco_polyakov(const lco_ctx *c, double *slice, double *corr, double *mean2) {
  const int L3 = c->L[2], nxy = c->nxy;
  for (int z = 0; z < L3; ++z) slice[z] = 0;
  for (int eo = 0; eo < 2; ++eo)
    for (int z = 0; z < L3; ++z)
      for (int i = 0; i < nxy; ++i) {
        const real *a = c->a + AIDX(c, eo, z * nxy + i);
        slice[z] += (double)(real)cos((real)4 * (real)sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
      }
  double tot = 0;
  for (int z = 0; z < L3; ++z) { slice[z] /= (double)c->L[0] * c->L[1]; tot += slice[z]; }
  for (int z = 0; z < L3; ++z) {
    double s = 0;
    for (int x0 = 0; x0 < L3; ++x0) s += slice[x0] * slice[(x0 + z) % L3];
    corr[z] = s / L3;
  }
  *mean2 = (tot / L3) * (tot / L3);
}

/* f/scalarcorr.f:43-104 */
void lco_scalarcorr(const lco_ctx *c, double *slice, double *corr, double *mean) {
  const int L3 = c->L[2], nxy = c->nxy;
  for (int z = 0; z < L3; ++z) slice[z] = 0;
  for (int eo = 0; eo < 2; ++eo)
    for (int z = 0; z < L3; ++z)
      for (int i = 0; i < nxy; ++i) {
        const real *a = c->a + AIDX(c, eo, z * nxy + i);
        slice[z] += (double)a[0] * a[0] + (double)a[1] * a[1] + (double)a[2] * a[2];
      }
  double tot = 0;
  for (int z = 0; z < L3; ++z) { slice[z] /= (double)c->L[0] * c->L[1]; tot += slice[z]; }
  for (int z = 0; z < L3; ++z) {
    double s = 0;
    for (int x0 = 0; x0 < L3; ++x0) s += slice[x0] * slice[(x0 + z) % L3];
    corr[z] = s / L3;
  }
  *mean = tot / L3;
}

/* f/meas2a.f:39-49 */
void lco_meas2(const lco_ctx *c, double af[3]) {
  af[0] = af[1] = af[2] = 0;
  for (int eo = 0; eo < 2; ++eo)
    for (int s = 0; s < c->nh; ++s)
      for (int k = 0; k < 3; ++k) af[k] += c->af[AIDX(c, eo, s) + k];
  for (int k = 0; k < 3; ++k) af[k] /= c->vol;
}

/* average plaquette of the current U, 1/2 Re Tr, over all 3V plaquettes */
double lco_plaquette(const lco_ctx *c) {
  double s = 0;
  for (int eo = 0; eo < 2; ++eo) {
    const int oe = 1 - eo;
    for (int mu = 0; mu < 3; ++mu)
      for (int nu = mu + 1; nu < 3; ++nu)
        for (int i = 0; i < c->nh; ++i) {
          /* U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ */
          su2 a = ld_su2(c->u + UIDX(c, mu, eo, i));
          su2 b = ld_su2(c->u + UIDX(c, nu, oe, UP(c, eo, mu, i)));
          su2 d = ld_su2(c->u + UIDX(c, mu, oe, UP(c, eo, nu, i)));
          su2 e = ld_su2(c->u + UIDX(c, nu, eo, i));
          su2 p = mul_nn(mul_nn(a, b), mul_dd(d, e));
          s += p.a.re;
        }
  }
  return s / (3.0 * c->vol);
}

void lco_get_meas(const lco_ctx *c, lco_meas *m) {
  m->plaq = c->plaq0; m->akin = c->a0kin; m->a2 = c->a02; m->a4 = c->a04;
  m->acc_gauge = c->acc_gauge; m->acc_hb = c->acc_hb; m->acc_or = c->acc_or;
  m->acc_metro = c->acc_metro;
  m->af[0] = c->a0f[0]; m->af[1] = c->a0f[1]; m->af[2] = c->a0f[2];
}
