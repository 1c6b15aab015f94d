// lce_gaugefix.cu -- overrelaxed Landau gauge fixing on the device, and the
// reference's iterative (steepest-descent) form, f/it_gauge_fixing.f.
//
// One iteration of f/or_gauge_fixing1.f:52-337 is two half-steps (eo = 0, 1).
// A half-step kernel gives one thread per site x of parity eo; the thread
//   * gathers w(x) = sum_mu c_mu [U_mu(x) + U_mu(x-mu)^+] (c_3 = alpha),
//   * on eo = 1 adds theta(x) = (Im w_a)^2 + |w_b|^2 to an FP64 partial sum,
//   * builds Omega = w/|w|, overrelaxes its angle by lambda,
//   * writes A_f(x) -> Omega A_f Omega^+, U_mu(x) -> Omega U_mu(x) and
//     U_mu(x-mu) -> U_mu(x-mu) Omega^+.
// Every link touched in a half-step belongs to exactly one thread, so the
// update is race free.  All links are rewritten in the eo = 1 half-step, so
// reunitarising there is exactly f/u_f_renorm.f after the iteration
// (f/landau_gauge.f:54-59).  A one-block check kernel sums the partials in a
// fixed order, counts the iteration and raises a device flag when theta <=
// limit_or (or the cap is reached); later kernels of a captured batch of
// iterations see the flag and return at once, so the host reads the state
// only once per batch.
#include <algorithm>

#include "lce_internal.hpp"

namespace lce {

template <typename R>
__device__ __forceinline__ su2<R> ldUf(const ChainDev& ch, int mu, int p, int s) {
  return LinkIO<R>::ld_cg(ch.uf, ((size_t)(mu * 2 + p)) * ch.nh + s);
}

template <int MU>
__device__ __forceinline__ int nbr_dn(const ChainDev& ch, Coord X) {
  int x = X.x, y = X.y, z = X.z;
  if (MU == 0) x = wrap(x - 1, ch.L1);
  if (MU == 1) y = wrap(y - 1, ch.L2);
  if (MU == 2) z = wrap(z - 1, ch.L3);
  return site_index(x, y, z, ch.hx, ch.nxy);
}

// w sums in FP64: t1 = sum_mu c_mu U_mu(x), t2 = sum_mu c_mu U_mu(x-mu)
// (f/or_gauge_fixing1.f:97-142)
template <typename R>
__device__ __forceinline__ void gf_sums(const ChainDev& ch, const su2<R> (&um)[3], const su2<R> (&ud)[3],
                                        su2<double>& t1, su2<double>& t2) {
  const double al = ch.alpha;
  t1 = su2<double>{{0, 0}, {0, 0}};
  t2 = t1;
#pragma unroll
  for (int mu = 0; mu < 2; ++mu) {
    t1.a = t1.a + mk<double>(um[mu].a.re, um[mu].a.im);
    t1.b = t1.b + mk<double>(um[mu].b.re, um[mu].b.im);
  }
  t1.a = t1.a + mk<double>(al * um[2].a.re, al * um[2].a.im);
  t1.b = t1.b + mk<double>(al * um[2].b.re, al * um[2].b.im);
#pragma unroll
  for (int mu = 0; mu < 2; ++mu) {
    t2.a = t2.a + mk<double>(ud[mu].a.re, ud[mu].a.im);
    t2.b = t2.b + mk<double>(ud[mu].b.re, ud[mu].b.im);
  }
  t2.a = t2.a + mk<double>(al * ud[2].a.re, al * ud[2].a.im);
  t2.b = t2.b + mk<double>(al * ud[2].b.re, al * ud[2].b.im);
}

// track != 0: also accumulate the gauge transform, G(x) -> Omega(x) G(x), so
// that U_f(x,mu) = G(x) U(x,mu) G(x+mu)^+ holds throughout.  FP32 is held to
// 64 registers (4 blocks per SM; 68 allowed 3): 8.5% less time per
// iteration at 128^3, the kernel being latency-bound.  s_lo: a z-slab's
// first visited site (its first and last planes are halos; sites
// [s_lo, nh - s_lo) are visited), 0 for a whole lattice.  last: the
// iteration's second half-step (the whole lattice's odd sites; a slab's
// local parity eo may be flipped), which sums theta and reunitarises.
template <typename R>
__global__ void __launch_bounds__(kBlock, sizeof(R) == 4 ? 4 : 1)
    gf_half_kernel(const ChainDev* chp, const ChainState* cst, int eo, double* part, int track, int s_lo, int last) {
  pdl_trigger();
  const ChainDev& ch = *chp;
  const int s = s_lo + blockIdx.x * kBlock + threadIdx.x;
  const int oe = 1 - eo, nh = ch.nh, s_hi = nh - s_lo;
  const Coord X = site_coord(eo, s < s_hi ? s : s_lo, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  const int xm[3] = {nbr_dn<0>(ch, X), nbr_dn<1>(ch, X), nbr_dn<2>(ch, X)};
  pdl_wait();
  if (cst->gf_done) return;
  double th[1] = {0.0};
  if (s < s_hi) {
    su2<R> um[3], ud[3];
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      um[mu] = ldUf<R>(ch, mu, eo, s);
      ud[mu] = ldUf<R>(ch, mu, oe, xm[mu]);
    }
    su2<double> t1, t2;
    gf_sums<R>(ch, um, ud, t1, t2);
    // (:145-146) w = first row of sum [U + U^+(x-mu)]
    const cpx<double> w1 = t1.a + cj(t2.a), w2 = t1.b - t2.b;
    if (last) {
      // (:153-158)
      const double d = t1.a.im - t2.a.im;
      th[0] = d * d + (w2.re * w2.re + w2.im * w2.im);
    }
    // (:162-184) Omega = w/|w| with its angle overrelaxed by lambda
    su2<R> o{{(R)w1.re, (R)w1.im}, {(R)w2.re, (R)w2.im}};
    const R sk = M<R>::sqrt(norm2(o));
    o = su2<R>{{M<R>::div(o.a.re, sk), M<R>::div(o.a.im, sk)}, {M<R>::div(o.b.re, sk), M<R>::div(o.b.im, sk)}};
    const R lam = (R)ch.lambda;
    if (ch.gf_angle == LCE_GF_ACOS) {
      // the reference's angle acos(Re Omega), clamped to the domain
      const R ca = o.a.re > (R)1 ? (R)1 : (o.a.re < (R)-1 ? (R)-1 : o.a.re);
      const R tht = acos(ca);
      if (tht != (R)0) {
        const R tho = lam * tht;
        const R q1 = cos(tho);
        const R q2 = sin(tho) / sin(tht) * o.a.im;
        const R f = -sin(tho) / sin(tht);
        o.a = mk<R>(q1, -q2);
        o.b = mk<R>(f * o.b.re, f * o.b.im);
      }
    } else {
      // same rotation, angle atan2(|vector part|, scalar part) of w: accurate
      // for the small angles that decide convergence below theta ~ 1e-7
      const double svd = sqrt(w1.im * w1.im + w2.re * w2.re + w2.im * w2.im);
      if (svd != 0.0) {
        const R sv = (R)svd;
        const R tho = lam * atan2(sv, (R)w1.re);
        R sn, cs;
        sincos(tho, &sn, &cs);
        const R f = sn / sv;
        o.a = mk<R>(cs, -f * (R)w1.im);
        o.b = mk<R>(-f * (R)w2.re, -f * (R)w2.im);
      }
    }
    // (:243-252) A_f(x) -> Omega (iA) Omega^+
    R* Af = reinterpret_cast<R*>(ch.af);
    const R a1 = Af[((size_t)(eo * 3 + 0)) * nh + s], a2 = Af[((size_t)(eo * 3 + 1)) * nh + s],
            a3 = Af[((size_t)(eo * 3 + 2)) * nh + s];
    const su2<R> ta = nn(o, ad(a1, a2, a3, o));
    Af[((size_t)(eo * 3 + 0)) * nh + s] = ta.b.im;
    Af[((size_t)(eo * 3 + 1)) * nh + s] = ta.b.re;
    Af[((size_t)(eo * 3 + 2)) * nh + s] = ta.a.im;
    // (:256-324) links at both ends; renormalise on the eo = 1 half-step
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      su2<R> a = nn(o, um[mu]);
      su2<R> b = nd(ud[mu], o);
      if (last) {
        a = unitarise64(a);
        b = unitarise64(b);
      }
      LinkIO<R>::st(ch.uf, ((size_t)(mu * 2 + eo)) * nh + s, a);
      LinkIO<R>::st(ch.uf, ((size_t)(mu * 2 + oe)) * nh + xm[mu], b);
    }
    if (track) {
      const size_t gi = (size_t)eo * nh + s;
      LinkIO<R>::st(ch.g, gi, unitarise64(nn(o, LinkIO<R>::ld_cg(ch.g, gi))));
    }
  }
  if (last) block_reduce_store<1>(th, part + blockIdx.x);
}

// One parity of f/it_gauge_fixing.f:52-206 (the reference's iterative gauge
// fixing): g = sum_mu (i Im a, b) of U_f(x,mu) minus the same of
// U_f(x-mu,mu) (:62-84), the second component as written g1(1) - g2(2)
// (:110) unless LCE_ITGF_FIX_COMPONENT; |g|^2 into the partial sums on the
// second parity (:116-120); Omega = exp(h), h = +-step g (:122-141); the
// transform of A_f and of the links at both ends (:143-210).  g, |g|^2 and
// Omega in FP64.  The step comes from the chain state (gf_step); renorm
// reunitarises the links on the second parity (u_f_renorm after the
// iteration, as f/landau_gauge.f:56-57 does for the overrelaxed form).
// s_lo and last as for gf_half_kernel (a z-slab's visited sites; the whole
// lattice's second half-step, which sums |g|^2 and reunitarises).
template <typename R>
__global__ void __launch_bounds__(kBlock) it_half_kernel(const ChainDev* chp, const ChainState* cst, int eo,
                                                         double* part, int flags, int renorm, int s_lo, int last) {
  pdl_trigger();
  const ChainDev& ch = *chp;
  const int s = s_lo + blockIdx.x * kBlock + threadIdx.x;
  const int oe = 1 - eo, nh = ch.nh, s_hi = nh - s_lo;
  const Coord X = site_coord(eo, s < s_hi ? s : s_lo, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  const int xm[3] = {nbr_dn<0>(ch, X), nbr_dn<1>(ch, X), nbr_dn<2>(ch, X)};
  pdl_wait();
  if (cst->gf_done) return;
  double th[1] = {0.0};
  if (s < s_hi) {
    su2<R> um[3], ud[3];
    double g1a = 0, g1br = 0, g1bi = 0, g2a = 0, g2br = 0, g2bi = 0;
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      um[mu] = ldUf<R>(ch, mu, eo, s);
      ud[mu] = ldUf<R>(ch, mu, oe, xm[mu]);
    }
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      g1a += (double)um[mu].a.im;
      g1br += (double)um[mu].b.re;
      g1bi += (double)um[mu].b.im;
    }
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      g2a += (double)ud[mu].a.im;
      g2br += (double)ud[mu].b.re;
      g2bi += (double)ud[mu].b.im;
    }
    const bool fix = (flags & LCE_ITGF_FIX_COMPONENT) != 0;
    const double ga = g1a - g2a;
    const double gbr = fix ? g1br - g2br : -g2br;
    const double gbi = fix ? g1bi - g2bi : g1a - g2bi;
    if (last) th[0] = ga * ga + (gbr * gbr + gbi * gbi);
    const double st = (flags & LCE_ITGF_ASCEND) ? -cst->gf_step : cst->gf_step;
    const double ha = st * ga, hbr = st * gbr, hbi = st * gbi;
    const double t1 = sqrt(ha * ha + hbr * hbr + hbi * hbi);
    // the reference divides 0 by 0 where g = 0; the limit is 1
    const double t2 = t1 > 0.0 ? sin(t1) / t1 : 1.0;
    const su2<R> o{{(R)cos(t1), (R)(ha * t2)}, {(R)(hbr * t2), (R)(hbi * t2)}};
    R* Af = reinterpret_cast<R*>(ch.af);
    const R a1 = Af[((size_t)(eo * 3 + 0)) * nh + s], a2 = Af[((size_t)(eo * 3 + 1)) * nh + s],
            a3 = Af[((size_t)(eo * 3 + 2)) * nh + s];
    const su2<R> ta = nn(o, ad(a1, a2, a3, o));
    Af[((size_t)(eo * 3 + 0)) * nh + s] = ta.b.im;
    Af[((size_t)(eo * 3 + 1)) * nh + s] = ta.b.re;
    Af[((size_t)(eo * 3 + 2)) * nh + s] = ta.a.im;
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      su2<R> a = nn(o, um[mu]);
      su2<R> b = nd(ud[mu], o);
      if (renorm && last) {
        a = unitarise64(a);
        b = unitarise64(b);
      }
      LinkIO<R>::st(ch.uf, ((size_t)(mu * 2 + eo)) * nh + s, a);
      LinkIO<R>::st(ch.uf, ((size_t)(mu * 2 + oe)) * nh + xm[mu], b);
    }
    if (flags & LCE_ITGF_TRACK) {
      const size_t gi = (size_t)eo * nh + s;
      LinkIO<R>::st(ch.g, gi, unitarise64(nn(o, LinkIO<R>::ld_cg(ch.g, gi))));
    }
  }
  if (last) block_reduce_store<1>(th, part + blockIdx.x);
}

// U_f(x,mu) = G(x) U(x,mu) G(x+mu)^+ and A_f(x) -> G(x) A(x) G(x)^+, one
// thread per site of both parities
template <typename R>
__global__ void __launch_bounds__(kBlock) gauge_apply_kernel(const ChainDev* chp) {
  const ChainDev& ch = *chp;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= 2 * ch.nh) return;
  const int eo = i >= ch.nh ? 1 : 0, oe = 1 - eo, s = i - eo * ch.nh, nh = ch.nh;
  const Coord X = site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  const su2<R> gx = LinkIO<R>::ld(ch.g, (size_t)eo * nh + s);
  const int L[3] = {ch.L1, ch.L2, ch.L3};
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    int c[3] = {X.x, X.y, X.z};
    c[mu] = wrap(c[mu] + 1, L[mu]);
    const int sp = site_index(c[0], c[1], c[2], ch.hx, ch.nxy);
    const su2<R> gp = LinkIO<R>::ld(ch.g, (size_t)oe * nh + sp);
    const size_t li = ((size_t)(mu * 2 + eo)) * nh + s;
    LinkIO<R>::st(ch.uf, li, unitarise64(nd(nn(gx, LinkIO<R>::ld(ch.u, li)), gp)));
  }
  const R* A = reinterpret_cast<const R*>(ch.a);
  R* Af = reinterpret_cast<R*>(ch.af);
  const su2<R> t = nn(gx, ad(A[((size_t)(eo * 3 + 0)) * nh + s], A[((size_t)(eo * 3 + 1)) * nh + s],
                             A[((size_t)(eo * 3 + 2)) * nh + s], gx));
  Af[((size_t)(eo * 3 + 0)) * nh + s] = t.b.im;
  Af[((size_t)(eo * 3 + 1)) * nh + s] = t.b.re;
  Af[((size_t)(eo * 3 + 2)) * nh + s] = t.a.im;
}

template <typename R>
__global__ void transform_identity_kernel(void* g, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    LinkIO<R>::st(g, i, su2<R>{{(R)1, (R)0}, {(R)0, (R)0}});
}

// sum the theta partials in block order, count the iteration, test convergence
__global__ void __launch_bounds__(1024) gf_check_kernel(const ChainDev* chp, ChainState* cst, const double* part,
                                                        int nblocks) {
  pdl_trigger();
  pdl_wait();
  if (cst->gf_done) return;
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v[0] += part[b];
  __shared__ double tot;
  block_reduce_store<1>(v, &tot);
  __syncthreads();
  if (threadIdx.x == 0) {
    const double theta = tot / chp->nh;
    const int it = cst->gf_iters + 1;
    cst->gf_iters = it;
    cst->gf_theta = theta;
    if (!(theta > chp->limit_or) || (cst->gf_cap > 0 && it >= cst->gf_cap)) cst->gf_done = 1;
  }
}

// the same test for a lattice split into z-slabs: the slabs' theta sums (in
// slab order) over the whole lattice's nh odd sites, counted into slab 0's
// chain state, which the host copies to the other slabs
// fa: the Fourier-accelerated iteration's check (stop at gf_limit; fa = 1
// also shortens the step after an overshoot, as fa_check_kernel, which the
// conjugate-gradient form, fa = 2, does not); fa = 0: the overrelaxed
// iteration's (stop at limit_or)
__global__ void gf_check_slabs_kernel(const ChainDev* chp, ChainState* cst, const double* sums, int nslabs,
                                      double nh, int fa) {
  if (cst->gf_done) return;
  double tot = 0.0;
  for (int j = 0; j < nslabs; ++j) tot += sums[j];
  const double theta = tot / nh;
  const int it = cst->gf_iters + 1;
  if (fa == 1 && it > 1 && theta > 2.0 * cst->gf_theta) cst->gf_step = fmax(0.1, 0.7 * cst->gf_step);
  cst->gf_iters = it;
  cst->gf_theta = theta;
  const double limit = fa ? cst->gf_limit : chp->limit_or;
  if (!(theta > limit) || (cst->gf_cap > 0 && it >= cst->gf_cap)) cst->gf_done = 1;
}

// theta of the current U_f without updating (odd sites)
template <typename R>
__global__ void __launch_bounds__(kBlock) gf_theta_kernel(const ChainDev* chp, double* part) {
  const ChainDev& ch = *chp;
  const int s = blockIdx.x * kBlock + threadIdx.x;
  double th[1] = {0.0};
  if (s < ch.nh) {
    const Coord X = site_coord(1, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
    const int xm[3] = {nbr_dn<0>(ch, X), nbr_dn<1>(ch, X), nbr_dn<2>(ch, X)};
    su2<R> um[3], ud[3];
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      um[mu] = ldUf<R>(ch, mu, 1, s);
      ud[mu] = ldUf<R>(ch, mu, 0, xm[mu]);
    }
    su2<double> t1, t2;
    gf_sums<R>(ch, um, ud, t1, t2);
    const cpx<double> w2 = t1.b - t2.b;
    const double d = t1.a.im - t2.a.im;
    th[0] = d * d + (w2.re * w2.re + w2.im * w2.im);
  }
  block_reduce_store<1>(th, part + blockIdx.x);
}

template <int NQ>
__global__ void __launch_bounds__(1024) sum_partials_kernel(const double* part, int nblocks, double* out) {
  double v[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] += part[(size_t)b * NQ + q];
  }
  block_reduce_store<NQ>(v, out);
}

template <typename R>
void launch_gf_iteration(const ChainDev* ch, ChainState* cst, int track, double* part, int nh, cudaStream_t s) {
  const int nb = ceil_div(nh, kBlock);
  // programmatic dependent launch: each kernel waits in griddepcontrol.wait
  (void)launch_pdl(gf_half_kernel<R>, nb, kBlock, 0, s, ch, (const ChainState*)cst, 0, part, track, 0, 0);
  (void)launch_pdl(gf_half_kernel<R>, nb, kBlock, 0, s, ch, (const ChainState*)cst, 1, part, track, 0, 1);
  (void)launch_pdl(gf_check_kernel, 1, 1024, 0, s, ch, cst, (const double*)part, nb);
}

template <typename R>
int launch_gf_half(const ChainDev* ch, ChainState* cst, int eo, int last, double* part, int nh, int s_lo, int track,
                   cudaStream_t s) {
  const int nb = ceil_div(nh - 2 * s_lo, kBlock);
  (void)launch_pdl(gf_half_kernel<R>, nb, kBlock, 0, s, ch, (const ChainState*)cst, eo, part, track, s_lo, last);
  return nb;
}

void launch_gf_check_slabs(const ChainDev* ch, ChainState* cst, const double* sums, int nslabs, double nh,
                           cudaStream_t s, int fa) {
  gf_check_slabs_kernel<<<1, 1, 0, s>>>(ch, cst, sums, nslabs, nh, fa);
}

template <typename R>
void launch_it_iteration(const ChainDev* ch, ChainState* cst, int flags, int renorm, double* part, int nh,
                         cudaStream_t s) {
  const int nb = ceil_div(nh, kBlock);
  (void)launch_pdl(it_half_kernel<R>, nb, kBlock, 0, s, ch, (const ChainState*)cst, 0, part, flags, renorm, 0, 0);
  (void)launch_pdl(it_half_kernel<R>, nb, kBlock, 0, s, ch, (const ChainState*)cst, 1, part, flags, renorm, 0, 1);
  (void)launch_pdl(gf_check_kernel, 1, 1024, 0, s, ch, cst, (const double*)part, nb);
}

template <typename R>
void launch_gauge_apply(const ChainDev* ch, int nh, cudaStream_t s) {
  gauge_apply_kernel<R><<<ceil_div(2L * nh, kBlock), kBlock, 0, s>>>(ch);
}

template <typename R>
void launch_transform_identity(void* g, int nh, cudaStream_t s) {
  transform_identity_kernel<R><<<ceil_div(2L * nh, 256), 256, 0, s>>>(g, (size_t)2 * nh);
}

template void launch_gauge_apply<float>(const ChainDev*, int, cudaStream_t);
template void launch_gauge_apply<double>(const ChainDev*, int, cudaStream_t);
template void launch_transform_identity<float>(void*, int, cudaStream_t);
template void launch_transform_identity<double>(void*, int, cudaStream_t);

template <typename R>
void launch_gf_theta(const ChainDev* ch, double* part, int nh, cudaStream_t s) {
  gf_theta_kernel<R><<<ceil_div(nh, kBlock), kBlock, 0, s>>>(ch, part);
}

void launch_sum_partials(const double* part, int nblocks, int nq, double* out, cudaStream_t s) {
  if (nq == 1) sum_partials_kernel<1><<<1, 1024, 0, s>>>(part, nblocks, out);
  else if (nq == 2) sum_partials_kernel<2><<<1, 1024, 0, s>>>(part, nblocks, out);
  else if (nq == 3) sum_partials_kernel<3><<<1, 1024, 0, s>>>(part, nblocks, out);
  else sum_partials_kernel<4><<<1, 1024, 0, s>>>(part, nblocks, out);
}

template void launch_gf_iteration<float>(const ChainDev*, ChainState*, int, double*, int, cudaStream_t);
template void launch_gf_iteration<double>(const ChainDev*, ChainState*, int, double*, int, cudaStream_t);
template int launch_gf_half<float>(const ChainDev*, ChainState*, int, int, double*, int, int, int, cudaStream_t);
template int launch_gf_half<double>(const ChainDev*, ChainState*, int, int, double*, int, int, int, cudaStream_t);
template <typename R>
int launch_it_half(const ChainDev* ch, ChainState* cst, int eo, int last, double* part, int nh, int s_lo, int flags,
                   cudaStream_t s) {
  const int nb = ceil_div(nh - 2 * s_lo, kBlock);
  (void)launch_pdl(it_half_kernel<R>, nb, kBlock, 0, s, ch, (const ChainState*)cst, eo, part, flags, 1, s_lo, last);
  return nb;
}
template int launch_it_half<float>(const ChainDev*, ChainState*, int, int, double*, int, int, int, cudaStream_t);
template int launch_it_half<double>(const ChainDev*, ChainState*, int, int, double*, int, int, int, cudaStream_t);

template void launch_it_iteration<float>(const ChainDev*, ChainState*, int, int, double*, int, cudaStream_t);
template void launch_it_iteration<double>(const ChainDev*, ChainState*, int, int, double*, int, cudaStream_t);
template void launch_gf_theta<float>(const ChainDev*, double*, int, cudaStream_t);
template void launch_gf_theta<double>(const ChainDev*, double*, int, cudaStream_t);

}  // namespace lce
