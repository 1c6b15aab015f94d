// lce_update.cu -- checkerboard Monte Carlo update kernels.
//
// One pass = one routine over one parity (and one mu for links), one thread
// per site (or two), sites grouped in tiles of consecutive sites of one chain
// (the tile shape -- threads per block and sites per thread -- is chosen per
// context; the persistent form uses kBlock threads and one site per thread).
// The per-tile bodies fuse what the reference does as a chain of whole-lattice
// array passes (multall*, halo exchanges, temporaries): neighbour gathers, the
// SU(2) algebra, the random proposal, the accept/reject and the FP64 partial
// sums of the measurements, so every field element is read from HBM once per
// pass.
//
//   higgs_tile<R, MODE>    f/a_force.f + f/ahiggs2.f (MODE 0, heatbath),
//                          f/ahiggs3.f (MODE 1, overrelaxation),
//                          f/ahiggs1.f (MODE 2, Metropolis)
//   link_tile<R, MU, OR>   f/staples.f + f/agauge.f + f/heat_kpi.f (OR = 0);
//                          link overrelaxation (OR = 1, no reference)
//   finalize_sum/combine   deterministic FP64 reduction of the per-tile
//                          partials into /aver_loc/-style results (f/meas1.f)
//
// Two execution forms share these bodies:
//   * one kernel per pass (higgs_kernel, link_kernel, finalize_kernel),
//     chained with programmatic dependent launch and captured in a graph;
//   * sweep_persistent_kernel: one cooperative launch per sweep whose blocks
//     loop over the tile work list of every pass, with a bounded grid barrier
//     between passes (no kernel boundaries inside the sweep).
//
// Random numbers: Philox4x32-10 keyed by the chain seed with counter
// (site, call, pass), or, in validation mode, the host-supplied stream indexed
// in the reference's consumption order (slot layouts in lce_common.cuh).
#include <algorithm>

#include "lce_internal.hpp"

namespace lce {

// The reference evaluates cos(tpi*u) and sin(tpi*u) with tpi = 2 acos(-1)
// (f/heat_kpi.f:29, f/gauss.f:17); M<R>::cos2pi / sincos2pi take u itself
// (lce_common.cuh).

__device__ __forceinline__ int find_chain(const int* blk_begin, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(blk_begin + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Field loads.  NC = true: the read-only (non-coherent) path, valid when no
// earlier writer runs in the same kernel (the per-pass form).  NC = false:
// L2 loads (ld.global.cg) for the persistent form, where fields written by
// other blocks before a grid barrier are read after it.  Ordinary cached
// loads are not enough there: measured on B200, lines an SM's L1 fetched
// before the barrier were still served after it (the persistent sweep then
// differs from the per-pass sweep), so L1 is bypassed.
template <typename R, bool NC = true>
__device__ __forceinline__ R ldA(const R* A, int nh, int p, int k, int s) {
  const R* q = A + ((size_t)(p * 3 + k)) * nh + s;
  return NC ? __ldg(q) : __ldcg(q);
}

// Neighbour offsets of one site.  The half-row index s = z*nxy + y*hx + (x>>1)
// of f/adresses.f is a sum of per-axis terms, so the index of any neighbour,
// one step or two steps along different axes, is s plus the steps' offsets;
// p[k] / m[k] are the offsets of +1 / -1 along axis k (periodic).  Computed
// once per site instead of re-deriving every neighbour from coordinates.
struct NbrOff {
  int p[3], m[3];
};
__device__ __forceinline__ NbrOff nbr_offsets(const ChainDev& ch, Coord X) {
  NbrOff o;
  const int xh = X.x >> 1;
  o.p[0] = X.x + 1 == ch.L1 ? -xh : ((X.x + 1) >> 1) - xh;
  o.m[0] = X.x == 0 ? ch.hx - 1 : ((X.x - 1) >> 1) - xh;
  o.p[1] = X.y + 1 == ch.L2 ? ch.hx - ch.nxy : ch.hx;
  o.m[1] = X.y == 0 ? ch.nxy - ch.hx : -ch.hx;
  o.p[2] = X.z + 1 == ch.L3 ? ch.nxy - ch.nh : ch.nxy;
  o.m[2] = X.z == 0 ? ch.nh - ch.nxy : -ch.nxy;
  return o;
}

template <typename R, bool NC = true>
__device__ __forceinline__ su2<R> ldU(const ChainDev& ch, int mu, int p, int s) {
  const size_t i = ((size_t)(mu * 2 + p)) * ch.nh + s;
  return NC ? LinkIO<R>::ld(ch.u, i) : LinkIO<R>::ld_cg(ch.u, i);
}

// f/staples.f:65-221: for each nu != mu (ascending),
//   upper  = U_nu(x+mu) [U_mu(x+nu)^+ U_nu(x)^+]          (NN of DD)
//   lower  = U_nu(x-nu+mu)^+ [U_mu(x-nu)^+ U_nu(x-nu)]    (DN of DN)
//   V      = (V + upper) + lower
template <typename R, int MU, int NU, bool NC>
__device__ __forceinline__ void staple_add(const ChainDev& ch, int eo, const NbrOff& o, int s, su2<R>& V) {
  const int oe = 1 - eo;
  const int xpmu = s + o.p[MU], xpnu = s + o.p[NU], xmnu = s + o.m[NU];
  const int xmnupmu = xmnu + o.p[MU];
  su2<R> up1 = dd(ldU<R, NC>(ch, MU, oe, xpnu), ldU<R, NC>(ch, NU, eo, s));
  su2<R> up2 = nn(ldU<R, NC>(ch, NU, oe, xpmu), up1);
  su2<R> bt1 = dn(ldU<R, NC>(ch, MU, oe, xmnu), ldU<R, NC>(ch, NU, oe, xmnu));
  su2<R> bt2 = dn(ldU<R, NC>(ch, NU, eo, xmnupmu), bt1);
  V.a = (V.a + up2.a) + bt2.a;
  V.b = (V.b + up2.b) + bt2.b;
}

template <typename R, int MU, bool NC = true>
__device__ __forceinline__ su2<R> staple(const ChainDev& ch, int eo, const NbrOff& o, int s) {
  su2<R> V{{(R)0, (R)0}, {(R)0, (R)0}};
  if (MU == 0) {
    staple_add<R, 0, 1, NC>(ch, eo, o, s, V);
    staple_add<R, 0, 2, NC>(ch, eo, o, s, V);
  } else if (MU == 1) {
    staple_add<R, 1, 0, NC>(ch, eo, o, s, V);
    staple_add<R, 1, 2, NC>(ch, eo, o, s, V);
  } else {
    staple_add<R, 2, 0, NC>(ch, eo, o, s, V);
    staple_add<R, 2, 1, NC>(ch, eo, o, s, V);
  }
  return V;
}

// f/a_force.f:54-110: F = sum_mu [U(x)(iA(x+mu))U(x)^+ + U(x-mu)^+(iA(x-mu))U(x-mu)],
// components F3 = Im(.)_a, F2 = Re(.)_b, F1 = Im(.)_b
template <typename R, int MU, bool NC>
__device__ __forceinline__ void force_add(const ChainDev& ch, int eo, const NbrOff& o, int s, R& f1, R& f2,
                                          R& f3) {
  const int oe = 1 - eo, nh = ch.nh;
  const R* A = reinterpret_cast<const R*>(ch.a);
  const int xp = s + o.p[MU], xm = s + o.m[MU];
  su2<R> ux = ldU<R, NC>(ch, MU, eo, s);
  su2<R> ud = ldU<R, NC>(ch, MU, oe, xm);
  su2<R> t1 = nn(ux, ad(ldA<R, NC>(A, nh, oe, 0, xp), ldA<R, NC>(A, nh, oe, 1, xp), ldA<R, NC>(A, nh, oe, 2, xp), ux));
  su2<R> tb = dn(ud, an(ldA<R, NC>(A, nh, oe, 0, xm), ldA<R, NC>(A, nh, oe, 1, xm), ldA<R, NC>(A, nh, oe, 2, xm), ud));
  f3 = f3 + (t1.a.im + tb.a.im);
  f2 = f2 + (t1.b.re + tb.b.re);
  f1 = f1 + (t1.b.im + tb.b.im);
}

template <typename R, bool NC = true>
__device__ __forceinline__ void higgs_force(const ChainDev& ch, int eo, const NbrOff& o, int s, R& f1, R& f2,
                                            R& f3) {
  f1 = f2 = f3 = (R)0;
  force_add<R, 0, NC>(ch, eo, o, s, f1, f2, f3);
  force_add<R, 1, NC>(ch, eo, o, s, f1, f2, f3);
  force_add<R, 2, NC>(ch, eo, o, s, f1, f2, f3);
}

// Set up the uniform source of this pass (of hit `hit` of a multi-hit pass:
// the next N*nh stream values, the next Philox pass).  Returns false (and
// flags the context) when the validation stream cannot cover the pass.
template <typename R, int N>
__device__ __forceinline__ bool setup_uniforms(const PassArgs& p, const ChainDev& ch, int s, int layout,
                                               Uniforms<R, N>& U, int hit = 0) {
  if (p.stream) {
    const int snh = p.stream_nh ? p.stream_nh : ch.nh;
    unsigned long long base = p.st->stream_pos + p.stream_off + (unsigned long long)hit * N * snh;
    if (base + (unsigned long long)N * snh > p.stream_n) {
      if (s == p.s_lo) atomicOr(&p.st->status, kStatusStreamExhausted);
      return false;
    }
    U.fill_stream(p.stream + base, snh, layout, s + p.site_off);
  } else {
    U.fill_philox(ch.key0, ch.key1, p.st->pass_ctr + p.pass_off + hit, s + p.site_off);
  }
  return true;
}

// ------------------------------------------------------------------ Higgs
// One tile (BS * SPT consecutive sites of one chain, BS threads) of a Higgs
// pass.  PDL: trigger dependents and wait for the previous kernel (per-pass
// form only).
template <typename R, int MODE, bool PDL, int SPT = 1, int BS = kBlock>
__device__ __forceinline__ void higgs_tile(const PassArgs& p, int tile) {
  if (PDL && !p.trigger_late) pdl_trigger();
  // the chain table is written once at context creation: safe before pdl_wait
  const int c = p.nchains > 1 ? find_chain(p.blk_begin, p.nchains, tile) : 0;
  const ChainDev& ch = p.chains[c];
  // a tile is BS * SPT consecutive sites; thread t takes t, t + BS, ...
  const int s0 = p.s_lo + (tile - __ldg(p.blk_begin + c)) * BS * SPT + threadIdx.x;
  const int eo = p.eo, nh = ch.nh, s_hi = nh - p.s_lo;
  const Coord X0 = site_coord(eo, s0 < s_hi ? s0 : p.s_lo, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  unsigned acc[1] = {0u};
  double q[3] = {0.0, 0.0, 0.0};
  constexpr int NS = MODE == 0 ? 7 : (MODE == 1 ? 1 : 4);
  const int layout = MODE == 2 ? kTriple : kPlanar;
  // the first site's uniforms, drawn before the wait when the counters are settled
  Uniforms<R, NS> Un0;
  const bool early = PDL && SPT == 1 && p.rng_early && s0 < s_hi;
  const bool ok0 = early ? setup_uniforms<R, NS>(p, ch, s0, layout, Un0) : false;
  if (PDL) {
    pdl_wait();
    if (p.trigger_late) pdl_trigger();
  }
#pragma unroll 1
  for (int r = 0; r < SPT; ++r) {
    const int s = s0 + r * BS;
    if (s >= s_hi) break;
    const Coord X = r == 0 ? X0 : site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
    const NbrOff no = nbr_offsets(ch, X);
    Uniforms<R, NS> Un = Un0;
    if (r == 0 && early ? ok0 : setup_uniforms<R, NS>(p, ch, s, layout, Un)) {
      R f[3];
      higgs_force<R, PDL>(ch, eo, no, s, f[0], f[1], f[2]);
      R* A = reinterpret_cast<R*>(ch.a);
      R ao[3], an_[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) ao[k] = PDL ? A[((size_t)(eo * 3 + k)) * nh + s] : __ldcg(A + ((size_t)(eo * 3 + k)) * nh + s);
      const R beta_a = (R)ch.beta_a, beta_2 = (R)ch.beta_2, beta_4 = (R)ch.beta_4;
      R alph = (R)0, sf_o = (R)0, sf_n = (R)0;
      if constexpr (MODE == 0 || MODE == 1) {
        // f/ahiggs2.f:52-77 width / cxval / alph
        R rr, cxval;
        if (ch.imode == 1) {
          R conf2 = (R)0;
#pragma unroll
          for (int i = 0; i < 3; ++i) conf2 = conf2 + beta_a * (f[i] * f[i]);
          R qq = beta_2 + beta_4 * conf2;
          alph = M<R>::div(beta_4 * conf2, (R)2 * (qq * qq));
          const R width = beta_2 + alph;
          rr = M<R>::div((R)1, width);
          cxval = M<R>::div(M<R>::div((R)1, (R)2), width);
        } else {
          rr = (R)ch.inv_beta2;      // 1/width, width = beta_2
          cxval = (R)ch.cxval0;      // 1/beta_2/2
        }
        if constexpr (MODE == 0) {
          // f/gauss.f:17-29: X = sqrt(-ln(W1)/R) cos(2 pi W2); f/ahiggs2.f:83-91
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const R w1 = -(R)1 * rr * M<R>::log(Un.v[2 * i]);
            const R g = M<R>::sqrt(w1) * M<R>::cos2pi(Un.v[2 * i + 1]);
            an_[i] = g + beta_a * f[i] * cxval;
          }
        } else {
          // f/ahiggs3.f:83-87
#pragma unroll
          for (int i = 0; i < 3; ++i) an_[i] = -ao[i] + (R)2 * beta_a * f[i] * cxval;
        }
      } else {
        // f/ahiggs1.f:51-56 box proposal
        const R delta = (R)p.cst[c].delta;
#pragma unroll
        for (int i = 0; i < 3; ++i) an_[i] = ao[i] + (Un.v[i] - (R)0.5) * delta;
      }
      R rho_o = (R)0, rho_n = (R)0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (MODE == 2) {
          sf_o = sf_o + ao[i] * f[i];
          sf_n = sf_n + an_[i] * f[i];
        }
        rho_o = rho_o + ao[i] * ao[i];
        rho_n = rho_n + an_[i] * an_[i];
      }
      R boltz;
      if constexpr (MODE == 2) {
        // f/ahiggs1.f:77-78
        boltz = M<R>::exp(-beta_a * (sf_o - sf_n) + beta_2 * (rho_o - rho_n) +
                          beta_4 * (rho_o * rho_o - rho_n * rho_n));
      } else {
        // f/ahiggs2.f:108-109
        boltz = M<R>::exp(-alph * (rho_o - rho_n) + beta_4 * (rho_o * rho_o - rho_n * rho_n));
      }
      constexpr int acc_slot = MODE == 0 ? 6 : (MODE == 1 ? 0 : 3);
      if (boltz >= Un.v[acc_slot]) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          A[((size_t)(eo * 3 + k)) * nh + s] = an_[k];
          ao[k] = an_[k];
        }
        rho_o = rho_n;
        sf_o = sf_n;
        acc[0] += 1u;
      }
      if (p.part) {
        q[0] += (double)rho_o;
        q[1] += (double)rho_o * (double)rho_o;
        if (MODE == 2) q[2] += (double)sf_o;
        else if constexpr (sizeof(R) == 4) q[2] += (double)(ao[0] * f[0] + ao[1] * f[1] + ao[2] * f[2]);
        else q[2] += (double)ao[0] * f[0] + (double)ao[1] * f[1] + (double)ao[2] * f[2];
      }
    }
  }
  // partials {accepted, sum rho, sum rho^2, sum a.F}
  if (p.part) block_reduce_cs<1, 3, kNQ, !PDL>(acc, q, p.part + (size_t)tile * kNQ);
}

// ------------------------------------------------------------------ links
// NHIT = 3 is f/agauge1.f: the staple is built once and the heatbath +
// Metropolis hit is repeated on the updated link, each hit with its own
// uniforms (f/agauge1.f:95-198).
template <typename R, int MU, int OR, bool PDL, int NHIT = 1, int SPT = 1, int BS = kBlock>
__device__ __forceinline__ void link_tile(const PassArgs& p, int tile) {
  if (PDL && !p.trigger_late) pdl_trigger();
  const int c = p.nchains > 1 ? find_chain(p.blk_begin, p.nchains, tile) : 0;
  const ChainDev& ch = p.chains[c];
  // a tile is BS * SPT consecutive sites; thread t takes t, t + BS, ...
  const int s0 = p.s_lo + (tile - __ldg(p.blk_begin + c)) * BS * SPT + threadIdx.x;
  const int eo = p.eo, oe = 1 - eo, nh = ch.nh, s_hi = nh - p.s_lo;
  const Coord X0 = site_coord(eo, s0 < s_hi ? s0 : p.s_lo, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  unsigned cnt[2] = {0u, 0u};
  double pl[1] = {0.0};
  // the first site's uniforms (of the first hit), drawn before the wait when
  // the counters are settled
  Uniforms<R, OR ? 1 : 7> Un0;
  const bool early = PDL && SPT == 1 && p.rng_early && s0 < s_hi;
  const bool ok0 = early ? setup_uniforms<R, OR ? 1 : 7>(p, ch, s0, OR ? kPlanar : kTriple, Un0) : false;
  if (PDL) {
    pdl_wait();
    if (p.trigger_late) pdl_trigger();
  }
#pragma unroll 1
  for (int r = 0; r < SPT; ++r) {
    const int s = s0 + r * BS;
    if (s >= s_hi) break;
    const Coord X = r == 0 ? X0 : site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
    const NbrOff no = nbr_offsets(ch, X);
    Uniforms<R, OR ? 1 : 7> Un = Un0;
    if (r == 0 && early ? ok0 : setup_uniforms<R, OR ? 1 : 7>(p, ch, s, OR ? kPlanar : kTriple, Un)) {
      const su2<R> V = staple<R, MU, PDL>(ch, eo, no, s);
      const size_t li = ((size_t)(MU * 2 + eo)) * nh + s;
      su2<R> uo = PDL ? LinkIO<R>::ld(ch.u, li) : LinkIO<R>::ld_cg(ch.u, li);
      // f/agauge.f:71-84: normalised staple, 1/(beta |V|), 1/2 Re Tr(U Vhat)
      const R tn = M<R>::rsqrt(norm2(V));
      const su2<R> vh{{tn * V.a.re, tn * V.a.im}, {tn * V.b.re, tn * V.b.im}};
      // f/agauge.f:126-174 hopping term beta_a Re[(iA(x) U)(iA(x+mu) U^+)]_11 and accept
      const R* A = reinterpret_cast<const R*>(ch.a);
      const int xp = s + no.p[MU];
      const R x1 = ldA<R, PDL>(A, nh, eo, 0, s), x2 = ldA<R, PDL>(A, nh, eo, 1, s), x3 = ldA<R, PDL>(A, nh, eo, 2, s);
      const R y1 = ldA<R, PDL>(A, nh, oe, 0, xp), y2 = ldA<R, PDL>(A, nh, oe, 1, xp), y3 = ldA<R, PDL>(A, nh, oe, 2, xp);
      const R beta_a = (R)ch.beta_a;
      bool changed = false;
#pragma unroll 1
      for (int hit = 0; hit < NHIT; ++hit) {
        if (hit > 0 && !setup_uniforms<R, OR ? 1 : 7>(p, ch, s, OR ? kPlanar : kTriple, Un, hit)) break;
        su2<R> hn;
        if constexpr (!OR) {
          const R t1 = M<R>::div(tn, (R)ch.beta);
          const R t2 = (uo.a * vh.a - uo.b * cj(vh.b)).re;
          // f/heat_kpi.f:33-98 single-trial Kennedy-Pendleton
          R a1 = Un.v[0], a2 = Un.v[1], a3 = Un.v[2];
          if (a1 == (R)0) a1 = (R)0.0000033;
          if (a2 == (R)0) a2 = (R)0.0000066;
          const R cc = M<R>::cos2pi(a3);
          R a0 = -(M<R>::log(a1) + M<R>::log(a2) * (cc * cc)) * t1;
          const R r4 = Un.v[3];
          const bool lacc = r4 * r4 <= ((R)1 - (R)0.5 * a0);
          a0 = lacc ? (R)1 - a0 : t2;
          cnt[0] += lacc ? 1u : 0u;
          R b1 = (R)1 - a0 * a0;
          b1 = b1 >= (R)0 ? M<R>::sqrt(b1) : (R)0;
          const R b2 = (R)2 * (Un.v[4] - (R)0.5);
          su2<R> Xk;
          Xk.a = mk<R>(a0, b1 * b2);
          R q0 = (R)1 - b2 * b2;
          q0 = q0 >= (R)0 ? b1 * M<R>::sqrt(q0) : (R)0;
          R sph, cph;
          M<R>::sincos2pi(Un.v[5], &sph, &cph);
          Xk.b = mk<R>(q0 * sph, q0 * cph);
          hn = nd(Xk, vh);  // f/agauge.f:98-99
        } else {
          // overrelaxation U' = (Vhat U Vhat)^+ leaves Re Tr(U V) unchanged
          const su2<R> w = nn(nn(vh, uo), vh);
          hn = su2<R>{cj(w.a), -w.b};
        }
        const R sa_old = beta_a * nn(an(x1, x2, x3, uo), ad(y1, y2, y3, uo)).a.re;
        const R sa_new = beta_a * nn(an(x1, x2, x3, hn), ad(y1, y2, y3, hn)).a.re;
        if (M<R>::exp(sa_old - sa_new) >= Un.v[OR ? 0 : 6]) {
          uo = hn;
          changed = true;
          cnt[OR ? 0 : 1] += 1u;
        }
      }
      if (changed) LinkIO<R>::st(ch.u, li, p.fuse_renorm ? unitarise64(uo) : uo);
      // f/agauge.f:179-185 plaquette against the staple
      if (!OR && p.part) pl[0] += (double)nn(uo, V).a.re;
    }
  }
  // partials {KP accepted, Metropolis accepted, sum plaquette} / {OR accepted}
  if (p.part) {
    if constexpr (!OR) block_reduce_cs<2, 1, kNQ, !PDL>(cnt, pl, p.part + (size_t)tile * kNQ);
    else {
      unsigned c1[1] = {cnt[0]};
      double d0[1] = {0.0};
      block_reduce_cs<1, 0, kNQ, !PDL>(c1, d0, p.part + (size_t)tile * kNQ);
    }
  }
}

// ------------------------------------------------------------------ finalize
// The partial sums of a reduction slot (kNQ doubles per tile) are added in two
// fixed levels, so the order of every FP64 addition depends only on the tile
// table, never on which warp or block does the work (the per-pass and the
// persistent forms give the same bits):
//   level 1  chunk k of chain c = the chain's tiles [k*128, (k+1)*128); lane l
//            adds the tiles l, l+32, l+64, l+96 of the chunk in order and the
//            lanes are combined by a fixed shuffle tree;
//   level 2  a chain of several chunks: lane l adds the chunk sums l, l+32,
//            ... in order, same tree.  A one-chunk chain's level-1 sum is its
//            total.
// One (chunk, slot) or (chain, slot) item per warp; the loads of four tiles
// (or chunk sums) are issued together before their in-order adds.  In the
// per-pass form level 1 of a pass's slot is done by extra blocks of the next
// pass (reduce-behind), so the finalize kernel is left with level 1 of the
// last pass's slot, level 2 and the combine.
__device__ __forceinline__ void warp_tree(double (&v)[kNQ]) {
#pragma unroll
  for (int q = 0; q < kNQ; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
}

// in-order sum over the strided elements e = e0 + lane, e0 + lane + 32, ...
// (e < e1) of an array of kNQ-double records with record stride `stride`
// (in double2), reading through L2
__device__ __forceinline__ void strided_sum(const double2* base, size_t stride, int e0, int e1, double (&v)[kNQ]) {
  static_assert(kNQ == 4, "a record is two double2");
  const int lane = threadIdx.x & 31;
  v[0] = v[1] = v[2] = v[3] = 0.0;
  constexpr int kBatch = 4;
  for (int b = e0 + lane; b < e1; b += 32 * kBatch) {
    double2 x[kBatch][2];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int e = b + 32 * j;
      x[j][0] = e < e1 ? __ldcg(base + (size_t)e * stride) : make_double2(0.0, 0.0);
      x[j][1] = e < e1 ? __ldcg(base + (size_t)e * stride + 1) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      if (b + 32 * j < e1) {
        v[0] += x[j][0].x;
        v[1] += x[j][0].y;
        v[2] += x[j][1].x;
        v[3] += x[j][1].y;
      }
    }
  }
  warp_tree(v);
}

// level 1 of slot i (partials at part_i), item g = chunk g over all chains:
// the chunk's sum goes to the chain's total when the chain is one chunk,
// else to chunks[g][i]
__device__ __forceinline__ void level1_item(const double* part_i, const int* blk_begin, const int* chunk_begin,
                                            int nchains, int g, int i, double* chunks, double* totals) {
  const int c = nchains > 1 ? find_chain(chunk_begin, nchains, g) : 0;
  const int t0 = __ldg(blk_begin + c) + (g - __ldg(chunk_begin + c)) * kChunkTiles;
  const int t1 = min(__ldg(blk_begin + c + 1), t0 + kChunkTiles);
  double v[kNQ];
  strided_sum(reinterpret_cast<const double2*>(part_i), 2, t0, t1, v);
  if ((threadIdx.x & 31) == 0) {
    const bool one = __ldg(chunk_begin + c + 1) - __ldg(chunk_begin + c) == 1;
    double* dst = one ? totals + ((size_t)c * kMaxSlots + i) * kNQ : chunks + ((size_t)g * kMaxSlots + i) * kNQ;
#pragma unroll
    for (int q = 0; q < kNQ; ++q) dst[q] = v[q];
  }
}

// level 1, item w = (chunk g over all chains, slot pre + w % (nslots - pre))
__device__ __forceinline__ void finalize_chunk_warp(const FinalizeArgs& f, int w) {
  const int nrem = f.nslots - f.pre;
  const int g = w / nrem, i = f.pre + w % nrem;
  level1_item(f.part + (size_t)i * f.slot_stride, f.blk_begin, f.chunk_begin, f.nchains, g, i, f.chunks, f.totals);
}

// The reduce-behind blocks of a per-pass launch (blockIdx.x >= p.ntiles):
// after the wait the previous pass has completed, and its slot's level-1
// items are spread over these blocks' warps.
__device__ __forceinline__ void reduce_behind(const PassArgs& p) {
  pdl_trigger();
  pdl_wait();
  const int nw = (int)(blockDim.x >> 5);
  const int nred = ((int)gridDim.x - p.ntiles) * nw;
  const CtxState& st = *p.st;
  const int slot = p.rb_slot & 0xff;
  const double* part = st.rb_part + (size_t)slot * st.rb_slot_stride;
  const int* chunk_begin = st.rb_chunk_begin[p.rb_slot >> 8];
  for (int g = ((int)blockIdx.x - p.ntiles) * nw + (int)(threadIdx.x >> 5); g < p.rb_nitems; g += nred)
    level1_item(part, p.blk_begin, chunk_begin, p.nchains, g, slot, st.rb_chunks, st.rb_totals);
}

// Reduce-behind blocks are compiled into the one-site-per-thread kernels:
// in the two-sites form, at its 64-register cap, the extra branch made the
// link kernels spill (56-76 bytes).
template <int SPT>
constexpr bool kReduceBehind = SPT == 1;

// Tile shape: BS threads per block, SPT sites per thread (1, or 2 for the
// LCE_SWEEP_PASSES2 form), and OCC resident threads per SM the register cap
// is set for: OCC = 0 keeps the cap of min_blocks<R>() blocks of kBlock
// threads (64 registers in FP32); OCC = 1152 is nine blocks of 128 (56).
template <typename R, int BS, int OCC>
constexpr int min_blocks_bs() {
  return OCC ? OCC / BS : (min_blocks<R>() * kBlock / BS > 0 ? min_blocks<R>() * kBlock / BS : 1);
}

template <typename R, int MODE, int SPT, int BS, int OCC = 0>
__global__ void __launch_bounds__(BS, min_blocks_bs<R, BS, OCC>()) higgs_kernel(PassArgs p) {
  if (kReduceBehind<SPT> && p.rb_nitems && (int)blockIdx.x >= p.ntiles) reduce_behind(p);
  else higgs_tile<R, MODE, true, SPT, BS>(p, blockIdx.x);
}

template <typename R, int MU, int OR, int SPT, int BS, int OCC = 0>
__global__ void __launch_bounds__(BS, min_blocks_bs<R, BS, OCC>()) link_kernel(PassArgs p) {
  if (kReduceBehind<SPT> && p.rb_nitems && (int)blockIdx.x >= p.ntiles) reduce_behind(p);
  else link_tile<R, MU, OR, true, 1, SPT, BS>(p, blockIdx.x);
}

// f/agauge1.f (3 hits)
template <typename R, int MU, int SPT, int BS, int OCC = 0>
__global__ void __launch_bounds__(BS, min_blocks_bs<R, BS, OCC>()) link3_kernel(PassArgs p) {
  if (kReduceBehind<SPT> && p.rb_nitems && (int)blockIdx.x >= p.ntiles) reduce_behind(p);
  else link_tile<R, MU, 0, true, 3, SPT, BS>(p, blockIdx.x);
}

// level 2, item w = (chain c, slot i); nothing to do for a one-chunk chain
__device__ __forceinline__ void finalize_chain_warp(const FinalizeArgs& f, int w) {
  const int c = w / f.nslots, i = w % f.nslots;
  const int g0 = __ldg(f.chunk_begin + c), g1 = __ldg(f.chunk_begin + c + 1);
  if (g1 - g0 <= 1) return;
  double v[kNQ];
  strided_sum(reinterpret_cast<const double2*>(f.chunks + (size_t)i * kNQ), kMaxSlots * kNQ / 2, g0, g1, v);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < kNQ; ++q) f.totals[((size_t)c * kMaxSlots + i) * kNQ + q] = v[q];
  }
}

// The combine's slot tables in shared memory, copied by the finalize kernels
// before their wait, while the previous pass still runs.
struct FinTables {
  unsigned char kinds[kMaxSlots], gid[kMaxSlots], gflags[kMaxSlots], gbeg[kMaxSlots], gend[kMaxSlots];
};
__device__ __forceinline__ void load_tables(const FinalizeArgs& f, FinTables& T) {
  for (int i = threadIdx.x; i < kMaxSlots; i += blockDim.x) {
    T.kinds[i] = f.kinds[i];
    T.gid[i] = f.gid[i];
    T.gflags[i] = f.gflags[i];
    T.gbeg[i] = f.gbeg[i];
    T.gend[i] = f.gend[i];
  }
}

// Per chain the reference's normalisations of the slot totals, then the RNG
// counters advance.  Run by one block after every total is complete, one
// warp per chain.  The routine groups (fin_groups) are independent: lane j
// sums the slots of groups j and j + 32 in slot order, and the divisions of
// the normalisations (up to four per group) run one per lane, lane 4 g' + d
// taking division d of group g = g' + 8 r, so that they overlap instead of
// following one another.  The additions and divisions are those of a scan
// over the slots in order, and each field is written by the last group that
// sets it.  Only the ahiggs1 step adaptation runs as a chain over the
// ahiggs1 groups in order.
// SM: a single chain whose totals are in shared memory (stot) instead of
// f.totals, with its volume, ahiggs1 step and RNG counters loaded at the
// kernel's start (pre = {2 nh, delta}, ctr = {pass_ctr, stream_pos}).
template <bool SM = false>
__device__ __forceinline__ void finalize_combine(const FinalizeArgs& f, const FinTables& T, const double* stot = nullptr,
                                                 const double* pre = nullptr, const unsigned long long* ctr = nullptr) {
  static_assert(kMaxSlots <= 64, "two slots (groups) per lane");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (int)(blockDim.x >> 5);
  for (int c = warp; c < f.nchains; c += nwarps) {
    const double V = SM ? pre[0] : 2.0 * f.chains[c].nh;
    const double* base = SM ? stot : f.totals + (size_t)c * kMaxSlots * kNQ;
    double t0[kNQ], t1[kNQ];
    bool bad = false;
#pragma unroll
    for (int q = 0; q < kNQ; ++q) {
      const size_t i0 = (size_t)lane * kNQ + q, i1 = (size_t)(lane + 32) * kNQ + q;
      t0[q] = lane < f.nslots ? (SM ? base[i0] : __ldcg(base + i0)) : 0.0;
      t1[q] = lane + 32 < f.nslots ? (SM ? base[i1] : __ldcg(base + i1)) : 0.0;
      bad = bad || !isfinite(t0[q]) || !isfinite(t1[q]);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&f.st->status, kStatusNaN);
    lce_meas& m = f.meas[c];
    // the group sums: lane j, groups j (hs[0]) and j + 32 (hs[1])
    double hs[2][kNQ] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    if (SM) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int g = lane + 32 * s;
        if (g >= f.ngroups) continue;
        for (int i = T.gbeg[g]; i <= T.gend[g]; ++i) {
          if (T.gid[i] != g) continue;
#pragma unroll
          for (int q = 0; q < kNQ; ++q) hs[s][q] += stot[i * kNQ + q];
        }
      }
    } else {
      // warp-uniform scan: slot i's totals by shuffle, added by its group's lane
      for (int i = 0; i < f.nslots; ++i) {
        const int g = T.gid[i];
        double t[kNQ];
#pragma unroll
        for (int q = 0; q < kNQ; ++q) t[q] = __shfl_sync(0xffffffffu, i < 32 ? t0[q] : t1[q], i & 31);
        if (g == kNoGroup || lane != (g & 31)) continue;
#pragma unroll
        for (int q = 0; q < kNQ; ++q) {
          if (g < 32) hs[0][q] += t[q];
          else hs[1][q] += t[q];
        }
      }
    }
    // the normalisations, one division per lane
    for (int g0 = 0; g0 < f.ngroups; g0 += 8) {
      const int g = g0 + (lane >> 2), d = lane & 3;
      double h[kNQ];
#pragma unroll
      for (int q = 0; q < kNQ; ++q) {
        const double x0 = __shfl_sync(0xffffffffu, hs[0][q], g & 31), x1 = __shfl_sync(0xffffffffu, hs[1][q], g & 31);
        h[q] = g < 32 ? x0 : x1;
      }
      const int kind = g < f.ngroups ? (T.kinds[T.gend[g]] & 0x7f) : -1;
      const unsigned fl = g < f.ngroups ? T.gflags[g] : 0u;
      const bool higgs = kind >= 0 && kind <= kHiggsMetro, link = kind == kLinkHB || kind == kLinkHB3;
      // f/ahiggs2.f:142-147 (same in ahiggs1/3): a2 = h1/V, a4 = h2/V, akin = h3/(6V), acc = h0/V;
      // f/agauge.f:195-200: plaq = l2/(12V), acc = (l0/(3V)) (l1/(12V)); f/agauge1.f:227-232
      // divides the Metropolis factor by the 3 hits; link overrelaxation: l0/(3V)
      double num = 1.0, den = 1.0;
      if (higgs) {
        num = d == 0 ? h[1] : (d == 1 ? h[2] : (d == 2 ? h[3] : h[0]));
        den = d == 2 ? 6.0 * V : V;
      } else if (link) {
        num = d == 0 ? h[2] : (d == 1 ? h[0] : h[1]);
        den = d == 1 ? 3.0 * V : 12.0 * V;
      } else if (kind == kLinkOR) {
        num = h[0];
        den = 3.0 * V;
      }
      double r = num / den;
      if (kind == kLinkHB3 && d == 2) r = r / 3.0;
      const double r2 = __shfl_down_sync(0xffffffffu, r, 1);  // division d + 1 of the same group
      if (higgs) {
        if (fl & kGrpHiggsLast) {
          if (d == 0) m.a2 = r;
          if (d == 1) m.a4 = r;
          if (d == 2) m.akin = r;
        }
        if ((fl & kGrpKindLast) && d == 3) {
          if (kind == kHiggsHB) m.acc_hb = r;
          if (kind == kHiggsOR) m.acc_or = r;
        }
      } else if (link) {
        if (fl & kGrpKindLast) {
          if (d == 0) m.plaq = r;
          if (d == 1) m.acc_gauge = r * r2;
        }
      } else if (kind == kLinkOR) {
        if ((fl & kGrpKindLast) && d == 0) m.acc_link_or = r;
      }
    }
    // f/ahiggs1.f:113-123 step adaptation after each ahiggs1 group, in order,
    // in the build's precision
    double delta = SM ? pre[1] : f.cst[c].delta;
    if (f.nmetro) {
      for (int g = 0; g < f.ngroups; ++g) {
        if (!(T.gflags[g] & kGrpMetro)) continue;
        const double h0 = __shfl_sync(0xffffffffu, g < 32 ? hs[0][0] : hs[1][0], g & 31);
        if (f.single) {
          float a = (float)h0 / (float)V, dl = (float)delta;
          if (fabsf(a - 0.5f) > 0.1f) dl = (a > 0.5f) ? 1.1131241f * dl : 0.8989669f * dl;
          if (lane == 0 && (T.gflags[g] & kGrpKindLast)) m.acc_metro = a;
          delta = dl;
        } else {
          const double a = h0 / V;
          double dl = delta;
          if (fabs(a - 0.5) > 0.1) dl = (a > 0.5) ? 1.1131241 * dl : 0.8989669 * dl;
          if (lane == 0 && (T.gflags[g] & kGrpKindLast)) m.acc_metro = a;
          delta = dl;
        }
      }
      if (lane == 0) f.cst[c].delta = delta;
    }
    if (lane == 0) m.delta = delta;
  }
  __syncthreads();
  if (threadIdx.x == 0 && (f.npasses || f.nstream)) {
    if (SM) {
      f.st->pass_ctr = ctr[0] + f.npasses;
      f.st->stream_pos = ctr[1] + f.nstream;
    } else {
      f.st->pass_ctr += f.npasses;
      f.st->stream_pos += f.nstream;
    }
  }
}

// One block for a single chain of at most kSmallChunks chunks, everything
// after the wait in one global round trip: warp w < (nslots - pre) * nch
// sums chunk w % nch of slot pre + w / nch (level 1, to shared memory) while
// the block loads the chunk sums of the slots [0, pre) that the passes
// summed behind; level 2 per slot (lane k holds chunk k, the fixed tree) and
// the combine then read shared memory.  Same additions, same order as the
// two-level kernel below.
constexpr int kFinSmallWarps = 16;
constexpr int kSmallChunks = 8;
struct SmallFinSmem {
  double tot[kMaxSlots * kNQ];
  double ck[kMaxSlots * kSmallChunks * kNQ];  // [slot][chunk][q]
  double pre[2];
  unsigned long long ctr[2];
  FinTables T;
};
// The single-chain finalize, run by one block of any number of warps: the
// finalize_small_kernel block, or the block a sweep's first pass carries for
// the previous sweep (DEFERRED: called after the caller's wait; the RNG
// counters are then left alone when f.npasses and f.nstream are 0).
template <bool DEFERRED>
__device__ __forceinline__ void finalize_small_body(const FinalizeArgs& f, SmallFinSmem& S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (int)(blockDim.x >> 5);
  // the slot tables, and the combine's inputs other than the totals -- the
  // volume, and the ahiggs1 step and the RNG counters, which only an earlier
  // finalize writes (before the wait in the finalize kernel: that finalize
  // completed before this queue's first pass went past its wait)
  load_tables(f, S.T);
  if ((int)threadIdx.x == (int)blockDim.x - 1) {
    S.pre[0] = 2.0 * f.chains[0].nh;
    S.pre[1] = f.cst[0].delta;
    S.ctr[0] = f.st->pass_ctr;
    S.ctr[1] = f.st->stream_pos;
  }
  if (!DEFERRED) pdl_wait();
  const int nch = f.nchunks, b1 = f.ntiles0;  // chain 0's chunks and tiles, from the host
  // chunk sums summed behind: one chunk -> the total, else chunks[k][i]
  // (the slots [0, pre) of one chunk are pre * kNQ consecutive doubles)
  if ((int)threadIdx.x < f.pre * kNQ) {
    const int i = threadIdx.x / kNQ, q = threadIdx.x % kNQ;
#pragma unroll
    for (int k = 0; k < kSmallChunks; ++k) {
      if (k < nch)
        S.ck[(i * kSmallChunks + k) * kNQ + q] =
            nch == 1 ? __ldcg(f.totals + threadIdx.x) : __ldcg(f.chunks + (size_t)k * kMaxSlots * kNQ + threadIdx.x);
    }
  }
  // level 1 of the remaining slots
  for (int w = warp; w < (f.nslots - f.pre) * nch; w += nwarps) {
    const int i = f.pre + w / nch, k = w % nch;
    const int t0 = k * kChunkTiles, t1 = min(b1, t0 + kChunkTiles);
    double v[kNQ];
    strided_sum(reinterpret_cast<const double2*>(f.part + (size_t)i * f.slot_stride), 2, t0, t1, v);
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < kNQ; ++q) S.ck[(i * kSmallChunks + k) * kNQ + q] = v[q];
    }
  }
  __syncthreads();
  // level 2: lane k adds chunk k to zero, then the tree (a one-chunk chain's
  // level-1 sum is its total)
  for (int i = warp; i < f.nslots; i += nwarps) {
    double v[kNQ];
#pragma unroll
    for (int q = 0; q < kNQ; ++q)
      v[q] = nch == 1 || lane < nch ? S.ck[(i * kSmallChunks + (nch == 1 ? 0 : lane)) * kNQ + q] : 0.0;
    if (nch > 1) {
#pragma unroll
      for (int q = 0; q < kNQ; ++q) v[q] = 0.0 + v[q];
      warp_tree(v);
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < kNQ; ++q) {
        S.tot[i * kNQ + q] = v[q];
        f.totals[(size_t)i * kNQ + q] = v[q];
      }
    }
  }
  __syncthreads();
  finalize_combine<true>(f, S.T, S.tot, S.pre, S.ctr);
}

__global__ void __launch_bounds__(kFinSmallWarps * 32) finalize_small_kernel(FinalizeArgs f) {
  __shared__ SmallFinSmem S;
  pdl_trigger();
  finalize_small_body<false>(f, S);
}

// The first pass (ahiggs2, eo 0) of a sweep inside a graph of several
// sweeps, with one extra block that runs the previous sweep's finalize (fp):
// its inputs -- the other slots' chunk sums and the last pass's partials --
// are not overwritten before this pass completes (the next pass's
// reduce-behind blocks write slot 0's chunk sums), and the RNG counters are
// not advanced inside such a graph (each sweep's passes take fixed offsets
// from its start; the graph's last finalize advances them), so the finalize
// runs beside this pass's tiles instead of between the sweeps.
template <typename R, int BS>
__global__ void __launch_bounds__(BS, min_blocks_bs<R, BS, 0>())
    higgs_fin_kernel(PassArgs p, const __grid_constant__ FinalizeArgs fp) {
  if ((int)blockIdx.x >= p.ntiles) {
    __shared__ SmallFinSmem S;
    pdl_wait();
    pdl_trigger();
    finalize_small_body<true>(fp, S);
  } else {
    higgs_tile<R, 0, true, 1, BS>(p, blockIdx.x);
  }
}

// kFinWarps warps per block, one level-1 item per warp.  One block: level 2
// and the combine follow in the same block (its own global writes are
// visible to it after the barrier).  Several blocks: the last block to finish
// level 1, by an atomic ticket, does level 2 and the combine.
constexpr int kFinWarps = 32;
__global__ void __launch_bounds__(kFinWarps * 32) finalize_kernel(FinalizeArgs f) {
  __shared__ FinTables T;
  pdl_trigger();
  load_tables(f, T);
  pdl_wait();
  const int warp = (int)(threadIdx.x >> 5);
  const int n1 = f.nchunks * (f.nslots - f.pre);
  for (int w = blockIdx.x * kFinWarps + warp; w < n1; w += gridDim.x * kFinWarps) finalize_chunk_warp(f, w);
  if (gridDim.x > 1) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned int t = atomicAdd(&f.st->ticket, 1u);
      last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
  } else {
    __syncthreads();
  }
  if (f.nchunks > f.nchains) {
    for (int w = warp; w < f.nchains * f.nslots; w += kFinWarps) finalize_chain_warp(f, w);
    __syncthreads();
  }
  finalize_combine(f, T);
  if (gridDim.x > 1 && threadIdx.x == 0) f.st->ticket = 0;
}

// ------------------------------------------------------------------ persistent sweep
// Grid barrier for a cooperative launch (every block resident).  The arrival
// counter only grows: barrier k of a launch waits for count >= base +
// (k+1)*nblocks, where base (the count when the launch began) is stored in
// device memory by block 0 at the end of the previous launch.  Thread 0 of
// each block makes the block's writes visible (acq_rel fence after the block
// barrier), arrives with a non-returning release add, and polls the count
// with acquire loads and a bounded number of short sleeps.  On timeout the
// block records the status bit and the kernel returns instead of spinning on.
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_sync(GridBar* bar, unsigned nblocks, unsigned& target, unsigned* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    fence_acq_rel_gpu();
    red_release_add(&bar->count, 1u);
    target += nblocks;
    unsigned spins = 0;
    while ((int)(ld_acquire(&bar->count) - target) < 0) {
      if (++spins > kBarrierSpinLimit) {
        ok = 0;
        atomicOr(status, kStatusBarrierTimeout);
        break;
      }
      __nanosleep(20);
    }
    fence_acq_rel_gpu();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <typename R>
__device__ __forceinline__ void persistent_pass(const PersistArgs& a, const PassArgs& p, const PlanEntry& e) {
  const int nt = a.ntiles;
  switch (e.kind) {
    case kHiggsHB:
      for (int t = blockIdx.x; t < nt; t += gridDim.x) higgs_tile<R, 0, false>(p, t);
      break;
    case kHiggsOR:
      for (int t = blockIdx.x; t < nt; t += gridDim.x) higgs_tile<R, 1, false>(p, t);
      break;
    case kHiggsMetro:
      for (int t = blockIdx.x; t < nt; t += gridDim.x) higgs_tile<R, 2, false>(p, t);
      break;
    case kLinkHB:
      if (e.mu == 0) for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 0, 0, false>(p, t);
      else if (e.mu == 1) for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 1, 0, false>(p, t);
      else for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 2, 0, false>(p, t);
      break;
    case kLinkHB3:
      if (e.mu == 0) for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 0, 0, false, 3>(p, t);
      else if (e.mu == 1) for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 1, 0, false, 3>(p, t);
      else for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 2, 0, false, 3>(p, t);
      break;
    default:
      if (e.mu == 0) for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 0, 1, false>(p, t);
      else if (e.mu == 1) for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 1, 1, false>(p, t);
      else for (int t = blockIdx.x; t < nt; t += gridDim.x) link_tile<R, 2, 1, false>(p, t);
      break;
  }
}

// One sweep: every pass over the (chain, tile) work list, a grid barrier
// between passes, then the finalize reduction -- a single cooperative launch.
template <typename R>
__global__ void __launch_bounds__(kBlock, kPersistMinBlocks) sweep_persistent_kernel(PersistArgs a) {
  // only thread 0 of each block tracks the barrier target
  unsigned target = 0;
  if (threadIdx.x == 0) target = *(volatile unsigned*)&a.bar->base;
  PassArgs p = a.base;
  for (int i = 0; i < a.npasses; ++i) {
    const PlanEntry e = a.plan[i];
    p.eo = e.eo;
    p.pass_off = a.pass_off[i];
    p.stream_off = a.stream_off[i];
    p.part = e.slot == kNoSlot ? nullptr : const_cast<double*>(a.fin.part) + (size_t)e.slot * a.fin.slot_stride;
    persistent_pass<R>(a, p, e);
    if (!grid_sync(a.bar, gridDim.x, target, &a.base.st->status)) return;
  }
  {
    const int nw = (int)(blockDim.x >> 5), w0 = blockIdx.x * nw + (int)(threadIdx.x >> 5);
    for (int w = w0; w < a.fin.nchunks * a.fin.nslots; w += gridDim.x * nw) finalize_chunk_warp(a.fin, w);
    if (!grid_sync(a.bar, gridDim.x, target, &a.base.st->status)) return;
    if (a.fin.nchunks > a.fin.nchains)
      for (int w = w0; w < a.fin.nchains * a.fin.nslots; w += gridDim.x * nw) finalize_chain_warp(a.fin, w);
  }
  if (!grid_sync(a.bar, gridDim.x, target, &a.base.st->status)) return;
  if (blockIdx.x == 0) {
    __shared__ FinTables T;
    load_tables(a.fin, T);
    __syncthreads();
    finalize_combine(a.fin, T);
    // every block has passed the last barrier: record where the count stands
    if (threadIdx.x == 0) *(volatile unsigned*)&a.bar->base = target;
  }
}

// ------------------------------------------------------------------ renorm
// f/renorm.f:24-34, in FP64 arithmetic for FP32 links
template <typename R>
__global__ void renorm_kernel(void* u, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    LinkIO<R>::st(u, i, unitarise64(LinkIO<R>::ld_cg(u, i)));
}

// ------------------------------------------------------------------ debug
template <typename R, int MU>
__global__ void debug_staple_kernel(const ChainDev* chp, int eo, double* out) {
  const ChainDev& ch = *chp;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ch.nh) return;
  Coord X = site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  su2<R> V = staple<R, MU>(ch, eo, nbr_offsets(ch, X), s);
  out[(size_t)s * 4 + 0] = V.a.re;
  out[(size_t)s * 4 + 1] = V.a.im;
  out[(size_t)s * 4 + 2] = V.b.re;
  out[(size_t)s * 4 + 3] = V.b.im;
}

template <typename R>
__global__ void debug_force_kernel(const ChainDev* chp, int eo, double* out) {
  const ChainDev& ch = *chp;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ch.nh) return;
  Coord X = site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  R f1, f2, f3;
  higgs_force<R>(ch, eo, nbr_offsets(ch, X), s, f1, f2, f3);
  out[(size_t)s * 3 + 0] = f1;
  out[(size_t)s * 3 + 1] = f2;
  out[(size_t)s * 3 + 2] = f3;
}

// ------------------------------------------------------------------ launchers
// The pass kernels and the finalize kernel are launched with programmatic
// dependent launch (lce_common.cuh: launch_pdl / pdl_wait).
template <typename R, int SPT, int BS, int OCC = 0>
void launch_higgs_t(int mode, const PassArgs& a, int nblocks, cudaStream_t s) {
  void (*k)(PassArgs) = mode == 0 ? higgs_kernel<R, 0, SPT, BS, OCC>
                                  : (mode == 1 ? higgs_kernel<R, 1, SPT, BS, OCC> : higgs_kernel<R, 2, SPT, BS, OCC>);
  (void)launch_pdl(k, nblocks, BS, 0, s, a);
}

template <typename R, int SPT, int BS, int OCC = 0>
void launch_link_t(int mode, int mu, const PassArgs& a, int nblocks, cudaStream_t s) {
  void (*k)(PassArgs);
  if (mode == 0)
    k = mu == 0 ? link_kernel<R, 0, 0, SPT, BS, OCC>
                : (mu == 1 ? link_kernel<R, 1, 0, SPT, BS, OCC> : link_kernel<R, 2, 0, SPT, BS, OCC>);
  else if (mode == 1)
    k = mu == 0 ? link_kernel<R, 0, 1, SPT, BS, OCC>
                : (mu == 1 ? link_kernel<R, 1, 1, SPT, BS, OCC> : link_kernel<R, 2, 1, SPT, BS, OCC>);
  else
    k = mu == 0 ? link3_kernel<R, 0, SPT, BS, OCC>
                : (mu == 1 ? link3_kernel<R, 1, SPT, BS, OCC> : link3_kernel<R, 2, SPT, BS, OCC>);
  (void)launch_pdl(k, nblocks, BS, 0, s, a);
}

// Tile shapes compiled: FP32 (BS, SPT) in {128, 256, 512} x {1} and
// {128, 256} x {2} at the 64-register cap, (448, 1) at two blocks per SM (72
// registers), and (128, 1) at 56 registers (a.occ = 1152); the FP64
// validation path only BS = 256.
template <typename R>
void launch_higgs(int mode, const PassArgs& a, int nblocks, cudaStream_t s) {
  if constexpr (sizeof(R) == 4) {
    if (a.bs == 128 && a.occ == 1152) {
      launch_higgs_t<R, 1, 128, 1152>(mode, a, nblocks, s);
      return;
    }
    if (a.bs == 128) {
      if (a.spt == 2) launch_higgs_t<R, 2, 128>(mode, a, nblocks, s);
      else launch_higgs_t<R, 1, 128>(mode, a, nblocks, s);
      return;
    }
    if (a.bs == 512) {
      launch_higgs_t<R, 1, 512>(mode, a, nblocks, s);
      return;
    }
    if (a.bs == 448) {
      launch_higgs_t<R, 1, 448>(mode, a, nblocks, s);
      return;
    }
  }
  if (a.spt == 2) launch_higgs_t<R, 2, 256>(mode, a, nblocks, s);
  else launch_higgs_t<R, 1, 256>(mode, a, nblocks, s);
}

template <typename R>
void launch_link(int mode, int mu, const PassArgs& a, int nblocks, cudaStream_t s) {
  if constexpr (sizeof(R) == 4) {
    if (a.bs == 128 && a.occ == 1152) {
      launch_link_t<R, 1, 128, 1152>(mode, mu, a, nblocks, s);
      return;
    }
    if (a.bs == 128) {
      if (a.spt == 2) launch_link_t<R, 2, 128>(mode, mu, a, nblocks, s);
      else launch_link_t<R, 1, 128>(mode, mu, a, nblocks, s);
      return;
    }
    if (a.bs == 512) {
      launch_link_t<R, 1, 512>(mode, mu, a, nblocks, s);
      return;
    }
    if (a.bs == 448) {
      launch_link_t<R, 1, 448>(mode, mu, a, nblocks, s);
      return;
    }
  }
  if (a.spt == 2) launch_link_t<R, 2, 256>(mode, mu, a, nblocks, s);
  else launch_link_t<R, 1, 256>(mode, mu, a, nblocks, s);
}

// the first pass of a sweep carrying the previous sweep's finalize (one site
// per thread, 128 (64 registers), 256, 448 or 512 threads in FP32; 256 in FP64)
template <typename R>
void launch_higgs_fin(const PassArgs& a, const FinalizeArgs& fp, int nblocks, cudaStream_t s) {
  if constexpr (sizeof(R) == 4) {
    if (a.bs == 128) {
      (void)launch_pdl(higgs_fin_kernel<R, 128>, nblocks, 128, 0, s, a, fp);
      return;
    }
    if (a.bs == 448) {
      (void)launch_pdl(higgs_fin_kernel<R, 448>, nblocks, 448, 0, s, a, fp);
      return;
    }
    if (a.bs == 512) {
      (void)launch_pdl(higgs_fin_kernel<R, 512>, nblocks, 512, 0, s, a, fp);
      return;
    }
  }
  (void)launch_pdl(higgs_fin_kernel<R, 256>, nblocks, 256, 0, s, a, fp);
}
template void launch_higgs_fin<float>(const PassArgs&, const FinalizeArgs&, int, cudaStream_t);
template void launch_higgs_fin<double>(const PassArgs&, const FinalizeArgs&, int, cudaStream_t);

void launch_finalize(const FinalizeArgs& f, cudaStream_t s) {
  if (f.nchains == 1 && f.nchunks <= kSmallChunks) {
    (void)launch_pdl(finalize_small_kernel, 1, kFinSmallWarps * 32, 0, s, f);
    return;
  }
  // one block for up to four level-1 items per warp (no ticket); beyond
  // that one item per warp, all loads in flight at once
  const int n1 = f.nchunks * f.nslots;
  int grid = n1 <= 4 * kFinWarps ? 1 : (n1 + kFinWarps - 1) / kFinWarps;
  if (grid < 1) grid = 1;
  (void)launch_pdl(finalize_kernel, grid, kFinWarps * 32, 0, s, f);
}

template <typename R>
int persistent_grid() {
  int dev = 0, nsm = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sweep_persistent_kernel<R>, kBlock, 0) != cudaSuccess)
    return 0;
  return per * nsm;
}

template <typename R>
cudaError_t launch_persistent(const PersistArgs& a, int grid, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = kBlock;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, sweep_persistent_kernel<R>, a);
}

template <typename R>
void launch_renorm(void* u, size_t nlinks, cudaStream_t s) {
  int grid = (int)std::min<size_t>((nlinks + 255) / 256, 148 * 16);
  renorm_kernel<R><<<grid, 256, 0, s>>>(u, nlinks);
}

template <typename R>
void launch_debug_staple(const ChainDev* ch, int eo, int mu, double* out, int nh, cudaStream_t s) {
  int grid = ceil_div(nh, 128);
  if (mu == 0) debug_staple_kernel<R, 0><<<grid, 128, 0, s>>>(ch, eo, out);
  else if (mu == 1) debug_staple_kernel<R, 1><<<grid, 128, 0, s>>>(ch, eo, out);
  else debug_staple_kernel<R, 2><<<grid, 128, 0, s>>>(ch, eo, out);
}

template <typename R>
void launch_debug_force(const ChainDev* ch, int eo, double* out, int nh, cudaStream_t s) {
  debug_force_kernel<R><<<ceil_div(nh, 128), 128, 0, s>>>(ch, eo, out);
}

#define LCE_INST(R)                                                                          \
  template void launch_higgs<R>(int, const PassArgs&, int, cudaStream_t);                  \
  template void launch_link<R>(int, int, const PassArgs&, int, cudaStream_t);              \
  template int persistent_grid<R>();                                                         \
  template cudaError_t launch_persistent<R>(const PersistArgs&, int, cudaStream_t);          \
  template void launch_renorm<R>(void*, size_t, cudaStream_t);                             \
  template void launch_debug_staple<R>(const ChainDev*, int, int, double*, int, cudaStream_t); \
  template void launch_debug_force<R>(const ChainDev*, int, double*, int, cudaStream_t);
LCE_INST(float)
LCE_INST(double)
#undef LCE_INST

}  // namespace lce
