// lce_fourier.cu -- Fourier-accelerated Landau gauge fixing (no reference
// counterpart; the reference iterates f/or_gauge_fixing1.f only).
//
// The overrelaxed iteration relaxes a gauge mode of lattice momentum p at a
// rate ~ p^2, so its iteration count grows like L^2 (L with overrelaxation)
// and is set by the longest wavelengths.  A Fourier-accelerated step
// (Davies et al., Phys. Rev. D 37 (1988) 1581) rotates every site by the
// divergence of the gauge field preconditioned with the inverse lattice
// Laplacian, so that all modes relax at a similar rate:
//
//   Delta(x)  = sum_mu c_mu [u_mu(x) - u_mu(x-mu)]   (vector parts, c = 1,1,alpha)
//   omega     = gamma F^-1[ F[Delta](p) / p_c^2 ],  p_c^2 = sum_mu c_mu 4 sin^2(p_mu/2)
//   g(x)      = exp(-i omega(x).sigma),   U_f(x,mu) -> g(x) U_f(x,mu) g(x+mu)^+
//
// Near the Landau gauge (links ~ 1) the divergence responds to omega as
// Delta -> Delta - (-laplacian_c) omega, so gamma = 1 is a Newton step for
// every mode at once; far from it (a random gauge) the same bounded step
// still raises the functional.  theta is the same quantity as in the
// overrelaxed iteration (odd sites, FP64), so both methods stop on one
// criterion.
//
// One iteration is seven kernels, captured in CUDA graphs like the plain
// iteration: (1) Delta on x-lines + forward FFT along x, with FP64 partials of
// theta; (2) the check (sum, count, done flag);
// (3) forward FFT along y; (4) forward FFT along z, scale, inverse FFT along
// z; (5) inverse FFT along y; (6) inverse FFT along x + build g; (7) apply g to
// U_f, A_f and the tracked transform G.  The FFTs are radix-2 in shared
// memory over a block of lines (1024 complex points per block; lines padded
// by one element against bank conflicts; radix-4 levels); extents must be
// powers of two up to 1024.  The divergence, g and its application to the fields are FP64 for
// either field precision (rounding the step's rotation to FP32 before
// applying it slowed the iteration below theta ~ 1e-8 at 64^3); the
// transforms themselves are FP32.  Two complex fields carry the three components:
// (Delta_b) and (Delta_a3 + 0i); the multiplier is real and even in p, so the
// inverse transform returns each component in its own slot.
#include <algorithm>

#include "lce_internal.hpp"

namespace lce {
namespace {

constexpr int kFaThreads = 256;
// complex type of the transforms: FP32 (timed on the B200: the same iteration
// counts as FP64 transforms at 64^3-256^3, 20-30% less time per iteration)
using FftR = float;
using FftC = float2;
// complex points per block and field, and the padded shared-memory size
constexpr int kFaPoints = 1024;
constexpr int kFaLogPoints = 10;
static_assert(1 << kFaLogPoints == kFaPoints, "points per block");
constexpr int kFaSmem = kFaPoints + kFaPoints / 2;

template <typename T>
__device__ __forceinline__ T cadd(T a, T b) { return T{a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ T csub(T a, T b) { return T{a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ T cmul(T a, T b) { return T{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }

__device__ __forceinline__ double sinpi_r(double x) { return sinpi(x); }

// tw[k] = exp(sign 2 pi i k / n), k < n/2, from the table tg[k] = exp(-2 pi i k / kFaPoints)
__device__ __forceinline__ void load_twiddles(FftC* tw, const double2* tg, int n, int sign) {
  const int stride = kFaPoints / n;
  for (int k = threadIdx.x; k < n / 2; k += blockDim.x) {
    const double2 t = __ldg(tg + k * stride);
    tw[k] = FftC{(FftR)t.x, (FftR)(sign > 0 ? -t.y : t.y)};
  }
}

// In-place decimation-in-time FFT of nl lines of length n = 2^logn held in
// shared memory at d[j*(n+1) + k], input in bit-reversed order, output
// natural.  Levels are fused in pairs (radix 4: two radix-2 levels per item,
// in registers) after one radix-2 level when logn is odd; tw[k] = exp(sign 2
// pi i k / n), k < n/2.  Ends with __syncthreads.
template <typename T>
__device__ __forceinline__ void fft_lines(T* d, int nl, int logn, const T* tw) {
  const int n = 1 << logn, ld = n + 1;
  int st = 0;
  if (logn & 1) {
    // level 0: pairs (2i, 2i+1), twiddle 1
    const int hn = n >> 1, nb = nl * hn;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int p = (b >> (logn - 1)) * ld + 2 * (b & (hn - 1));
      const T u = d[p], v = d[p + 1];
      d[p] = cadd(u, v);
      d[p + 1] = csub(u, v);
    }
    __syncthreads();
    st = 1;
  }
  for (; st < logn; st += 2) {
    // levels st (pairs at distance m) and st + 1 (distance 2m) on groups of 4m
    const int m = 1 << st, q = n >> 2, nb = nl * q;
    const int t1 = n >> (st + 1), t2 = n >> (st + 2);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int r = b & (q - 1), i = r & (m - 1);
      const int base = (b >> (logn - 2)) * ld + (r >> st) * 4 * m + i;
      const T a0 = d[base], a1 = d[base + m], a2 = d[base + 2 * m], a3 = d[base + 3 * m];
      const T w = tw[i * t1];
      const T wa1 = cmul(w, a1), wa3 = cmul(w, a3);
      const T b0 = cadd(a0, wa1), b1 = csub(a0, wa1), b2 = cadd(a2, wa3), b3 = csub(a2, wa3);
      const T x2 = cmul(tw[i * t2], b2), x3 = cmul(tw[(i + m) * t2], b3);
      d[base] = cadd(b0, x2);
      d[base + 2 * m] = csub(b0, x2);
      d[base + m] = cadd(b1, x3);
      d[base + 3 * m] = csub(b1, x3);
    }
    __syncthreads();
  }
}

template <typename R>
__device__ __forceinline__ su2<double> to_d(su2<R> u) {
  return su2<double>{{(double)u.a.re, (double)u.a.im}, {(double)u.b.re, (double)u.b.im}};
}
template <typename R>
__device__ __forceinline__ su2<R> to_r(su2<double> u) {
  return su2<R>{{(R)u.a.re, (R)u.a.im}, {(R)u.b.re, (R)u.b.im}};
}

__device__ __forceinline__ int brev(int k, int logn) { return logn ? (int)(__brev((unsigned)k) >> (32 - logn)) : 0; }

struct FaArgs {
  const ChainDev* ch;
  const ChainState* cst;  // done flag and step; NULL: never done, step gamma
  double gamma;
  void* fft;              // 2 fields x V complex, natural order (x fastest)
  void* gstep;            // g per site, [parity][site], link layout
  double* part;           // [block]: theta (odd sites)
  double* omega_out;      // debug: omega per site [parity][site][3], or NULL
  const double2* tw;      // exp(-2 pi i k / kFaPoints), k < kFaPoints / 2
  int L[3], logL[3];
  int track;
};

__device__ __forceinline__ bool fa_done(const FaArgs& a) { return a.cst && a.cst->gf_done; }

// line l of axis AX and position k along it -> natural index
// (all extents are powers of two: divisions are shifts)
template <int AX>
__device__ __forceinline__ size_t nat_index(const FaArgs& a, int l, int k) {
  const int s1 = a.logL[0], s2 = a.logL[1], m1 = a.L[0] - 1;
  if (AX == 0) return ((size_t)l << s1) + k;                                          // l = y + L2 z
  if (AX == 1) return ((((size_t)(l >> s1) << s2) + k) << s1) + (l & m1);             // l = x + L1 z
  return ((((size_t)k << s2) + (l >> s1)) << s1) + (l & m1);                          // l = x + L1 y
}

// (1) Delta on x-lines, forward FFT along x; partials of theta
template <typename R>
__global__ void __launch_bounds__(kFaThreads) fa_div_kernel(FaArgs a) {
  using T = FftC;
  __shared__ T sm[2][kFaSmem];
  __shared__ T tw[kFaPoints / 2];
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int n = a.L[0], logn = a.logL[0], ld = n + 1;
  const int nl = kFaPoints >> logn, nlines = a.L[1] * a.L[2];
  const int l0 = blockIdx.x * nl;
  load_twiddles(tw, a.tw, n, -1);
  const double al = ch.alpha;
  double q[1] = {0.0};
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int j = e >> logn, x = e & (n - 1), l = l0 + j;
    T v0{0, 0}, v1{0, 0};
    if (l < nlines) {
      const int y = l & (a.L[1] - 1), z = l >> a.logL[1];
      const int p = (x + y + z) & 1, op = 1 - p;
      const int s = site_index(x, y, z, ch.hx, ch.nxy);
      const int xm[3] = {site_index(wrap(x - 1, ch.L1), y, z, ch.hx, ch.nxy),
                         site_index(x, wrap(y - 1, ch.L2), z, ch.hx, ch.nxy),
                         site_index(x, y, wrap(z - 1, ch.L3), ch.hx, ch.nxy)};
      double d3 = 0.0, dbr = 0.0, dbi = 0.0;
#pragma unroll
      for (int mu = 0; mu < 3; ++mu) {
        const double c = mu == 2 ? al : 1.0;
        const su2<R> u = LinkIO<R>::ld_cg(ch.uf, ((size_t)(mu * 2 + p)) * ch.nh + s);
        const su2<R> w = LinkIO<R>::ld_cg(ch.uf, ((size_t)(mu * 2 + op)) * ch.nh + xm[mu]);
        d3 += c * ((double)u.a.im - (double)w.a.im);
        dbr += c * ((double)u.b.re - (double)w.b.re);
        dbi += c * ((double)u.b.im - (double)w.b.im);
      }
      if (p == 1) q[0] += d3 * d3 + dbr * dbr + dbi * dbi;
      v0 = T{(FftR)dbr, (FftR)dbi};
      v1 = T{(FftR)d3, (FftR)0};
    }
    const int pos = j * ld + brev(x, logn);
    sm[0][pos] = v0;
    sm[1][pos] = v1;
  }
  block_reduce_store<1>(q, a.part + blockIdx.x);
  __syncthreads();
  fft_lines<T>(sm[0], nl, logn, tw);
  fft_lines<T>(sm[1], nl, logn, tw);
  const size_t V = (size_t)a.L[0] * a.L[1] * a.L[2];
  T* F = reinterpret_cast<T*>(a.fft);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int j = e >> logn, k = e & (n - 1), l = l0 + j;
    if (l >= nlines) continue;
    const size_t gi = nat_index<0>(a, l, k);
    F[gi] = sm[0][j * ld + k];
    F[V + gi] = sm[1][j * ld + k];
  }
}

// (2) theta = sum / nh (odd sites); count; done flag at theta <= gf_limit or
// the cap
__global__ void __launch_bounds__(1024) fa_check_kernel(const ChainDev* chp, ChainState* cst, const double* part,
                                                        int nblocks) {
  if (cst->gf_done) return;
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v[0] += part[b];
  __shared__ double tot[1];
  block_reduce_store<1>(v, tot);
  __syncthreads();
  if (threadIdx.x == 0) {
    const double theta = tot[0] / chp->nh;
    const int it = cst->gf_iters + 1;
    // a step that doubled theta overshot (far from the Landau gauge the
    // linearised step can be too long): shorten it for the rest of the run
    if (it > 1 && theta > 2.0 * cst->gf_theta) cst->gf_step = fmax(0.1, 0.7 * cst->gf_step);
    cst->gf_iters = it;
    cst->gf_theta = theta;
    if (!(theta > cst->gf_limit) || (cst->gf_cap > 0 && it >= cst->gf_cap)) cst->gf_done = 1;
  }
}

// (3)-(5) FFT of both fields along axis AX (1: y, 2: z); for AX = 2 with
// SCALE: forward, multiply by gamma / (p_c^2 V), inverse
template <typename R, int AX, int SIGN, bool SCALE>
__global__ void __launch_bounds__(kFaThreads) fa_fft_kernel(FaArgs a) {
  using T = FftC;
  __shared__ T sm[kFaSmem];
  __shared__ T tw[kFaPoints / 2];
  __shared__ T twi[SCALE ? kFaPoints / 2 : 1];
  if (fa_done(a)) return;
  const int n = a.L[AX], logn = a.logL[AX], ld = n + 1;
  const int lnl = kFaLogPoints - logn, nl = 1 << lnl;
  const int nlines = (a.L[0] * a.L[1] * a.L[2]) >> logn;
  const int l0 = blockIdx.x * nl;
  const int fld = blockIdx.y;
  const size_t V = (size_t)a.L[0] * a.L[1] * a.L[2];
  T* F = reinterpret_cast<T*>(a.fft) + fld * V;
  __shared__ double sz2[SCALE ? kFaPoints : 1];  // alpha sin^2(pi kz / L3)
  __shared__ double sxy[SCALE ? kFaPoints : 1];  // sin^2(pi kx / L1) + sin^2(pi ky / L2) per line
  load_twiddles(tw, a.tw, n, SIGN);
  if (SCALE) {
    load_twiddles(twi, a.tw, n, -SIGN);
    const double al = a.ch->alpha;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const double sz = sinpi_r((double)k / a.L[2]);
      sz2[k] = al * sz * sz;
    }
    for (int j = threadIdx.x; j < nl; j += blockDim.x) {
      const int l = l0 + j, kx = l & (a.L[0] - 1), ky = l >> a.logL[0];
      const double sx = sinpi_r((double)kx / a.L[0]), sy = sinpi_r((double)ky / a.L[1]);
      sxy[j] = sx * sx + sy * sy;
    }
  }
  // element e -> (line j = e % nl, position k = e / nl): consecutive threads
  // read consecutive lines, i.e. consecutive x
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int j = e & (nl - 1), k = e >> lnl, l = l0 + j;
    sm[j * ld + brev(k, logn)] = l < nlines ? F[nat_index<AX>(a, l, k)] : T{0, 0};
  }
  __syncthreads();
  fft_lines<T>(sm, nl, logn, tw);
  if (SCALE) {
    const double gv = (a.cst ? a.cst->gf_step : a.gamma) / (4.0 * (double)V);
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int j = e >> logn, kz = e & (n - 1), l = l0 + j;
      const double p2 = sxy[j] + sz2[kz];
      const double m = (l | kz) ? gv / p2 : 0.0;
      const int q = j * ld + kz;
      sm[q] = T{(FftR)(sm[q].x * m), (FftR)(sm[q].y * m)};
    }
    __syncthreads();
    // bit-reverse permutation for the inverse transform
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int j = e >> logn, k = e & (n - 1), r = brev(k, logn);
      if (r > k) {
        const T t = sm[j * ld + k];
        sm[j * ld + k] = sm[j * ld + r];
        sm[j * ld + r] = t;
      }
    }
    __syncthreads();
    fft_lines<T>(sm, nl, logn, twi);
  }
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int j = e & (nl - 1), k = e >> lnl, l = l0 + j;
    if (l < nlines) F[nat_index<AX>(a, l, k)] = sm[j * ld + k];
  }
}

// (6) inverse FFT along x; g(x) = exp(-i omega.sigma) per site
template <typename R>
__global__ void __launch_bounds__(kFaThreads) fa_g_kernel(FaArgs a) {
  using T = FftC;
  __shared__ T sm[2][kFaSmem];
  __shared__ T tw[kFaPoints / 2];
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int n = a.L[0], logn = a.logL[0], ld = n + 1;
  const int nl = kFaPoints >> logn, nlines = a.L[1] * a.L[2];
  const int l0 = blockIdx.x * nl;
  const size_t V = (size_t)a.L[0] * a.L[1] * a.L[2];
  const T* F = reinterpret_cast<const T*>(a.fft);
  load_twiddles(tw, a.tw, n, +1);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int j = e >> logn, k = e & (n - 1), l = l0 + j;
    const size_t gi = l < nlines ? nat_index<0>(a, l, k) : 0;
    sm[0][j * ld + brev(k, logn)] = l < nlines ? F[gi] : T{0, 0};
    sm[1][j * ld + brev(k, logn)] = l < nlines ? F[V + gi] : T{0, 0};
  }
  __syncthreads();
  fft_lines<T>(sm[0], nl, logn, tw);
  fft_lines<T>(sm[1], nl, logn, tw);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    const int j = e >> logn, x = e & (n - 1), l = l0 + j;
    if (l >= nlines) continue;
    const int y = l & (a.L[1] - 1), z = l >> a.logL[1];
    const int p = (x + y + z) & 1, s = site_index(x, y, z, ch.hx, ch.nxy);
    const double w3 = sm[1][j * ld + x].x, wbr = sm[0][j * ld + x].x, wbi = sm[0][j * ld + x].y;
    const double nw = sqrt(w3 * w3 + wbr * wbr + wbi * wbi);
    su2<double> g{{1.0, 0.0}, {0.0, 0.0}};
    if (nw > 0.0) {
      double sn, cs;
      sincos(nw, &sn, &cs);
      const double f = sn / nw;
      g = su2<double>{{cs, -f * w3}, {-f * wbr, -f * wbi}};
    }
    LinkIO<double>::st(a.gstep, (size_t)p * ch.nh + s, g);
    if (a.omega_out) {
      double* o = a.omega_out + ((size_t)p * ch.nh + s) * 3;
      o[0] = (double)w3;
      o[1] = (double)wbr;
      o[2] = (double)wbi;
    }
  }
}

// (7) U_f(x,mu) -> g(x) U_f(x,mu) g(x+mu)^+, A_f -> g A_f g^+, G -> g G
template <typename R>
__global__ void __launch_bounds__(kBlock) fa_apply_kernel(FaArgs a) {
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= 2 * ch.nh) return;
  const int eo = i >= ch.nh ? 1 : 0, oe = 1 - eo, s = i - eo * ch.nh, nh = ch.nh;
  const Coord X = site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
  const su2<double> gx = LinkIO<double>::ld_cg(a.gstep, (size_t)eo * nh + s);
  const int L[3] = {ch.L1, ch.L2, ch.L3};
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    int c[3] = {X.x, X.y, X.z};
    c[mu] = wrap(c[mu] + 1, L[mu]);
    const int sp = site_index(c[0], c[1], c[2], ch.hx, ch.nxy);
    const su2<double> gp = LinkIO<double>::ld_cg(a.gstep, (size_t)oe * nh + sp);
    const size_t li = ((size_t)(mu * 2 + eo)) * nh + s;
    LinkIO<R>::st(ch.uf, li, to_r<R>(unitarise64(nd(nn(gx, to_d(LinkIO<R>::ld_cg(ch.uf, li))), gp))));
  }
  R* Af = reinterpret_cast<R*>(ch.af);
  const su2<double> t =
      nn(gx, ad((double)__ldcg(Af + ((size_t)(eo * 3 + 0)) * nh + s), (double)__ldcg(Af + ((size_t)(eo * 3 + 1)) * nh + s),
                (double)__ldcg(Af + ((size_t)(eo * 3 + 2)) * nh + s), gx));
  Af[((size_t)(eo * 3 + 0)) * nh + s] = (R)t.b.im;
  Af[((size_t)(eo * 3 + 1)) * nh + s] = (R)t.b.re;
  Af[((size_t)(eo * 3 + 2)) * nh + s] = (R)t.a.im;
  if (a.track) {
    const size_t gi = (size_t)eo * nh + s;
    LinkIO<R>::st(ch.g, gi, to_r<R>(unitarise64(nn(gx, to_d(LinkIO<R>::ld_cg(ch.g, gi))))));
  }
}

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return (1 << l) == n ? l : -1;
}

}  // namespace

bool fa_supported(const ChainDev& ch) {
  const int L[3] = {ch.L1, ch.L2, ch.L3};
  for (int d = 0; d < 3; ++d) {
    const int lg = ilog2_exact(L[d]);
    if (lg < 1 || L[d] > kFaPoints) return false;
  }
  return true;
}

// two FP64 complex fields and the FP64 step transform
// Buffer layout for chains of up to vcap sites: two FP64 complex fields,
// the FP64 step transform and the twiddle table (fixed offsets, so graphs
// captured for one chain stay valid while others use the same buffer)
size_t fa_buffer_bytes(size_t vcap) {
  return 2 * vcap * sizeof(FftC) + vcap * 32 + kFaPoints / 2 * sizeof(double2) + 256;
}
namespace {
void* fa_gstep(void* buf, size_t vcap) { return reinterpret_cast<char*>(buf) + 2 * vcap * sizeof(FftC); }
double2* fa_table(void* buf, size_t vcap) {
  return reinterpret_cast<double2*>(reinterpret_cast<char*>(buf) + 2 * vcap * sizeof(FftC) + vcap * 32);
}
}  // namespace

namespace {
__global__ void fa_twiddle_table_kernel(double2* tg) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kFaPoints / 2) return;
  double s, c;
  sincospi((double)(2 * k) / kFaPoints, &s, &c);
  tg[k] = double2{c, -s};
}
}  // namespace

void fa_init_table(void* buf, size_t vcap, cudaStream_t s) {
  fa_twiddle_table_kernel<<<1, kFaPoints / 2, 0, s>>>(fa_table(buf, vcap));
}

template <typename R>
int fa_blocks_div(const ChainDev& ch) { return ceil_div((long)ch.L2 * ch.L3, kFaPoints / ch.L1); }

// enqueue one Fourier-accelerated iteration (kernels 1-7)
template <typename R>
void launch_fa_iteration(const ChainDev* chd, const ChainDev& ch, ChainState* cst, double gamma, void* buf,
                         size_t vcap, double* part, double* omega_out, int track, bool with_check, bool with_apply,
                         cudaStream_t s) {
  FaArgs a;
  a.ch = chd;
  a.cst = cst;
  a.gamma = gamma;
  a.fft = buf;
  const size_t V = 2 * (size_t)ch.nh;
  a.gstep = fa_gstep(buf, vcap);
  a.part = part;
  a.omega_out = omega_out;
  a.tw = fa_table(buf, vcap);
  a.L[0] = ch.L1;
  a.L[1] = ch.L2;
  a.L[2] = ch.L3;
  for (int d = 0; d < 3; ++d) a.logL[d] = ilog2_exact(a.L[d]);
  a.track = track;
  const int nbd = fa_blocks_div<R>(ch);
  fa_div_kernel<R><<<nbd, kFaThreads, 0, s>>>(a);
  if (with_check) fa_check_kernel<<<1, 1024, 0, s>>>(chd, cst, part, nbd);
  constexpr int P = kFaPoints;
  const dim3 gy(ceil_div((long)V / ch.L2, P / ch.L2), 2), gz(ceil_div((long)V / ch.L3, P / ch.L3), 2);
  fa_fft_kernel<R, 1, -1, false><<<gy, kFaThreads, 0, s>>>(a);
  fa_fft_kernel<R, 2, -1, true><<<gz, kFaThreads, 0, s>>>(a);
  fa_fft_kernel<R, 1, +1, false><<<gy, kFaThreads, 0, s>>>(a);
  fa_g_kernel<R><<<nbd, kFaThreads, 0, s>>>(a);
  if (with_apply) fa_apply_kernel<R><<<ceil_div((long)V, kBlock), kBlock, 0, s>>>(a);
}

template void launch_fa_iteration<float>(const ChainDev*, const ChainDev&, ChainState*, double, void*, size_t,
                                         double*, double*, int, bool, bool, cudaStream_t);
template void launch_fa_iteration<double>(const ChainDev*, const ChainDev&, ChainState*, double, void*, size_t,
                                          double*, double*, int, bool, bool, cudaStream_t);

}  // namespace lce
