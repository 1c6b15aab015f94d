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
// U_f, A_f and the tracked transform G.  A block transforms 4096 complex
// points (lines of one axis, one or both fields) held in shared memory.  A
// line of n = N1 x N2 points is transformed in two steps: N2 threads each
// take N1 points of stride N2 into registers, do an N1-point DFT there
// (radix-2 butterflies, fully unrolled), multiply by the twiddles
// W_n^(n2 k1) and store a row; then N1 threads each take a row of N2 points,
// do the N2-point DFT and store the results in natural order (N1, N2 <= 32).
// Both steps read into registers before writing, so the two layouts share
// the buffer.  Threads walk the lines fastest, and the padded line stride
// keeps the shared-memory accesses free of bank conflicts.  Extents must be
// powers of two up to 1024.  The divergence, g and its application to the
// fields are FP64 for either field precision (rounding the step's rotation to FP32 before
// applying it slowed the iteration below theta ~ 1e-8 at 64^3); the
// transforms themselves are FP32.  Two complex fields carry the three components:
// (Delta_b) and (Delta_a3 + 0i); the multiplier is real and even in p, so the
// inverse transform returns each component in its own slot.
//
// Conjugate-gradient form (nonlinear CG on the gauge functional with the same
// Fourier preconditioner, after Hudspith, Comput. Phys. Commun. 187 (2015)
// 115): the preconditioned gradient g_k = F^-1[F[Delta_k] / p_c^2] enters a
// direction s_k = g_k + beta_k s_(k-1), beta_k = max(0, Polak-Ribiere) with
// its inner products sum_x Delta_k.g_k and sum_x Delta_k.g_(k-1) taken in
// momentum space (Parseval: sum_p |F_k|^2 / p_c^2 and
// sum_p Re(F_k^* F_(k-1)) / p_c^2, the previous F kept), and the step along
// s_k maximises the second-order expansion of the functional
// F(alpha) = sum_(x,mu) c_mu Re a[g_a(x) U(x,mu) g_a(x+mu)^+], g_a = exp(alpha X),
// X = -i s.sigma: with Y = X(x+mu),
//   F'(0)  = sum c_mu Re a[X U - U Y]
//   F''(0) = sum c_mu Re a[X^2 U + U Y^2 - 2 X U Y],
// alpha = F'(0) / -F''(0) (exact per link to second order).  Four more
// kernels per iteration: the beta reduction, the line derivatives, the alpha
// reduction and g = exp(alpha X) per site.  The step is bounded by a trust
// region (fa_alpha_kernel).
#include <algorithm>
#include <cstring>

#include <string>

#include "lce_internal.hpp"

namespace lce {
namespace {

constexpr int kFaThreads = 256;
// complex type of the transforms: FP32 (timed on the B200: the same iteration
// counts as FP64 transforms at 64^3-256^3, 20-30% less time per iteration)
using FftR = float;
using FftC = float2;
// longest line (and size of the twiddle table exp(-2 pi i k / kFaPoints))
constexpr int kFaPoints = 1024;
// complex points transformed per block (all fields), 2^kFaBlockLog
constexpr int kFaBlockLog = 12;
constexpr int kFaBlockPts = 1 << kFaBlockLog;

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

// n = 2^LOGN = N1 x N2, N1 points per thread in the first step
template <int LOGN>
struct FaLines {
  static constexpr int n = 1 << LOGN;
  static constexpr int N1 = LOGN <= 4 ? n : (LOGN <= 8 ? 16 : 32);
  static constexpr int N2 = n / N1;
  static constexpr int NLT = kFaBlockPts >> LOGN;               // lines per block (all fields)
  // line stride: a line in natural order, or (between the two steps) N1 rows
  // of N2 points, each row padded by one; n + N1 + 1 = 2 mod 32 words apart
  static constexpr int ld = N2 > 1 ? N1 * (N2 + 1) + 1 : n + 1;
  static constexpr int ntw = n / 2 > 0 ? n / 2 : 1;              // twiddle table entries
  // lines, ntab twiddle tables and nd doubles
  static constexpr size_t smem(int ntab, int nd) {
    return ((size_t)NLT * ld + (size_t)ntab * ntw) * sizeof(FftC) + (size_t)nd * sizeof(double);
  }
};

__host__ __device__ constexpr int cbrev(int k, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r = (r << 1) | ((k >> i) & 1);
  return r;
}
template <int N>
struct ILog2 {
  static constexpr int v = 1 + ILog2<N / 2>::v;
};
template <>
struct ILog2<1> {
  static constexpr int v = 0;
};

// radix-2 stages S, S+1, ... of an N-point decimation-in-time DFT in
// registers; one loop of constant trip count per stage, so that every index
// is a compile-time constant after unrolling.  tw[k] = exp(sign 2 pi i k / n),
// k < n/2: W_2m^j = tw[j n / 2m].
template <int N, int n, int S>
__device__ __forceinline__ void dft_stages(FftC (&t)[N], const FftC* tw) {
  if constexpr ((1 << S) < N) {
    constexpr int m = 1 << S;
#pragma unroll
    for (int b = 0; b < N / 2; ++b) {
      const int j = b % m, k = (b / m) * 2 * m;
      FftC u = t[k + j + m];
      if (j > 0) u = cmul(tw[j * (n / (2 * m))], u);
      t[k + j + m] = csub(t[k + j], u);
      t[k + j] = cadd(t[k + j], u);
    }
    dft_stages<N, n, S + 1>(t, tw);
  }
}

// N-point DFT in registers, natural order in and out (decimation in time on
// the bit-reversed copy)
template <int N, int n>
__device__ __forceinline__ void dft_reg(FftC (&v)[N], const FftC* tw) {
  constexpr int LG = ILog2<N>::v;
  FftC t[N];
#pragma unroll
  for (int i = 0; i < N; ++i) t[cbrev(i, LG)] = v[i];
  dft_stages<N, n, 0>(t, tw);
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = t[i];
}

// In-place FFT of the block's NLT lines at d[j*ld + x] (natural order in and
// out).  Each step reads its items into registers, transforms them, waits for
// the block and writes back, so the two layouts share one buffer.  Ends with
// __syncthreads.
template <int LOGN>
__device__ __forceinline__ void fft2_lines(FftC* d, const FftC* tw) {
  using G = FaLines<LOGN>;
  constexpr int n = G::n, N1 = G::N1, N2 = G::N2, NLT = G::NLT, ld = G::ld;
  if constexpr (N2 == 1) {
    // one thread per line
    for (int j = threadIdx.x; j < NLT; j += blockDim.x) {
      FftC v[N1];
#pragma unroll
      for (int i = 0; i < N1; ++i) v[i] = d[j * ld + i];
      dft_reg<N1, n>(v, tw);
#pragma unroll
      for (int k = 0; k < N1; ++k) d[j * ld + k] = v[k];
    }
  } else {
    // items per thread of the two steps
    constexpr int IA = (NLT * N2 + kFaThreads - 1) / kFaThreads;
    constexpr int IB = (NLT * N1 + kFaThreads - 1) / kFaThreads;
    // step 1: item (line j, column n2), lines fastest: N1 points of stride N2,
    // DFT, twiddles W_n^(n2 k1); stored as row k1, column n2
    FftC r[IA][N1];
#pragma unroll
    for (int q = 0; q < IA; ++q) {
      const int it = threadIdx.x + q * kFaThreads;
      if (it < NLT * N2) {
        const int j = it % NLT, n2 = it / NLT;
#pragma unroll
        for (int i = 0; i < N1; ++i) r[q][i] = d[j * ld + i * N2 + n2];
        dft_reg<N1, n>(r[q], tw);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) {
          const int e = n2 * k1;  // < n; W_n^e = -W_n^(e - n/2) for e >= n/2
          const FftC w = e < n / 2 ? tw[e] : FftC{-tw[e - n / 2].x, -tw[e - n / 2].y};
          r[q][k1] = cmul(w, r[q][k1]);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < IA; ++q) {
      const int it = threadIdx.x + q * kFaThreads;
      if (it < NLT * N2) {
        const int j = it % NLT, n2 = it / NLT;
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) d[j * ld + k1 * (N2 + 1) + n2] = r[q][k1];
      }
    }
    __syncthreads();
    // step 2: item (line j, row k1): N2-point DFT, X[k1 + N1 k2] in natural order
    FftC w2[IB][N2];
#pragma unroll
    for (int q = 0; q < IB; ++q) {
      const int it = threadIdx.x + q * kFaThreads;
      if (it < NLT * N1) {
        const int j = it % NLT, k1 = it / NLT;
#pragma unroll
        for (int i = 0; i < N2; ++i) w2[q][i] = d[j * ld + k1 * (N2 + 1) + i];
        dft_reg<N2, n>(w2[q], tw);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < IB; ++q) {
      const int it = threadIdx.x + q * kFaThreads;
      if (it < NLT * N1) {
        const int j = it % NLT, k1 = it / NLT;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) d[j * ld + k1 + k2 * N1] = w2[q][k2];
      }
    }
  }
  __syncthreads();
}

template <typename R>
__device__ __forceinline__ su2<double> to_d(su2<R> u) {
  return su2<double>{{(double)u.a.re, (double)u.a.im}, {(double)u.b.re, (double)u.b.im}};
}
template <typename R>
__device__ __forceinline__ su2<R> to_r(su2<double> u) {
  return su2<R>{{(R)u.a.re, (R)u.a.im}, {(R)u.b.re, (R)u.b.im}};
}

// state of the conjugate-gradient form (device, in the buffer)
struct FaCg {
  double s_prev;  // sum_p |F_(k-1)|^2 / p_c^2
  double beta;    // this iteration's Polak-Ribiere coefficient
  double alpha;   // this iteration's step along the direction
  int restart;    // the next direction is the preconditioned gradient alone
  int n_restart;  // directions that did not ascend (diagnostic)
  int parity;     // F_k goes to prev[parity], F_(k-1) is read from prev[parity ^ 1]
  int pad;
};

struct FaArgs {
  const ChainDev* ch;
  const ChainState* cst;  // done flag and step; NULL: never done, step gamma
  double gamma;
  void* fft;              // 2 fields x V complex, natural order (x fastest)
  void* gstep;            // g per site, [parity][site], link layout
  double* part;           // [block]: theta (odd sites)
  double* omega_out;      // debug: omega per site [parity][site][3], or NULL
  const double2* tw;      // exp(-2 pi i k / kFaPoints), k < kFaPoints / 2
  void* prev;             // CG: F of this and the previous iteration, [2][2 fields][V] complex, natural order
  float* sdir;            // CG: direction s, [component][parity][site]
  double* cgpart;         // CG: per-block pairs of sums
  FaCg* cg;               // CG: state
  int L[3], logL[3];      // the transformed (whole) lattice
  int track;
  // the planes the per-site kernels visit (a z-slab: its interior planes).
  // zl0: first visited local plane, nzl: their number, zg0: the whole
  // lattice's z of plane zl0, s_lo: first visited site of each parity.
  // A whole lattice: 0, L3, 0, 0.
  int zl0, nzl, zg0, s_lo;
  // CG: sites per parity of the whole lattice for the step's rms angle
  // (0: the chain's)
  double nh_all;
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

// (1) Delta on x-lines, forward FFT along x; partials of theta.  A block
// takes NL x-lines of both fields: lines 0 .. NL-1 hold Delta_b, NL .. 2NL-1
// hold Delta_a3.
template <typename R, int LOGN>
__global__ void __launch_bounds__(kFaThreads) fa_div_kernel(FaArgs a) {
  using G = FaLines<LOGN>;
  constexpr int n = G::n, ld = G::ld, NL = G::NLT / 2;
  extern __shared__ __align__(16) FftC fa_sm[];
  FftC* d = fa_sm;
  FftC* tw = d + G::NLT * ld;
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int nlines = a.L[1] * a.nzl;
  const int l0 = blockIdx.x * NL;
  load_twiddles(tw, a.tw, n, -1);
  const double al = ch.alpha;
  double q[1] = {0.0};
  for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
    const int j = e >> LOGN, x = e & (n - 1), l = l0 + j;
    FftC v0{0, 0}, v1{0, 0};
    if (l < nlines) {
      // z: the local plane (field arrays), zg: the whole lattice's (theta's
      // odd sites)
      const int y = l & (a.L[1] - 1), zi = l >> a.logL[1], z = zi + a.zl0, zg = zi + a.zg0;
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
      if (((x + y + zg) & 1) == 1) q[0] += d3 * d3 + dbr * dbr + dbi * dbi;
      v0 = FftC{(FftR)dbr, (FftR)dbi};
      v1 = FftC{(FftR)d3, (FftR)0};
    }
    d[j * ld + x] = v0;
    d[(NL + j) * ld + x] = v1;
  }
  block_reduce_store<1>(q, a.part + blockIdx.x);
  __syncthreads();
  fft2_lines<LOGN>(d, tw);
  const size_t V = (size_t)a.L[0] * a.L[1] * a.L[2];
  FftC* F = reinterpret_cast<FftC*>(a.fft);
  const int lg0 = a.zg0 * a.L[1];  // the whole lattice's line of local line 0
  for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
    const int j = e >> LOGN, k = e & (n - 1), l = l0 + j;
    if (l >= nlines) continue;
    const size_t gi = nat_index<0>(a, lg0 + l, k);
    F[gi] = d[j * ld + k];
    F[V + gi] = d[(NL + j) * ld + k];
  }
}

// (2) theta = sum / nh (odd sites); count; done flag at theta <= gf_limit or
// the cap
__global__ void __launch_bounds__(1024) fa_check_kernel(const ChainDev* chp, ChainState* cst, const double* part,
                                                        int nblocks, int adapt) {
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
    // (the conjugate-gradient form chooses its own step)
    if (adapt && it > 1 && theta > 2.0 * cst->gf_theta) cst->gf_step = fmax(0.1, 0.7 * cst->gf_step);
    cst->gf_iters = it;
    cst->gf_theta = theta;
    if (!(theta > cst->gf_limit) || (cst->gf_cap > 0 && it >= cst->gf_cap)) cst->gf_done = 1;
  }
}

// (3)-(5) FFT of one field (blockIdx.y) along axis AX (1: y, 2: z); for
// AX = 2 with SCALE: forward, multiply by gamma / (p_c^2 V), inverse
// (the forward-scale-inverse form is held to 64 registers, 4 blocks per SM)
// CG (with SCALE): the block's sums of |F|^2 / p_c^2 and Re(F^* F_prev) / p_c^2
// into cgpart, and F kept as the next F_prev
template <int AX, int SIGN, bool SCALE, int LOGN, bool CG = false>
__global__ void __launch_bounds__(kFaThreads, LOGN <= 8 ? 4 : 1) fa_fft_kernel(FaArgs a) {
  using G = FaLines<LOGN>;
  constexpr int n = G::n, ld = G::ld, NL = G::NLT, LNL = kFaBlockLog - LOGN;
  extern __shared__ __align__(16) FftC fa_sm[];
  FftC* d = fa_sm;
  FftC* tw = d + NL * ld;
  FftC* twi = tw + G::ntw;                                       // SCALE: inverse twiddles
  double* sz2 = reinterpret_cast<double*>(twi + G::ntw);         // SCALE: alpha sin^2(pi kz / L3)
  double* sxy = sz2 + n;                                         // SCALE: sin^2(pi kx/L1) + sin^2(pi ky/L2)
  if (fa_done(a)) return;
  const int nlines = (a.L[0] * a.L[1] * a.L[2]) >> LOGN;
  const int l0 = blockIdx.x * NL;
  const size_t V = (size_t)a.L[0] * a.L[1] * a.L[2];
  FftC* F = reinterpret_cast<FftC*>(a.fft) + blockIdx.y * V;
  load_twiddles(tw, a.tw, n, SIGN);
  if (SCALE) {
    load_twiddles(twi, a.tw, n, -SIGN);
    const double al = a.ch->alpha;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const double sz = sinpi_r((double)k / a.L[2]);
      sz2[k] = al * sz * sz;
    }
    for (int j = threadIdx.x; j < NL; j += blockDim.x) {
      const int l = l0 + j, kx = l & (a.L[0] - 1), ky = l >> a.logL[0];
      const double sx = sinpi_r((double)kx / a.L[0]), sy = sinpi_r((double)ky / a.L[1]);
      sxy[j] = sx * sx + sy * sy;
    }
  }
  // element e -> (line j = e % NL, position k = e / NL): consecutive threads
  // read consecutive lines, i.e. consecutive x
  for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
    const int j = e & (NL - 1), k = e >> LNL, l = l0 + j;
    d[j * ld + k] = l < nlines ? F[nat_index<AX>(a, l, k)] : FftC{0, 0};
  }
  __syncthreads();
  fft2_lines<LOGN>(d, tw);
  if (CG) {
    // two buffers: a read-modify-write of one stalled every element on its
    // own load (5x the kernel's time at 128^3).  One pass: the sums with the
    // weight 1/(4 p^2) = (1/p^2) / 4 (exact), then the element scaled by
    // gamma / (4 V p^2) = gv (1/p^2) -- one FP64 division per element
    const int par = a.cg->parity;
    FftC* Pn = reinterpret_cast<FftC*>(a.prev) + ((size_t)par * 2 + blockIdx.y) * V;
    const FftC* Po = reinterpret_cast<const FftC*>(a.prev) + ((size_t)(par ^ 1) * 2 + blockIdx.y) * V;
    const double gv = (a.cst ? a.cst->gf_step : a.gamma) / (4.0 * (double)V);
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
      const int j = e & (NL - 1), k = e >> LNL, l = l0 + j;
      const int q = j * ld + k;
      if (l >= nlines) continue;
      const size_t gi = nat_index<AX>(a, l, k);
      const FftC f = d[q], pv = __ldg(Po + gi);
      Pn[gi] = f;
      if ((l | k) == 0) {
        d[q] = FftC{0, 0};
        continue;
      }
      const double r = 1.0 / (sxy[j] + sz2[k]), m0 = 0.25 * r, m = gv * r;
      v[0] += m0 * ((double)f.x * f.x + (double)f.y * f.y);
      v[1] += m0 * ((double)f.x * pv.x + (double)f.y * pv.y);
      d[q] = FftC{(FftR)(f.x * m), (FftR)(f.y * m)};
    }
    block_reduce_store<2>(v, a.cgpart + 2 * ((size_t)blockIdx.y * gridDim.x + blockIdx.x));
    __syncthreads();
    fft2_lines<LOGN>(d, twi);
  } else if (SCALE) {
    const double gv = (a.cst ? a.cst->gf_step : a.gamma) / (4.0 * (double)V);
    for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
      const int j = e >> LOGN, kz = e & (n - 1), l = l0 + j;
      const double p2 = sxy[j] + sz2[kz];
      const double m = (l | kz) ? gv / p2 : 0.0;
      const int q = j * ld + kz;
      d[q] = FftC{(FftR)(d[q].x * m), (FftR)(d[q].y * m)};
    }
    __syncthreads();
    fft2_lines<LOGN>(d, twi);
  }
  for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
    const int j = e & (NL - 1), k = e >> LNL, l = l0 + j;
    if (l < nlines) F[nat_index<AX>(a, l, k)] = d[j * ld + k];
  }
}

// (6) inverse FFT along x; g(x) = exp(-i omega.sigma) per site (CG: the
// direction s = omega + beta s instead)
template <typename R, int LOGN, bool CG = false>
__global__ void __launch_bounds__(kFaThreads) fa_g_kernel(FaArgs a) {
  using G = FaLines<LOGN>;
  constexpr int n = G::n, ld = G::ld, NL = G::NLT / 2;
  extern __shared__ __align__(16) FftC fa_sm[];
  FftC* d = fa_sm;
  FftC* tw = d + G::NLT * ld;
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int nlines = a.L[1] * a.nzl;
  const int l0 = blockIdx.x * NL;
  const size_t V = (size_t)a.L[0] * a.L[1] * a.L[2];
  const FftC* F = reinterpret_cast<const FftC*>(a.fft);
  const int lg0 = a.zg0 * a.L[1];
  load_twiddles(tw, a.tw, n, +1);
  for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
    const int j = e >> LOGN, k = e & (n - 1), l = l0 + j;
    const size_t gi = l < nlines ? nat_index<0>(a, lg0 + l, k) : 0;
    d[j * ld + k] = l < nlines ? F[gi] : FftC{0, 0};
    d[(NL + j) * ld + k] = l < nlines ? F[V + gi] : FftC{0, 0};
  }
  __syncthreads();
  fft2_lines<LOGN>(d, tw);
  for (int e = threadIdx.x; e < NL * n; e += blockDim.x) {
    const int j = e >> LOGN, x = e & (n - 1), l = l0 + j;
    if (l >= nlines) continue;
    const int y = l & (a.L[1] - 1), z = (l >> a.logL[1]) + a.zl0;
    const int p = (x + y + z) & 1, s = site_index(x, y, z, ch.hx, ch.nxy);
    const double w3 = d[(NL + j) * ld + x].x, wbr = d[j * ld + x].x, wbi = d[j * ld + x].y;
    if (CG) {
      const double beta = a.cg->beta;
      const size_t V2 = 2 * (size_t)ch.nh, gi = (size_t)p * ch.nh + s;
      float* S = a.sdir;
      // beta = 0 starts afresh (the old direction is not read)
      S[gi] = (float)(beta > 0.0 ? w3 + beta * (double)S[gi] : w3);
      S[V2 + gi] = (float)(beta > 0.0 ? wbr + beta * (double)S[V2 + gi] : wbr);
      S[2 * V2 + gi] = (float)(beta > 0.0 ? wbi + beta * (double)S[2 * V2 + gi] : wbi);
      continue;
    }
    const double nw = sqrt(w3 * w3 + wbr * wbr + wbi * wbi);
    su2<double> gg{{1.0, 0.0}, {0.0, 0.0}};
    if (nw > 0.0) {
      double sn, cs;
      sincos(nw, &sn, &cs);
      const double f = sn / nw;
      gg = su2<double>{{cs, -f * w3}, {-f * wbr, -f * wbi}};
    }
    LinkIO<double>::st(a.gstep, (size_t)p * ch.nh + s, gg);
    if (a.omega_out) {
      double* o = a.omega_out + ((size_t)p * ch.nh + s) * 3;
      o[0] = (double)w3;
      o[1] = (double)wbr;
      o[2] = (double)wbi;
    }
  }
}

// CG: g = exp(alpha X) at flat index gi of the direction, X = -i s.sigma:
// cos n - (sin n / n) i (alpha s).sigma, n = alpha |s|; below n = 0.05 by the
// Taylor series of cos n and sin n / n through n^8 (the first term left out
// is below 3e-20), else by sincos
__device__ __forceinline__ su2<double> fa_exp_dir(const float* S, size_t V2, size_t gi, double al) {
  const double w3 = al * S[gi], wbr = al * S[V2 + gi], wbi = al * S[2 * V2 + gi];
  const double n2 = w3 * w3 + wbr * wbr + wbi * wbi;
  double c, f;
  if (n2 < 0.0025) {
    c = 1.0 + n2 * (-1.0 / 2.0 + n2 * (1.0 / 24.0 + n2 * (-1.0 / 720.0 + n2 * (1.0 / 40320.0))));
    f = 1.0 + n2 * (-1.0 / 6.0 + n2 * (1.0 / 120.0 + n2 * (-1.0 / 5040.0 + n2 * (1.0 / 362880.0))));
  } else {
    const double n = sqrt(n2);
    double sn;
    sincos(n, &sn, &c);
    f = sn / n;
  }
  return su2<double>{{c, -f * w3}, {-f * wbr, -f * wbi}};
}

// CG: g(x) = exp(alpha X(x)) per site.  (Forming it inside the apply kernel
// instead, four exponentials per site, took 108 us against 17 + 69 us at
// 128^3 for the first iterations from G = 1, whose large angles take sincos.)
__global__ void __launch_bounds__(kBlock) fa_gstep_kernel(FaArgs a) {
  if (fa_done(a)) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= 2 * a.ch->nh) return;
  LinkIO<double>::st(a.gstep, (size_t)i, fa_exp_dir(a.sdir, 2 * (size_t)a.ch->nh, (size_t)i, a.cg->alpha));
}

// (7) U_f(x,mu) -> g(x) U_f(x,mu) g(x+mu)^+, A_f -> g A_f g^+, G -> g G
template <typename R>
__global__ void __launch_bounds__(kBlock) fa_apply_kernel(FaArgs a) {
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  const int nvis = ch.nh - 2 * a.s_lo;  // visited sites per parity
  if (i >= 2 * nvis) return;
  const int eo = i >= nvis ? 1 : 0, oe = 1 - eo, s = a.s_lo + i - eo * nvis, nh = ch.nh;
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

// CG: beta = max(0, (S_k - C_k) / S_(k-1)) from the scale kernel's sums
__global__ void __launch_bounds__(1024) fa_beta_kernel(FaArgs a, int nparts) {
  if (fa_done(a)) return;
  double v[2] = {0.0, 0.0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
    v[0] += a.cgpart[2 * b];
    v[1] += a.cgpart[2 * b + 1];
  }
  __shared__ double t[2];
  block_reduce_store<2>(v, t);
  __syncthreads();
  if (threadIdx.x == 0) {
    FaCg* g = a.cg;
    double beta = 0.0;
    if (!g->restart && g->s_prev > 0.0) beta = fmax(0.0, (t[0] - t[1]) / g->s_prev);
    g->beta = beta;
    g->s_prev = t[0];
    g->restart = 0;
    g->parity ^= 1;
  }
}

// X = -i s.sigma in first-row form (the generator of exp(-i omega.sigma) above)
template <typename R>
__device__ __forceinline__ su2<R> fa_gen(const float* S, size_t V2, size_t gi) {
  return su2<R>{{(R)0, -(R)S[gi]}, {-(R)S[V2 + gi], -(R)S[2 * V2 + gi]}};
}

// CG: per-block F'(0), F''(0) along s and sum |s|^2 (one thread per site,
// both parities).  Per link in the fields' precision (they only set the step
// length; the cancellation in F'' ~ |s(x) - s(x+mu)|^2 loses at most ~(L/2pi)^2
// of the relative precision), summed in FP64.
template <typename R>
__global__ void __launch_bounds__(kBlock) fa_line_kernel(FaArgs a) {
  if (fa_done(a)) return;
  const ChainDev& ch = *a.ch;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  const int nvis = ch.nh - 2 * a.s_lo;  // visited sites per parity
  double v[3] = {0.0, 0.0, 0.0};
  if (i < 2 * nvis) {
    const int eo = i >= nvis ? 1 : 0, oe = 1 - eo, s = a.s_lo + i - eo * nvis, nh = ch.nh;
    const size_t V2 = 2 * (size_t)nh;
    const Coord X = site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
    const su2<R> gx = fa_gen<R>(a.sdir, V2, (size_t)eo * nh + s);
    const R xx = gx.a.im * gx.a.im + gx.b.re * gx.b.re + gx.b.im * gx.b.im;
    v[2] = (double)xx;
    const int L[3] = {ch.L1, ch.L2, ch.L3};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      int c[3] = {X.x, X.y, X.z};
      c[mu] = wrap(c[mu] + 1, L[mu]);
      const int sp = site_index(c[0], c[1], c[2], ch.hx, ch.nxy);
      const su2<R> gy = fa_gen<R>(a.sdir, V2, (size_t)oe * nh + sp);
      const R yy = gy.a.im * gy.a.im + gy.b.re * gy.b.re + gy.b.im * gy.b.im;
      const su2<R> u = LinkIO<R>::ld_cg(ch.uf, ((size_t)(mu * 2 + eo)) * nh + s);
      const double w = mu == 2 ? ch.alpha : 1.0;
      const su2<R> xu = nn(gx, u);
      v[0] += w * (double)(xu.a.re - nn(u, gy).a.re);
      v[1] += w * (double)(-(xx + yy) * u.a.re - (R)2 * nn(xu, gy).a.re);
    }
  }
  block_reduce_store<3>(v, a.cgpart + 3 * (size_t)blockIdx.x);
}

// CG step: the maximum of the quadratic model, alpha = F'(0) / -F''(0), inside
// a trust region: at most 10, and an rms rotation angle alpha |s|_rms of at
// most 0.5 (far from the Landau gauge the model's maximum lies where the
// functional is no longer quadratic).  Near the gauge the slow modes are the
// low modes of the Faddeev-Popov operator, for which the free Laplacian
// overestimates the curvature: alpha ~ 4 there, where the steepest-ascent form
// takes 1.  A non-concave line takes alpha = 1 (within the angle bound), one
// that does not ascend moves nothing; both restart from the gradient.
__global__ void __launch_bounds__(1024) fa_alpha_kernel(FaArgs a, int nparts) {
  if (fa_done(a)) return;
  double v[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
    v[0] += a.cgpart[3 * b];
    v[1] += a.cgpart[3 * b + 1];
    v[2] += a.cgpart[3 * b + 2];
  }
  __shared__ double t[3];
  block_reduce_store<3>(v, t);
  __syncthreads();
  if (threadIdx.x == 0) {
    FaCg* g = a.cg;
    const double nh = a.nh_all > 0.0 ? a.nh_all : (double)a.ch->nh;
    const double d1 = t[0], d2 = t[1], rms = sqrt(t[2] / (2.0 * nh));
    const double amax = rms > 0.0 ? fmin(10.0, 0.5 / rms) : 10.0;
    double al;
    if (d1 > 0.0 && d2 < 0.0) {
      al = fmin(d1 / -d2, amax);
    } else {
      al = d1 > 0.0 ? fmin(1.0, amax) : 0.0;
      g->restart = 1;
      g->n_restart += 1;
    }
    g->alpha = al;
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

// Buffer layout for chains of up to vcap sites: two complex fields, the
// FP64 step transform, the twiddle table, then the conjugate-gradient form's
// state, this and the previous F (two complex fields each), direction (3
// FP32 per site) and per-block sums (fixed offsets, so graphs captured for
// one chain stay valid while others use the same buffer)
namespace {
size_t fa_off_table(size_t vcap) { return 2 * vcap * sizeof(FftC) + vcap * 32; }
size_t fa_off_cg(size_t vcap) { return (fa_off_table(vcap) + kFaPoints / 2 * sizeof(double2) + 255) & ~(size_t)255; }
size_t fa_off_prev(size_t vcap) { return fa_off_cg(vcap) + 256; }
size_t fa_off_sdir(size_t vcap) { return fa_off_prev(vcap) + 4 * vcap * sizeof(FftC); }
size_t fa_off_cgpart(size_t vcap) { return (fa_off_sdir(vcap) + 3 * vcap * sizeof(float) + 255) & ~(size_t)255; }
size_t fa_cgpart_n(size_t vcap) { return 3 * (vcap / 128 + 64); }  // doubles: triples for >= V/256 + 64 blocks
}  // namespace
size_t fa_buffer_bytes(size_t vcap) { return fa_off_cgpart(vcap) + fa_cgpart_n(vcap) * sizeof(double) + 256; }
void* fa_gstep_ptr(void* buf, size_t vcap) { return reinterpret_cast<char*>(buf) + 2 * vcap * sizeof(FftC); }
namespace {
char* fa_at(void* buf, size_t off) { return reinterpret_cast<char*>(buf) + off; }
void* fa_gstep(void* buf, size_t vcap) { return fa_at(buf, 2 * vcap * sizeof(FftC)); }
double2* fa_table(void* buf, size_t vcap) { return reinterpret_cast<double2*>(fa_at(buf, fa_off_table(vcap))); }
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

namespace {
__global__ void fa_cg_reset_kernel(FaCg* g) {
  g->s_prev = 0.0;
  g->beta = 0.0;
  g->alpha = 0.0;
  g->restart = 1;
  g->n_restart = 0;
  g->parity = 0;
}
}  // namespace

void fa_cg_reset(void* buf, size_t vcap, cudaStream_t s) {
  fa_cg_reset_kernel<<<1, 1, 0, s>>>(reinterpret_cast<FaCg*>(fa_at(buf, fa_off_cg(vcap))));
}
void* fa_cg_state(void* buf, size_t vcap) { return fa_at(buf, fa_off_cg(vcap)); }
void fa_cg_reset_state(void* cg, cudaStream_t s) { fa_cg_reset_kernel<<<1, 1, 0, s>>>(reinterpret_cast<FaCg*>(cg)); }
size_t fa_cg_state_bytes() { return sizeof(FaCg); }
void* fa_sdir_ptr(void* buf, size_t vcap) { return fa_at(buf, fa_off_sdir(vcap)); }
double* fa_cgpart_ptr(void* buf, size_t vcap) { return reinterpret_cast<double*>(fa_at(buf, fa_off_cgpart(vcap))); }

// The first failed launch set-up of this host thread since the last
// fa_take_error(): which kernel, its line length and the shared memory it
// asked for.  A kernel whose set-up failed is not launched.
namespace {
thread_local std::string t_fa_error;
}

std::string fa_take_error() {
  std::string e;
  e.swap(t_fa_error);
  return e;
}

// launchers per line length (the kernels are compiled for each power of two)
template <typename K>
void fa_launch(K kernel, const char* what, int logn, dim3 grid, size_t smem, const FaArgs& a, cudaStream_t s) {
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    if (t_fa_error.empty())
      t_fa_error = std::string(what) + " for lines of " + std::to_string(1 << logn) +
                   " points: cudaFuncSetAttribute(MaxDynamicSharedMemorySize = " + std::to_string(smem) +
                   " bytes): " + cudaGetErrorString(e);
    return;
  }
  kernel<<<grid, kFaThreads, smem, s>>>(a);
}
template <typename R, int LOGN>
void fa_div_launch(const FaArgs& a, int nb, cudaStream_t s) {
  fa_launch(fa_div_kernel<R, LOGN>, "fa_div_kernel", LOGN, dim3(nb), FaLines<LOGN>::smem(1, 0), a, s);
}
template <typename R, int LOGN, bool CG = false>
void fa_g_launch(const FaArgs& a, int nb, cudaStream_t s) {
  fa_launch(fa_g_kernel<R, LOGN, CG>, "fa_g_kernel", LOGN, dim3(nb), FaLines<LOGN>::smem(1, 0), a, s);
}
template <int AX, int SIGN, bool SCALE, int LOGN, bool CG = false>
void fa_fft_launch(const FaArgs& a, int nb, cudaStream_t s) {
  using G = FaLines<LOGN>;
  fa_launch(fa_fft_kernel<AX, SIGN, SCALE, LOGN, CG>, "fa_fft_kernel", LOGN, dim3(nb, 2),
            G::smem(SCALE ? 2 : 1, SCALE ? G::n + G::NLT : 0), a, s);
}
#define LCE_FA_SWITCH(logn, CALL) \
  switch (logn) {                 \
    case 1: CALL(1); break;       \
    case 2: CALL(2); break;       \
    case 3: CALL(3); break;       \
    case 4: CALL(4); break;       \
    case 5: CALL(5); break;       \
    case 6: CALL(6); break;       \
    case 7: CALL(7); break;       \
    case 8: CALL(8); break;       \
    case 9: CALL(9); break;       \
    case 10: CALL(10); break;     \
    default: break;               \
  }

// blocks of a transform kernel over lines of length 2^logn (all fields of
// the block share its 4096 points)
int fa_blocks(long nlines, int logn, int fields) {
  return ceil_div(nlines, (long)(kFaBlockPts >> logn) / fields);
}

// enqueue one Fourier-accelerated iteration (kernels 1-7; cg: the
// conjugate-gradient form, 11 kernels)
template <typename R>
void launch_fa_iteration(const ChainDev* chd, const ChainDev& ch, ChainState* cst, double gamma, void* buf,
                         size_t vcap, double* part, double* omega_out, int track, bool with_check, bool with_apply,
                         bool cg, cudaStream_t s) {
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
  a.zl0 = 0;
  a.nzl = ch.L3;
  a.zg0 = 0;
  a.s_lo = 0;
  a.nh_all = 0.0;
  a.cg = reinterpret_cast<FaCg*>(fa_at(buf, fa_off_cg(vcap)));
  a.prev = fa_at(buf, fa_off_prev(vcap));
  a.sdir = reinterpret_cast<float*>(fa_at(buf, fa_off_sdir(vcap)));
  a.cgpart = reinterpret_cast<double*>(fa_at(buf, fa_off_cgpart(vcap)));
  const int nbd = fa_blocks((long)ch.L2 * ch.L3, a.logL[0], 2);
#define LCE_FA_DIV(L) fa_div_launch<R, L>(a, nbd, s)
  LCE_FA_SWITCH(a.logL[0], LCE_FA_DIV)
#undef LCE_FA_DIV
  if (with_check) fa_check_kernel<<<1, 1024, 0, s>>>(chd, cst, part, nbd, cg ? 0 : 1);
  const int nby = fa_blocks((long)V / ch.L2, a.logL[1], 1), nbz = fa_blocks((long)V / ch.L3, a.logL[2], 1);
#define LCE_FA_Y(L) fa_fft_launch<1, -1, false, L>(a, nby, s)
  LCE_FA_SWITCH(a.logL[1], LCE_FA_Y)
#undef LCE_FA_Y
  if (cg) {
#define LCE_FA_ZC(L) fa_fft_launch<2, -1, true, L, true>(a, nbz, s)
    LCE_FA_SWITCH(a.logL[2], LCE_FA_ZC)
#undef LCE_FA_ZC
    fa_beta_kernel<<<1, 1024, 0, s>>>(a, 2 * nbz);
  } else {
#define LCE_FA_Z(L) fa_fft_launch<2, -1, true, L>(a, nbz, s)
    LCE_FA_SWITCH(a.logL[2], LCE_FA_Z)
#undef LCE_FA_Z
  }
#define LCE_FA_YI(L) fa_fft_launch<1, +1, false, L>(a, nby, s)
  LCE_FA_SWITCH(a.logL[1], LCE_FA_YI)
#undef LCE_FA_YI
  const int nbv = ceil_div((long)V, kBlock);
  if (cg) {
#define LCE_FA_GC(L) fa_g_launch<R, L, true>(a, nbd, s)
    LCE_FA_SWITCH(a.logL[0], LCE_FA_GC)
#undef LCE_FA_GC
    fa_line_kernel<R><<<nbv, kBlock, 0, s>>>(a);
    fa_alpha_kernel<<<1, 1024, 0, s>>>(a, nbv);
    fa_gstep_kernel<<<nbv, kBlock, 0, s>>>(a);
  } else {
#define LCE_FA_G(L) fa_g_launch<R, L>(a, nbd, s)
    LCE_FA_SWITCH(a.logL[0], LCE_FA_G)
#undef LCE_FA_G
  }
  if (with_apply) fa_apply_kernel<R><<<nbv, kBlock, 0, s>>>(a);
}

// One stage of a Fourier-accelerated iteration on a z-slab decomposed
// lattice.  Each slab holds its own step transform and twiddle table (buf);
// the whole lattice's two transformed fields are one buffer (fft) on the
// first slab's device.  stage 0: Delta and the x transforms of the slab's
// interior x-lines into fft, theta partials into part (returns their
// number); stage 1: the y and z transforms of the whole of fft (on its
// device; ch, cst: the first slab's); stage 2: the inverse x transforms of the
// slab's lines and g at its interior sites; stage 3: g applied at its
// interior sites, the transform G tracked.
template <typename R>
int launch_fa_slab_stage(int stage, const ChainDev* chd, const ChainDev& ch, ChainState* cst, void* fft, void* buf,
                         size_t vcap, double* part, const int Lg[3], int zl0, int nzl, int zg0, int s_lo,
                         cudaStream_t s, const FaSlabCg* cgw) {
  FaArgs a;
  std::memset(&a, 0, sizeof(a));
  a.ch = chd;
  a.cst = cst;
  a.gamma = 1.0;
  a.fft = fft;
  a.gstep = fa_gstep(buf, vcap);
  a.part = part;
  a.omega_out = nullptr;
  a.tw = fa_table(buf, vcap);
  for (int d = 0; d < 3; ++d) {
    a.L[d] = Lg[d];
    a.logL[d] = ilog2_exact(Lg[d]);
  }
  a.track = 1;
  a.zl0 = zl0;
  a.nzl = nzl;
  a.zg0 = zg0;
  a.s_lo = s_lo;
  a.cg = reinterpret_cast<FaCg*>(fa_at(buf, fa_off_cg(vcap)));
  a.prev = fa_at(buf, fa_off_prev(vcap));
  a.sdir = reinterpret_cast<float*>(fa_at(buf, fa_off_sdir(vcap)));
  a.cgpart = reinterpret_cast<double*>(fa_at(buf, fa_off_cgpart(vcap)));
  a.nh_all = 0.0;
  const bool cg = cgw != nullptr;
  if (cg && (stage == 1 || stage == 5)) {
    // the whole lattice's CG state, F of this and the previous iteration and
    // the sums, on the first slab's device
    a.cg = reinterpret_cast<FaCg*>(cgw->cg);
    a.prev = cgw->prev;
    a.cgpart = stage == 1 ? cgw->pairs : cgw->tri;
    a.nh_all = cgw->nh_all;
  }
  const size_t V = (size_t)Lg[0] * Lg[1] * Lg[2];
  const int nbd = fa_blocks((long)Lg[1] * nzl, a.logL[0], 2);
  if (stage == 0) {
#define LCE_FA_DIV(L) fa_div_launch<R, L>(a, nbd, s)
    LCE_FA_SWITCH(a.logL[0], LCE_FA_DIV)
#undef LCE_FA_DIV
    return nbd;
  }
  if (stage == 1) {
    const int nby = fa_blocks((long)V / Lg[1], a.logL[1], 1), nbz = fa_blocks((long)V / Lg[2], a.logL[2], 1);
#define LCE_FA_Y(L) fa_fft_launch<1, -1, false, L>(a, nby, s)
    LCE_FA_SWITCH(a.logL[1], LCE_FA_Y)
#undef LCE_FA_Y
    if (cg) {
#define LCE_FA_ZC(L) fa_fft_launch<2, -1, true, L, true>(a, nbz, s)
      LCE_FA_SWITCH(a.logL[2], LCE_FA_ZC)
#undef LCE_FA_ZC
      fa_beta_kernel<<<1, 1024, 0, s>>>(a, 2 * nbz);
    } else {
#define LCE_FA_Z(L) fa_fft_launch<2, -1, true, L>(a, nbz, s)
      LCE_FA_SWITCH(a.logL[2], LCE_FA_Z)
#undef LCE_FA_Z
    }
#define LCE_FA_YI(L) fa_fft_launch<1, +1, false, L>(a, nby, s)
    LCE_FA_SWITCH(a.logL[1], LCE_FA_YI)
#undef LCE_FA_YI
    return 0;
  }
  if (stage == 2) {
    if (cg) {
#define LCE_FA_GC(L) fa_g_launch<R, L, true>(a, nbd, s)
      LCE_FA_SWITCH(a.logL[0], LCE_FA_GC)
#undef LCE_FA_GC
    } else {
#define LCE_FA_G(L) fa_g_launch<R, L>(a, nbd, s)
      LCE_FA_SWITCH(a.logL[0], LCE_FA_G)
#undef LCE_FA_G
    }
    return 0;
  }
  const int nbv = ceil_div(2L * (ch.nh - 2 * s_lo), kBlock);
  if (stage == 4) {
    // CG: the line derivatives at the slab's interior sites, one triple per
    // block into the buffer's own per-block sums (fa_cgpart_ptr)
    fa_line_kernel<R><<<nbv, kBlock, 0, s>>>(a);
    return nbv;
  }
  if (stage == 5) {
    // CG: the step from the slabs' sums (cgw->sums, one triple per slab)
    fa_alpha_kernel<<<1, 1024, 0, s>>>(a, cgw->nslabs);
    return 0;
  }
  if (stage == 6) {
    // CG: g = exp(alpha X) at every local site (the halo planes included)
    fa_gstep_kernel<<<ceil_div(2L * ch.nh, kBlock), kBlock, 0, s>>>(a);
    return 0;
  }
  fa_apply_kernel<R><<<nbv, kBlock, 0, s>>>(a);
  return 0;
}

template int launch_fa_slab_stage<float>(int, const ChainDev*, const ChainDev&, ChainState*, void*, void*, size_t,
                                         double*, const int*, int, int, int, int, cudaStream_t, const FaSlabCg*);
template int launch_fa_slab_stage<double>(int, const ChainDev*, const ChainDev&, ChainState*, void*, void*, size_t,
                                          double*, const int*, int, int, int, int, cudaStream_t, const FaSlabCg*);

template void launch_fa_iteration<float>(const ChainDev*, const ChainDev&, ChainState*, double, void*, size_t,
                                         double*, double*, int, bool, bool, bool, cudaStream_t);
template void launch_fa_iteration<double>(const ChainDev*, const ChainDev&, ChainState*, double, void*, size_t,
                                          double*, double*, int, bool, bool, bool, cudaStream_t);

}  // namespace lce
