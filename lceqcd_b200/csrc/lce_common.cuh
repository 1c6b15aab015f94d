// lce_common.cuh -- device building blocks shared by every lceqcd kernel.
//
//  * SU(2) links in the reference's first-row convention: U = {{a, b}, {-b*, a*}}
//    stored as (Re a, Im a, Re b, Im b) (f/INCLUDE/gaugefield.inc:39-51), with the
//    six products of f/matmul.f written exactly as the reference forms them.
//  * The adjoint Higgs field A = a_k sigma_k enters products as iA, whose first
//    row is (i a3, a2 + i a1) (f/matmul.f:150-154).
//  * Parity-split half-row site order of f/adresses.f: parity p = 0 holds the
//    sites with (x+y+z) even (0-based coordinates), and inside a parity
//    s = z*(L1*L2/2) + y*(L1/2) + x/2.
//  * Philox4x32-10 counter-based uniforms for production runs.
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#define LCE_HD __host__ __device__ __forceinline__

namespace lce {

// ------------------------------------------------------------------ complex
template <typename R>
struct cpx {
  R re, im;
};
template <typename R>
LCE_HD cpx<R> mk(R re, R im) { return cpx<R>{re, im}; }
template <typename R>
LCE_HD cpx<R> operator*(cpx<R> x, cpx<R> y) {
  return cpx<R>{x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re};
}
template <typename R>
LCE_HD cpx<R> operator+(cpx<R> x, cpx<R> y) { return cpx<R>{x.re + y.re, x.im + y.im}; }
template <typename R>
LCE_HD cpx<R> operator-(cpx<R> x, cpx<R> y) { return cpx<R>{x.re - y.re, x.im - y.im}; }
template <typename R>
LCE_HD cpx<R> operator-(cpx<R> x) { return cpx<R>{-x.re, -x.im}; }
template <typename R>
LCE_HD cpx<R> cj(cpx<R> x) { return cpx<R>{x.re, -x.im}; }

// SU(2) (or quaternion-proportional) matrix by its first row
template <typename R>
struct su2 {
  cpx<R> a, b;
};

// f/matmul.f MULTALLNN:22-23   U1 U2
template <typename R>
LCE_HD su2<R> nn(su2<R> u1, su2<R> u2) {
  return su2<R>{u1.a * u2.a - u1.b * cj(u2.b), u1.a * u2.b + u1.b * cj(u2.a)};
}
// MULTALLDN:52-56   U1^+ U2
template <typename R>
LCE_HD su2<R> dn(su2<R> u1, su2<R> u2) {
  return su2<R>{cj(u1.a) * u2.a + u1.b * cj(u2.b), cj(u1.a) * u2.b - u1.b * cj(u2.a)};
}
// MULTALLND:85-89   U1 U2^+
template <typename R>
LCE_HD su2<R> nd(su2<R> u1, su2<R> u2) {
  return su2<R>{u1.a * cj(u2.a) + u1.b * cj(u2.b), -(u1.a * u2.b) + u1.b * u2.a};
}
// MULTALLDD:118-122   U1^+ U2^+
template <typename R>
LCE_HD su2<R> dd(su2<R> u1, su2<R> u2) {
  return su2<R>{cj(u1.a) * cj(u2.a) - u1.b * cj(u2.b), -(cj(u1.a) * u2.b) - u1.b * u2.a};
}
// i a3 z for real a3: the product by the purely imaginary diagonal entry of
// iA without its zero real part (equal to (0, a3) * z but for the sign of a
// zero)
template <typename R>
LCE_HD cpx<R> imul(R a3, cpx<R> z) { return cpx<R>{-(a3 * z.im), a3 * z.re}; }
// MULTALLAD:150-154   (iA) U^+
template <typename R>
LCE_HD su2<R> ad(R a1, R a2, R a3, su2<R> u) {
  cpx<R> y = mk<R>(a2, a1);
  return su2<R>{imul(a3, cj(u.a)) + y * cj(u.b), -imul(a3, u.b) + y * u.a};
}
// MULTALLAN:183-187   (iA) U
template <typename R>
LCE_HD su2<R> an(R a1, R a2, R a3, su2<R> u) {
  cpx<R> y = mk<R>(a2, a1);
  return su2<R>{imul(a3, u.a) - y * cj(u.b), imul(a3, u.b) + y * cj(u.a)};
}

template <typename R>
LCE_HD R norm2(su2<R> u) {
  return u.a.re * u.a.re + u.a.im * u.a.im + u.b.re * u.b.re + u.b.im * u.b.im;
}

// ------------------------------------------------------------------ link I/O
// A link plane is nh consecutive links of one (mu, parity).  FP32 links are a
// 16-byte float4; FP64 links are two 16-byte double2.
template <typename R>
struct LinkIO;

template <>
struct LinkIO<float> {
  static constexpr int kBytes = 16;
  __device__ static su2<float> ld(const void* base, size_t i) {
    float4 v = __ldg(reinterpret_cast<const float4*>(base) + i);
    return su2<float>{{v.x, v.y}, {v.z, v.w}};
  }
  __device__ static su2<float> ld_cg(const void* base, size_t i) {
    float4 v = __ldcg(reinterpret_cast<const float4*>(base) + i);
    return su2<float>{{v.x, v.y}, {v.z, v.w}};
  }  __device__ static void st(void* base, size_t i, su2<float> u) {
    reinterpret_cast<float4*>(base)[i] = make_float4(u.a.re, u.a.im, u.b.re, u.b.im);
  }
};

template <>
struct LinkIO<double> {
  static constexpr int kBytes = 32;
  __device__ static su2<double> ld(const void* base, size_t i) {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * i;
    double2 x = __ldg(p), y = __ldg(p + 1);
    return su2<double>{{x.x, x.y}, {y.x, y.y}};
  }
  __device__ static su2<double> ld_cg(const void* base, size_t i) {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * i;
    double2 x = __ldcg(p), y = __ldcg(p + 1);
    return su2<double>{{x.x, x.y}, {y.x, y.y}};
  }
  __device__ static void st(void* base, size_t i, su2<double> u) {
    double2* p = reinterpret_cast<double2*>(base) + 2 * i;
    p[0] = make_double2(u.a.re, u.a.im);
    p[1] = make_double2(u.b.re, u.b.im);
  }
};

// Reunitarise in FP64 before storing (f/renorm.f:27-31 fused into the writer).
// The norm is formed in FP64 from the stored components; for n = 1 + e with
// |e| < 1e-4 (every link written by an update) 1/sqrt(n) is the series
// 1 - e/2 + 3e^2/8 - 5e^3/16, whose truncation error (35/128) e^4 < 3e-17 is
// below FP64 rounding; otherwise the division is taken.
template <typename R>
__device__ __forceinline__ su2<R> unitarise64(su2<R> u) {
  const double n = (double)u.a.re * u.a.re + (double)u.a.im * u.a.im + (double)u.b.re * u.b.re +
                   (double)u.b.im * u.b.im;
  const double e = n - 1.0;
  double t;
  if (fabs(e) < 1.0e-4) t = fma(e, fma(e, fma(e, -0.3125, 0.375), -0.5), 1.0);
  else t = 1.0 / sqrt(n);
  return su2<R>{{(R)(u.a.re * t), (R)(u.a.im * t)}, {(R)(u.b.re * t), (R)(u.b.im * t)}};
}

// ------------------------------------------------------------------ math policy
// M<double>: the library functions (validation mode, compared with the FP64
// oracle at 1e-12).  M<float>: the SFU (MUFU) forms for the production path;
// their errors (a few 1e-7 relative or absolute, CUDA C Programming Guide
// intrinsic-function tables) sit at the level of FP32 storage rounding.
// Arguments of the trigonometric forms are 2*pi*u with u in (0,1), reduced
// to [-pi, pi] where the SFU error bound holds: cos(2 pi u) = -cos(2 pi (u - 1/2)).
template <typename R>
struct M;

template <>
struct M<double> {
  __device__ static double log(double x) { return ::log(x); }
  __device__ static double exp(double x) { return ::exp(x); }
  __device__ static double sqrt(double x) { return ::sqrt(x); }
  __device__ static double rsqrt(double x) { return 1.0 / ::sqrt(x); }
  __device__ static double div(double a, double b) { return a / b; }
  __device__ static double cos2pi(double u) { return ::cospi(2.0 * u); }
  __device__ static void sincos2pi(double u, double* s, double* c) { ::sincospi(2.0 * u, s, c); }
  __device__ static double acos(double x) { return ::acos(x); }
  __device__ static double atan2(double y, double x) { return ::atan2(y, x); }
  __device__ static void sincos(double x, double* s, double* c) { ::sincos(x, s, c); }
  __device__ static double sin(double x) { return ::sin(x); }
  __device__ static double cos(double x) { return ::cos(x); }
};

template <>
struct M<float> {
  __device__ static float log(float x) { return __logf(x); }
  __device__ static float exp(float x) { return __expf(x); }
  __device__ static float sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
  __device__ static float rsqrt(float x) { return rsqrtf(x); }
  __device__ static float div(float a, float b) { return __fdividef(a, b); }
  __device__ static float cos2pi(float u) { return -__cosf(6.28318530717958647692f * (u - 0.5f)); }
  __device__ static void sincos2pi(float u, float* s, float* c) {
    __sincosf(6.28318530717958647692f * (u - 0.5f), s, c);
    *s = -*s;
    *c = -*c;
  }
  __device__ static float acos(float x) { return acosf(x); }
  __device__ static float atan2(float y, float x) { return atan2f(y, x); }
  __device__ static void sincos(float x, float* s, float* c) { sincosf(x, s, c); }
  __device__ static float sin(float x) { return sinf(x); }
  __device__ static float cos(float x) { return cosf(x); }
};

// ------------------------------------------------------------------ geometry
// Division by a runtime constant with one high multiply (round-up method of
// Granlund & Montgomery, PLDI 1994); valid for n < 2^31.
struct FastDiv {
  uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t s = 0;
  while ((1ull << s) < d) ++s;
  uint64_t m = ((1ull << 32) * ((1ull << s) - d)) / d + 1;
  return FastDiv{d, (uint32_t)m, s};
}
LCE_HD uint32_t fdiv(uint32_t n, FastDiv f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(n, f.m) + n) >> f.s;
#else
  return (uint32_t)((((uint64_t)n * f.m) >> 32) + n) >> f.s;
#endif
}

// Coordinates of site s of parity p.
struct Coord {
  int x, y, z;
};
LCE_HD Coord site_coord(int p, int s, int hx, int nxy, FastDiv dhx, FastDiv dnxy) {
  int z = (int)fdiv((uint32_t)s, dnxy);
  int r = s - z * nxy;
  int y = (int)fdiv((uint32_t)r, dhx);
  int xh = r - y * hx;
  return Coord{2 * xh + ((p + y + z) & 1), y, z};
}
LCE_HD int wrap(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }
// Index inside its parity of the site at (x, y, z), coordinates already in range.
LCE_HD int site_index(int x, int y, int z, int hx, int nxy) { return z * nxy + y * hx + (x >> 1); }

// ------------------------------------------------------------------ RNG
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
LCE_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    // one 32x32 -> 64-bit multiply gives both halves
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}
// (2k+1)/2^24 with k the top 23 bits: strictly inside (0,1), exact in FP32.
// On the device it is built without an integer-to-float conversion: the bits
// 0x3f800000 | k are the float 1 + k 2^-23, and subtracting 1 - 2^-24 (the
// float below 1) leaves (2k+1) 2^-24 exactly (the operands are within a
// factor 2 of each other, so the difference is exact -- Sterbenz's lemma).
LCE_HD float u01(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(0x3f800000u | (x >> 9)) - 0.999999940395355224609375f;
#else
  return (float)((x >> 9) * 2u + 1u) * 5.9604644775390625e-8f;
#endif
}

// Uniform slot layouts of one update pass in the reference's consumption
// order: PLANAR puts slot k of site s at k*nh + s; TRIPLE interleaves slots
// 0..2 per site (3s + k) and keeps later slots planar (f/heat_kpi.f:33-40,
// f/ahiggs1.f:51-56).
enum Layout : int { kPlanar = 0, kTriple = 1 };
LCE_HD size_t slot_off(int layout, int nh, int k, int s) {
  return (layout == kTriple && k < 3) ? (size_t)3 * s + k : (size_t)k * nh + s;
}

// The N uniforms one site draws in one pass, held in registers.  Philox
// mode: slot k is word k&3 of Philox4x32-10(key, {site, k>>2, pass_lo,
// pass_hi}).  Stream mode: slot k is stream[slot_off(layout, nh, k, site)].
template <typename R, int N>
struct Uniforms {
  R v[N];
  __device__ __forceinline__ void fill_philox(uint32_t k0, uint32_t k1, unsigned long long pass, int s) {
#pragma unroll
    for (int q = 0; q < (N + 3) / 4; ++q) {
      uint32_t c[4] = {(uint32_t)s, (uint32_t)q, (uint32_t)pass, (uint32_t)(pass >> 32)};
      philox4x32_10(c, k0, k1);
#pragma unroll
      for (int w = 0; w < 4; ++w)
        if (4 * q + w < N) v[4 * q + w] = (R)u01(c[w]);
    }
  }
  __device__ __forceinline__ void fill_stream(const double* st, int nh, int layout, int s) {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = (R)__ldg(st + slot_off(layout, nh, k, s));
  }
};

// ------------------------------------------------------------------ PDL
// Programmatic dependent launch (sm_90+): a kernel lets the next kernel of
// its stream begin launching once every block of it has started, and the
// next kernel blocks in griddepcontrol.wait until this grid has completed
// and its writes are visible.  Kernels call pdl_trigger() first, do
// data-independent set-up, and call pdl_wait() before their first read of
// anything an earlier kernel writes.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// ------------------------------------------------------------------ reductions
// Block partials of NC event counts (reduced as 32-bit integers) and ND FP64
// sums; out[0..NC) = counts, out[NC..NC+ND) = sums, out[NC+ND..NQ) = 0.
// REUSE: the block calls it more than once (the persistent form's tile loop),
// so the shared slots are first waited free.
template <int NC, int ND, int NQ, bool REUSE = true>
__device__ __forceinline__ void block_reduce_cs(const unsigned (&cnt)[NC > 0 ? NC : 1], double (&v)[ND > 0 ? ND : 1],
                                                double* out) {
  static_assert(NC + ND <= NQ, "too many partials");
  __shared__ unsigned redc[32][NC > 0 ? NC : 1];
  __shared__ double redd[32][ND > 0 ? ND : 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (REUSE) __syncthreads();  // a previous call's readers are done with the shared slots
  unsigned cw[NC > 0 ? NC : 1];
#pragma unroll
  for (int q = 0; q < NC; ++q) cw[q] = __reduce_add_sync(0xffffffffu, cnt[q]);
#pragma unroll
  for (int q = 0; q < ND; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NC; ++q) redc[w][q] = cw[q];
#pragma unroll
    for (int q = 0; q < ND; ++q) redd[w][q] = v[q];
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      unsigned t = __reduce_add_sync(0xffffffffu, lane < nw ? redc[lane][q] : 0u);
      if (lane == 0) out[q] = (double)t;
    }
#pragma unroll
    for (int q = 0; q < ND; ++q) {
      double t = lane < nw ? redd[lane][q] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) out[NC + q] = t;
    }
    if (lane == 0) {
#pragma unroll
      for (int q = NC + ND; q < NQ; ++q) out[q] = 0.0;
    }
  }
}

template <int NQ>
__device__ __forceinline__ void block_reduce_store(double (&v)[NQ], double* out) {
  __shared__ double red[32][NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) red[w][q] = v[q];
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double t = lane < nw ? red[lane][q] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) out[q] = t;
    }
  }
}

}  // namespace lce
