// lce_fields.cu -- moving fields between the reference's array order and the
// device planes, and device-side initial configurations.
//
// Reference order (compacted to ld = nh by the caller's 2D copy):
//   links  [mu][eo][site][4]   (the COMMON u(2, site, eo, mu) COMPLEX layout)
//   Higgs  [eo][site][3]       (REAL a(3, site, eo))
// Device planes: links [mu][eo][site] (float4 or 2 x double2), Higgs
// [eo][k][site] SoA.
#include <algorithm>

#include <atomic>

#include "lce_internal.hpp"

namespace lce {

namespace {
inline int grid_for(size_t n, int bs) { return (int)std::min<size_t>((n + bs - 1) / bs, 148 * 32); }
}  // namespace

template <typename Rin, typename R>
__global__ void links_in_kernel(const Rin* __restrict__ src, void* dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Rin* q = src + i * 4;
    LinkIO<R>::st(dst, i, su2<R>{{(R)q[0], (R)q[1]}, {(R)q[2], (R)q[3]}});
  }
}

template <typename R, typename Rout>
__global__ void links_out_kernel(const void* src, Rout* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    su2<R> u = LinkIO<R>::ld_cg(src, i);
    Rout* q = dst + i * 4;
    q[0] = (Rout)u.a.re;
    q[1] = (Rout)u.a.im;
    q[2] = (Rout)u.b.re;
    q[3] = (Rout)u.b.im;
  }
}

// [eo][site][3] -> [eo][k][site]
template <typename Rin, typename R>
__global__ void higgs_in_kernel(const Rin* __restrict__ src, R* __restrict__ dst, int nh) {
  const size_t n = (size_t)2 * nh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t eo = i / nh, s = i - eo * nh;
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[(eo * 3 + k) * nh + s] = (R)src[i * 3 + k];
  }
}

template <typename R, typename Rout>
__global__ void higgs_out_kernel(const R* __restrict__ src, Rout* __restrict__ dst, int nh) {
  const size_t n = (size_t)2 * nh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t eo = i / nh, s = i - eo * nh;
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[i * 3 + k] = (Rout)src[(eo * 3 + k) * nh + s];
  }
}

template <typename R>
__global__ void init_unit_kernel(void* u, R* a, int nh, R a3) {
  const size_t nl = (size_t)6 * nh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nl; i += (size_t)gridDim.x * blockDim.x) {
    LinkIO<R>::st(u, i, su2<R>{{(R)1, (R)0}, {(R)0, (R)0}});
    if (i < (size_t)2 * nh) {
      const size_t eo = i / nh, s = i - eo * nh;
      a[(eo * 3 + 0) * nh + s] = (R)0;
      a[(eo * 3 + 1) * nh + s] = (R)0;
      a[(eo * 3 + 2) * nh + s] = a3;
    }
  }
}

// Box-Muller pair from two Philox words
__device__ __forceinline__ void gauss2(uint32_t w0, uint32_t w1, double& g0, double& g1) {
  const double u1 = (double)u01(w0), u2 = (double)u01(w1);
  const double r = sqrt(-2.0 * log(u1));
  double sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  g0 = r * cs;
  g1 = r * sn;
}

// Haar links as normalised 4-vectors of Gaussians; A components N(0,1).
// Counter (index, field tag, 0, 0) with the chain key.
template <typename R>
__global__ void init_hot_kernel(void* u, R* a, int nh, uint32_t k0, uint32_t k1) {
  const size_t nl = (size_t)6 * nh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nl; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0x484f54u, 0u};
    philox4x32_10(c, k0, k1);
    double g[4];
    gauss2(c[0], c[1], g[0], g[1]);
    gauss2(c[2], c[3], g[2], g[3]);
    const double n = 1.0 / sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + g[3] * g[3]);
    LinkIO<R>::st(u, i, su2<R>{{(R)(g[0] * n), (R)(g[1] * n)}, {(R)(g[2] * n), (R)(g[3] * n)}});
    if (i < (size_t)2 * nh) {
      uint32_t d[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0x41304bu, 1u};
      philox4x32_10(d, k0, k1);
      double h[4];
      gauss2(d[0], d[1], h[0], h[1]);
      gauss2(d[2], d[3], h[2], h[3]);
      const size_t eo = i / nh, s = i - eo * nh;
      a[(eo * 3 + 0) * nh + s] = (R)h[0];
      a[(eo * 3 + 1) * nh + s] = (R)h[1];
      a[(eo * 3 + 2) * nh + s] = (R)h[2];
    }
  }
}

__global__ void flush_kernel(uint4* buf, size_t n, uint32_t tag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    buf[i] = make_uint4(tag, (uint32_t)i, tag, (uint32_t)i);
}

// Reads a second buffer larger than L2: the dirty lines left by the write
// are evicted (written back) here, so the next timed kernel starts with an
// L2 holding clean lines of unrelated data.  The sink keeps the loads alive.
__global__ void flush_read_kernel(const uint4* __restrict__ buf, size_t n, uint32_t* sink) {
  uint32_t acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint4 v = __ldcg(buf + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9E3779B9u) sink[0] = acc;
}

template <typename Rin, typename R>
void launch_links_in(const Rin* src, void* dst, int nh, cudaStream_t s) {
  size_t n = (size_t)6 * nh;
  links_in_kernel<Rin, R><<<grid_for(n, 256), 256, 0, s>>>(src, dst, n);
}
template <typename R, typename Rout>
void launch_links_out(const void* src, Rout* dst, int nh, cudaStream_t s) {
  size_t n = (size_t)6 * nh;
  links_out_kernel<R, Rout><<<grid_for(n, 256), 256, 0, s>>>(src, dst, n);
}
template <typename Rin, typename R>
void launch_higgs_in(const Rin* src, void* dst, int nh, cudaStream_t s) {
  higgs_in_kernel<Rin, R><<<grid_for((size_t)2 * nh, 256), 256, 0, s>>>(src, reinterpret_cast<R*>(dst), nh);
}
template <typename R, typename Rout>
void launch_higgs_out(const void* src, Rout* dst, int nh, cudaStream_t s) {
  higgs_out_kernel<R, Rout><<<grid_for((size_t)2 * nh, 256), 256, 0, s>>>(reinterpret_cast<const R*>(src), dst, nh);
}
template <typename R>
void launch_init_unit(void* u, void* a, int nh, double a3, cudaStream_t s) {
  init_unit_kernel<R><<<grid_for((size_t)6 * nh, 256), 256, 0, s>>>(u, reinterpret_cast<R*>(a), nh, (R)a3);
}
template <typename R>
void launch_init_hot(void* u, void* a, int nh, uint32_t k0, uint32_t k1, cudaStream_t s) {
  init_hot_kernel<R><<<grid_for((size_t)6 * nh, 256), 256, 0, s>>>(u, reinterpret_cast<R*>(a), nh, k0, k1);
}
// buf holds 2 x bytes: the first half is written, the second half read.
void launch_flush(void* buf, size_t bytes, cudaStream_t s) {
  static std::atomic<uint32_t> tag{1};  // a new value per flush, from any host thread
  size_t n = bytes / sizeof(uint4);
  uint4* b = reinterpret_cast<uint4*>(buf);
  flush_kernel<<<148 * 8, 512, 0, s>>>(b, n, tag.fetch_add(1, std::memory_order_relaxed));
  flush_read_kernel<<<148 * 8, 512, 0, s>>>(b + n, n, reinterpret_cast<uint32_t*>(b));
}

#define LCE_INST2(A, B)                                                         \
  template void launch_links_in<A, B>(const A*, void*, int, cudaStream_t);     \
  template void launch_links_out<B, A>(const void*, A*, int, cudaStream_t);    \
  template void launch_higgs_in<A, B>(const A*, void*, int, cudaStream_t);     \
  template void launch_higgs_out<B, A>(const void*, A*, int, cudaStream_t);
LCE_INST2(float, float)
LCE_INST2(float, double)
LCE_INST2(double, float)
LCE_INST2(double, double)
#undef LCE_INST2
template void launch_init_unit<float>(void*, void*, int, double, cudaStream_t);
template void launch_init_unit<double>(void*, void*, int, double, cudaStream_t);
template void launch_init_hot<float>(void*, void*, int, uint32_t, uint32_t, cudaStream_t);
template void launch_init_hot<double>(void*, void*, int, uint32_t, uint32_t, cudaStream_t);

}  // namespace lce
