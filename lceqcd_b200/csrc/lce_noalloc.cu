// lce_noalloc.cu -- average plaquette of a caller-owned link field, with no
// device allocation.
//
// Some callers cannot let this library call cudaMalloc: a driver whose device
// memory is owned by another allocator (a PyTorch caching allocator, a CUDA
// Fortran memory pool, a fixed budget carved out up front), or code that runs
// between asynchronous launches where cudaMalloc/cudaFree could synchronise
// the device.  lce_plaquette_noalloc serves them: the caller passes the link
// field and the output in its own device memory, and the only scratch -- one
// FP64 partial sum per thread block -- lives in a file-scope __device__ array
// that every GPU loading this library holds until the process exits.
//
// That array is shared by every call on a device and keeps the last call's
// contents; each call overwrites every entry it reads, so nothing needs to
// start at zero.  Calls whose kernels overlap on the GPU (different streams,
// or different host threads) race on the array and must be serialised by the
// caller.  The array's device address is looked up on a device's first call
// and kept until the process exits: after a cudaDeviceReset (which tears down
// the primary context and reloads this module) the kept address is stale, so
// the entry point must not be used across a device reset.
#include <mutex>

#include "lce_internal.hpp"

namespace lce {

namespace {

constexpr int kNaBlock = 256;                  // sites per thread block
constexpr int kNaMaxBlocks = 65536;            // scratch capacity (512 KiB)
constexpr long kNaMaxSites = (long)kNaBlock * kNaMaxBlocks;  // 16,777,216 = 256^3

static __device__ __align__(256) double g_noalloc_partials[kNaMaxBlocks];

struct NaGeom {
  int L1, L2, L3, hx, nxy, nh;
  long ld;
  FastDiv dhx, dnxy;
};

// one thread per site (both parities); the block's sum of the three
// plaquettes 1/2 Re Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ at its sites
__global__ void __launch_bounds__(kNaBlock) noalloc_plaquette_partials(const float4* __restrict__ u, NaGeom g,
                                                                       double* part) {
  const int i = blockIdx.x * kNaBlock + threadIdx.x;
  double v[1] = {0.0};
  if (i < 2 * g.nh) {
    const int eo = i >= g.nh ? 1 : 0, oe = 1 - eo, s = i - eo * g.nh;
    const Coord X = site_coord(eo, s, g.hx, g.nxy, g.dhx, g.dnxy);
    const int L[3] = {g.L1, g.L2, g.L3};
    int up[3];
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      int c[3] = {X.x, X.y, X.z};
      c[mu] = wrap(c[mu] + 1, L[mu]);
      up[mu] = site_index(c[0], c[1], c[2], g.hx, g.nxy);
    }
#pragma unroll
    for (int mu = 0; mu < 3; ++mu)
#pragma unroll
      for (int nu = mu + 1; nu < 3; ++nu) {
        su2<float> a = LinkIO<float>::ld(u, (size_t)(mu * 2 + eo) * g.ld + s);
        su2<float> b = LinkIO<float>::ld(u, (size_t)(nu * 2 + oe) * g.ld + up[mu]);
        su2<float> d = LinkIO<float>::ld(u, (size_t)(mu * 2 + oe) * g.ld + up[nu]);
        su2<float> e = LinkIO<float>::ld(u, (size_t)(nu * 2 + eo) * g.ld + s);
        v[0] += (double)nn(nn(a, b), dd(d, e)).a.re;
      }
  }
  block_reduce_store<1>(v, part + blockIdx.x);
}

// sums the partials in block order and writes the average to the caller
__global__ void __launch_bounds__(1024) noalloc_plaquette_sum(const double* part, int nblocks, double norm,
                                                             double* out) {
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v[0] += part[b];
  __shared__ double tot;
  block_reduce_store<1>(v, &tot);
  __syncthreads();
  if (threadIdx.x == 0) out[0] = tot * norm;
}

std::mutex g_na_mu;
double* g_na_scratch[256] = {nullptr};

}  // namespace
}  // namespace lce

extern "C" int lce_plaquette_noalloc(const float* u, long ld, int L1, int L2, int L3, double* plaq,
                                     void* stream) {
  using namespace lce;
  if (!u || !plaq) {
    set_thread_error("lce_plaquette_noalloc: null field or output pointer");
    return LCE_ERR_INVALID;
  }
  if (L1 < 2 || L2 < 2 || L3 < 2 || ((L1 | L2 | L3) & 1)) {
    set_thread_error("lce_plaquette_noalloc: lattice extents must be even and >= 2");
    return LCE_ERR_INVALID;
  }
  const long vol = (long)L1 * L2 * L3;
  if (vol > kNaMaxSites) {
    set_thread_error("lce_plaquette_noalloc: lattice volume " + std::to_string(vol) +
                     " exceeds the fixed scratch capacity of " + std::to_string(kNaMaxSites) +
                     " sites (256^3); use lce_plaquette on a context instead");
    return LCE_ERR_INVALID;
  }
  const int nh = (int)(vol / 2);
  if (ld < nh || (reinterpret_cast<uintptr_t>(u) & 15u)) {
    set_thread_error("lce_plaquette_noalloc: ld must be >= L1*L2*L3/2 and the field 16-byte aligned");
    return LCE_ERR_INVALID;
  }
  // Set-up, once per device with that device current: the host-side name of
  // the __device__ array is not a device address; ask the runtime for it.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 256) {
    set_thread_error(std::string("lce_plaquette_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return LCE_ERR_CUDA;
  }
  double* scratch;
  {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_scratch[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess || !p) {
        set_thread_error(std::string("lce_plaquette_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return LCE_ERR_CUDA;
      }
      g_na_scratch[dev] = static_cast<double*>(p);
    }
    scratch = g_na_scratch[dev];
  }
  NaGeom g;
  g.L1 = L1;
  g.L2 = L2;
  g.L3 = L3;
  g.hx = L1 / 2;
  g.nxy = L1 * L2 / 2;
  g.nh = nh;
  g.ld = ld;
  g.dhx = make_fastdiv((uint32_t)g.hx);
  g.dnxy = make_fastdiv((uint32_t)g.nxy);
  const int nb = ceil_div(vol, kNaBlock);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  noalloc_plaquette_partials<<<nb, kNaBlock, 0, s>>>(reinterpret_cast<const float4*>(u), g, scratch);
  noalloc_plaquette_sum<<<1, 1024, 0, s>>>(scratch, nb, 1.0 / (3.0 * (double)vol), plaq);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_thread_error(std::string("lce_plaquette_noalloc: launch: ") + cudaGetErrorString(e));
    return LCE_ERR_CUDA;
  }
  return LCE_OK;
}
