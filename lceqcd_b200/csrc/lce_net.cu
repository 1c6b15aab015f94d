// lce_net.cu -- learned warm start for Landau gauge fixing (no reference
// counterpart).
//
// A 3D convolutional network, 4 layers x 16 channels x 3^3 kernels, periodic
// boundaries, on the parity-split lattice (site i = eo*nh + s, the fields'
// order).  Inputs (16 channels): the 12 link components of U_f = U^G_prev and
// the 3 components of A_f, i.e. the configuration in the gauge of the previous
// measurement's converged transform G_prev.  Output: 4 channels, normalised
// to a unit quaternion Omega(x); the warm start is G = Omega G_prev.  Trained
// on (configuration in G_prev gauge, converged relative transform
// G_new G_prev^+) pairs recorded from the plain overrelaxed gauge fixing, with
// the loss 1 - Omega . T per site.
//
// Arithmetic: BF16 weights and activations, FP32 accumulation, on the tensor
// cores.  When L1 is a multiple of 128 all three contractions (forward, input
// gradient, weight gradient) run on tcgen05 with tensor-memory accumulators
// (conv_tc_kernel, wgrad_tc_kernel below); other extents use mma.sync.m16n8k16
// (bf16 x bf16 -> f32), which this paragraph describes.  A convolution is 27
// shifted 16x16 products: a warp owns 16 sites x 16 output channels (two
// m16n8 tiles), gathers the 16 neighbour rows of each offset straight into
// A fragments and takes the offset's weights (B) from shared memory.  The
// input gradient is the same kernel with the flipped, transposed weights; the
// weight gradient contracts over sites (M = out channel, N = in channel,
// K = 16 sites per step) into per-chunk partials summed in a fixed order.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lce_internal.hpp"

namespace lce {
namespace {

constexpr int kC = 16;            // channels (inputs padded to 16)
constexpr int kK = 27;            // kernel offsets
constexpr int kLayers = 4;
constexpr int kOut = 4;           // output channels used (quaternion)
constexpr int kWl = kK * kC * kC;  // weights per layer [k][co][ci]
constexpr int kPl = kWl + kC;      // + bias
constexpr int kNParam = kLayers * kPl;
constexpr int kConvWarps = 4;
constexpr int kChunk = 4096;       // sites per weight-gradient block

struct NetGeom {
  int L1, L2, L3, hx, nxy, nh;
  FastDiv dhx, dnxy;
};

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// flat index of the neighbour at offset (dx, dy, dz) of flat site i
__device__ __forceinline__ int nbr3(const NetGeom& g, int i, int dx, int dy, int dz) {
  const int eo = i >= g.nh ? 1 : 0, s = i - eo * g.nh;
  const Coord X = site_coord(eo, s, g.hx, g.nxy, g.dhx, g.dnxy);
  const int x = wrap(X.x + dx, g.L1), y = wrap(X.y + dy, g.L2), z = wrap(X.z + dz, g.L3);
  return ((eo + dx + dy + dz) & 1) * g.nh + site_index(x, y, z, g.hx, g.nxy);
}

// out[i][co] = act( bias[co] + sum_k sum_ci in[nbr_k(i)][ci] W[k][co][ci] ) (* mask)
// MODE 0: hidden layer (ReLU, BF16 out); 1: output layer (FP32 out, first 8
// channels); 2: input gradient (BF16 out times (mask_src > 0), no bias)
template <int MODE>
__global__ void __launch_bounds__(32 * kConvWarps) conv_kernel(const __nv_bfloat16* __restrict__ in,
                                                               const __nv_bfloat16* __restrict__ W,
                                                               const float* __restrict__ bias,
                                                               __nv_bfloat16* __restrict__ out16,
                                                               float* __restrict__ out32,
                                                               const __nv_bfloat16* __restrict__ mask_src, NetGeom g) {
  __shared__ uint32_t sw[kK * kC * kC / 2];  // W as bf16 pairs [k][co][ci/2]
  const uint32_t* W32 = reinterpret_cast<const uint32_t*>(W);
  for (int j = threadIdx.x; j < kK * kC * kC / 2; j += blockDim.x) sw[j] = W32[j];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gr = lane >> 2, tq = lane & 3;
  const int nsites = 2 * g.nh, ntiles = (nsites + 15) / 16;
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  for (int tile = blockIdx.x * kConvWarps + warp; tile < ntiles; tile += gridDim.x * kConvWarps) {
    const int r0 = tile * 16 + gr, r1 = r0 + 8;
    const bool v0 = r0 < nsites, v1 = r1 < nsites;
    float acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll 1
    for (int k = 0; k < kK; ++k) {
      const int dx = k / 9 - 1, dy = (k / 3) % 3 - 1, dz = k % 3 - 1;
      const int i0 = v0 ? nbr3(g, r0, dx, dy, dz) : 0, i1 = v1 ? nbr3(g, r1, dx, dy, dz) : 0;
      uint32_t a[4];
      a[0] = v0 ? __ldg(in32 + (size_t)i0 * 8 + tq) : 0u;
      a[1] = v1 ? __ldg(in32 + (size_t)i1 * 8 + tq) : 0u;
      a[2] = v0 ? __ldg(in32 + (size_t)i0 * 8 + tq + 4) : 0u;
      a[3] = v1 ? __ldg(in32 + (size_t)i1 * 8 + tq + 4) : 0u;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const uint32_t* wk = sw + (k * kC + 8 * j + gr) * (kC / 2);
        mma16816(acc[j], a, wk[tq], wk[tq + 4]);
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = 8 * j + 2 * tq;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = h ? r1 : r0;
        if (!(h ? v1 : v0)) continue;
        float x0 = acc[j][2 * h], x1 = acc[j][2 * h + 1];
        if (MODE != 2) {
          x0 += bias[c];
          x1 += bias[c + 1];
        }
        if (MODE == 0) {
          x0 = fmaxf(x0, 0.f);
          x1 = fmaxf(x1, 0.f);
          reinterpret_cast<uint32_t*>(out16)[(size_t)r * 8 + c / 2] =
              pack2(__float2bfloat16_rn(x0), __float2bfloat16_rn(x1));
        } else if (MODE == 1) {
          if (j == 0) {
            out32[(size_t)r * 8 + c] = x0;
            out32[(size_t)r * 8 + c + 1] = x1;
          }
        } else {
          const __nv_bfloat16* m = mask_src + (size_t)r * kC + c;
          if (!(__bfloat162float(m[0]) > 0.f)) x0 = 0.f;
          if (!(__bfloat162float(m[1]) > 0.f)) x1 = 0.f;
          reinterpret_cast<uint32_t*>(out16)[(size_t)r * 8 + c / 2] =
              pack2(__float2bfloat16_rn(x0), __float2bfloat16_rn(x1));
        }
      }
    }
  }
}

// ------------------------------------------------------------------ tcgen05 path
// The same convolution on the 5th-generation tensor cores when L1 is a
// multiple of 128.  A tile is 128 consecutive sites j = x0 .. x0+127 of one
// x-line (y, z).  Moving the x offset out of the operand,
//   P_dx[j][co] = sum_{(dy,dz)} sum_ci in[(j, y+dy, z+dz)][ci] W[dx,dy,dz][co][ci]
//   out[i][co]  = P_-1[i-1][co] + P_0[i][co] + P_+1[i+1][co],
// makes the tile one GEMM: M = 128 sites, K = 9 lines x 16 channels,
// N = 3 dx x 16 output channels -- 9 tcgen05.mma of M 128, N 48, K 16 (BF16
// in, FP32 accumulate in 48 tensor-memory columns) instead of 27 of N 16.
// The 9 (dy, dz) lines sit in shared memory as channel planes (channels 0-7
// and 8-15, 16-byte rows): the canonical K-major layout without swizzle
// (8-row core matrices of 128 B, the second K chunk one plane further); the
// weights, staged once per CTA, in the same layout with N = 48 rows per line.
// The epilogue reads each warp's 32 rows out of tensor memory and forms the
// x-shifted sum with warp shuffles; the rows across warp boundaries go
// through shared memory, and the two rows outside the tile (P_-1 at x0-1,
// P_+1 at x0+128) are computed on the CUDA cores from staged halo sites.
// CTAs are persistent (4 per SM) and loop over tiles.
constexpr int kTcRows = 128;                          // sites per tile
constexpr int kTcN = 3 * kC;                          // N: 3 dx x 16 output channels
constexpr int kTcActBytes = 18 * kTcRows * 16;        // 9 lines x 2 planes
constexpr int kTcWtBytes = 9 * 2 * kTcN * 16;         // 9 lines x 2 planes x 48 rows
constexpr int kTcHaloBytes = 2 * 9 * 2 * 16;          // x0-1 and x0+128: 9 lines x 2 planes
constexpr int kTcXchBytes = (2 * 4 + 2) * kC * 4;     // warp-boundary and edge rows (FP32)
constexpr int kTcSmem = kTcActBytes + kTcWtBytes + kTcHaloBytes + kTcXchBytes + 16;
constexpr int kTcCtasPerSm = 4;
static_assert(kTcCtasPerSm * (kTcSmem + 1024) <= 228 * 1024, "conv CTAs per SM");
constexpr unsigned kTcSpin = 1u << 24;                // mbarrier polls before giving up

// tcgen05.mma instruction descriptor: BF16 A and B (K-major), FP32 D, M 128, N 48
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((kTcN >> 3) << 17) | ((128u >> 4) << 24);

// shared-memory matrix descriptor, no swizzle: start address, leading-dimension
// byte offset (between the two K chunks), stride-dimension byte offset
// (between 8-row core matrices), all in 16 B units; version 1
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 16-byte asynchronous global -> shared copy (L2 only): a thread issues all of
// its staging copies before waiting once, instead of one load round trip each
__device__ __forceinline__ void cp16(void* dst_smem, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst_smem)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ bool tc_try_wait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(mbar), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase) {
  for (unsigned i = 0; i < kTcSpin; ++i)
    if (tc_try_wait(mbar, phase)) return true;
  return false;
}

// flat (parity-split) index of site (x, y, z), coordinates in range
__device__ __forceinline__ int tc_flat(const NetGeom& g, int x, int y, int z) {
  return ((x + y + z) & 1) * g.nh + site_index(x, y, z, g.hx, g.nxy);
}

// x-line tile t -> (x0, y, z)
__device__ __forceinline__ void tc_tile(const NetGeom& g, int t, int& x0, int& y, int& z) {
  const int segs = g.L1 >> 7;
  x0 = (t % segs) << 7;
  t /= segs;
  y = t % g.L2;
  z = t / g.L2;
}

template <int MODE>
__global__ void __launch_bounds__(128) conv_tc_kernel(const __nv_bfloat16* __restrict__ in,
                                                      const __nv_bfloat16* __restrict__ W,
                                                      const float* __restrict__ bias,
                                                      __nv_bfloat16* __restrict__ out16, float* __restrict__ out32,
                                                      const __nv_bfloat16* __restrict__ mask_src, NetGeom g,
                                                      unsigned* status) {
  extern __shared__ __align__(1024) uint8_t tc_sm[];
  uint8_t* act = tc_sm;
  uint8_t* wts = act + kTcActBytes;
  uint8_t* halo = wts + kTcWtBytes;                          // [side][line][plane] 16 B
  float* xch = reinterpret_cast<float*>(halo + kTcHaloBytes);  // [0..3] P_-1 of lane 31, [4..7] P_+1 of lane 0, [8] edge lo, [9] edge hi
  uint64_t* mbar = reinterpret_cast<uint64_t*>(xch + (2 * 4 + 2) * kC);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = (g.L1 >> 7) * g.L2 * g.L3;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(64)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights once per CTA: line s, plane c, row n = dx_index * 16 + o holds
  // inputs 8c .. 8c+7 of output o at offset k = dx_index * 9 + s
  const uint4* W4 = reinterpret_cast<const uint4*>(W);
  for (int e = tid; e < 9 * 2 * kTcN; e += blockDim.x) {
    const int sg = e / (2 * kTcN), c = (e / kTcN) & 1, n = e % kTcN;
    const int k = (n >> 4) * 9 + sg, o = n & 15;
    cp16(reinterpret_cast<uint4*>(wts) + e, W4 + (k * kC + o) * 2 + c);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint4* in4 = reinterpret_cast<const uint4*>(in);
  const __nv_bfloat16* wb = reinterpret_cast<const __nv_bfloat16*>(wts);
  const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(halo);
  uint32_t phase = 0;

  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int x0, y, z;
    tc_tile(g, t, x0, y, z);
    // line s = (dy, dz), plane c, row r = site x0 + r; halo sites x0-1, x0+128
#pragma unroll
    for (int sg = 0; sg < 9; ++sg) {
      const int yy = wrap(y + sg / 3 - 1, g.L2), zz = wrap(z + sg % 3 - 1, g.L3);
      const size_t f = (size_t)tc_flat(g, x0 + tid, yy, zz) * 2;
      cp16(reinterpret_cast<uint4*>(act) + (sg * 2) * kTcRows + tid, in4 + f);
      cp16(reinterpret_cast<uint4*>(act) + (sg * 2 + 1) * kTcRows + tid, in4 + f + 1);
    }
    if (tid < 36) {
      const int side = tid / 18, sg = (tid >> 1) % 9, c = tid & 1;
      const int yy = wrap(y + sg / 3 - 1, g.L2), zz = wrap(z + sg % 3 - 1, g.L3);
      const int xx = wrap(side ? x0 + kTcRows : x0 - 1, g.L1);
      cp16(reinterpret_cast<uint4*>(halo) + tid, in4 + (size_t)tc_flat(g, xx, yy, zz) * 2 + c);
    }
    cp_wait_all();
    // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (tid == 0) {
      const uint32_t a0 = smem_u32(act), b0 = smem_u32(wts);
#pragma unroll 1
      for (int sg = 0; sg < 9; ++sg) {
        const uint64_t ad = tc_desc(a0 + (sg * 2 * kTcRows) * 16, kTcRows * 16, 128);
        const uint64_t bd = tc_desc(b0 + (sg * 2 * kTcN) * 16, kTcN * 16, 128);
        const uint32_t acc = sg > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mbar))
                   : "memory");
    }
    if (warp == 1) {
      // the rows outside the tile on the CUDA cores: lanes 0-15 P_-1[x0-1][o],
      // lanes 16-31 P_+1[x0+128][o]
      const int side = lane >> 4, o = lane & 15, n = (side ? 2 : 0) * kC + o;
      float v = 0.f;
#pragma unroll 1
      for (int sg = 0; sg < 9; ++sg) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const __nv_bfloat16* xr = hb + ((side * 9 + sg) * 2 + c) * 8;
          const __nv_bfloat16* wr = wb + ((size_t)(sg * 2 + c) * kTcN + n) * 8;
#pragma unroll
          for (int q = 0; q < 8; ++q) v = fmaf(__bfloat162float(xr[q]), __bfloat162float(wr[q]), v);
        }
      }
      xch[(8 + side) * kC + o] = v;
    }
    const uint32_t ph = phase;
    phase ^= 1u;
    const bool done = tc_wait(smem_u32(mbar), ph);
    if (__syncthreads_or(!done)) {
      // record the failure, give the MMAs a second bounded wait, then stop
      if (!done) {
        if (lane == 0) atomicOr(status, 1u);
        tc_wait(smem_u32(mbar), ph);
      }
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // row j = 32 warp + lane: P_-1[j] (columns 0-15), P_0[j] (16-31), P_+1[j] (32-47)
    uint32_t vm[16], v0[16], vp[16];
    const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16);
#define LCE_TC_LD16(dst, col)                                                                                   \
  asm volatile(                                                                                                 \
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, " \
      "%15}, [%16];"                                                                                            \
      : "=r"(dst[0]), "=r"(dst[1]), "=r"(dst[2]), "=r"(dst[3]), "=r"(dst[4]), "=r"(dst[5]), "=r"(dst[6]),       \
        "=r"(dst[7]), "=r"(dst[8]), "=r"(dst[9]), "=r"(dst[10]), "=r"(dst[11]), "=r"(dst[12]), "=r"(dst[13]),   \
        "=r"(dst[14]), "=r"(dst[15])                                                                            \
      : "r"(ta + (col)))
    LCE_TC_LD16(vm, 0);
    LCE_TC_LD16(v0, 16);
    LCE_TC_LD16(vp, 32);
#undef LCE_TC_LD16
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    // rows across warp boundaries
    if (lane == 31) {
#pragma unroll
      for (int c = 0; c < kC; ++c) xch[warp * kC + c] = __uint_as_float(vm[c]);
    }
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < kC; ++c) xch[(4 + warp) * kC + c] = __uint_as_float(vp[c]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    const float* lo = lane == 0 ? (warp == 0 ? xch + 8 * kC : xch + (warp - 1) * kC) : nullptr;
    const float* hi = lane == 31 ? (warp == 3 ? xch + 9 * kC : xch + (4 + warp + 1) * kC) : nullptr;
    float o[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) {
      const float pm = __shfl_up_sync(0xffffffffu, __uint_as_float(vm[c]), 1);
      const float pp = __shfl_down_sync(0xffffffffu, __uint_as_float(vp[c]), 1);
      o[c] = (lo ? lo[c] : pm) + __uint_as_float(v0[c]) + (hi ? hi[c] : pp) + (MODE != 2 ? bias[c] : 0.f);
    }
    const int f = tc_flat(g, x0 + tid, y, z);
    if (MODE == 1) {
      float4* d = reinterpret_cast<float4*>(out32 + (size_t)f * 8);
      d[0] = make_float4(o[0], o[1], o[2], o[3]);
      d[1] = make_float4(o[4], o[5], o[6], o[7]);
    } else {
      if (MODE == 0) {
#pragma unroll
        for (int c = 0; c < kC; ++c) o[c] = fmaxf(o[c], 0.f);
      } else {
        const __nv_bfloat16* m = mask_src + (size_t)f * kC;
#pragma unroll
        for (int c = 0; c < kC; ++c)
          if (!(__bfloat162float(m[c]) > 0.f)) o[c] = 0.f;
      }
      uint4 w0, w1;
      w0.x = pack2(__float2bfloat16_rn(o[0]), __float2bfloat16_rn(o[1]));
      w0.y = pack2(__float2bfloat16_rn(o[2]), __float2bfloat16_rn(o[3]));
      w0.z = pack2(__float2bfloat16_rn(o[4]), __float2bfloat16_rn(o[5]));
      w0.w = pack2(__float2bfloat16_rn(o[6]), __float2bfloat16_rn(o[7]));
      w1.x = pack2(__float2bfloat16_rn(o[8]), __float2bfloat16_rn(o[9]));
      w1.y = pack2(__float2bfloat16_rn(o[10]), __float2bfloat16_rn(o[11]));
      w1.z = pack2(__float2bfloat16_rn(o[12]), __float2bfloat16_rn(o[13]));
      w1.w = pack2(__float2bfloat16_rn(o[14]), __float2bfloat16_rn(o[15]));
      uint4* d = reinterpret_cast<uint4*>(out16) + (size_t)f * 2;
      d[0] = w0;
      d[1] = w1;
    }
    // the exchange rows, the staged tile and the accumulator are reused by the next tile
    __syncthreads();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
  }
}

// ------------------------------------------------------------------ tcgen05 weight gradient
// gW[k][co][ci] = sum_i gz[i][co] x[i + d_k][ci], d_k = (dx, dy, dz), when L1
// is a multiple of 128.  Substituting j = i + dx e_x turns every x offset into
// a shift of gz: gW = sum_j x[j + (0, dy, dz)][ci] gz[j - dx e_x][co].  A tile
// is 128 consecutive sites j of one x-line; a CTA (at most 4 per SM, each with
// 128 tensor-memory columns) loops over tiles and accumulates in tensor
// memory:
//   A (M 128 = 8 (dy, dz) lines x 16 ci, K = 128 sites), MN-major: the 9 lines
//     of x staged as 18 channel planes of 128 rows (16 B each); M groups of 8
//     channels are one plane apart.  M = 128 covers lines 0-7; lines 1-8 form
//     the second accumulator, of which only line 8's 16 rows are used;
//   B (K = 128 sites, N 48 = 3 dx x 16 co), MN-major: gz staged three times,
//     shifted by -dx, as 6 channel planes of 128 rows;
//   2 accumulators x 48 FP32 columns, 8 K steps of 16 sites: 16 MMAs per tile.
// The partial sums of each CTA go to part[k][cta][co][ci] (bias: sum of gz)
// and are reduced in a fixed order by wgrad_sum_kernel.
constexpr int kTgRows = 128;                            // sites per tile
constexpr int kTgActBytes = 18 * kTgRows * 16;          // 9 lines x 2 planes
constexpr int kTgGzBytes = 6 * kTgRows * 16;            // 3 shifts x 2 planes
constexpr int kTgSmem = 52 * 1024;  // padded so that at most 4 CTAs (4 x 128 columns) share an SM
static_assert(kTgActBytes + kTgGzBytes + 16 + 16 + 8 * kC * 4 <= kTgSmem, "wgrad shared memory");
constexpr int kTgMaxCtasPerSm = 4;
// BF16 A and B, both MN-major, FP32 D, M 128, N 48
constexpr uint32_t kTgIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((48u >> 3) << 17) | ((128u >> 4) << 24);

__global__ void __launch_bounds__(128) wgrad_tc_kernel(const __nv_bfloat16* __restrict__ gz,
                                                       const __nv_bfloat16* __restrict__ x, float* __restrict__ part,
                                                       int nchunk, NetGeom g, unsigned* status) {
  extern __shared__ __align__(1024) uint8_t tg_sm[];
  uint8_t* act = tg_sm;
  uint8_t* gzs = tg_sm + kTgActBytes;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(gzs + kTgGzBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  float* bred = reinterpret_cast<float*>(tslot + 4);  // [8][16]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int segs = g.L1 >> 7, ntiles = segs * g.L2 * g.L3;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  const uint4* x4 = reinterpret_cast<const uint4*>(x);
  const uint4* gz4 = reinterpret_cast<const uint4*>(gz);
  const int bco = tid & 15, brow = tid >> 4;  // bias: channel, row group
  float bsum = 0.f;
  uint32_t phase = 0;
  bool ok = true;
  int ndone = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int x0 = (t % segs) << 7, y = (t / segs) % g.L2, z = (t / segs) / g.L2;
    // x: line (dy, dz) = seg, plane c, row r = site x0 + r
#pragma unroll
    for (int seg = 0; seg < 9; ++seg) {
      const int yy = wrap(y + seg / 3 - 1, g.L2), zz = wrap(z + seg % 3 - 1, g.L3);
      const int f = tc_flat(g, x0 + tid, yy, zz);
      cp16(reinterpret_cast<uint4*>(act) + (seg * 2) * kTgRows + tid, x4 + (size_t)f * 2);
      cp16(reinterpret_cast<uint4*>(act) + (seg * 2 + 1) * kTgRows + tid, x4 + (size_t)f * 2 + 1);
    }
    // gz: shift s = dx + 1, plane c, row r = site x0 + r - dx
#pragma unroll
    for (int sh = 0; sh < 3; ++sh) {
      const int f = tc_flat(g, wrap(x0 + tid - (sh - 1), g.L1), y, z);
      cp16(reinterpret_cast<uint4*>(gzs) + (sh * 2) * kTgRows + tid, gz4 + (size_t)f * 2);
      cp16(reinterpret_cast<uint4*>(gzs) + (sh * 2 + 1) * kTgRows + tid, gz4 + (size_t)f * 2 + 1);
    }
    cp_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t a0 = smem_u32(act), b0 = smem_u32(gzs);
#pragma unroll 1
      for (int kk = 0; kk < kTgRows / 16; ++kk) {
        const uint64_t bd = tc_desc(b0 + kk * 16 * 16, 128, kTgRows * 16);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint64_t ad = tc_desc(a0 + ((2 * h) * kTgRows + kk * 16) * 16, 128, kTgRows * 16);
          const uint32_t acc = (ndone > 0 || kk > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
              ::"r"(tmem + (uint32_t)(h * 48)), "l"(ad), "l"(bd), "r"(kTgIdesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                   : "memory");
    }
    // bias gradient from the unshifted gz planes (generic reads beside the MMAs)
    {
      const __nv_bfloat16* p = reinterpret_cast<const __nv_bfloat16*>(gzs) + (size_t)(2 + (bco >> 3)) * kTgRows * 8;
#pragma unroll
      for (int j = 0; j < 16; ++j) bsum += __bfloat162float(p[(brow + 8 * j) * 8 + (bco & 7)]);
    }
    const uint32_t ph = phase;
    phase ^= 1u;
    const bool done = tc_wait(smem_u32(mbar), ph);
    ++ndone;
    if (__syncthreads_or(!done)) {
      // record the failure, give the MMAs a second bounded wait, then stop
      if (!done) {
        if (lane == 0) atomicOr(status, 1u);
        tc_wait(smem_u32(mbar), ph);
      }
      ok = false;
      break;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  // epilogue: warp w reads tensor-memory lanes 32w .. 32w+31 (M rows)
  const int m = warp * 32 + lane, ci = m & 15;
  const bool valid = ok && ndone > 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (h == 1 && warp != 3) continue;  // second accumulator: only line 8 (rows 112-127)
#pragma unroll
    for (int sh = 0; sh < 3; ++sh) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * 48 + sh * 16)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int seg = h + (m >> 4);
      if (h == 0 || m >= 112) {
        const int k = sh * 9 + seg;
        float* d = part + ((size_t)k * nchunk + blockIdx.x) * kC * kC + ci;
#pragma unroll
        for (int co = 0; co < kC; ++co) d[co * kC] = valid ? __uint_as_float(v[co]) : 0.f;
      }
    }
  }
  bred[brow * kC + bco] = bsum;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid < kC) {
    float b = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) b += bred[q * kC + tid];
    part[(size_t)kK * nchunk * kC * kC + (size_t)blockIdx.x * kC + tid] = valid ? b : 0.f;
  }
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
  }
}

// partial[k][chunk][co][ci] = sum over the chunk's sites of gz[i][co] x[nbr_k(i)][ci]
__global__ void __launch_bounds__(128) wgrad_kernel(const __nv_bfloat16* __restrict__ gz,
                                                    const __nv_bfloat16* __restrict__ x, float* __restrict__ part,
                                                    int nchunk, NetGeom g) {
  const int chunk = blockIdx.x, k = blockIdx.y;
  const int dx = k / 9 - 1, dy = (k / 3) % 3 - 1, dz = k % 3 - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gr = lane >> 2, tq = lane & 3;
  const int nsites = 2 * g.nh;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
  float acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
  const int base = chunk * kChunk + warp * (kChunk / 4);
  for (int s0 = base; s0 < base + kChunk / 4 && s0 < nsites; s0 += 16) {
    const int sa = s0 + 2 * tq, sb = sa + 1, sc = sa + 8, sd = sa + 9;
    auto gzv = [&](int s, int co) { return s < nsites ? gz[(size_t)s * kC + co] : zero; };
    uint32_t a[4];
    a[0] = pack2(gzv(sa, gr), gzv(sb, gr));
    a[1] = pack2(gzv(sa, gr + 8), gzv(sb, gr + 8));
    a[2] = pack2(gzv(sc, gr), gzv(sd, gr));
    a[3] = pack2(gzv(sc, gr + 8), gzv(sd, gr + 8));
    const int na = sa < nsites ? nbr3(g, sa, dx, dy, dz) : -1, nb = sb < nsites ? nbr3(g, sb, dx, dy, dz) : -1;
    const int nc = sc < nsites ? nbr3(g, sc, dx, dy, dz) : -1, nd = sd < nsites ? nbr3(g, sd, dx, dy, dz) : -1;
    auto xv = [&](int n, int ci) { return n >= 0 ? x[(size_t)n * kC + ci] : zero; };
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int ci = 8 * j + gr;
      mma16816(acc[j], a, pack2(xv(na, ci), xv(nb, ci)), pack2(xv(nc, ci), xv(nd, ci)));
    }
  }
  __shared__ float red[4][kC * kC];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    red[warp][gr * kC + 8 * j + 2 * tq] = acc[j][0];
    red[warp][gr * kC + 8 * j + 2 * tq + 1] = acc[j][1];
    red[warp][(gr + 8) * kC + 8 * j + 2 * tq] = acc[j][2];
    red[warp][(gr + 8) * kC + 8 * j + 2 * tq + 1] = acc[j][3];
  }
  if (k == 0) {
    // bias partial of the chunk: bpart[chunk][co] = sum_i gz[i][co]
    float b = 0.f;
    const int co = threadIdx.x & 15, grp = threadIdx.x >> 4;  // 8 groups
    for (int s = chunk * kChunk + grp; s < (chunk + 1) * kChunk && s < nsites; s += 8)
      b += __bfloat162float(gz[(size_t)s * kC + co]);
    __shared__ float bred[8][kC];
    bred[grp][co] = b;
    __syncthreads();
    if (threadIdx.x < kC) {
      float t = 0.f;
      for (int q = 0; q < 8; ++q) t += bred[q][threadIdx.x];
      part[(size_t)kK * nchunk * kC * kC + (size_t)chunk * kC + threadIdx.x] = t;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kC * kC; e += blockDim.x)
    part[((size_t)k * nchunk + chunk) * kC * kC + e] = red[0][e] + red[1][e] + red[2][e] + red[3][e];
}

// grad W[k][co][ci] = sum over chunks of part (blocks 0..26); grad b[co]
// (block 27) -- fixed summation order, so the gradient is deterministic
__global__ void wgrad_sum_kernel(const float* part, int nchunk, float* gW) {
  const int k = blockIdx.x, e = threadIdx.x;  // 256 threads
  float s = 0.f;
  if (k < kK) {
    for (int c = 0; c < nchunk; ++c) s += part[((size_t)k * nchunk + c) * kC * kC + e];
    gW[(size_t)k * kC * kC + e] = s;
  } else if (e < kC) {
    const float* bp = part + (size_t)kK * nchunk * kC * kC;
    for (int c = 0; c < nchunk; ++c) s += bp[(size_t)c * kC + e];
    gW[(size_t)kK * kC * kC + e] = s;
  }
}

// loss 1 - q . t per site, q = o/|o|; gz = dL/do = -(t - (q.t) q) / (|o| N)
__global__ void loss_kernel(const float* out, const float* target, int nsites, __nv_bfloat16* gz, double* part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l[1] = {0.0};
  if (i < nsites) {
    const float* o = out + (size_t)i * 8;
    const float* t = target + (size_t)i * 4;
    const float n = sqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + o[3] * o[3]) + 1e-12f;
    float q[4], qt = 0.f;
    for (int c = 0; c < 4; ++c) {
      q[c] = o[c] / n;
      qt += q[c] * t[c];
    }
    l[0] = 1.0 - qt;
    const float sc = -1.0f / (n * (float)nsites);
    uint32_t* gz32 = reinterpret_cast<uint32_t*>(gz) + (size_t)i * 8;
    gz32[0] = pack2(__float2bfloat16_rn(sc * (t[0] - qt * q[0])), __float2bfloat16_rn(sc * (t[1] - qt * q[1])));
    gz32[1] = pack2(__float2bfloat16_rn(sc * (t[2] - qt * q[2])), __float2bfloat16_rn(sc * (t[3] - qt * q[3])));
    for (int w = 2; w < 8; ++w) gz32[w] = 0u;
  }
  block_reduce_store<1>(l, part + blockIdx.x);
}

// W16 = bf16(W32), WT16[k'][ci][co] = bf16(W32[26-k'][co][ci]); output-layer
// rows co >= kOut and their biases are kept at zero
__global__ void refresh_kernel(float* w32, __nv_bfloat16* w16, __nv_bfloat16* wt16) {
  const int l = blockIdx.x;
  float* W = w32 + (size_t)l * kPl;
  for (int e = threadIdx.x; e < kWl; e += blockDim.x) {
    const int k = e / (kC * kC), co = (e / kC) % kC, ci = e % kC;
    if (l == kLayers - 1 && co >= kOut) W[e] = 0.f;
    w16[(size_t)l * kWl + e] = __float2bfloat16_rn(W[e]);
    wt16[(size_t)l * kWl + ((size_t)(kK - 1 - k) * kC + ci) * kC + co] = __float2bfloat16_rn(W[e]);
  }
  if (l == kLayers - 1 && threadIdx.x >= kOut && threadIdx.x < kC) W[kWl + threadIdx.x] = 0.f;
}

__global__ void adam_kernel(float* w, float* m, float* v, const float* grad, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// features: 12 link components of U_f and 3 of A_f per site (channel 15 = 0)
template <typename R>
__global__ void features_kernel(const ChainDev* chp, __nv_bfloat16* feat) {
  const ChainDev& ch = *chp;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * ch.nh) return;
  const int eo = i >= ch.nh ? 1 : 0, s = i - eo * ch.nh, nh = ch.nh;
  float f[kC];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    const su2<R> u = LinkIO<R>::ld(ch.uf, ((size_t)(mu * 2 + eo)) * nh + s);
    f[4 * mu + 0] = (float)u.a.re;
    f[4 * mu + 1] = (float)u.a.im;
    f[4 * mu + 2] = (float)u.b.re;
    f[4 * mu + 3] = (float)u.b.im;
  }
  const R* Af = reinterpret_cast<const R*>(ch.af);
#pragma unroll
  for (int k = 0; k < 3; ++k) f[12 + k] = (float)Af[((size_t)(eo * 3 + k)) * nh + s];
  f[15] = 0.f;
  uint32_t* o = reinterpret_cast<uint32_t*>(feat) + (size_t)i * 8;
#pragma unroll
  for (int w = 0; w < 8; ++w) o[w] = pack2(__float2bfloat16_rn(f[2 * w]), __float2bfloat16_rn(f[2 * w + 1]));
}

// G(x) = (o/|o|) G_prev(x) with o the network output as a first row
template <typename R>
__global__ void compose_kernel(const float* out, const void* gprev, void* g, int nsites) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsites) return;
  const float* o = out + (size_t)i * 8;
  const float n = rsqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + o[3] * o[3] + 1e-30f);
  const su2<R> om{{(R)(o[0] * n), (R)(o[1] * n)}, {(R)(o[2] * n), (R)(o[3] * n)}};
  LinkIO<R>::st(g, i, unitarise64(nn(om, LinkIO<R>::ld(gprev, i))));
}

// T(x) = G_new(x) G_prev(x)^+ as a quaternion target
template <typename R>
__global__ void target_kernel(const void* gnew, const void* gprev, float* t, int nsites) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsites) return;
  const su2<R> r = nd(LinkIO<R>::ld(gnew, i), LinkIO<R>::ld(gprev, i));
  t[(size_t)i * 4 + 0] = (float)r.a.re;
  t[(size_t)i * 4 + 1] = (float)r.a.im;
  t[(size_t)i * 4 + 2] = (float)r.b.re;
  t[(size_t)i * 4 + 3] = (float)r.b.im;
}

__global__ void init_params_kernel(float* w, uint32_t k0, uint32_t k1) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNParam; i += gridDim.x * blockDim.x) {
    const int l = i / kPl, e = i % kPl;
    uint32_t c[4] = {(uint32_t)i, 0x4e4554u, 0u, 0u};
    philox4x32_10(c, k0, k1);
    const float u1 = u01(c[0]), u2 = u01(c[1]);
    const float gauss = sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
    float v;
    if (e >= kWl) v = (l == kLayers - 1 && e - kWl == 0) ? 1.f : 0.f;       // output bias: identity
    else if (l == kLayers - 1) v = 0.f;  // output = bias: the untrained network predicts Omega = 1
    else v = gauss * sqrtf(2.f / (kK * kC));                                   // He
    w[i] = v;
  }
}

NetGeom make_geom(int L1, int L2, int L3) {
  NetGeom g;
  g.L1 = L1;
  g.L2 = L2;
  g.L3 = L3;
  g.hx = L1 / 2;
  g.nxy = L1 * L2 / 2;
  g.nh = g.nxy * L3;
  g.dhx = make_fastdiv((uint32_t)g.hx);
  g.dnxy = make_fastdiv((uint32_t)g.nxy);
  return g;
}

}  // namespace
}  // namespace lce

using namespace lce;

struct lce_net {
  int device = 0;
  cudaStream_t stream = nullptr;
  float *w32 = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  __nv_bfloat16 *w16 = nullptr, *wt16 = nullptr;
  int step = 0;
  // work buffers for the current volume
  long nsites = 0;
  __nv_bfloat16* act[kLayers] = {nullptr, nullptr, nullptr, nullptr};
  __nv_bfloat16 *gz = nullptr, *gy = nullptr;
  float* out = nullptr;
  float* target = nullptr;
  double* part = nullptr;
  float* wpart = nullptr;
  int nchunk = 0;
  int tg_grid = 0;   // CTAs of the tcgen05 weight gradient
  unsigned* flag = nullptr;  // set on the device when a tensor-core wait gave up
  // recorded training pairs
  struct Pair {
    NetGeom g;
    __nv_bfloat16* feat;
    float* target;
  };
  std::vector<Pair> pairs;
  std::string err;
};

namespace {

int net_fail(lce_net* n, int code, const std::string& m) {
  if (n) n->err = m;
  set_thread_error(m);
  return code;
}
#define NCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return net_fail(n, LCE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// CTAs of the tcgen05 weight gradient: 4 per SM, all resident (4 x 53 KB of
// shared memory; tensor memory: 4 x 128 columns).  The runtime's occupancy
// query reported 1 per SM for this kernel where the launch itself holds 4.
static_assert(kTgMaxCtasPerSm * (kTgSmem + 1024) <= 228 * 1024, "wgrad CTAs per SM");
static_assert(kTcCtasPerSm == kTgMaxCtasPerSm, "the convolution uses the weight gradient's grid");
template <typename K>
void tc_attributes(K kernel, int smem) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  // all of the unified L1 / shared memory as shared memory
  cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
}

// the grid of the persistent tcgen05 kernels; the first call for a network
// (on its device) also sets their shared-memory attributes there
int wgrad_tc_grid(lce_net* n) {
  if (n->tg_grid > 0) return n->tg_grid;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, n->device);
  tc_attributes(wgrad_tc_kernel, kTgSmem);
  tc_attributes(conv_tc_kernel<0>, kTcSmem);
  tc_attributes(conv_tc_kernel<1>, kTcSmem);
  tc_attributes(conv_tc_kernel<2>, kTcSmem);
  n->tg_grid = std::max(1, nsm) * kTgMaxCtasPerSm;
  return n->tg_grid;
}

int net_buffers(lce_net* n, long nsites) {
  if (n->nsites == nsites) return LCE_OK;
  // the buffers may still be in use by work queued on a context's stream
  NCK(cudaDeviceSynchronize());
  n->nsites = 0;
  for (auto& a : n->act) {
    if (a) cudaFree(a);
    a = nullptr;
  }
  void* ptrs[] = {n->gz, n->gy, n->out, n->target, n->part, n->wpart};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  n->gz = n->gy = nullptr;
  n->out = n->target = nullptr;
  n->part = nullptr;
  n->wpart = nullptr;
  for (auto& a : n->act) NCK(cudaMalloc(&a, (size_t)nsites * kC * sizeof(__nv_bfloat16)));
  NCK(cudaMalloc(&n->gz, (size_t)nsites * kC * sizeof(__nv_bfloat16)));
  NCK(cudaMalloc(&n->gy, (size_t)nsites * kC * sizeof(__nv_bfloat16)));
  NCK(cudaMalloc(&n->out, (size_t)nsites * 8 * sizeof(float)));
  NCK(cudaMalloc(&n->target, (size_t)nsites * 4 * sizeof(float)));
  NCK(cudaMalloc(&n->part, (size_t)ceil_div(nsites, 256) * sizeof(double) + 64));
  n->nchunk = ceil_div(nsites, kChunk);
  // partial sums of the mma.sync (per chunk) or the tcgen05 (per CTA) weight gradient
  const size_t nparts = std::max(n->nchunk, wgrad_tc_grid(n));
  NCK(cudaMalloc(&n->wpart, ((size_t)kK * nparts * kC * kC + nparts * kC) * sizeof(float)));
  n->nsites = nsites;
  return LCE_OK;
}

int conv_grid(long nsites) {
  const int ntiles = ceil_div(nsites, 16);
  return std::max(1, std::min(ceil_div(ntiles, kConvWarps), 148 * 8));
}

// forward through all layers from act[0]; output in n->out
// one convolution: the tcgen05 kernel when L1 is a multiple of 128, else the
// mma.sync kernel
template <int MODE>
void launch_conv(lce_net* n, const __nv_bfloat16* in, const __nv_bfloat16* W, const float* bias,
                 __nv_bfloat16* out16, float* out32, const __nv_bfloat16* mask, const NetGeom& g, cudaStream_t s) {
  if (g.L1 % 128 == 0) {
    // persistent CTAs, 4 per SM, like the weight gradient
    const int grid = std::min(wgrad_tc_grid(n), (g.L1 / 128) * g.L2 * g.L3);
    conv_tc_kernel<MODE><<<grid, 128, kTcSmem, s>>>(in, W, bias, out16, out32, mask, g, n->flag);
  } else {
    conv_kernel<MODE><<<conv_grid(2L * g.nh), 32 * kConvWarps, 0, s>>>(in, W, bias, out16, out32, mask, g);
  }
}

void net_forward(lce_net* n, const NetGeom& g, cudaStream_t s) {
  for (int l = 0; l < kLayers; ++l) {
    const __nv_bfloat16* W = n->w16 + (size_t)l * kWl;
    const float* b = n->w32 + (size_t)l * kPl + kWl;
    if (l < kLayers - 1) launch_conv<0>(n, n->act[l], W, b, n->act[l + 1], nullptr, nullptr, g, s);
    else launch_conv<1>(n, n->act[l], W, b, nullptr, n->out, nullptr, g, s);
  }
}

// loss and gradients (into n->grad) for act[0] and n->target; returns the
// loss through part (device) -- caller sums
void net_backward(lce_net* n, const NetGeom& g, cudaStream_t s) {
  const long ns = 2L * g.nh;
  loss_kernel<<<ceil_div(ns, 256), 256, 0, s>>>(n->out, n->target, (int)ns, n->gz, n->part);
  __nv_bfloat16* gz = n->gz;   // gradient at the output of layer l (pre-activation)
  __nv_bfloat16* gy = n->gy;
  for (int l = kLayers - 1; l >= 0; --l) {
    float* gW = n->grad + (size_t)l * kPl;
    if (g.L1 % 128 == 0) {
      const int grid = std::min(wgrad_tc_grid(n), (g.L1 / 128) * g.L2 * g.L3);
      wgrad_tc_kernel<<<grid, 128, kTgSmem, s>>>(gz, n->act[l], n->wpart, grid, g, n->flag);
      wgrad_sum_kernel<<<kK + 1, kC * kC, 0, s>>>(n->wpart, grid, gW);
    } else {
      wgrad_kernel<<<dim3(n->nchunk, kK), 128, 0, s>>>(gz, n->act[l], n->wpart, n->nchunk, g);
      wgrad_sum_kernel<<<kK + 1, kC * kC, 0, s>>>(n->wpart, n->nchunk, gW);
    }
    if (l > 0) {
      // gradient w.r.t. act[l] = conv_T(gz, W_l), times relu'(layer l-1) = (act[l] > 0)
      launch_conv<2>(n, gz, n->wt16 + (size_t)l * kWl, nullptr, gy, nullptr, n->act[l], g, s);
      __nv_bfloat16* t = gz;
      gz = gy;
      gy = t;
    }
  }
}

void net_refresh(lce_net* n, cudaStream_t s) { refresh_kernel<<<kLayers, 256, 0, s>>>(n->w32, n->w16, n->wt16); }

}  // namespace

// the device flag of the tensor-core kernels (a wait that gave up), read and
// cleared; the work of the network's stream and of the caller's stream must
// have completed
int lce::net_status(lce_net* n) {
  unsigned f = 0;
  NCK(cudaMemcpy(&f, n->flag, sizeof(f), cudaMemcpyDeviceToHost));
  if (!f) return LCE_OK;
  NCK(cudaMemset(n->flag, 0, sizeof(unsigned)));
  return net_fail(n, LCE_ERR_CUDA, "warm-start network: a tensor-core completion wait timed out");
}

namespace {

}  // namespace

extern "C" {

lce_net* lce_net_create(int device, unsigned long long seed) {
  DeviceScope ds_(device);
  lce_net* n = new lce_net();
  n->device = device;
  auto bad = [&](cudaError_t e, const char* w) -> lce_net* {
    set_thread_error(std::string("lce_net_create: ") + w + ": " + cudaGetErrorString(e));
    lce_net_destroy(n);
    return nullptr;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return bad(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking)) != cudaSuccess) return bad(e, "stream");
  if ((e = cudaMalloc(&n->w32, sizeof(float) * kNParam)) != cudaSuccess) return bad(e, "cudaMalloc");
  if ((e = cudaMalloc(&n->m, sizeof(float) * kNParam)) != cudaSuccess) return bad(e, "cudaMalloc");
  if ((e = cudaMalloc(&n->v, sizeof(float) * kNParam)) != cudaSuccess) return bad(e, "cudaMalloc");
  if ((e = cudaMalloc(&n->grad, sizeof(float) * kNParam)) != cudaSuccess) return bad(e, "cudaMalloc");
  if ((e = cudaMalloc(&n->w16, sizeof(__nv_bfloat16) * kLayers * kWl)) != cudaSuccess) return bad(e, "cudaMalloc");
  if ((e = cudaMalloc(&n->wt16, sizeof(__nv_bfloat16) * kLayers * kWl)) != cudaSuccess) return bad(e, "cudaMalloc");
  if ((e = cudaMalloc(&n->flag, sizeof(unsigned))) != cudaSuccess) return bad(e, "cudaMalloc");
  cudaMemsetAsync(n->flag, 0, sizeof(unsigned), n->stream);
  cudaMemsetAsync(n->m, 0, sizeof(float) * kNParam, n->stream);
  cudaMemsetAsync(n->v, 0, sizeof(float) * kNParam, n->stream);
  init_params_kernel<<<64, 256, 0, n->stream>>>(n->w32, (uint32_t)seed, (uint32_t)(seed >> 32));
  net_refresh(n, n->stream);
  if ((e = cudaStreamSynchronize(n->stream)) != cudaSuccess) return bad(e, "init");
  return n;
}

void lce_net_destroy(lce_net* n) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n) return;
  cudaSetDevice(n->device);
  if (n->stream) cudaStreamSynchronize(n->stream);
  for (auto& p : n->pairs) {
    cudaFree(p.feat);
    cudaFree(p.target);
  }
  for (auto& a : n->act)
    if (a) cudaFree(a);
  void* ptrs[] = {n->w32, n->m, n->v, n->grad, n->w16, n->wt16, n->gz, n->gy, n->out, n->target, n->part, n->wpart,
                  n->flag};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
}

int lce_net_num_params(lce_net* n) { return n ? kNParam : LCE_ERR_INVALID; }

int lce_net_get_params(lce_net* n, float* w) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n || !w) return LCE_ERR_INVALID;
  NCK(cudaMemcpyAsync(w, n->w32, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, n->stream));
  NCK(cudaStreamSynchronize(n->stream));
  return LCE_OK;
}

int lce_net_set_params(lce_net* n, const float* w) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n || !w) return LCE_ERR_INVALID;
  NCK(cudaMemcpyAsync(n->w32, w, sizeof(float) * kNParam, cudaMemcpyHostToDevice, n->stream));
  net_refresh(n, n->stream);
  NCK(cudaStreamSynchronize(n->stream));
  return LCE_OK;
}

int lce_net_save(lce_net* n, const char* path) {
  DeviceScope ds_(n ? n->device : -1);
  std::vector<float> w(kNParam);
  int rc = lce_net_get_params(n, w.data());
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return net_fail(n, LCE_ERR_INVALID, std::string("lce_net_save: cannot open ") + path);
  const char magic[8] = {'L', 'C', 'E', 'N', 'E', 'T', '0', '1'};
  bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(w.data(), sizeof(float), w.size(), f) == w.size();
  ok = std::fclose(f) == 0 && ok;
  return ok ? LCE_OK : net_fail(n, LCE_ERR_INVALID, "lce_net_save: write failed");
}

int lce_net_load(lce_net* n, const char* path) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n || !path) return LCE_ERR_INVALID;
  FILE* f = std::fopen(path, "rb");
  if (!f) return net_fail(n, LCE_ERR_INVALID, std::string("lce_net_load: cannot open ") + path);
  char magic[8];
  std::vector<float> w(kNParam);
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "LCENET01", 8) == 0 &&
            std::fread(w.data(), sizeof(float), w.size(), f) == w.size();
  std::fclose(f);
  if (!ok) return net_fail(n, LCE_ERR_INVALID, "lce_net_load: not a network file of this format");
  return lce_net_set_params(n, w.data());
}

// forward, loss and gradients on caller data (no update): feat [2][nh][16]
// float (rounded to BF16 here), target [2][nh][4]; out [2][nh][4] and grad
// [nparam] may be NULL
int lce_net_eval(lce_net* n, int L1, int L2, int L3, const float* feat, const float* target, float* out, float* grad,
                 double* loss) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n || !feat || !target || L1 < 2 || L2 < 2 || L3 < 2 || ((L1 | L2 | L3) & 1)) return LCE_ERR_INVALID;
  const NetGeom g = make_geom(L1, L2, L3);
  const long ns = 2L * g.nh;
  int rc = net_buffers(n, ns);
  if (rc) return rc;
  std::vector<uint16_t> fb((size_t)ns * kC);
  for (size_t i = 0; i < fb.size(); ++i) fb[i] = __bfloat16_as_ushort(__float2bfloat16_rn(feat[i]));
  NCK(cudaMemcpyAsync(n->act[0], fb.data(), fb.size() * 2, cudaMemcpyHostToDevice, n->stream));
  NCK(cudaMemcpyAsync(n->target, target, sizeof(float) * ns * 4, cudaMemcpyHostToDevice, n->stream));
  net_forward(n, g, n->stream);
  net_backward(n, g, n->stream);
  NCK(cudaGetLastError());
  std::vector<double> lp(ceil_div(ns, 256));
  NCK(cudaMemcpyAsync(lp.data(), n->part, lp.size() * sizeof(double), cudaMemcpyDeviceToHost, n->stream));
  if (out) {
    std::vector<float> o((size_t)ns * 8);
    NCK(cudaMemcpyAsync(o.data(), n->out, o.size() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    for (long i = 0; i < ns; ++i)
      for (int c = 0; c < 4; ++c) out[i * 4 + c] = o[(size_t)i * 8 + c];
  }
  if (grad) NCK(cudaMemcpyAsync(grad, n->grad, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, n->stream));
  NCK(cudaStreamSynchronize(n->stream));
  double l = 0;
  for (double x : lp) l += x;
  if (loss) *loss = l / ns;
  if (int rc = lce::net_status(n)) return rc;
  return LCE_OK;
}

int lce_net_num_pairs(lce_net* n) { return n ? (int)n->pairs.size() : LCE_ERR_INVALID; }

int lce_net_clear_pairs(lce_net* n) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n) return LCE_ERR_INVALID;
  NCK(cudaStreamSynchronize(n->stream));
  for (auto& p : n->pairs) {
    cudaFree(p.feat);
    cudaFree(p.target);
  }
  n->pairs.clear();
  return LCE_OK;
}

// Adam over the recorded pairs, `epochs` passes in an order shuffled per epoch
int lce_net_train(lce_net* n, int epochs, double lr, double* mean_loss) {
  DeviceScope ds_(n ? n->device : -1);
  if (!n || epochs < 0 || n->pairs.empty()) return LCE_ERR_INVALID;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  std::vector<int> order(n->pairs.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  uint32_t rs = 0x12345u;
  double last_epoch = 0.0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (size_t i = order.size(); i > 1; --i) {
      rs = rs * 1664525u + 1013904223u;
      std::swap(order[i - 1], order[rs % i]);
    }
    double tot = 0.0;
    for (int idx : order) {
      const auto& p = n->pairs[idx];
      const long ns = 2L * p.g.nh;
      int rc = net_buffers(n, ns);
      if (rc) return rc;
      NCK(cudaMemcpyAsync(n->act[0], p.feat, (size_t)ns * kC * 2, cudaMemcpyDeviceToDevice, n->stream));
      NCK(cudaMemcpyAsync(n->target, p.target, (size_t)ns * 16, cudaMemcpyDeviceToDevice, n->stream));
      net_forward(n, p.g, n->stream);
      net_backward(n, p.g, n->stream);
      ++n->step;
      const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
      adam_kernel<<<64, 256, 0, n->stream>>>(n->w32, n->m, n->v, n->grad, kNParam, (float)lr, b1, b2, eps, c1, c2);
      net_refresh(n, n->stream);
      NCK(cudaGetLastError());
      std::vector<double> lp(ceil_div(ns, 256));
      NCK(cudaMemcpyAsync(lp.data(), n->part, lp.size() * sizeof(double), cudaMemcpyDeviceToHost, n->stream));
      NCK(cudaStreamSynchronize(n->stream));
      double l = 0;
      for (double x : lp) l += x;
      tot += l / ns;
    }
    last_epoch = tot / order.size();
  }
  if (mean_loss) *mean_loss = last_epoch;
  if (int rc = lce::net_status(n)) return rc;
  return LCE_OK;
}

}  // extern "C"

// ---- used by the gauge-fixing warm start in lce_capi.cu
namespace lce {

int net_features(lce_net* n, const ChainDev* chd, const ChainDev& ch, bool f64, cudaStream_t s) {
  const long ns = 2L * ch.nh;
  int rc = net_buffers(n, ns);
  if (rc) return rc;
  if (f64) features_kernel<double><<<ceil_div(ns, 256), 256, 0, s>>>(chd, n->act[0]);
  else features_kernel<float><<<ceil_div(ns, 256), 256, 0, s>>>(chd, n->act[0]);
  return cudaGetLastError() == cudaSuccess ? LCE_OK : LCE_ERR_CUDA;
}

void net_predict(lce_net* n, const ChainDev& ch, cudaStream_t s) {
  net_forward(n, make_geom(ch.L1, ch.L2, ch.L3), s);
}

// ch.g = Omega G_prev from the last net_predict
int net_compose(lce_net* n, const ChainDev& ch, const void* gprev, bool f64, cudaStream_t s) {
  const long ns = 2L * ch.nh;
  if (f64) compose_kernel<double><<<ceil_div(ns, 256), 256, 0, s>>>(n->out, gprev, ch.g, (int)ns);
  else compose_kernel<float><<<ceil_div(ns, 256), 256, 0, s>>>(n->out, gprev, ch.g, (int)ns);
  return cudaGetLastError() == cudaSuccess ? LCE_OK : LCE_ERR_CUDA;
}

int net_device(lce_net* n) { return n->device; }

// store (current features, T = G_new G_prev^+) as a training pair
int net_record(lce_net* n, const ChainDev& ch, const void* gprev, bool f64, cudaStream_t s) {
  const long ns = 2L * ch.nh;
  lce_net::Pair p;
  p.g = make_geom(ch.L1, ch.L2, ch.L3);
  if (cudaMalloc(&p.feat, (size_t)ns * kC * 2) != cudaSuccess) return LCE_ERR_NOMEM;
  if (cudaMalloc(&p.target, (size_t)ns * 16) != cudaSuccess) {
    cudaFree(p.feat);
    return LCE_ERR_NOMEM;
  }
  cudaMemcpyAsync(p.feat, n->act[0], (size_t)ns * kC * 2, cudaMemcpyDeviceToDevice, s);
  if (f64) target_kernel<double><<<ceil_div(ns, 256), 256, 0, s>>>(ch.g, gprev, p.target, (int)ns);
  else target_kernel<float><<<ceil_div(ns, 256), 256, 0, s>>>(ch.g, gprev, p.target, (int)ns);
  if (cudaGetLastError() != cudaSuccess) return LCE_ERR_CUDA;
  n->pairs.push_back(p);
  return LCE_OK;
}

}  // namespace lce
