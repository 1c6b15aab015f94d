// lce_meas.cu -- device reductions for the measurements.
//
// slice_sums_kernel: one block per z slice sums, over both parities and in
// FP64, the quantities the reference accumulates per slice:
//   0..2   A_f                        f/correlator.f:58-59
//   3..11  per mu: Im a, Im b, -Re b  of U_f  (Im a and -i b, :61-74)
//   12     cos(4 |A|) on the un-fixed A     f/polyakov.f:52-55
//   13     |A|^2 on the un-fixed A          f/scalarcorr.f:48-51
// correlators_kernel then forms the periodic z autocorrelations of
// f/correlator.f:139-164, f/polyakov.f:100-108 and f/scalarcorr.f:96-104
// (all z = 0..L3-1, as the reference writes them) and the meas2a average.
#include "lce_internal.hpp"

namespace lce {

constexpr int kSliceQ = 14;

template <typename R>
__global__ void __launch_bounds__(256) slice_sums_kernel(const ChainDev* chp, double* slices) {
  const ChainDev& ch = *chp;
  const int z = blockIdx.x, nh = ch.nh, nxy = ch.nxy;
  const R* Af = reinterpret_cast<const R*>(ch.af);
  const R* A = reinterpret_cast<const R*>(ch.a);
  double v[kSliceQ];
#pragma unroll
  for (int q = 0; q < kSliceQ; ++q) v[q] = 0.0;
  for (int i = threadIdx.x; i < 2 * nxy; i += blockDim.x) {
    const int eo = i >= nxy ? 1 : 0;
    const int s = z * nxy + (i - eo * nxy);
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] += (double)__ldg(Af + ((size_t)(eo * 3 + k)) * nh + s);
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      su2<R> u = LinkIO<R>::ld(ch.uf, ((size_t)(mu * 2 + eo)) * nh + s);
      v[3 + 3 * mu] += (double)u.a.im;
      v[4 + 3 * mu] += (double)u.b.im;
      v[5 + 3 * mu] += -(double)u.b.re;
    }
    const R a1 = __ldg(A + ((size_t)(eo * 3 + 0)) * nh + s), a2 = __ldg(A + ((size_t)(eo * 3 + 1)) * nh + s),
            a3 = __ldg(A + ((size_t)(eo * 3 + 2)) * nh + s);
    const R r2 = a1 * a1 + a2 * a2 + a3 * a3;
    v[12] += (double)cos((R)4 * sqrt(r2));
    v[13] += (double)a1 * a1 + (double)a2 * a2 + (double)a3 * a3;
  }
  block_reduce_store<kSliceQ>(v, slices + (size_t)z * kSliceQ);
}

// out: corr_a[L3], corr_u[L3], corr_3[L3], pol_slice[L3], pol_corr[L3],
//      sc_slice[L3], sc_corr[L3], af[3], pol_mean2, sc_mean
__global__ void __launch_bounds__(256) correlators_kernel(const double* slices, int L1, int L2, int L3,
                                                          double* out) {
  extern __shared__ double sh[];  // [L3][kSliceQ], normalised by L1*L2
  const double norm = 1.0 / ((double)L1 * (double)L2);
  for (int i = threadIdx.x; i < L3 * kSliceQ; i += blockDim.x) sh[i] = slices[i] * norm;
  __syncthreads();
  double* corr_a = out;
  double* corr_u = out + L3;
  double* corr_3 = out + 2 * L3;
  double* pol_slice = out + 3 * L3;
  double* pol_corr = out + 4 * L3;
  double* sc_slice = out + 5 * L3;
  double* sc_corr = out + 6 * L3;
  double* tail = out + 7 * L3;
  for (int z = threadIdx.x; z < L3; z += blockDim.x) {
    double ca = 0, cu = 0, c3 = 0, cp = 0, cs = 0;
    for (int x0 = 0; x0 < L3; ++x0) {
      const double* p = sh + x0 * kSliceQ;
      const double* q = sh + ((x0 + z) % L3) * kSliceQ;
      ca += p[0] * q[0] + p[1] * q[1] + p[2] * q[2];
      // Re[s1 s1' + s2 conj(s2')], s1 = sum Im a (real), s2 = sum -i b
      cu += p[3] * q[3] + (p[4] * q[4] + p[5] * q[5]);
      cu += p[6] * q[6] + (p[7] * q[7] + p[8] * q[8]);
      c3 += p[9] * q[9] + (p[10] * q[10] + p[11] * q[11]);
      cp += p[12] * q[12];
      cs += p[13] * q[13];
    }
    corr_a[z] = ca / L3;
    corr_u[z] = cu / (L3 * 2.0);
    corr_3[z] = c3 / L3;
    pol_corr[z] = cp / L3;
    sc_corr[z] = cs / L3;
    pol_slice[z] = sh[z * kSliceQ + 12];
    sc_slice[z] = sh[z * kSliceQ + 13];
  }
  if (threadIdx.x == 0) {
    double af0 = 0, af1 = 0, af2 = 0, ps = 0, ss = 0;
    for (int z = 0; z < L3; ++z) {
      af0 += sh[z * kSliceQ + 0];
      af1 += sh[z * kSliceQ + 1];
      af2 += sh[z * kSliceQ + 2];
      ps += sh[z * kSliceQ + 12];
      ss += sh[z * kSliceQ + 13];
    }
    tail[0] = af0 / L3;
    tail[1] = af1 / L3;
    tail[2] = af2 / L3;
    tail[3] = (ps / L3) * (ps / L3);
    tail[4] = ss / L3;
  }
}

// plaquette 1/2 Re Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ over both parities
template <typename R>
__global__ void __launch_bounds__(256) plaquette_kernel(const ChainDev* chp, double* part) {
  const ChainDev& ch = *chp;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (i < 2 * ch.nh) {
    const int eo = i >= ch.nh ? 1 : 0, oe = 1 - eo, s = i - eo * ch.nh;
    const Coord X = site_coord(eo, s, ch.hx, ch.nxy, ch.dhx, ch.dnxy);
    const int L[3] = {ch.L1, ch.L2, ch.L3};
    int up[3];
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      int c[3] = {X.x, X.y, X.z};
      c[mu] = wrap(c[mu] + 1, L[mu]);
      up[mu] = site_index(c[0], c[1], c[2], ch.hx, ch.nxy);
    }
#pragma unroll
    for (int mu = 0; mu < 3; ++mu)
#pragma unroll
      for (int nu = mu + 1; nu < 3; ++nu) {
        su2<R> a = LinkIO<R>::ld(ch.u, ((size_t)(mu * 2 + eo)) * ch.nh + s);
        su2<R> b = LinkIO<R>::ld(ch.u, ((size_t)(nu * 2 + oe)) * ch.nh + up[mu]);
        su2<R> d = LinkIO<R>::ld(ch.u, ((size_t)(mu * 2 + oe)) * ch.nh + up[nu]);
        su2<R> e = LinkIO<R>::ld(ch.u, ((size_t)(nu * 2 + eo)) * ch.nh + s);
        v[0] += (double)nn(nn(a, b), dd(d, e)).a.re;
      }
  }
  block_reduce_store<1>(v, part + blockIdx.x);
}

// Landau functional: sum over links of U_f of c_mu Re a
template <typename R>
__global__ void __launch_bounds__(256) functional_kernel(const ChainDev* chp, double* part) {
  const ChainDev& ch = *chp;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (i < 2 * ch.nh) {
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      const double w = mu == 2 ? ch.alpha : 1.0;
      su2<R> u = LinkIO<R>::ld(ch.uf, (size_t)mu * 2 * ch.nh + i);
      v[0] += w * (double)u.a.re;
    }
  }
  block_reduce_store<1>(v, part + blockIdx.x);
}

template <typename R>
void launch_slice_sums(const ChainDev* ch, int L3, double* slices, cudaStream_t s) {
  slice_sums_kernel<R><<<L3, 256, 0, s>>>(ch, slices);
}
void launch_correlators(const double* slices, int L1, int L2, int L3, double* out, cudaStream_t s) {
  const size_t smem = (size_t)L3 * kSliceQ * sizeof(double);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(correlators_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  correlators_kernel<<<1, 256, smem, s>>>(slices, L1, L2, L3, out);
}
template <typename R>
void launch_plaquette(const ChainDev* ch, double* part, int nh, cudaStream_t s) {
  plaquette_kernel<R><<<ceil_div(2L * nh, 256), 256, 0, s>>>(ch, part);
}
template <typename R>
void launch_functional(const ChainDev* ch, double* part, int nh, cudaStream_t s) {
  functional_kernel<R><<<ceil_div(2L * nh, 256), 256, 0, s>>>(ch, part);
}

template void launch_slice_sums<float>(const ChainDev*, int, double*, cudaStream_t);
template void launch_slice_sums<double>(const ChainDev*, int, double*, cudaStream_t);
template void launch_plaquette<float>(const ChainDev*, double*, int, cudaStream_t);
template void launch_plaquette<double>(const ChainDev*, double*, int, cudaStream_t);
template void launch_functional<float>(const ChainDev*, double*, int, cudaStream_t);
template void launch_functional<double>(const ChainDev*, double*, int, cudaStream_t);

}  // namespace lce
