// lbm_verify.cu -- the -verify check on the device: the x-velocity slice and
// the Poiseuille error of the reference's KernelGetXSlice / KernelVerifiy
// (src/Kernel.c:456-625), computed where the PDFs live, so that a check of a
// large instance moves the nY x nZ slice to the host instead of the field.
//
// Pass 1 (one thread per slice cell): u_x = sum_i c_ix f_i + F/2 at x = nX/2,
// in the reference's summation order (E + NE + SE + TE + BE - W - NW - SW -
// TW - BW), from the logical PDFs in the instance's storage (FP64, or FP32 /
// FP16 deviations restored to w_i + delta_i in FP64 as the host mirror does);
// 0 at obstacles. Pass 2 (one block): the relative error of the profile
// through the channel centre against the analytic one, squared and summed
// over z with warp shuffles, then the square root.
#include <cuda_fp16.h>

#include "lbm_kernels.cuh"

namespace lbm {

// Logical PDF `d` of element `e` in storage `storage` (the FP64 value the
// host mirror holds).
__device__ __forceinline__ double logical_pdf(const void* f, int storage, unsigned long long e, int d) {
  if (storage == kStoreF64) return static_cast<const double*>(f)[e];
  const double w = d == DC ? 1.0 / 3.0 : ((cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
  if (storage == kStoreF32) return w + static_cast<double>(static_cast<const float*>(f)[e]);
  const double scale = d == DC ? 32768.0 : ((cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 1 ? 262144.0 : 524288.0);
  return w + static_cast<double>(__half2float(static_cast<const __half*>(f)[e])) / scale;
}

__global__ void k_verify_slice(const VerifyArgs a, double* slice) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nY * a.nZ) return;
  const long long b = a.base[i];
  if (b < 0) {
    slice[i] = 0.0;
    return;
  }
  double p[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d)
    p[d] = cx(d) != 0 ? logical_pdf(a.f, a.storage, static_cast<unsigned long long>(b + a.off[d]), d) : 0.0;
  double u = p[E] + p[NE] + p[SE] + p[TE] + p[BE] - p[W] - p[NW] - p[SW] - p[TW] - p[BW];
  u += 0.5 * a.xforce;
  slice[i] = u;
}

// Profile error (src/Kernel.c:547-616): at y = ym (and ym + 1 averaged when
// nY is even), for each z: analytic u_a = F (r_max^2 - r^2) / (2 nu) inside
// the channel, r = z - nY/2 + 1/2, r_max = nY/2 - 1; deviation sum of
// ((u_a - u_s) / u_a)^2 over the z with u_a != 0.
__global__ void __launch_bounds__(256) k_verify_error(const VerifyArgs a, const double* slice, double* out) {
  __shared__ double part[8];
  const int evenNy = a.nY % 2 == 0;
  const int ym = (a.nY - evenNy - 1) / 2;
  const double center = a.nY / 2.0;
  const double rmax = (double)a.nY / 2.0 - 1.0;
  const double r2max = rmax * rmax;
  double dev = 0.0;
  for (int z = threadIdx.x; z < a.nZ; z += blockDim.x) {
    const double r = z - center + 0.5;
    const double r2 = r * r;
    const double ua = r2 >= r2max ? 0.0 : a.xforce * (r2max - r2) / (2.0 * a.visc);
    const double us = evenNy ? (slice[ym * a.nZ + z] + slice[(ym + 1) * a.nZ + z]) / 2.0 : slice[ym * a.nZ + z];
    if (ua != 0.0) {
      const double rel = fabs(ua - us) / ua;
      dev += rel * rel;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dev += __shfl_down_sync(0xffffffffu, dev, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = dev;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
    out[0] = sqrt(s);
  }
}

void verify_device(const VerifyArgs& a, double* slice, double* err, cudaStream_t s) {
  const int n = a.nY * a.nZ;
  if (n > 0) k_verify_slice<<<(n + 255) / 256, 256, 0, s>>>(a, slice);
  k_verify_error<<<1, 256, 0, s>>>(a, slice, err);
}

}  // namespace lbm
