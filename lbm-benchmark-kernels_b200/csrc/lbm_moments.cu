// lbm_moments.cu -- FP64 conservation sums of a list-layout PDF field on the
// GPU: total mass sum_n sum_i f_i and momentum sum_n sum_i c_i f_i over the
// fluid nodes (the quantities KernelDensity / KernelStatisticsAdv sum on the
// host through GetNode, src/Kernel.c:209-254,633-755).
//
// Two passes, both with a fixed reduction tree (so the result depends only on
// the field and nFluid, not on scheduling): pass 1, one block per tile of
// kListTile nodes, writes 4 partial sums per block to a scratch array; pass 2,
// one block, folds the partials into the 4 outputs.
// The entry point allocates the scratch (4 doubles per block) with cudaMalloc
// for each call.
#include "lbm_kernels.cuh"
#include "lbm_store.cuh"

namespace lbm {

constexpr int kMomentTile = kListTile;  // nodes per block in pass 1

__device__ __forceinline__ void node_moments(const double* f, long long nCells, int n, double& rho, double& jx,
                                             double& jy, double& jz) {
  double v[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) v[d] = f[d * nCells + n];
  rho = v[C] + v[N] + v[E] + v[S] + v[W] + v[NE] + v[SE] + v[SW] + v[NW] + v[T] + v[TN] + v[TE] + v[TS] + v[TW] +
        v[B] + v[BN] + v[BE] + v[BS] + v[BW];
  jx = v[E] + v[NE] + v[SE] + v[TE] + v[BE] - v[W] - v[NW] - v[SW] - v[TW] - v[BW];
  jy = v[N] + v[NE] + v[NW] + v[TN] + v[BN] - v[S] - v[SE] - v[SW] - v[TS] - v[BS];
  jz = v[T] + v[TE] + v[TW] + v[TN] + v[TS] - v[B] - v[BE] - v[BW] - v[BN] - v[BS];
}

// Sums 4 values over the block (blockDim.x == kMomentTile) with warp
// shuffles and one shared-memory round; the result is valid in thread 0.
__device__ __forceinline__ void block_sum4(double s[4]) {
  __shared__ double part[kMomentTile / 32][4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) part[warp][k] = s[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double acc = part[0][k];
      for (int w = 1; w < kMomentTile / 32; ++w) acc += part[w][k];
      s[k] = acc;
    }
  }
}

__global__ void __launch_bounds__(kMomentTile) k_moments_partial(const double* f, long long nCells, int nFluid,
                                                                 double* partials) {
  const int n = blockIdx.x * kMomentTile + threadIdx.x;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  if (n < nFluid) node_moments(f, nCells, n, s[0], s[1], s[2], s[3]);
  block_sum4(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) partials[blockIdx.x * 4 + k] = s[k];
}

__global__ void __launch_bounds__(kMomentTile) k_moments_final(const double* partials, int nBlocks, double* out) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nBlocks; b += kMomentTile)
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] += partials[b * 4 + k];
  block_sum4(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = s[k];
}

// Launchers shared by the entry points (declared in lbm_kernels.cuh).
int moment_blocks(int nFluid) { return nFluid > 0 ? (nFluid + kMomentTile - 1) / kMomentTile : 1; }

void moments_enqueue(const double* f, long long nCells, int nFluid, double* partials, double* out, cudaStream_t s) {
  const int nb = moment_blocks(nFluid);
  k_moments_partial<<<nb, kMomentTile, 0, s>>>(f, nCells, nFluid, partials);
  k_moments_final<<<1, kMomentTile, 0, s>>>(partials, nb, out);
}

// Reduced storage (FP32 or FP16 deviations delta_i = f_i - w_i): per node,
// sum_i delta_i (= rho - 1) and the momentum sum_i c_i delta_i (the weights'
// momentum vanishes), each stored element converted exactly to FP64; pass 2
// adds nFluid to the mass, so out[0] = sum rho as for FP64 storage.
template <class St>
__global__ void __launch_bounds__(kMomentTile) k_moments_partial_lp(const void* fv, long long nCells, int nFluid,
                                                                    double* partials) {
  using Elem = typename St::T;
  const Elem* f = static_cast<const Elem*>(fv);
  const int n = blockIdx.x * kMomentTile + threadIdx.x;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  if (n < nFluid) {
    double v[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) v[d] = static_cast<double>(St::dev(f[d * nCells + n], d));
    s[0] = v[C] + v[N] + v[E] + v[S] + v[W] + v[NE] + v[SE] + v[SW] + v[NW] + v[T] + v[TN] + v[TE] + v[TS] + v[TW] +
           v[B] + v[BN] + v[BE] + v[BS] + v[BW];
    s[1] = v[E] + v[NE] + v[SE] + v[TE] + v[BE] - v[W] - v[NW] - v[SW] - v[TW] - v[BW];
    s[2] = v[N] + v[NE] + v[NW] + v[TN] + v[BN] - v[S] - v[SE] - v[SW] - v[TS] - v[BS];
    s[3] = v[T] + v[TE] + v[TW] + v[TN] + v[TS] - v[B] - v[BE] - v[BW] - v[BN] - v[BS];
  }
  block_sum4(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) partials[blockIdx.x * 4 + k] = s[k];
}

__global__ void k_moments_add_mass(double* out, int nFluid) { out[0] = static_cast<double>(nFluid) + out[0]; }

void moments_enqueue_lp(const void* f, int storage, long long nCells, int nFluid, double* partials, double* out,
                        cudaStream_t s) {
  const int nb = moment_blocks(nFluid);
  if (storage == kStoreF16)
    k_moments_partial_lp<StoreF16><<<nb, kMomentTile, 0, s>>>(f, nCells, nFluid, partials);
  else
    k_moments_partial_lp<StoreF32><<<nb, kMomentTile, 0, s>>>(f, nCells, nFluid, partials);
  k_moments_final<<<1, kMomentTile, 0, s>>>(partials, nb, out);
  k_moments_add_mass<<<1, 1, 0, s>>>(out, nFluid);
}

}  // namespace lbm

extern "C" {

// Declared in include/lbm_b200.h.
int lbm_b200_moments_device(const double* pdfs, long long nCells, int nFluid, double* out_device, void* stream) {
  if (nFluid < 0 || nCells < nFluid || pdfs == nullptr || out_device == nullptr) return -1;
  double* partials = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMalloc(&partials, sizeof(double) * 4 * lbm::moment_blocks(nFluid));
  if (e != cudaSuccess) return (int)e;
  lbm::moments_enqueue(pdfs, nCells, nFluid, partials, out_device, s);
  e = cudaGetLastError();
  cudaError_t e2 = cudaStreamSynchronize(s);
  cudaFree(partials);
  return (int)(e != cudaSuccess ? e : e2);
}

}  // extern "C"
