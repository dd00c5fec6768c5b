// lbm_batch_lp.cu -- persistent list AA kernels over a batch of domains
// (FP32 arithmetic on FP32 or FP16-deviation storage, as lbm_kernels_lp.cu).
//
// Every block walks the tile table with a grid stride. The odd step stages a
// tile's adjacency (256 nodes x 18 entries, 18 KB, contiguous) into shared
// memory with one bulk copy, double buffered: while a tile is relaxed, the
// bulk copy of the block's next tile is already in flight.
#include <cuda_fp16.h>

#include "lbm_batch.cuh"
#include "lbm_bulk.cuh"

namespace lbm {

__device__ __forceinline__ float bweight(int d) {
  return d == DC ? 1.0f / 3.0f : (d == N || d == S || d == E || d == W || d == T || d == B) ? 1.0f / 18.0f : 1.0f / 36.0f;
}

struct BStoreF32 {
  using T = float;
  __device__ static float dev(T raw, int d) { return raw - bweight(d); }
  __device__ static T raw(float delta, int d) { return bweight(d) + delta; }
};

struct BStoreF16 {
  using T = __half;
  __device__ static float scale(int d) { return d == DC ? 32768.0f : (bweight(d) > 0.05f ? 262144.0f : 524288.0f); }
  __device__ static float dev(T raw, int d) { return __half2float(raw) * (1.0f / scale(d)); }
  __device__ static T raw(float delta, int d) { return __float2half_rn(delta * scale(d)); }
};

template <class St>
__device__ __forceinline__ void batch_even_node(const BatchDomain& D, int n) {
  using T = typename St::T;
  T* const f = static_cast<T*>(D.f) + n;
  T* const fs = launder(f);
  const long long S = D.nCells;
  trt_update(D.trt, [&](int d) { return St::dev(f[d * S], d); },
             [&](int d, float v) { fs[inv(d) * S] = St::raw(v, inv(d)); });
}

template <class St>
__global__ void __launch_bounds__(256) k_batch_even(const BatchArgs a) {
  const int nT = *a.nTiles;
  for (int tile = blockIdx.x; tile < nT; tile += gridDim.x) {
    const BatchDomain& D = a.doms[a.tileDom[tile]];
    const int base = (tile - D.tileStart) * kBatchTileNodes + threadIdx.x;
    for (int k = 0; k < a.nodesPerThread; ++k) {
      const int n = base + k * blockDim.x;
      if (n < D.nFluid) batch_even_node<St>(D, n);
    }
  }
}

template <class St>
__device__ __forceinline__ void batch_odd_node(const BatchDomain& D, const uint32_t* e, int n) {
  using T = typename St::T;
  T* const f = static_cast<T*>(D.f);
  const long long S = D.nCells;
  const Trt<float>& t = D.trt;
  auto load = [&](int d) -> float { return St::dev(d == DC ? f[DC * S + n] : f[e[inv(d)]], d) + t.force[d]; };
  auto store = [&](int d, float v) {
    if (d == DC) {
      f[DC * S + n] = St::raw(v + t.force[DC], DC);
      return;
    }
    const uint32_t dst = reinterpret_cast<const volatile uint32_t*>(e)[d];
    const int j = inv(d);
    const bool bounce = dst == static_cast<uint32_t>(j * S + n);
    f[dst] = St::raw(v + (bounce ? t.force[j] : t.force[d]), d);
  };
  trt_update(t, load, store);
}

constexpr uint32_t kTileAdjBytes = kBatchTileNodes * QM * 4;

template <class St>
__global__ void __launch_bounds__(256) k_batch_odd(const BatchArgs a) {
  extern __shared__ __align__(128) uint32_t sadj[];  // 2 x kBatchTileNodes x 18
  __shared__ alignas(8) uint64_t bar[2];
  const int nT = *a.nTiles;
  if (blockIdx.x >= nT) return;

  auto issue = [&](int tile, int buf) {
    const BatchDomain& D = a.doms[a.tileDom[tile]];
    const uint32_t* src = D.adj + static_cast<size_t>(tile - D.tileStart) * kBatchTileNodes * QM;
    mbar_arrive_expect_tx(&bar[buf], kTileAdjBytes);
    bulk_g2s(sadj + buf * kBatchTileNodes * QM, src, kTileAdjBytes, &bar[buf]);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    issue(blockIdx.x, 0);
  }

  int it = 0;
  for (int tile = blockIdx.x; tile < nT; tile += gridDim.x, ++it) {
    const int buf = it & 1;
    __syncthreads();  // every thread is done with buffer buf ^ 1 (the previous tile)
    const int next = tile + gridDim.x;
    if (threadIdx.x == 0 && next < nT) issue(next, buf ^ 1);
    if (!mbar_wait_bounded(&bar[buf], (it >> 1) & 1)) {
      if (threadIdx.x == 0) atomicOr(a.err, 1);
      return;
    }
    const BatchDomain& D = a.doms[a.tileDom[tile]];
    const uint32_t* tileAdj = sadj + buf * kBatchTileNodes * QM;
    for (int k = 0; k < a.nodesPerThread; ++k) {
      const int local = threadIdx.x + k * blockDim.x;
      const int n = (tile - D.tileStart) * kBatchTileNodes + local;
      if (n < D.nFluid) batch_odd_node<St>(D, tileAdj + local * QM, n);
    }
  }
  // a block that exits early on a failed wait leaves its other copy unwaited;
  // here every issued copy has been waited for
}

void batch_even_lp(const BatchArgs& a, const BatchLaunch& l, cudaStream_t s) {
  if (a.storage == kStoreF16)
    k_batch_even<BStoreF16><<<l.blocks, l.threads, 0, s>>>(a);
  else
    k_batch_even<BStoreF32><<<l.blocks, l.threads, 0, s>>>(a);
}

void batch_odd_lp(const BatchArgs& a, const BatchLaunch& l, cudaStream_t s) {
  const size_t smem = 2 * (size_t)kTileAdjBytes;
  if (a.storage == kStoreF16)
    k_batch_odd<BStoreF16><<<l.blocks, l.threads, smem, s>>>(a);
  else
    k_batch_odd<BStoreF32><<<l.blocks, l.threads, smem, s>>>(a);
}

// ---------------------------------------------------------------------------
// FP64 per-domain sums.

template <class St>
__global__ void __launch_bounds__(256) k_batch_moments_tile(const BatchArgs a, int maxTiles, double* partials) {
  __shared__ double part[8][4];
  const int nT = *a.nTiles;
  for (int tile = blockIdx.x; tile < nT && tile < maxTiles; tile += gridDim.x) {
    const BatchDomain& D = a.doms[a.tileDom[tile]];
    const int n = (tile - D.tileStart) * kBatchTileNodes + threadIdx.x;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (n < D.nFluid) {
      using T = typename St::T;
      const T* f = static_cast<const T*>(D.f) + n;
      float v[Q];
#pragma unroll
      for (int d = 0; d < Q; ++d) v[d] = St::dev(f[d * D.nCells], d);
      // rho - 1 and momentum from the deviations, accumulated in FP64
#pragma unroll
      for (int d = 0; d < Q; ++d) {
        s[0] += (double)v[d];
        s[1] += (double)(cx(d) * v[d]);
        s[2] += (double)(cy(d) * v[d]);
        s[3] += (double)(cz(d) * v[d]);
      }
      s[0] += 1.0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
      for (int k = 0; k < 4; ++k) part[threadIdx.x >> 5][k] = s[k];
    __syncthreads();
    if (threadIdx.x < 4) {
      double acc = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) acc += part[w][threadIdx.x];
      partials[(size_t)tile * 4 + threadIdx.x] = acc;
    }
    __syncthreads();
  }
}

__global__ void k_batch_moments_dom(const double* partials, const int* domTileStart, const int* domTileCount,
                                    int nDomSlots, double* out) {
  const int dslot = blockIdx.x * blockDim.x + threadIdx.x;
  if (dslot >= nDomSlots) return;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  const int t0 = domTileStart[dslot], nt = domTileCount[dslot];
  for (int t = t0; t < t0 + nt; ++t)
#pragma unroll
    for (int k = 0; k < 4; ++k) s[k] += partials[(size_t)t * 4 + k];
#pragma unroll
  for (int k = 0; k < 4; ++k) out[dslot * 4 + k] = s[k];
}

void batch_moments(const BatchArgs& a, int maxTiles, double* tilePartials, const int* domTileStart,
                   const int* domTileCount, int nDomSlots, double* out, cudaStream_t s) {
  const int blocks = maxTiles < 4096 ? (maxTiles > 0 ? maxTiles : 1) : 4096;
  if (a.storage == kStoreF16)
    k_batch_moments_tile<BStoreF16><<<blocks, kBatchTileNodes, 0, s>>>(a, maxTiles, tilePartials);
  else
    k_batch_moments_tile<BStoreF32><<<blocks, kBatchTileNodes, 0, s>>>(a, maxTiles, tilePartials);
  k_batch_moments_dom<<<(nDomSlots + 127) / 128, 128, 0, s>>>(tilePartials, domTileStart, domTileCount, nDomSlots, out);
}

}  // namespace lbm
