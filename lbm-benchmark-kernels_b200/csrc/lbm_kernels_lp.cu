// lbm_kernels_lp.cu -- reduced-storage list AA kernels for sm_100a: PDFs kept
// in HBM as FP32, or as FP16 deviations from the lattice weights, with the
// collision evaluated in FP32 (FMA contraction allowed in this file).
//
// Deviation form. With f_i = w_i + delta_i, the TRT update of
// lbm_d3q19.cuh holds unchanged for the deltas once "dens" is replaced by
// sum_i delta_i (= rho - 1): the momentum sum_i c_i w_i vanishes and the
// weight terms cancel in both parts of each pair. Working on deltas keeps the
// O(1) background out of the FP32 arithmetic.
//
// Storage:
//   StoreF32  raw = w_i + delta_i as float (delta = raw - w_i is exact while
//             raw stays within a factor 2 of w_i)
//   StoreF16  raw = half(delta_i * 2^k_i), k_i fixed per direction class
//             (k = 15, 18, 19 for w = 1/3, 1/18, 1/36), so that |delta| up to
//             ~4.5 w_i is representable and deltas down to ~2e-10 stay normal.
// Bytes per fluid-lattice update: even 19*2*s, odd 19*2*s + 72 (s = 4 or 2).
#include <cuda_fp16.h>

#include "lbm_bulk.cuh"
#include "lbm_kernels.cuh"

namespace lbm {

__device__ __forceinline__ float weight_f(int d) { return d == DC ? 1.0f / 3.0f : (d == N || d == S || d == E || d == W || d == T || d == B) ? 1.0f / 18.0f : 1.0f / 36.0f; }

struct StoreF32 {
  using T = float;
  __device__ static float dev(T raw, int d) { return raw - weight_f(d); }
  __device__ static T raw(float delta, int d) { return weight_f(d) + delta; }
};

struct StoreF16 {
  using T = __half;
  __device__ static float scale(int d) { return d == DC ? 32768.0f : (weight_f(d) > 0.05f ? 262144.0f : 524288.0f); }
  __device__ static float dev(T raw, int d) { return __half2float(raw) * (1.0f / scale(d)); }
  __device__ static T raw(float delta, int d) { return __float2half_rn(delta * scale(d)); }
};

template <class St>
__global__ void __launch_bounds__(kListTile) k_list_even_lp(const ListArgsLp a, const Trt<float> t) {
  using T = typename St::T;
  const int n = blockIdx.x * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  T* const f = static_cast<T*>(a.f) + n;
  T* const fs = launder(f);
  const long long S = a.nCells;
  trt_update(t, [&](int d) { return St::dev(f[d * S], d); },
             [&](int d, float v) { fs[inv(d) * S] = St::raw(v, inv(d)); });
}

__device__ __forceinline__ bool stage_adj_tile_lp(const ListArgsLp& a, uint32_t* sadj, uint64_t* bar) {
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, kListTile * QM * 4);
    bulk_g2s(sadj, a.adj + static_cast<size_t>(blockIdx.x) * kListTile * QM, kListTile * QM * 4, bar);
  }
  __syncthreads();
  if (!mbar_wait_bounded(bar, 0)) {
    if (threadIdx.x == 0) atomicOr(a.err, 1);
    return false;
  }
  return true;
}

template <class St>
__global__ void __launch_bounds__(kListTile) k_list_odd_lp(const ListArgsLp a, const Trt<float> t) {
  using T = typename St::T;
  __shared__ alignas(128) uint32_t sadj[kListTile * QM];
  __shared__ alignas(8) uint64_t bar;
  if (!stage_adj_tile_lp(a, sadj, &bar)) return;
  const int n = blockIdx.x * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  const uint32_t* e = sadj + threadIdx.x * QM;
  T* const f = static_cast<T*>(a.f);
  const long long S = a.nCells;
  auto load = [&](int d) -> float { return St::dev(d == DC ? f[DC * S + n] : f[e[inv(d)]], d) + t.force[d]; };
  auto store = [&](int d, float v) {
    if (d == DC) {
      f[DC * S + n] = St::raw(v + t.force[DC], DC);
      return;
    }
    const uint32_t dst = reinterpret_cast<const volatile uint32_t*>(e)[d];  // re-read: keeps no 64-bit addresses live across the collision
    const int j = inv(d);
    const bool bounce = dst == static_cast<uint32_t>(j * S + n);
    f[dst] = St::raw(v + (bounce ? t.force[j] : t.force[d]), d);  // w and the scale are equal for d and inv(d)
  };
  trt_update(t, load, store);
}

static unsigned lp_blocks(const ListArgsLp& a) { return (a.nFluid + kListTile - 1) / kListTile; }

void list_even_lp(const ListArgsLp& a, const Trt<float>& t, int storage, cudaStream_t s) {
  if (a.nFluid <= 0) return;
  if (storage == kStoreF16)
    k_list_even_lp<StoreF16><<<lp_blocks(a), kListTile, 0, s>>>(a, t);
  else
    k_list_even_lp<StoreF32><<<lp_blocks(a), kListTile, 0, s>>>(a, t);
}

void list_odd_lp(const ListArgsLp& a, const Trt<float>& t, int storage, cudaStream_t s) {
  if (a.nFluid <= 0) return;
  if (storage == kStoreF16)
    k_list_odd_lp<StoreF16><<<lp_blocks(a), kListTile, 0, s>>>(a, t);
  else
    k_list_odd_lp<StoreF32><<<lp_blocks(a), kListTile, 0, s>>>(a, t);
}

}  // namespace lbm
