// lbm_kernels_lp.cu -- reduced-storage list AA kernels for sm_100a: PDFs kept
// in HBM as FP32 or FP16 deviations from the lattice weights (lbm_store.cuh),
// with the collision evaluated in FP32 (FMA contraction allowed in this file).
// Bytes per fluid-lattice update: even 19*2*s, odd 19*2*s + 72 (s = 4 or 2).
#include "lbm_bulk.cuh"
#include "lbm_kernels.cuh"
#include "lbm_store.cuh"

namespace lbm {

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
    f[dst] = St::raw(v + (bounce ? t.force[j] : t.force[d]), d);  // the scale is equal for d and inv(d)
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
