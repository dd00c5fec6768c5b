// lbm_store.cuh -- reduced-precision PDF storage of the list AA kernels
// (single-domain and batched): PDFs kept in HBM as deviations from the lattice
// weights, delta_i = f_i - w_i, with the collision evaluated in FP32.
//
// Deviation form. With f_i = w_i + delta_i, the TRT update of lbm_d3q19.cuh
// holds unchanged for the deltas once "dens" is replaced by sum_i delta_i
// (= rho - 1): the momentum sum_i c_i w_i vanishes and the weight terms cancel
// in both parts of each pair. Working on deltas keeps the O(1) background out
// of the FP32 arithmetic and out of the stored bits.
//
//   StoreF32  raw = delta_i as float: 24 significant bits of the deviation
//             itself (storing w_i + delta_i instead would leave only
//             ulp(w_i) ~ 4e-9 of absolute resolution for delta_i).
//   StoreF16  raw = half(delta_i * 2^k_i), k_i fixed per direction class
//             (k = 15, 18, 19 for w = 1/3, 1/18, 1/36), so that |delta| up to
//             ~4.5 w_i is representable and deltas down to ~2e-10 stay normal.
#pragma once
#include <cuda_fp16.h>

#include "lbm_d3q19.cuh"

namespace lbm {

// Directions along a lattice axis (weight 1/18).
__device__ __forceinline__ bool axis_dir(int d) { return d == N || d == S || d == E || d == W || d == T || d == B; }

struct StoreF32 {
  using T = float;
  __device__ static float dev(T raw, int) { return raw; }
  __device__ static T raw(float delta, int) { return delta; }
};

struct StoreF16 {
  using T = __half;
  __device__ static float scale(int d) {
    return d == DC ? 32768.0f : (axis_dir(d) ? 262144.0f : 524288.0f);
  }
  __device__ static float dev(T raw, int d) { return __half2float(raw) * (1.0f / scale(d)); }
  __device__ static T raw(float delta, int d) { return __float2half_rn(delta * scale(d)); }
};

}  // namespace lbm
