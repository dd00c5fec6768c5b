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
//
// Working unit. The time-step kernels relax U_i = delta_i * kUnit (FP32:
// kUnit = 1; FP16: kUnit = 2^19, the diagonal directions' scale), so that a
// diagonal FP16 PDF converts to and from the working unit with no multiply
// and the others with one power-of-two multiply (x2 / x16 in, x0.5 / x1/16
// out). The TRT update is linear in the PDFs apart from the u^2 terms, whose
// constants carry the 1/kUnit (TrtDev); all scalings are powers of two, so
// the FP16 results equal those of a plain deviation update up to the rounding
// of the FP32 arithmetic.
#pragma once
#include <cuda_fp16.h>

#include "lbm_d3q19.cuh"

namespace lbm {

// Directions along a lattice axis (weight 1/18).
__host__ __device__ constexpr bool axis_dir(int d) {
  return d == N || d == S || d == E || d == W || d == T || d == B;
}

struct StoreF32 {
  using T = float;
  static constexpr float kUnit = 1.0f;
  __device__ static float dev(T raw, int) { return raw; }
  __device__ static T raw(float delta, int) { return delta; }
  // raw <-> working unit
  __device__ static float in(T raw, int) { return raw; }
  __device__ static T out(float u, int) { return u; }
};

struct StoreF16 {
  using T = __half;
  static constexpr float kUnit = 524288.0f;  // 2^19
  __host__ __device__ static constexpr float scale(int d) {
    return d == DC ? 32768.0f : (axis_dir(d) ? 262144.0f : 524288.0f);
  }
  __device__ static float dev(T raw, int d) { return __half2float(raw) * (1.0f / scale(d)); }
  __device__ static T raw(float delta, int d) { return __float2half_rn(delta * scale(d)); }
  // raw <-> working unit: kUnit / scale(d) is 1, 2 or 16
  __device__ static float in(T raw, int d) {
    const float v = __half2float(raw);
    return d == DC ? v * 16.0f : (axis_dir(d) ? v * 2.0f : v);
  }
  __device__ static T out(float u, int d) {
    return __float2half_rn(d == DC ? u * 0.0625f : (axis_dir(d) ? u * 0.5f : u));
  }
  __device__ static float2 in2(__half2 raw, int d) {
    const float2 v = __half22float2(raw);
    const float k = d == DC ? 16.0f : (axis_dir(d) ? 2.0f : 1.0f);
    return k == 1.0f ? v : make_float2(v.x * k, v.y * k);
  }
  __device__ static __half2 out2(float a, float b, int d) {
    const float k = d == DC ? 0.0625f : (axis_dir(d) ? 0.5f : 1.0f);
    return k == 1.0f ? __floats2half2_rn(a, b) : __floats2half2_rn(a * k, b * k);
  }
};

// FP32 TRT constants in the working unit of storage St. The weights are
// compile-time constants; the u^2 terms carry 1/kUnit; the body force is
// c_ix times the class increment 3 w F_x in the working unit (only the ten
// directions with c_x != 0 get one).
template <class St>
struct TrtDev {
  float omegaEven, omegaOdd;
  float fx1, fx2;  // 3 w F_x for w = 1/18 and 1/36, times kUnit
  static constexpr float w0 = static_cast<float>(1.0 / 3.0);
  static constexpr float w1 = static_cast<float>(1.0 / 18.0);
  static constexpr float w2 = static_cast<float>(1.0 / 36.0);
  static constexpr float w1x3 = static_cast<float>(1.0 / 18.0 * 3.0);
  static constexpr float w2x3 = static_cast<float>(1.0 / 36.0 * 3.0);
  static constexpr float w1nh = static_cast<float>(1.0 / 18.0 * 9.0 / 2.0) / St::kUnit;
  static constexpr float w2nh = static_cast<float>(1.0 / 36.0 * 9.0 / 2.0) / St::kUnit;
  static constexpr float kDit = 1.5f / St::kUnit;
  __device__ __forceinline__ TrtDev(const TrtW& w)
      : omegaEven(w.omegaEven), omegaOdd(w.omegaOdd), fx1(w.fx1 * St::kUnit), fx2(w.fx2 * St::kUnit) {}
  __device__ __forceinline__ float force(int d) const {
    const float v = axis_dir(d) ? fx1 : fx2;
    return cx(d) > 0 ? v : -v;  // call only for c_x(d) != 0
  }
};

__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }

// Two TRT pairs (a0, b0) and (a1, b1) of one weight class relaxed together
// on packed FP32x2 arithmetic (sm_100: one instruction for two lanes; lane 0
// = pair 0, lane 1 = pair 1), each lane in the operation order of trt_pair.
template <class P>
__device__ __forceinline__ void trt_pair2(const P& t, const float* f, float* out, int a0, int b0, int a1, int b1,
                                          float2 u, float wnh, float wx3, float windep) {
  const float2 fa = make_float2(f[a0], f[a1]), fb = make_float2(f[b0], f[b1]);
  const float2 half = make_float2(0.5f, 0.5f);
  const float2 s = __fadd2_rn(fa, fb);
  const float2 d = __fadd2_rn(fa, neg2(fb));
  const float2 c = __ffma2_rn(__fmul2_rn(u, u), make_float2(wnh, wnh), make_float2(windep, windep));
  const float2 ev = __fmul2_rn(make_float2(t.omegaEven, t.omegaEven), __ffma2_rn(s, half, neg2(c)));
  const float2 uw = __fmul2_rn(u, make_float2(wx3, wx3));
  const float2 od = __fmul2_rn(make_float2(t.omegaOdd, t.omegaOdd), __ffma2_rn(d, half, neg2(uw)));
  const float2 oa = __fadd2_rn(fa, neg2(__fadd2_rn(ev, od)));
  const float2 ob = __fadd2_rn(fb, neg2(__fadd2_rn(ev, neg2(od))));
  out[a0] = oa.x;
  out[a1] = oa.y;
  out[b0] = ob.x;
  out[b1] = ob.y;
}

// One TRT relaxation in the working unit in the order of trt_collide.
// kPacked: eight of the nine direction pairs are relaxed two at a time on
// packed FP32x2 arithmetic (trt_pair2); the single-domain kernels use it
// (FP16 odd step 0.171 -> 0.165 ms, FP32 0.220 -> 0.217 ms at the 256^3
// packing). The batched kernels relax pair by pair: under their register cap
// the packed form spills (batched FP32 34.7 -> 32.0 GFLUP/s at 64 domains).
// The moments stay scalar sums in both: forming them from packed pair sums
// and differences keeps 18 more values live and spills (FP16 odd step 0.165
// -> 0.201 ms).
template <class St, bool kPacked = true>
__device__ __forceinline__ void trt_collide_dev(const TrtDev<St>& t, const float* f, float* out) {
  using P = TrtDev<St>;
  float ux = f[E] + f[NE] + f[SE] + f[TE] + f[BE] - f[W] - f[NW] - f[SW] - f[TW] - f[BW];
  float uy = f[N] + f[NE] + f[NW] + f[TN] + f[BN] - f[S] - f[SE] - f[SW] - f[TS] - f[BS];
  float uz = f[T] + f[TE] + f[TW] + f[TN] + f[TS] - f[B] - f[BE] - f[BW] - f[BN] - f[BS];
  float dens = f[C] + f[N] + f[E] + f[S] + f[W] + f[NE] + f[SE] + f[SW] + f[NW] + f[T] + f[TN] + f[TE] + f[TS] +
               f[TW] + f[B] + f[BN] + f[BE] + f[BS] + f[BW];
  float dit = dens - (ux * ux + uy * uy + uz * uz) * P::kDit;
  out[C] = f[C] - t.omegaEven * (f[C] - P::w0 * dit);
  const float w1i = P::w1 * dit;
  const float w2i = P::w2 * dit;
  if constexpr (kPacked) {
    trt_pair2(t, f, out, N, S, E, W, make_float2(uy, ux), P::w1nh, P::w1x3, w1i);
    trt_pair(t, f, out, T, B, uz, P::w1nh, P::w1x3, w1i);
    trt_pair2(t, f, out, NW, SE, NE, SW, make_float2(-ux + uy, ux + uy), P::w2nh, P::w2x3, w2i);
    trt_pair2(t, f, out, TW, BE, TE, BW, make_float2(-ux + uz, ux + uz), P::w2nh, P::w2x3, w2i);
    trt_pair2(t, f, out, TS, BN, TN, BS, make_float2(-uy + uz, uy + uz), P::w2nh, P::w2x3, w2i);
  } else {
    trt_pair(t, f, out, N, S, uy, P::w1nh, P::w1x3, w1i);
    trt_pair(t, f, out, E, W, ux, P::w1nh, P::w1x3, w1i);
    trt_pair(t, f, out, T, B, uz, P::w1nh, P::w1x3, w1i);
    trt_pair(t, f, out, NW, SE, -ux + uy, P::w2nh, P::w2x3, w2i);
    trt_pair(t, f, out, NE, SW, ux + uy, P::w2nh, P::w2x3, w2i);
    trt_pair(t, f, out, TW, BE, -ux + uz, P::w2nh, P::w2x3, w2i);
    trt_pair(t, f, out, TE, BW, ux + uz, P::w2nh, P::w2x3, w2i);
    trt_pair(t, f, out, TS, BN, -uy + uz, P::w2nh, P::w2x3, w2i);
    trt_pair(t, f, out, TN, BS, uy + uz, P::w2nh, P::w2x3, w2i);
  }
}

// Even step of node n (local collide, swapped store): f[d * S + n].
template <class St, bool kPacked = true>
__device__ __forceinline__ void lp_even_node(typename St::T* f, long long S, int n, const TrtDev<St>& t) {
  using T = typename St::T;
  const T* const src = f + n;
  T* const dst = launder(f + n);
  float x[Q], o[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) x[d] = St::in(src[d * S], d);
  trt_collide_dev<St, kPacked>(t, x, o);
#pragma unroll
  for (int d = 0; d < Q; ++d) dst[inv(d) * S] = St::out(o[d], inv(d));
}

// Odd step of node n, whose links come run-compressed: link d = e[d] + off
// (e: the run's adjacency row in shared memory). The node reads f_d from link inv(d)
// plus its body-force increment and writes f_d to link d. A link is either
// the neighbour's slot in plane d or -- bounce back -- the node's own slot
// in plane inv(d); the PDF then gets the increment of inv(d), which differs
// from d's only for c_x != 0, so only those ten directions test it, by the
// link's plane (one compare against a constant per direction). Addresses
// are formed from f + off, so a link costs one index on top of its
// shared-memory read.
template <class St, bool kPacked = true>
__device__ __forceinline__ void lp_odd_node(typename St::T* f, uint32_t S, uint32_t n, const uint32_t* e,
                                            uint32_t off, const TrtDev<St>& t) {
  using T = typename St::T;
  T* const fo = f + off;  // every address below is fo + 32-bit index (the node itself: DC * S + head)
  const uint32_t head = n - off;
  uint32_t l[QM];
#pragma unroll
  for (int k = 0; k < QM; ++k) l[k] = e[k];
  float x[Q], o[Q];
  x[DC] = St::in(fo[DC * S + head], DC);
#pragma unroll
  for (int d = 0; d < QM; ++d) {
    const float v = St::in(fo[l[inv(d)]], d);
    x[d] = cx(d) != 0 ? v + t.force(d) : v;
  }
  trt_collide_dev<St, kPacked>(t, x, o);
  T* const fs = launder(fo);
  fs[DC * S + head] = St::out(o[DC], DC);
#pragma unroll
  for (int d = 0; d < QM; ++d) {
    // re-read from shared memory: keeps no links live across the collision
    const uint32_t ed = reinterpret_cast<const volatile uint32_t*>(e)[d];
    float v = o[d];
    if (cx(d) != 0) {
      // plane inv(d) lies below plane d when inv(d) < d, above it otherwise
      const bool bounce = inv(d) < d ? ed < static_cast<uint32_t>(d) * S : ed >= static_cast<uint32_t>(d + 1) * S;
      v += bounce ? t.force(inv(d)) : t.force(d);
    }
    fs[ed] = St::out(v, d);  // the scale is equal for d and inv(d)
  }
}

}  // namespace lbm
