// lbm_d3q19.cuh -- D3Q19 tables and the TRT collision shared by the sm_100a
// kernels.
//
// Direction order and inverse table follow the reference's D3Q19_LIST
// (src/Kernel.h:89-140): N,S,E,W,NE,SE,NW,SW,T,TN,TE,TW,TS,B,BS,BN,BW,BE,C.
// The order is part of the interface (it is the SoA plane order of every PDF
// array and the order of GetNode/SetNode arrays), so it is kept.
#pragma once
#include <cstdint>

namespace lbm {

constexpr int Q = 19;
constexpr int QM = 18;  // directions with a neighbour (all but the centre)
constexpr int DC = 18;  // centre direction index

enum Dir { N = 0, S, E, W, NE, SE, NW, SW, T, TN, TE, TW, TS, B, BS, BN, BW, BE, C };

__host__ __device__ constexpr int cx(int d) {
  constexpr int v[Q] = {0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0};
  return v[d];
}
__host__ __device__ constexpr int cy(int d) {
  constexpr int v[Q] = {1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0};
  return v[d];
}
__host__ __device__ constexpr int cz(int d) {
  constexpr int v[Q] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0};
  return v[d];
}
__host__ __device__ constexpr int inv(int d) {
  constexpr int v[Q] = {1, 0, 3, 2, 7, 6, 5, 4, 13, 14, 16, 17, 15, 8, 9, 12, 10, 11, 18};
  return v[d];
}

// Relaxation constants of one run, evaluated on the host exactly as the
// reference evaluates them at the top of each kernel
// (src/BenchKernelD3Q19Aa.c:69-88), plus the 19 body-force increments
// 3 w_i c_ix F (src/Kernel.c:772-795).
template <typename R>
struct Trt {
  R omegaEven, omegaOdd;
  R w0, w1, w2;
  R w1x3, w2x3, w1nh, w2nh;
  R force[Q];
};

// FP32 relaxation constants with the lattice weights as compile-time
// constants (the same values as a host-built Trt<float>). Per-run data are the
// two rates and the x body force as its two increments 3 w F_x (w = 1/18,
// 1/36); force(d) = c_dx times the increment of d's class, which equals the
// Trt<float> table entry bit for bit. Used where the per-run part sits in
// shared memory rather than in the kernel's parameter bank.
struct TrtW {
  float omegaEven, omegaOdd;
  float fx1, fx2;
  __device__ __forceinline__ float force(int d) const {
    const float v = (d == N || d == S || d == E || d == W || d == T || d == B) ? fx1 : fx2;
    return cx(d) > 0 ? v : (cx(d) < 0 ? -v : 0.0f);
  }
  static constexpr float w0 = static_cast<float>(1.0 / 3.0);
  static constexpr float w1 = static_cast<float>(1.0 / 18.0);
  static constexpr float w2 = static_cast<float>(1.0 / 36.0);
  static constexpr float w1x3 = static_cast<float>(1.0 / 18.0 * 3.0);
  static constexpr float w2x3 = static_cast<float>(1.0 / 36.0 * 3.0);
  static constexpr float w1nh = static_cast<float>(1.0 / 18.0 * 9.0 / 2.0);
  static constexpr float w2nh = static_cast<float>(1.0 / 36.0 * 9.0 / 2.0);
};

template <class P>
struct TrtReal;
template <typename R>
struct TrtReal<Trt<R>> {
  using type = R;
};
template <>
struct TrtReal<TrtW> {
  using type = float;
};

// One TRT relaxation of a node (src/BenchKernelD3Q19Aa.c:205-284), written as
// a straight-line function of the 19 incoming PDFs. The operation order is the
// reference's scalar order; FP64 builds compile this file without FMA
// contraction, so the results are bit-identical to the reference's scalar
// kernels. out[i] is the post-collision PDF of direction i (unswapped).
template <typename R, class P>
__device__ __forceinline__ void trt_pair(const P& t, const R* f, R* out, int a, int b, R ui, R wnh, R wx3,
                                         R windep) {
  R evenPart = t.omegaEven * (R(0.5) * (f[a] + f[b]) - ui * ui * wnh - windep);
  R oddPart = t.omegaOdd * (R(0.5) * (f[a] - f[b]) - ui * wx3);
  out[a] = f[a] - evenPart - oddPart;
  out[b] = f[b] - evenPart + oddPart;
}

template <typename R, class P>
__device__ __forceinline__ void trt_collide(const P& t, const R* f, R* out) {
  R ux = f[E] + f[NE] + f[SE] + f[TE] + f[BE] - f[W] - f[NW] - f[SW] - f[TW] - f[BW];
  R uy = f[N] + f[NE] + f[NW] + f[TN] + f[BN] - f[S] - f[SE] - f[SW] - f[TS] - f[BS];
  R uz = f[T] + f[TE] + f[TW] + f[TN] + f[TS] - f[B] - f[BE] - f[BW] - f[BN] - f[BS];
  R dens = f[C] + f[N] + f[E] + f[S] + f[W] + f[NE] + f[SE] + f[SW] + f[NW] + f[T] + f[TN] + f[TE] + f[TS] + f[TW] +
           f[B] + f[BN] + f[BE] + f[BS] + f[BW];
  R dit = dens - (ux * ux + uy * uy + uz * uz) * R(3.0) / R(2.0);

  out[C] = f[C] - t.omegaEven * (f[C] - t.w0 * dit);

  R w1i = t.w1 * dit;
  trt_pair(t, f, out, N, S, uy, t.w1nh, t.w1x3, w1i);
  trt_pair(t, f, out, E, W, ux, t.w1nh, t.w1x3, w1i);
  trt_pair(t, f, out, T, B, uz, t.w1nh, t.w1x3, w1i);

  R w2i = t.w2 * dit;
  trt_pair(t, f, out, NW, SE, -ux + uy, t.w2nh, t.w2x3, w2i);
  trt_pair(t, f, out, NE, SW, ux + uy, t.w2nh, t.w2x3, w2i);
  trt_pair(t, f, out, TW, BE, -ux + uz, t.w2nh, t.w2x3, w2i);
  trt_pair(t, f, out, TE, BW, ux + uz, t.w2nh, t.w2x3, w2i);
  trt_pair(t, f, out, TS, BN, -uy + uz, t.w2nh, t.w2x3, w2i);
  trt_pair(t, f, out, TN, BS, uy + uz, t.w2nh, t.w2x3, w2i);
}

// An opaque copy of a pointer: the compiler cannot tell that it equals its
// source, so addresses formed from it are not shared with (and do not keep
// alive) addresses formed from the original. Used to give the store phase its
// own addresses, which frees the load addresses' registers across the
// collision.
template <typename P>
__device__ __forceinline__ P* launder(P* p) {
  P* q;
  asm volatile("mov.b64 %0, %1;" : "=l"(q) : "l"(p));
  return q;
}

// One node update through accessors: all 19 loads are issued first (they are
// independent, so they are in flight together), then the relaxation, then
// the 19 stores. `load(d)` returns the incoming PDF of direction d,
// `store(d, v)` writes the post-collision PDF of direction d to its
// destination.
template <class P, class Load, class Store>
__device__ __forceinline__ void trt_update(const P& t, Load load, Store store) {
  using R = typename TrtReal<P>::type;
  R f[Q], o[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) f[d] = load(d);
  trt_collide(t, f, o);
#pragma unroll
  for (int d = 0; d < Q; ++d) store(d, o[d]);
}

}  // namespace lbm
