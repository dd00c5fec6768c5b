// lbm_bulk.cuh -- one-dimensional bulk copies global -> shared (sm_90+
// cp.async.bulk, issued by one thread, completion tracked by an mbarrier).
// Used to stage the contiguous adjacency tile of a block of list nodes.
// No cluster multicast anywhere: every copy reads this GPU's own memory into
// its own CTA.
#pragma once
#include <cstdint>

#include "lbm_kernels.cuh"

namespace lbm {

constexpr uint32_t kBulkSpinLimit = 1u << 22;  // try_wait rounds before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// dst, src 16 B aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Hint: bring [src, src + bytes) into L2 ahead of its bulk copy (16 B
// aligned, a multiple of 16 bytes; no completion to wait for).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on phase `parity`; false after kBulkSpinLimit rounds.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kBulkSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Stages the run record of tile blockIdx.x + a.tileBase (run-compressed adjacency, see
// kRunHdrWords) into srun (kRunTileWords words) with one bulk copy, in two
// halves: stage_run_tile_issue starts the copy (thread 0; a record whose size
// does not fit flags error bit 4 and is not copied) and makes the barrier
// visible to the block; stage_run_tile_wait waits for it. Work that does not
// need the record (a node's own PDFs) may run between the two. After the
// wait, warp 1 prefetches into L2 the record of the tile kWaves x
// `a.prefetch` tiles ahead (kWaves = 1: the block that will take this one's
// place), off the block's critical path. Both return false (error word set)
// if the copy was refused or did not arrive within the spin limit; every
// thread returns the same from the issue half.
template <class A>
__device__ __forceinline__ bool stage_run_tile_issue(const A& a, uint32_t* srun, uint64_t* bar, int* ok) {
  const unsigned tile = blockIdx.x + static_cast<unsigned>(a.tileBase);
  if (threadIdx.x == 0) {
    const uint32_t o0 = a.runOff[tile], o1 = a.runOff[tile + 1];
    const uint32_t bytes = (o1 - o0) * 16u;
    *ok = o1 > o0 && bytes <= static_cast<uint32_t>(kRunTileWords) * 4u;
    mbar_init(bar, 1);
    if (*ok) {
      mbar_arrive_expect_tx(bar, bytes);
      bulk_g2s(srun, a.runs + static_cast<size_t>(o0) * 4, bytes, bar);
    } else {
      atomicOr(a.err, 4);
    }
  }
  __syncthreads();
  return *ok != 0;
}

template <int kWaves = 1, class A>
__device__ __forceinline__ bool stage_run_tile_wait(const A& a, uint64_t* bar) {
  if (!mbar_wait_bounded(bar, 0)) {
    atomicOr(a.err, 1);
    return false;
  }
  const unsigned tile = blockIdx.x + static_cast<unsigned>(a.tileBase);
  const unsigned nTiles = static_cast<unsigned>((a.nFluid + kListTile - 1) / kListTile);
  if (threadIdx.x == 32 && a.prefetch > 0 && tile + kWaves * static_cast<unsigned>(a.prefetch) < nTiles) {
    const unsigned t = tile + kWaves * a.prefetch;
    const uint32_t o0 = a.runOff[t], o1 = a.runOff[t + 1];
    if (o1 > o0 && (o1 - o0) * 16u <= static_cast<uint32_t>(kRunTileWords) * 4u)
      bulk_prefetch_l2(a.runs + static_cast<size_t>(o0) * 4, (o1 - o0) * 16u);
  }
  return true;
}

// Both halves back to back (the record is needed from the start).
template <int kWaves = 1, class A>
__device__ __forceinline__ bool stage_run_tile(const A& a, uint32_t* srun, uint64_t* bar, int* ok) {
  if (!stage_run_tile_issue(a, srun, bar, ok)) return false;
  return stage_run_tile_wait<kWaves>(a, bar);
}

// The adjacency row of node `tid` of a staged run record and the node's
// distance from its run's head: link d of the node is row[d] + off.
__device__ __forceinline__ const uint32_t* run_row(const uint32_t* srun, int tid, uint32_t& off) {
  const int w = tid >> 5, b = tid & 31;
  // heads before word w (header byte w of words 8-9), then those up to tid
  int rank = static_cast<int>((srun[8 + (w >> 2)] >> (8 * (w & 3))) & 0xffu);
  uint32_t mk = srun[w] & ((2u << b) - 1u);
  rank += __popc(mk);
  int k = w;
  while (mk == 0u && k > 0) mk = srun[--k];  // node 0 of a tile always heads a run
  off = mk ? static_cast<uint32_t>(tid - (32 * k + 31 - __clz(mk))) : 0u;
  return srun + kRunHdrWords + (rank > 0 ? rank - 1 : 0) * 18;
}

}  // namespace lbm
