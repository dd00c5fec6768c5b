// lbm_kernels_lp.cu -- reduced-storage list AA kernels for sm_100a: PDFs kept
// in HBM as FP32 or FP16 deviations from the lattice weights (lbm_store.cuh),
// with the collision evaluated in FP32 (FMA contraction allowed in this file).
// Bytes per fluid-lattice update: even 19*2*s, odd 19*2*s + 72 (s = 4 or 2).
#include <atomic>
#include <type_traits>

#include "lbm_bulk.cuh"
#include "lbm_kernels.cuh"
#include "lbm_store.cuh"

namespace lbm {

template <class St>
__global__ void __launch_bounds__(kListTile) k_list_even_lp(const ListArgsLp a, const TrtW w) {
  const int n = (blockIdx.x + a.tileBase) * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  lp_even_node<St>(static_cast<typename St::T*>(a.f), a.nCells, n, TrtDev<St>(w));
}

// Even step with the PDF planes staged through shared memory by bulk copies
// (TMA, cp.async.bulk): each tile of TN = StageBytes / sizeof(T) nodes is 19
// contiguous plane segments, copied by one thread into one of Stages buffers
// with an mbarrier per buffer; Stages - 1 tiles are in flight while one is
// relaxed, so the bytes in flight per SM do not depend on registers. Stores
// go straight to global memory (coalesced, swapped planes). Requires the
// plane stride nCells to be a multiple of TN (the reduced-storage layout pads
// it to whole kLpTileNodes tiles).
template <class St, int StageBytes, int Stages>
__global__ void __launch_bounds__(256, 2) k_list_even_staged(const ListArgsLp a, const TrtW w) {
  using T = typename St::T;
  const TrtDev<St> t(w);
  constexpr int TN = StageBytes / (int)sizeof(T);
  constexpr int NPT = TN / 256;
  static_assert(TN % 256 == 0 && StageBytes % 16 == 0, "stage layout");
  extern __shared__ __align__(128) unsigned char stage[];  // Stages x Q x StageBytes
  __shared__ alignas(8) uint64_t full[Stages];
  const int nTiles = (a.nFluid + TN - 1) / TN;
  T* const f = static_cast<T*>(a.f);
  const long long S = a.nCells;
  auto issue = [&](int tile, int st) {  // thread 0
    mbar_arrive_expect_tx(&full[st], Q * StageBytes);
    unsigned char* dst = stage + (size_t)st * Q * StageBytes;
    for (int d = 0; d < Q; ++d) bulk_g2s(dst + d * StageBytes, f + d * S + (long long)tile * TN, StageBytes, &full[st]);
  };
  if (threadIdx.x == 0) {
    for (int st = 0; st < Stages; ++st) mbar_init(&full[st], 1);
    for (int st = 0; st < Stages - 1; ++st)
      if (blockIdx.x + st * gridDim.x < nTiles) issue(blockIdx.x + st * gridDim.x, st);
  }
  int i = 0;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++i) {
    const int st = i % Stages;
    __syncthreads();  // the buffer refilled below was read by everyone in the previous iteration
    if (threadIdx.x == 0) {
      const long long ahead = tile + (long long)(Stages - 1) * gridDim.x;
      if (ahead < nTiles) issue((int)ahead, (i + Stages - 1) % Stages);
    }
    if (!mbar_wait_bounded(&full[st], (i / Stages) & 1)) {
      if (threadIdx.x == 0) {
        atomicOr(a.err, 1);
        // let the copies already issued for later tiles land before the
        // block's shared memory is released
        for (int j = 1; j < Stages; ++j)
          if (tile + (long long)j * gridDim.x < nTiles)
            mbar_wait_bounded(&full[(i + j) % Stages], ((i + j) / Stages) & 1);
      }
      return;
    }
    const T* buf = reinterpret_cast<const T*>(stage + (size_t)st * Q * StageBytes);
    if constexpr (std::is_same<St, StoreF16>::value) {
      // FP16: two neighbouring nodes per thread, moved as half2 (one shared
      // memory load, one conversion and one 4-byte store per direction for
      // both); a pair's second node past nFluid is a padding node, whose
      // zero deviations relax to zero
#pragma unroll 1
      for (int k = 0; k < NPT / 2; ++k) {
        const int local = 2 * (threadIdx.x + k * 256);
        const int n = tile * TN + local;
        if (n >= a.nFluid) break;
        float fa[Q], fb[Q], oa[Q], ob[Q];
#pragma unroll
        for (int d = 0; d < Q; ++d) {
          const float2 v = StoreF16::in2(*reinterpret_cast<const __half2*>(buf + d * TN + local), d);
          fa[d] = v.x;
          fb[d] = v.y;
        }
        trt_collide_dev(t, fa, oa);
        trt_collide_dev(t, fb, ob);
        T* const fs = launder(f + n);
#pragma unroll
        for (int d = 0; d < Q; ++d)
          *reinterpret_cast<__half2*>(fs + inv(d) * S) = StoreF16::out2(oa[d], ob[d], inv(d));
      }
    } else {
#pragma unroll 1
      for (int k = 0; k < NPT; ++k) {
        const int local = threadIdx.x + k * 256;
        const int n = tile * TN + local;
        if (n >= a.nFluid) break;
        T* const fs = launder(f + n);
        float x[Q], o[Q];
#pragma unroll
        for (int d = 0; d < Q; ++d) x[d] = St::in(buf[d * TN + local], d);
        trt_collide_dev(t, x, o);
#pragma unroll
        for (int d = 0; d < Q; ++d) fs[inv(d) * S] = St::out(o[d], inv(d));
      }
    }
  }
}

// Resident blocks per SM the odd step is compiled for (6: the shared-memory
// limit of its staged run record; the register cap follows from it).
#ifndef LBM_LP_ODD_BLOCKS
#define LBM_LP_ODD_BLOCKS 6
#endif

template <class St>
__global__ void __launch_bounds__(kListTile, LBM_LP_ODD_BLOCKS) k_list_odd_lp(const ListArgsLp a, const TrtW w) {
  __shared__ alignas(128) uint32_t srun[kRunTileWords];
  __shared__ alignas(8) uint64_t bar;
  __shared__ int ok;
  if (!stage_run_tile(a, srun, &bar, &ok)) return;
  const int n = (blockIdx.x + a.tileBase) * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  uint32_t off;
  const uint32_t* e = run_row(srun, threadIdx.x, off);  // link d = e[d] + off (run-compressed adjacency)
  lp_odd_node<St>(static_cast<typename St::T*>(a.f), static_cast<uint32_t>(a.nCells), n, e, off, TrtDev<St>(w));
}

static unsigned lp_blocks(const ListArgsLp& a) { return (a.nFluid + kListTile - 1) / kListTile; }

// Staging geometry of the even step: 2 KB plane segments (1024 FP16 or 512
// FP32 nodes per tile), 2 buffers, 2 resident blocks of 256 threads per SM.
constexpr int kEvenStageBytes = 2048, kEvenStages = 2, kEvenBlocksPerSM = 2;

// The kernel's shared-memory opt-in is a per-device attribute: it is set once
// per device (and per storage type), with the grid sized to that device.
template <class St>
static void launch_even_staged(const ListArgsLp& a, const TrtW& t, cudaStream_t s) {
  constexpr int kMaxDevices = 64;
  static std::atomic<int> grid[kMaxDevices];
  constexpr size_t smem = (size_t)kEvenStages * Q * kEvenStageBytes;
  auto kern = k_list_even_staged<St, kEvenStageBytes, kEvenStages>;
  int dev = 0;
  cudaGetDevice(&dev);
  int g = dev < kMaxDevices ? grid[dev].load(std::memory_order_acquire) : 0;
  if (g == 0) {
    // idempotent: concurrent first launches on a device set the same values
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    g = sms * kEvenBlocksPerSM;
    if (dev < kMaxDevices) grid[dev].store(g, std::memory_order_release);
  }
  kern<<<g, 256, smem, s>>>(a, t);
}

// FP16: the staged even step (0.118 -> 0.100 ms at 6.7M nodes on B200, 66 ->
// 78 % of the measured HBM bandwidth). FP32: the direct kernel, whose 4-byte
// loads already keep enough bytes in flight (0.162 ms direct, 0.174 staged).
void list_even_lp(const ListArgsLp& a, const TrtW& t, int storage, cudaStream_t s) {
  if (a.nFluid <= 0) return;
  ListArgsLp b = a;
  b.tileBase = 0;
  if (storage == kStoreF16)
    launch_even_staged<StoreF16>(b, t, s);
  else
    k_list_even_lp<StoreF32><<<lp_blocks(b), kListTile, 0, s>>>(b, t);
}

// Tile ranges run the per-node kernel for both storages (the FP16 staged
// kernel works on whole 1024-node tiles).
void list_even_lp_tiles(const ListArgsLp& a, const TrtW& t, int storage, int t0, int t1, cudaStream_t s) {
  if (a.nFluid <= 0 || t1 <= t0) return;
  ListArgsLp b = a;
  b.tileBase = t0;
  if (storage == kStoreF16)
    k_list_even_lp<StoreF16><<<(unsigned)(t1 - t0), kListTile, 0, s>>>(b, t);
  else
    k_list_even_lp<StoreF32><<<(unsigned)(t1 - t0), kListTile, 0, s>>>(b, t);
}

static std::atomic<int> ahead16{0}, ahead32{0};

void list_odd_lp_tiles(const ListArgsLp& a, const TrtW& t, int storage, int t0, int t1, cudaStream_t s) {
  if (a.nFluid <= 0 || t1 <= t0) return;
  ListArgsLp b = a;
  b.tileBase = t0;
  if (storage == kStoreF16) {
    b.prefetch = prefetch_distance(ahead16, k_list_odd_lp<StoreF16>, kListTile, a.prefetch != 0);
    k_list_odd_lp<StoreF16><<<(unsigned)(t1 - t0), kListTile, 0, s>>>(b, t);
  } else {
    b.prefetch = prefetch_distance(ahead32, k_list_odd_lp<StoreF32>, kListTile, a.prefetch != 0);
    k_list_odd_lp<StoreF32><<<(unsigned)(t1 - t0), kListTile, 0, s>>>(b, t);
  }
}

void list_odd_lp(const ListArgsLp& a, const TrtW& t, int storage, cudaStream_t s) {
  if (a.nFluid <= 0) return;
  ListArgsLp b = a;
  b.tileBase = 0;
  if (storage == kStoreF16) {
    b.prefetch = prefetch_distance(ahead16, k_list_odd_lp<StoreF16>, kListTile, a.prefetch != 0);
    k_list_odd_lp<StoreF16><<<lp_blocks(b), kListTile, 0, s>>>(b, t);
  } else {
    b.prefetch = prefetch_distance(ahead32, k_list_odd_lp<StoreF32>, kListTile, a.prefetch != 0);
    k_list_odd_lp<StoreF32><<<lp_blocks(b), kListTile, 0, s>>>(b, t);
  }
}

}  // namespace lbm
