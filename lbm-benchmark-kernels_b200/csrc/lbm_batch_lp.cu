// lbm_batch_lp.cu -- persistent list AA kernels over a batch of domains
// (FP32 arithmetic on FP32 or FP16-deviation storage, as lbm_kernels_lp.cu).
//
// Every block walks the tile records with a grid stride (one tile per block
// when the grid covers the table). The odd step stages a tile's run record
// (run-compressed adjacency of 256 nodes, at most 18480 bytes, contiguous)
// into shared memory with one bulk copy, double buffered in the persistent
// kernel: while a tile is relaxed, the bulk copy of the block's next tile is
// already in flight.
#include "lbm_batch.cuh"
#include "lbm_bulk.cuh"
#include "lbm_store.cuh"

namespace lbm {

// Warp 0 moves tile records: each lane loads one 32-bit word (the load of the
// block's next-but-one record is issued before the current tile is updated
// and consumed after it), then stores it to shared memory.
__device__ __forceinline__ uint32_t tile_load(const BatchTile* tiles, int tile) {
  const int lane = threadIdx.x;
  return lane < kTileWords ? __ldg(reinterpret_cast<const uint32_t*>(tiles + tile) + lane) : 0u;
}

__device__ __forceinline__ void tile_store(BatchTile* dst, uint32_t w) {
  const int lane = threadIdx.x;
  if (lane < kTileWords) reinterpret_cast<uint32_t*>(dst)[lane] = w;
}

template <class St>
__device__ __forceinline__ void batch_even_node(const BatchTile& T, int n) {
  lp_even_node<St, false>(static_cast<typename St::T*>(T.f), T.nCells, n, TrtDev<St>(T.trt));
}

// Grid-stride over the tiles; with one block per tile the loop runs once.
template <class St>
__global__ void __launch_bounds__(256) k_batch_even(const BatchArgs a) {
  __shared__ __align__(16) BatchTile st[2];
  const int nT = *a.nTiles;
  if (static_cast<int>(blockIdx.x) >= nT) return;
  const bool warp0 = threadIdx.x < 32;
  uint32_t r = 0;
  if (warp0) {
    r = tile_load(a.tiles, blockIdx.x);
    tile_store(&st[0], r);
    if (static_cast<int>(blockIdx.x + gridDim.x) < nT) r = tile_load(a.tiles, blockIdx.x + gridDim.x);
  }
  int it = 0;
  for (int tile = blockIdx.x; tile < nT; tile += gridDim.x, ++it) {
    const int buf = it & 1;
    __syncthreads();  // st[buf] is written; every thread is done with st[buf ^ 1]
    const int next = tile + gridDim.x;
    if (warp0 && next < nT) {
      tile_store(&st[buf ^ 1], r);
      if (next + static_cast<int>(gridDim.x) < nT) r = tile_load(a.tiles, next + gridDim.x);
    }
    const BatchTile& T = st[buf];
    for (int k = 0; k < a.nodesPerThread; ++k) {
      const int local = threadIdx.x + k * blockDim.x;
      if (local < T.nValid) batch_even_node<St>(T, T.n0 + local);
    }
  }
}

// One node of a tile whose run record is staged in srun (local = the node's
// index in the tile): link d is e[d] + off.
template <class St>
__device__ __forceinline__ void batch_odd_node(const BatchTile& T, const uint32_t* srun, int local) {
  uint32_t off;
  const uint32_t* e = run_row(srun, local, off);
  lp_odd_node<St, false>(static_cast<typename St::T*>(T.f), static_cast<uint32_t>(T.nCells), T.n0 + local, e, off,
                  TrtDev<St>(T.trt));
}

static_assert(kBatchTileNodes == kListTile, "batch tiles are the run records' tiles");
constexpr uint32_t kRunRecordMax = kRunTileWords * 4;  // largest run record, bytes

__device__ __forceinline__ bool run_bytes_ok(uint32_t bytes) { return bytes > 0 && bytes <= kRunRecordMax; }

// As k_batch_even, with the tile's adjacency staged into shared memory by one
// bulk copy, double buffered: the copy of the block's next tile is issued
// before the current tile is updated.
template <class St>
__global__ void __launch_bounds__(256) k_batch_odd(const BatchArgs a) {
  extern __shared__ __align__(128) uint32_t sadj[];  // 2 x kRunTileWords
  __shared__ alignas(8) uint64_t bar[2];
  __shared__ __align__(16) BatchTile st[2];
  const int nT = *a.nTiles;
  if (static_cast<int>(blockIdx.x) >= nT) return;
  const bool warp0 = threadIdx.x < 32;
  uint32_t r = 0;
  auto issue = [&](int buf) {  // thread 0, once st[buf] holds the tile's record
    // a record that does not fit is not copied: 0 bytes complete the phase
    // at once, and the tile is skipped below with error bit 4
    const uint32_t bytes = run_bytes_ok(st[buf].runBytes) ? st[buf].runBytes : 0u;
    if (bytes) {
      mbar_arrive_expect_tx(&bar[buf], bytes);
      bulk_g2s(sadj + buf * kRunTileWords, st[buf].run, bytes, &bar[buf]);
    } else {
      atomicOr(a.err, 4);
      mbar_arrive_expect_tx(&bar[buf], 0);
    }
  };
  if (warp0) {
    r = tile_load(a.tiles, blockIdx.x);
    tile_store(&st[0], r);
    __syncwarp();
    if (threadIdx.x == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      issue(0);
    }
    if (static_cast<int>(blockIdx.x + gridDim.x) < nT) r = tile_load(a.tiles, blockIdx.x + gridDim.x);
  }
  int it = 0;
  for (int tile = blockIdx.x; tile < nT; tile += gridDim.x, ++it) {
    const int buf = it & 1;
    __syncthreads();  // st[buf] is written; every thread is done with buffers buf ^ 1
    const int next = tile + gridDim.x;
    if (warp0 && next < nT) {
      tile_store(&st[buf ^ 1], r);
      __syncwarp();
      if (threadIdx.x == 0) issue(buf ^ 1);
      if (next + static_cast<int>(gridDim.x) < nT) r = tile_load(a.tiles, next + gridDim.x);
    }
    if (!mbar_wait_bounded(&bar[buf], (it >> 1) & 1)) {
      if (threadIdx.x == 0) {
        atomicOr(a.err, 1);
        // let the copy already issued for the next tile land before the
        // block's shared memory is released
        if (next < nT) mbar_wait_bounded(&bar[buf ^ 1], ((it + 1) >> 1) & 1);
      }
      return;
    }
    const BatchTile& T = st[buf];
    if (!run_bytes_ok(T.runBytes)) continue;
    const uint32_t* srun = sadj + buf * kRunTileWords;
    for (int k = 0; k < a.nodesPerThread; ++k) {
      const int local = threadIdx.x + k * blockDim.x;
      if (local < T.nValid) batch_odd_node<St>(T, srun, local);
    }
  }
}

// One block per tile: no loop state stays live across the node update, so
// these take fewer registers (more resident blocks) than the persistent
// kernels. NPT nodes per thread, blockDim = kBatchTileNodes / NPT.
template <class St, int NPT>
__global__ void __launch_bounds__(kBatchTileNodes / NPT) k_batch_even_tile(const BatchArgs a) {
  __shared__ __align__(16) BatchTile st;
  if (static_cast<int>(blockIdx.x) >= *a.nTiles) return;
  if (threadIdx.x < 32) tile_store(&st, tile_load(a.tiles, blockIdx.x));
  __syncthreads();
#pragma unroll 1
  for (int k = 0; k < NPT; ++k) {
    const int local = threadIdx.x + k * (kBatchTileNodes / NPT);
    if (local < st.nValid) batch_even_node<St>(st, st.n0 + local);
  }
}

// 6 tiles' blocks resident per SM (the shared-memory limit of the staged run
// records), which caps the registers at 40.
template <class St, int NPT>
__global__ void __launch_bounds__(kBatchTileNodes / NPT, 6 * NPT) k_batch_odd_tile(const BatchArgs a) {
  __shared__ __align__(128) uint32_t srun[kRunTileWords];
  __shared__ alignas(8) uint64_t bar;
  __shared__ __align__(16) BatchTile st;
  if (static_cast<int>(blockIdx.x) >= *a.nTiles) return;
  if (threadIdx.x < 32) {
    tile_store(&st, tile_load(a.tiles, blockIdx.x));
    __syncwarp();
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      if (run_bytes_ok(st.runBytes)) {
        mbar_arrive_expect_tx(&bar, st.runBytes);
        bulk_g2s(srun, st.run, st.runBytes, &bar);
      } else {
        atomicOr(a.err, 4);
      }
    }
  }
  __syncthreads();
  if (!run_bytes_ok(st.runBytes)) return;
  if (!mbar_wait_bounded(&bar, 0)) {
    if (threadIdx.x == 0) atomicOr(a.err, 1);
    return;
  }
#pragma unroll 1
  for (int k = 0; k < NPT; ++k) {
    const int local = threadIdx.x + k * (kBatchTileNodes / NPT);
    if (local < st.nValid) batch_odd_node<St>(st, srun, local);
  }
}

template <class St>
static void launch_even(const BatchArgs& a, const BatchLaunch& l, int grid, cudaStream_t s) {
  if (l.blocks > 0)
    k_batch_even<St><<<grid, l.threads, 0, s>>>(a);
  else if (l.nodesPerThread == 4)
    k_batch_even_tile<St, 4><<<grid, kBatchTileNodes / 4, 0, s>>>(a);
  else if (l.nodesPerThread == 2)
    k_batch_even_tile<St, 2><<<grid, kBatchTileNodes / 2, 0, s>>>(a);
  else
    k_batch_even_tile<St, 1><<<grid, kBatchTileNodes, 0, s>>>(a);
}

template <class St>
static void launch_odd(const BatchArgs& a, const BatchLaunch& l, int grid, cudaStream_t s) {
  if (l.blocks > 0)
    k_batch_odd<St><<<grid, l.threads, 2 * (size_t)kRunRecordMax, s>>>(a);
  else if (l.nodesPerThread == 4)
    k_batch_odd_tile<St, 4><<<grid, kBatchTileNodes / 4, 0, s>>>(a);
  else if (l.nodesPerThread == 2)
    k_batch_odd_tile<St, 2><<<grid, kBatchTileNodes / 2, 0, s>>>(a);
  else
    k_batch_odd_tile<St, 1><<<grid, kBatchTileNodes, 0, s>>>(a);
}

void batch_even_lp(const BatchArgs& a, const BatchLaunch& l, int grid, cudaStream_t s) {
  if (a.storage == kStoreF16)
    launch_even<StoreF16>(a, l, grid, s);
  else
    launch_even<StoreF32>(a, l, grid, s);
}

void batch_odd_lp(const BatchArgs& a, const BatchLaunch& l, int grid, cudaStream_t s) {
  if (a.storage == kStoreF16)
    launch_odd<StoreF16>(a, l, grid, s);
  else
    launch_odd<StoreF32>(a, l, grid, s);
}

__global__ void k_batch_tiles(const BatchDomain* doms, const int* tileDom, int nTiles, BatchTile* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nTiles) return;
  const BatchDomain& D = doms[tileDom[t]];
  const int lt = t - D.tileStart;
  BatchTile r;
  const uint32_t o0 = D.runOff[lt], o1 = D.runOff[lt + 1];
  r.run = D.runs + static_cast<size_t>(o0) * 4;
  r.runBytes = (o1 - o0) * 16u;
  r.f = D.f;
  r.nCells = static_cast<int>(D.nCells);
  r.n0 = lt * kBatchTileNodes;
  r.nValid = max(0, min(kBatchTileNodes, D.nFluid - r.n0));
  r.trt = D.trt;
  out[t] = r;
}

__global__ void k_batch_pad_adjacency(uint32_t* adj, int nFluid, long long nCells) {
  const long long n = nFluid + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nCells) return;
#pragma unroll
  for (int q = 0; q < QM; ++q) adj[n * QM + q] = (uint32_t)(inv(q) * nCells + n);
}

void batch_pad_adjacency(uint32_t* adj, int nFluid, long long nCells, cudaStream_t s) {
  const long long pad = nCells - nFluid;
  if (pad > 0) k_batch_pad_adjacency<<<(unsigned)((pad + 255) / 256), 256, 0, s>>>(adj, nFluid, nCells);
}

void batch_build_tiles(const BatchDomain* doms, const int* tileDom, int nTiles, BatchTile* out, cudaStream_t s) {
  if (nTiles > 0) k_batch_tiles<<<(nTiles + 255) / 256, 256, 0, s>>>(doms, tileDom, nTiles, out);
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
    k_batch_moments_tile<StoreF16><<<blocks, kBatchTileNodes, 0, s>>>(a, maxTiles, tilePartials);
  else
    k_batch_moments_tile<StoreF32><<<blocks, kBatchTileNodes, 0, s>>>(a, maxTiles, tilePartials);
  k_batch_moments_dom<<<(nDomSlots + 127) / 128, 128, 0, s>>>(tilePartials, domTileStart, domTileCount, nDomSlots, out);
}

}  // namespace lbm
