// lbm_batch.cuh -- device side of the batched list AA form: many independent
// porous domains of uneven size advanced by one persistent launch per time
// step (no counterpart in the reference, which runs one domain per process).
//
// Each domain keeps its own list layout (fluid nodes numbered as the
// reference's list kernels, adjacency with 32-bit PDF indices relative to the
// domain's own PDF array) in its own allocations. Its node range is padded to
// whole tiles of kBatchTileNodes nodes, so that a tile never straddles two
// domains; a device tile table maps tiles to domains. Kernels read the tile
// count and the tables from device memory, so a CUDA graph captured once
// stays valid when domains are admitted or retired.
#pragma once
#include <cstdint>

#include "lbm_kernels.cuh"

namespace lbm {

constexpr int kBatchTileNodes = 256;  // node granularity of a domain's tiles

struct BatchDomain {
  void* f;                // PDFs, storage format of the batch, f[d * nCells + n]
  const uint32_t* adj;    // nTiles * kBatchTileNodes * 18 entries
  long long nCells;       // padded node count (a multiple of kBatchTileNodes)
  int nFluid;
  int tileStart;          // first tile of this domain in the tile table
  Trt<float> trt;         // relaxation and body force of this domain
};

struct BatchArgs {
  const BatchDomain* doms;   // indexed by domain slot
  const int* tileDom;        // tile -> domain slot
  const int* nTiles;         // device word: number of tiles in the table
  int* err;
  int storage;               // kStoreF32 or kStoreF16
  int blockNodes;            // nodes per block per tile pass: blockDim.x * nodesPerThread
  int nodesPerThread;
};

// Launch configuration picked by the autotuner.
struct BatchLaunch {
  int threads;         // block size
  int nodesPerThread;  // nodes each thread updates per tile
  int blocks;          // persistent grid size
};

void batch_even_lp(const BatchArgs& a, const BatchLaunch& l, cudaStream_t s);
void batch_odd_lp(const BatchArgs& a, const BatchLaunch& l, cudaStream_t s);
// FP64 sums {rho, jx, jy, jz} per tile (pass 1) and per domain slot (pass 2).
void batch_moments(const BatchArgs& a, int maxTiles, double* tilePartials, const int* domTileStart,
                   const int* domTileCount, int nDomSlots, double* out, cudaStream_t s);

}  // namespace lbm
