// lbm_batch.cuh -- device side of the batched list AA form: many independent
// porous domains of uneven size advanced by one launch per time step (a
// persistent grid, or one block per tile) (no counterpart in the reference, which runs one domain per process).
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
  const uint32_t* runs;   // run-compressed adjacency of the nCells nodes (kRunHdrWords)
  const uint32_t* runOff; // nTiles + 1 record offsets, 16-byte units
  long long nCells;       // padded node count (a multiple of kBatchTileNodes)
  int nFluid;
  int tileStart;          // first tile of this domain in the tile table
  TrtW trt;               // relaxation rates and body force of this domain
};

// Everything a block needs to update one tile, built on the device from the
// slot table whenever membership changes: the step kernels load one record
// per tile, from an address that depends on the tile index alone, so the
// record of a block's next tile is fetched while the current one is updated.
struct BatchTile {
  const uint32_t* run;  // this tile's run record (run-compressed adjacency)
  void* f;              // the domain's PDFs
  int nCells;           // PDF plane stride of the domain (nCells * 19 < 2^32)
  int n0;               // domain-local index of the tile's first node
  int nValid;           // fluid nodes in the tile (0..kBatchTileNodes)
  uint32_t runBytes;    // size of the run record (a multiple of 16)
  TrtW trt;             // relaxation rates and body force of the domain
};
constexpr int kTileWords = static_cast<int>(sizeof(BatchTile) / 4);  // one word per lane of a warp
static_assert(sizeof(BatchTile) % 8 == 0 && kTileWords <= 32, "tile record layout");

struct BatchArgs {
  const BatchDomain* doms;   // indexed by domain slot
  const int* tileDom;        // tile -> domain slot
  const BatchTile* tiles;    // tile records (same order as tileDom)
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
  int blocks;          // persistent grid size; 0 = one block per tile
};

// Adjacency rows of the padding nodes [nFluid, nCells): each entry points at
// the node's own slot of the inverse direction (always in range, never read
// back into a fluid node). Padding rows advance by one from node to node, so
// a tile's padding is one run in the run-compressed form.
void batch_pad_adjacency(uint32_t* adj, int nFluid, long long nCells, cudaStream_t s);

// Builds the tile records of tiles [0, nTiles).
void batch_build_tiles(const BatchDomain* doms, const int* tileDom, int nTiles, BatchTile* out, cudaStream_t s);

// grid: the launch's block count (l.blocks, or the tile-grid size when
// l.blocks is 0).
void batch_even_lp(const BatchArgs& a, const BatchLaunch& l, int grid, cudaStream_t s);
void batch_odd_lp(const BatchArgs& a, const BatchLaunch& l, int grid, cudaStream_t s);
// FP64 sums {rho, jx, jy, jz} per tile (pass 1) and per domain slot (pass 2).
void batch_moments(const BatchArgs& a, int maxTiles, double* tilePartials, const int* domTileStart,
                   const int* domTileCount, int nDomSlots, double* out, cudaStream_t s);

}  // namespace lbm
