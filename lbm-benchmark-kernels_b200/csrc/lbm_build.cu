// lbm_build.cu -- the list layout built on the GPU: fluid-node numbering in
// the reference's blocked order and the 18-link push or pull adjacency
// (src/BenchKernelD3Q19ListAaPvCommon.c:587-792,
// src/BenchKernelD3Q19ListPullSplitNtCommon.c:548-755), bit-identical to the
// host builder lbmh_list_build (lbm_host.c), in a few milliseconds instead of
// seconds at 256^3.
//
// Three passes over the cells in numbering order (position p):
//   1. flag[p] = the cell at p is not an obstacle;
//   2. exclusive prefix sum of the flags = the node index of each fluid cell;
//   3. grid[cell] = node; then, once the grid is complete, each node's 18
//      adjacency entries from its neighbours' node indices.
#include <cstdint>
#include <cstdio>

#include <cub/device/device_scan.cuh>

#include "../../include/lbm_b200.h"
#include "lbm_d3q19.cuh"
#include "lbm_kernels.cuh"

namespace lbm {

struct BuildGeom {
  int nx, ny, nz;
  int bx, by, bz;  // block extents of the numbering
  int per[3];
  long long n;     // cells
};

// Cell (x, y, z) at numbering position p: blocks of bx x by x bz cells in
// x -> y -> z order (edge blocks smaller), x -> y -> z inside a block, z
// innermost.
__device__ __forceinline__ void build_cell_of(const BuildGeom& g, long long p, int& x, int& y, int& z) {
  const long long slabX = (long long)g.bx * g.ny * g.nz;
  const int x0 = (int)(p / slabX) * g.bx;
  long long r = p % slabX;
  const int wx = min(g.bx, g.nx - x0);
  const long long slabY = (long long)wx * g.by * g.nz;
  const int y0 = (int)(r / slabY) * g.by;
  r %= slabY;
  const int wy = min(g.by, g.ny - y0);
  const long long slabZ = (long long)wx * wy * g.bz;
  const int z0 = (int)(r / slabZ) * g.bz;
  r %= slabZ;
  const int wz = min(g.bz, g.nz - z0);
  x = x0 + (int)(r / ((long long)wy * wz));
  y = y0 + (int)(r / wz % wy);
  z = z0 + (int)(r % wz);
}

__device__ __forceinline__ long long build_lidx(const BuildGeom& g, int x, int y, int z) {
  return ((long long)z * g.ny + y) * g.nx + x;
}

__global__ void k_build_flags(BuildGeom g, const int* mask, uint32_t* flag, uint32_t* grid) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.n) return;
  int x, y, z;
  build_cell_of(g, p, x, y, z);
  flag[p] = mask[build_lidx(g, x, y, z)] != LAT_CELL_OBSTACLE ? 1u : 0u;
  grid[p] = 0xffffffffu;  // grid is indexed by cell; every entry is reset here
}

__global__ void k_build_grid(BuildGeom g, const uint32_t* flag, const uint32_t* node, uint32_t* grid) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.n || !flag[p]) return;
  int x, y, z;
  build_cell_of(g, p, x, y, z);
  grid[build_lidx(g, x, y, z)] = node[p];
}

__global__ void k_build_adj(BuildGeom g, int pull, uint32_t nCells, const uint32_t* flag, const uint32_t* node,
                            const uint32_t* grid, uint32_t* adj) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= g.n || !flag[p]) return;
  int x, y, z;
  build_cell_of(g, p, x, y, z);
  const uint32_t self = node[p];
  const int sign = pull ? -1 : 1;
  const int dims[3] = {g.nx, g.ny, g.nz};
  uint32_t* row = adj + (size_t)self * QM;
#pragma unroll
  for (int d = 0; d < QM; ++d) {
    int q[3] = {x + sign * cx(d), y + sign * cy(d), z + sign * cz(d)};
    bool out = false, crossPer = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool o = q[a] < 0 || q[a] >= dims[a];
      out = out || o;
      crossPer = crossPer || (o && g.per[a]);
    }
    uint32_t dst = (uint32_t)inv(d) * nCells + self;  // bounce back by default
    if (crossPer) {
      // every crossed axis wraps once a periodic one is crossed
#pragma unroll
      for (int a = 0; a < 3; ++a) q[a] = q[a] < 0 ? dims[a] - 1 : (q[a] >= dims[a] ? 0 : q[a]);
      out = false;
    }
    if (!out) {
      const uint32_t m = grid[build_lidx(g, q[0], q[1], q[2])];
      if (m != 0xffffffffu) dst = (uint32_t)d * nCells + m;
    }
    row[d] = dst;
  }
}

// Device build. mask: nx*ny*nz ints (x fastest); grid: same count of
// uint32; adj: room for adjCap nodes (18 entries each). Temporary device
// memory is allocated and freed here; synchronises the stream. Returns the
// fluid node count; -1 on a CUDA error (message in *err); -2 (adjacency not
// written) when the mask has more fluid cells than adjCap.
long long list_build_device(const int* mask, const int dims[3], const int periodic[3], int pull, const int blk[3],
                            int nCells, uint32_t* grid, uint32_t* adj, long long adjCap, cudaStream_t s,
                            const char** err) {
  BuildGeom g;
  g.nx = dims[0];
  g.ny = dims[1];
  g.nz = dims[2];
  g.bx = blk && blk[0] > 0 ? blk[0] : g.nx;
  g.by = blk && blk[1] > 0 ? blk[1] : g.ny;
  g.bz = blk && blk[2] > 0 ? blk[2] : g.nz;
  for (int a = 0; a < 3; ++a) g.per[a] = periodic[a];
  g.n = (long long)g.nx * g.ny * g.nz;
  *err = "";
  if (g.n <= 0) return 0;
  uint32_t *flag = nullptr, *node = nullptr;
  void* tmp = nullptr;
  size_t tmpBytes = 0;
  long long count = -1;
  uint32_t last[2] = {0, 0};
  const unsigned blocks = (unsigned)((g.n + 255) / 256);
  cudaError_t e = cudaMallocAsync(&flag, sizeof(uint32_t) * g.n, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&node, sizeof(uint32_t) * g.n, s);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, flag, node, (int)g.n, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&tmp, tmpBytes, s);
  if (e == cudaSuccess) {
    k_build_flags<<<blocks, 256, 0, s>>>(g, mask, flag, grid);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmpBytes, flag, node, (int)g.n, s);
  if (e == cudaSuccess) {
    k_build_grid<<<blocks, 256, 0, s>>>(g, flag, node, grid);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&last[0], flag + g.n - 1, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&last[1], node + g.n - 1, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) count = (long long)last[0] + last[1];
  if (e == cudaSuccess && count > adjCap) {
    count = -2;
    *err = "the mask has more fluid cells than the adjacency holds";
  }
  if (e == cudaSuccess && count > 0) {
    k_build_adj<<<blocks, 256, 0, s>>>(g, pull, (uint32_t)nCells, flag, node, grid, adj);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  cudaFreeAsync(tmp, s);
  cudaFreeAsync(node, s);
  cudaFreeAsync(flag, s);
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return -1;
  }
  return count;
}

// --- run-compressed adjacency ----------------------------------------------------

// One block of kListTile threads per tile: the tile's head mask.
__global__ void k_run_heads(const uint32_t* __restrict__ adj, int nFluid, uint32_t* __restrict__ mask) {
  const long long n = (long long)blockIdx.x * kListTile + threadIdx.x;
  bool head = false;
  if (n < nFluid) {
    head = threadIdx.x == 0;
    for (int d = 0; d < QM && !head; ++d) head = adj[n * QM + d] != adj[(n - 1) * QM + d] + 1u;
  }
  const uint32_t m = __ballot_sync(0xffffffffu, head);
  if ((threadIdx.x & 31) == 0) mask[(size_t)blockIdx.x * (kListTile / 32) + (threadIdx.x >> 5)] = m;
}

// Size of each tile's record in 16-byte units (entry nTiles: 0, so that the
// exclusive sum ends with the total).
__global__ void k_run_sizes(const uint32_t* __restrict__ mask, int nTiles, uint32_t* __restrict__ size16) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > nTiles) return;
  if (t == nTiles) { size16[t] = 0; return; }
  int h = 0;
  for (int k = 0; k < kListTile / 32; ++k) h += __popc(mask[(size_t)t * (kListTile / 32) + k]);
  const int h2 = (h + 1) & ~1;
  size16[t] = (uint32_t)(kRunHdrWords / 4 + h2 * QM / 4);
}

__global__ void k_run_fill(const uint32_t* __restrict__ adj, int nFluid, const uint32_t* __restrict__ mask,
                           const uint32_t* __restrict__ runOff, uint32_t* __restrict__ runs) {
  const int t = blockIdx.x;
  uint32_t* const rec = runs + (size_t)runOff[t] * 4;
  const uint32_t* const m = mask + (size_t)t * (kListTile / 32);
  if (threadIdx.x < kRunHdrWords) {
    uint32_t v = 0u;
    if (threadIdx.x < kListTile / 32) {
      v = m[threadIdx.x];
    } else if (threadIdx.x < kListTile / 32 + 2) {
      // heads before mask words 4 q .. 4 q + 3, one byte each (at most 224)
      const int q = threadIdx.x - kListTile / 32;
      int before = 0;
      for (int k = 0; k < 4 * q; ++k) before += __popc(m[k]);
      for (int k = 0; k < 4; ++k) {
        v |= static_cast<uint32_t>(before) << (8 * k);
        before += __popc(m[4 * q + k]);
      }
    }
    rec[threadIdx.x] = v;
  }
  const long long n = (long long)t * kListTile + threadIdx.x;
  if (n >= nFluid) return;
  const int w = threadIdx.x >> 5, b = threadIdx.x & 31;
  if (!((m[w] >> b) & 1u)) return;
  int rank = 0;
  for (int k = 0; k < w; ++k) rank += __popc(m[k]);
  rank += __popc(m[w] & ((2u << b) - 1u)) - 1;  // heads before this one
  uint32_t* const row = rec + kRunHdrWords + rank * QM;
  for (int d = 0; d < QM; ++d) row[d] = adj[n * QM + d];
}

int list_runs_device(const uint32_t* adj, int nFluid, cudaStream_t s, uint32_t** runs, uint32_t** runOff,
                     size_t* runBytes) {
  *runs = nullptr;
  *runOff = nullptr;
  *runBytes = 0;
  const int nTiles = (nFluid + kListTile - 1) / kListTile;
  uint32_t *mask = nullptr, *size16 = nullptr;
  void* tmp = nullptr;
  size_t tmpBytes = 0;
  uint32_t total = 0;
  cudaError_t e = cudaMalloc(runOff, sizeof(uint32_t) * (nTiles + 1));
  if (e == cudaSuccess) e = cudaMallocAsync(&mask, sizeof(uint32_t) * (size_t)(nTiles > 0 ? nTiles : 1) * 8, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&size16, sizeof(uint32_t) * (nTiles + 1), s);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, size16, *runOff, nTiles + 1, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&tmp, tmpBytes, s);
  if (e == cudaSuccess && nTiles > 0) {
    k_run_heads<<<nTiles, kListTile, 0, s>>>(adj, nFluid, mask);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_run_sizes<<<(nTiles + 1 + 255) / 256, 256, 0, s>>>(mask, nTiles, size16);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmpBytes, size16, *runOff, nTiles + 1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, *runOff + nTiles, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    *runBytes = (size_t)(total > 0 ? total : 1) * 16;
    e = cudaMalloc(runs, *runBytes);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(*runs, 0, *runBytes, s);
  if (e == cudaSuccess && nTiles > 0) {
    k_run_fill<<<nTiles, kListTile, 0, s>>>(adj, nFluid, mask, *runOff, *runs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(tmp, s);
  cudaFreeAsync(size16, s);
  cudaFreeAsync(mask, s);
  cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaFree(*runs);
    cudaFree(*runOff);
    *runs = nullptr;
    *runOff = nullptr;
    return (int)e;
  }
  return 0;
}

}  // namespace lbm

extern "C" {

// Declared in include/lbm_b200.h.
int lbm_b200_list_build(const LatticeDesc* ld, int pull, const int blk[3], int nCells, uint32_t* grid,
                        uint32_t* adj) {
  const long long n = (long long)ld->Dims[0] * ld->Dims[1] * ld->Dims[2];
  const int per[3] = {ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ};
  int* dMask = nullptr;
  uint32_t *dGrid = nullptr, *dAdj = nullptr;
  const size_t adjN = (size_t)(ld->nFluid > 0 ? ld->nFluid : 1) * lbm::QM;
  cudaStream_t s = nullptr;
  long long count = -1;
  const char* err = "";
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&dMask, sizeof(int) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dGrid, sizeof(uint32_t) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dAdj, sizeof(uint32_t) * adjN);
  if (e == cudaSuccess) e = cudaMemcpy(dMask, ld->Lattice, sizeof(int) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    count = lbm::list_build_device(dMask, ld->Dims, per, pull, blk, nCells, dGrid, dAdj,
                                   ld->nFluid > 0 ? ld->nFluid : 0, s, &err);
    if (count < 0) std::fprintf(stderr, "lbm_b200_list_build: %s\n", err);
  }
  if (e == cudaSuccess && count >= 0) {
    e = cudaMemcpy(grid, dGrid, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && count > 0) e = cudaMemcpy(adj, dAdj, sizeof(uint32_t) * count * lbm::QM, cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) std::fprintf(stderr, "lbm_b200_list_build: %s\n", cudaGetErrorString(e));
  cudaFree(dAdj);
  cudaFree(dGrid);
  cudaFree(dMask);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) return -1;
  return (int)count;
}

}  // extern "C"
