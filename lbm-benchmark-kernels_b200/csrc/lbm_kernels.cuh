// lbm_kernels.cuh -- argument blocks and launchers of the sm_100a D3Q19 TRT
// time-step kernels (definitions in lbm_kernels_fp64.cu).
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "lbm_d3q19.cuh"

namespace lbm {

// ---------------------------------------------------------------------------
// Full-array AA layout on the device.
//
// SoA, one plane per direction. Cells carry the reference's one-cell ghost
// layer ((nX+2) x (nY+2) x (nZ+2), src/BenchKernelD3Q19AaCommon.c:331-337) so
// that non-periodic fluid faces keep the reference's semantics, but the z rows
// are padded: interior z = 0 sits at element kZOff of a row whose pitch is a
// multiple of 4 doubles, so every warp's 32 consecutive z cells start on a 32 B
// sector boundary.
//   cell(x, y, z) = (x + 1) * xs + (y + 1) * pitch + z + kZOff   (x,y,z interior coords)
//   pdf(d, cell)  = f[d * dstride + cell]
// link[cell] (uint32): bit 31 = fluid cell; bit d (d < 18) = the neighbour
// x + c_d is not a fluid node reached directly or through a periodic wrap
// (a wall: bounce back, or an open non-periodic face).
constexpr int kZOff = 4;
constexpr uint32_t kFluidBit = 0x80000000u;
constexpr uint32_t kLinkBits = 0x3ffffu;  // the 18 reversed-link bits

struct AaArgs {
  double* f;
  double* g;  // two-grid full-array kernels: the destination grid (same layout)
  long long dstride;
  const uint32_t* link;
  int nX, nY, nZ;
  int xs, pitch;
  int perX, perY, perZ;
  // element offsets from a cell's slot of plane 0, per direction d, read from
  // the parameter bank: the odd step's load of d (slot inv(d) of x + c_inv(d))
  // and store of d (slot d of x + c_d); the centre uses its own slot
  int ldOff[Q], stOff[Q];
  // x-slab of a larger lattice: a halo face (haloLo at x = 0, haloHi at
  // x = nX-1) borders the neighbouring slab, whose face plane the ghost plane
  // mirrors (exchanged around the odd step); cross* marks a halo face that is
  // also the lattice's periodic x boundary. All 0 for a whole lattice.
  int haloLo, haloHi, crossLo, crossHi;
  int xBase;  // even step: first x plane of the launch (grid z = planes launched)
};

// x-slab halo exchange (lbm_kernels_fp64.cu). A message is the 5 PDFs that
// cross one x face, over the face's nY x nZ cells: [k][y][z]. side 0 = the
// x = 0 face, 1 = the x = nX-1 face. Phase 0 (after the even step): pack the
// face plane's slots that the neighbour's cells read and write in the odd
// step / unpack them into the ghost plane. Phase 1 (after the odd step): pack
// the ghost plane's slots this slab's cells wrote / unpack them into the face
// plane.
void aa_halo_pack(const AaArgs& a, int side, int phase, double* buf, cudaStream_t s);
void aa_halo_unpack(const AaArgs& a, int side, int phase, const double* buf, cudaStream_t s);

// ---------------------------------------------------------------------------
// Fluid-node list layout (the reference's list kernels).
//   pdf(d, n) = f[d * nCells + n], nCells = padded cell count
//   adj[n * 18 + d] = PDF index (d' * nCells + m) of link d of node n, push or
//   pull as in src/BenchKernelD3Q19ListAaPvCommon.c:700-792 /
//   src/BenchKernelD3Q19ListPullSplitNtCommon.c:662-755.
// The adjacency allocation holds whole tiles of kListTile nodes so that every
// tile can be fetched with one bulk copy.
constexpr int kListTile = 256;

// Run-compressed adjacency (the reference's consecutive nodes,
// src/BenchKernelD3Q19ListAaPvCommon.c:326-469, cut at tiles of kListTile
// nodes): node n starts a run unless every link of n is the same link of
// n - 1 plus one, and a tile's first node always starts one. Per tile, at
// runs + 4 * runOff[t] (16-byte units): a header of kRunHdrWords words (the
// head mask: bit k of word w = node 32 w + k of the tile starts a run; then
// the heads before each mask word, byte w of words 8-9; 2 zero words) and
// one 18-entry row per head, the head count rounded up to even (a multiple
// of 16 bytes). A node's link d is its head's link d plus its distance from
// the head.
constexpr int kRunHdrWords = 12;
constexpr int kRunTileWords = kRunHdrWords + kListTile * 18;

struct ListArgs {
  double* f;      // list AA: the one grid; pull: source grid
  double* g;      // pull: destination grid
  const uint32_t* adj;
  long long nCells;
  int nFluid;
  int* err;       // device error word (bounded waits)
  int prefetch;   // tiles ahead whose adjacency a block prefetches into L2 (0: none)
  const uint32_t* runs;    // run-compressed adjacency (list AA odd step, list push)
  const uint32_t* runOff;  // nTiles + 1 tile offsets into runs, 16-byte units
  int tileBase;            // first tile of the launch (block b updates tile tileBase + b)
};

// The prefetch distance of a launch of `kernel` (threads per block): its
// resident blocks across the device, so that a block prefetches the tile of
// the block that takes its place when the first wave retires. `ahead` caches
// it per launcher; `enabled` false gives 0 (no prefetch).
template <class K>
int prefetch_distance(std::atomic<int>& ahead, K kernel, int threads, bool enabled) {
  if (!enabled) return 0;
  int v = ahead.load(std::memory_order_acquire);
  if (v <= 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0);
    v = sms * per;
    ahead.store(v, std::memory_order_release);
  }
  return v;
}

// Reduced-storage list AA (lbm_kernels_lp.cu): PDFs stored as FP32 or as
// scaled FP16 deviations from the weights, collision in FP32.
constexpr int kStoreF64 = 0;
constexpr int kStoreF32 = 1;
constexpr int kStoreF16 = 2;

// Plane stride granularity of the reduced-storage list layout: nCells is a
// multiple of this, so that every plane segment of an even-step tile is one
// aligned bulk copy inside the array.
constexpr int kLpTileNodes = 1024;

struct ListArgsLp {
  void* f;  // float or __half, f[d * nCells + n]
  const uint32_t* adj;
  const uint32_t* runs;    // as ListArgs
  const uint32_t* runOff;
  long long nCells;
  int nFluid;
  int* err;
  int prefetch;  // as ListArgs::prefetch
  int tileBase;  // as ListArgs::tileBase
};

// List layout built on the device (lbm_build.cu): numbering into grid (one
// entry per cell), adjacency for up to adjCap nodes. Synchronises s. Returns
// the fluid node count, -1 on a CUDA error, -2 if adjCap is too small.
long long list_build_device(const int* mask, const int dims[3], const int periodic[3], int pull, const int blk[3],
                            int nCells, uint32_t* grid, uint32_t* adj, long long adjCap, cudaStream_t s,
                            const char** err);

// Halo messages of a list slab: buf[k] = f[idx[k]] (gather) and
// f[idx[k]] = buf[k] (scatter) for k < n, elements of elemBytes (8, 4 or 2:
// the slab's PDF storage) moved bit for bit.
void slot_gather(const void* f, const uint32_t* idx, long long n, void* buf, int elemBytes, cudaStream_t s);
void slot_scatter(void* f, const uint32_t* idx, long long n, const void* buf, int elemBytes, cudaStream_t s);

// Run-compressed adjacency of the nFluid nodes of adj (device, 18 entries
// per node): allocates *runs (cudaMalloc, *runBytes bytes) and *runOff
// (nTiles + 1 entries) and fills them; synchronises s. Returns 0 or a CUDA
// error code.
int list_runs_device(const uint32_t* adj, int nFluid, cudaStream_t s, uint32_t** runs, uint32_t** runOff,
                     size_t* runBytes);

// Launchers (stream-ordered, no synchronisation).
void list_even_lp(const ListArgsLp& a, const TrtW& t, int storage, cudaStream_t s);
void list_odd_lp(const ListArgsLp& a, const TrtW& t, int storage, cudaStream_t s);
// The odd steps over tiles [t0, t1) only (slabs overlap their halo exchange
// with the tiles that read no ghost node).
void list_odd_fp64_tiles(const ListArgs& a, const Trt<double>& t, int t0, int t1, cudaStream_t s);
// The even steps over tiles [t0, t1) (reduced storage: the per-node kernel,
// also for FP16, whose whole-array step is the staged kernel) and the
// full-array even step over x planes [x0, x1).
void list_even_fp64_tiles(const ListArgs& a, const Trt<double>& t, int t0, int t1, cudaStream_t s);
void list_even_lp_tiles(const ListArgsLp& a, const TrtW& t, int storage, int t0, int t1, cudaStream_t s);
void aa_even_fp64_planes(const AaArgs& a, const Trt<double>& t, int x0, int x1, cudaStream_t s);
void list_odd_lp_tiles(const ListArgsLp& a, const TrtW& t, int storage, int t0, int t1, cudaStream_t s);
void aa_even_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s);
// The AA odd step: the interior launch over a list of work items (built by
// aa_interior_items), then the face shell.
void aa_odd_interior_fp64(const AaArgs& a, const Trt<double>& t, const int* items, int nItems, const int* cells,
                          cudaStream_t s);
// Host: the interior work items of the odd step from the link words (link:
// the host copy of the device link array), in x-plane order. Per plane:
// the ids of the interior blocks that hold at least one direct fluid cell
// (no reversed link), then one item ~k per chunk k of 128 entries of `cells`
// (the cell indices of the plane's interior fluid cells with a reversed
// link, ascending, the last chunk padded with -1).
long long aa_interior_block_count(const AaArgs& a);
void aa_interior_items(const AaArgs& a, const uint32_t* link, std::vector<int>& items, std::vector<int>& cells);
void aa_odd_face_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s);
bool aa_has_interior(const AaArgs& a);
// Two-grid full-array push / pull steps (push-soa / pull-soa): every fluid
// cell from grid a.f into grid a.g.
void fa_push_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s);
void fa_pull_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s);
long long aa_shell_cells(const AaArgs& a);
// Whether the face kernel has cells to take: the shell exists and the
// interior launch does not cover the whole lattice (it does when every axis
// is periodic and no x face is a halo face).
bool aa_shell_needed(const AaArgs& a);
void list_even_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s);
void list_odd_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s);
void list_pull_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s);
void list_push_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s);

// The -verify check on the device (lbm_verify.cu). A slice cell i = y * nZ +
// z at x = nX/2 reads PDF d at element base[i] + off[d] of f (storage
// kStoreF64/F32/F16); base[i] < 0 marks an obstacle. Writes the x-velocity
// slice (nY * nZ doubles) and err[0] = the Poiseuille error norm.
struct VerifyArgs {
  const void* f;
  int storage;
  const long long* base;
  long long off[Q];
  int nY, nZ;
  double xforce, visc;
};
void verify_device(const VerifyArgs& a, double* slice, double* err, cudaStream_t s);

// FP64 mass and momentum sums of a list-layout field (lbm_moments.cu):
// pass 1 writes 4 partial sums per block of kListTile nodes into `partials`
// (moment_blocks(nFluid) * 4 doubles), pass 2 folds them into out[0..3] =
// {sum rho, sum j_x, sum j_y, sum j_z}.
int moment_blocks(int nFluid);
void moments_enqueue(const double* f, long long nCells, int nFluid, double* partials, double* out, cudaStream_t s);
// The same sums over reduced storage (kStoreF32 / kStoreF16 deviations).
void moments_enqueue_lp(const void* f, int storage, long long nCells, int nFluid, double* partials, double* out,
                        cudaStream_t s);

}  // namespace lbm
