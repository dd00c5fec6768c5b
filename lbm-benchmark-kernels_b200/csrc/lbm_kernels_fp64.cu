// lbm_kernels_fp64.cu -- FP64 D3Q19 TRT time-step kernels for sm_100a.
//
// Compiled with --fmad=false: every add and multiply rounds on its own, in the
// reference's scalar order (lbm_d3q19.cuh), so the PDFs are bit-identical to
// the reference's scalar CPU kernels.
//
// One thread per lattice cell (full array) or fluid node (lists). The work is
// HBM bound: a time step moves 19 PDFs in and 19 out per fluid node; no
// tensor-core path applies (the collision is not a contraction).
//
// Body force. The reference adds f_i += 3 w_i c_ix F to every logical PDF of a
// fluid node after each step (KernelAddBodyForce, src/Kernel.c:759-803) in a
// separate pass. Here the increment travels with the data instead:
//  * AA kernels: the even step stores plain post-collision values; the odd
//    step adds the increment of each PDF when it loads it (the logical
//    post-even PDF) and adds the increment of its destination when it stores
//    it (a PDF that bounces back becomes direction inv(i), so it gets the
//    increment of inv(i)). After every even/odd pair the device state equals
//    the reference's state bit for bit.
//  * pull kernel: the increment is added at the store.
// Obstacle cells are skipped in both AA steps. The reference relaxes them in
// its odd step and then overwrites what they wrote with the fix-up lists
// (src/BenchKernelD3Q19Aa.c:301-311,501-511); here periodic wraps and bounce
// back are resolved at the load/store itself, so no fix-up pass exists.
#include "lbm_bulk.cuh"
#include "lbm_kernels.cuh"

namespace lbm {

// ---------------------------------------------------------------------------
// Full array, AA pattern.

__device__ __forceinline__ int aa_cell(const AaArgs& a, int x, int y, int z) {
  return (x + 1) * a.xs + (y + 1) * a.pitch + z + kZOff;
}

// Offset of the neighbour in direction d, in cells.
__device__ __forceinline__ int aa_off(const AaArgs& a, int d) { return cx(d) * a.xs + cy(d) * a.pitch + cz(d); }

// Cell of x + c_d with every out-of-range coordinate wrapped (the reference
// wraps all crossed axes once one periodic axis is crossed,
// src/BenchKernelD3Q19AaCommon.c:522-578). Only called for links that do
// reach a fluid node, i.e. in-range or periodic ones.
__device__ __forceinline__ int aa_wrapped(const AaArgs& a, int x, int y, int z, int d) {
  int nx = x + cx(d), ny = y + cy(d), nz = z + cz(d);
  nx = nx < 0 ? a.nX - 1 : (nx >= a.nX ? 0 : nx);
  ny = ny < 0 ? a.nY - 1 : (ny >= a.nY ? 0 : ny);
  nz = nz < 0 ? a.nZ - 1 : (nz >= a.nZ ? 0 : nz);
  return aa_cell(a, nx, ny, nz);
}

// A reversed link (bit set) is open when x + c_d leaves the domain only
// through non-periodic faces: the PDF then goes to the ghost layer, as in the
// reference, instead of bouncing back.
__device__ __forceinline__ bool aa_open(const AaArgs& a, int x, int y, int z, int d) {
  int nx = x + cx(d), ny = y + cy(d), nz = z + cz(d);
  bool ox = nx < 0 || nx >= a.nX, oy = ny < 0 || ny >= a.nY, oz = nz < 0 || nz >= a.nZ;
  bool crossesPeriodic = (ox && a.perX) || (oy && a.perY) || (oz && a.perZ);
  return (ox || oy || oz) && !crossesPeriodic;
}

__global__ void __launch_bounds__(128) k_aa_even_fp64(const AaArgs a, const Trt<double> t) {
  const int z = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 4 + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= a.nZ || y >= a.nY) return;
  const int c = aa_cell(a, x, y, z);
  if (!(__ldg(a.link + c) & kFluidBit)) return;

  double f[Q], o[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) f[d] = a.f[d * a.dstride + c];
  trt_collide(t, f, o);
#pragma unroll
  for (int d = 0; d < Q; ++d) a.f[inv(d) * a.dstride + c] = o[d];
}

__global__ void __launch_bounds__(128) k_aa_odd_fp64(const AaArgs a, const Trt<double> t) {
  const int z = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 4 + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= a.nZ || y >= a.nY) return;
  const int c = aa_cell(a, x, y, z);
  const uint32_t w = __ldg(a.link + c);
  if (!(w & kFluidBit)) return;
  const bool edge = x == 0 || y == 0 || z == 0 || x == a.nX - 1 || y == a.nY - 1 || z == a.nZ - 1;

  double f[Q], o[Q];
  // Incoming PDF of direction i comes from x - c_i = x + c_inv(i).
#pragma unroll
  for (int i = 0; i < QM; ++i) {
    const int j = inv(i);
    double v;
    if ((w >> j) & 1u) {
      if (edge && aa_open(a, x, y, z, j))
        v = a.f[j * a.dstride + c + aa_off(a, j)];  // ghost slot, as the reference
      else
        v = a.f[i * a.dstride + c];  // bounce back: own slot of direction i
    } else {
      const int nc = edge ? aa_wrapped(a, x, y, z, j) : c + aa_off(a, j);
      v = a.f[j * a.dstride + nc];
    }
    f[i] = v + t.force[i];
  }
  f[DC] = a.f[DC * a.dstride + c] + t.force[DC];

  trt_collide(t, f, o);

#pragma unroll
  for (int i = 0; i < QM; ++i) {
    const int j = inv(i);
    if ((w >> i) & 1u) {
      if (edge && aa_open(a, x, y, z, i)) {
        a.f[i * a.dstride + c + aa_off(a, i)] = o[i];
        double* own = a.f + j * a.dstride + c;
        *own = *own + t.force[j];
      } else {
        a.f[j * a.dstride + c] = o[i] + t.force[j];
      }
    } else {
      const int nc = edge ? aa_wrapped(a, x, y, z, i) : c + aa_off(a, i);
      a.f[i * a.dstride + nc] = o[i] + t.force[i];
    }
  }
  a.f[DC * a.dstride + c] = o[DC] + t.force[DC];
}

static dim3 aa_grid(const AaArgs& a) { return dim3((a.nZ + 31) / 32, (a.nY + 3) / 4, a.nX); }

void aa_even_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s) {
  k_aa_even_fp64<<<aa_grid(a), dim3(32, 4), 0, s>>>(a, t);
}

void aa_odd_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s) {
  k_aa_odd_fp64<<<aa_grid(a), dim3(32, 4), 0, s>>>(a, t);
}

// ---------------------------------------------------------------------------
// Fluid-node lists.

__global__ void __launch_bounds__(kListTile) k_list_even_fp64(const ListArgs a, const Trt<double> t) {
  const int n = blockIdx.x * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  double f[Q], o[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) f[d] = a.f[d * a.nCells + n];
  trt_collide(t, f, o);
#pragma unroll
  for (int d = 0; d < Q; ++d) a.f[inv(d) * a.nCells + n] = o[d];
}

// Stages the block's adjacency tile (kListTile nodes x 18 entries, contiguous)
// into shared memory with one bulk copy. Returns false (and flags the error
// word) if the copy does not complete within the spin limit.
__device__ __forceinline__ bool stage_adj_tile(const ListArgs& a, uint32_t* sadj, uint64_t* bar) {
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, kListTile * QM * 4);
    bulk_g2s(sadj, a.adj + static_cast<size_t>(blockIdx.x) * kListTile * QM, kListTile * QM * 4, bar);
  }
  __syncthreads();
  if (!mbar_wait_bounded(bar, 0)) {
    if (threadIdx.x == 0) atomicOr(a.err, 1);
    return false;
  }
  return true;
}

// Reads the 18 entries of node `t` of the tile as 9 8-byte words (conflict
// free: 18 words apart per thread).
__device__ __forceinline__ void load_adj(const uint32_t* sadj, int t, uint32_t* e) {
  const uint2* p = reinterpret_cast<const uint2*>(sadj + t * QM);
#pragma unroll
  for (int k = 0; k < QM / 2; ++k) {
    uint2 v = p[k];
    e[2 * k] = v.x;
    e[2 * k + 1] = v.y;
  }
}

__global__ void __launch_bounds__(kListTile) k_list_odd_fp64(const ListArgs a, const Trt<double> t) {
  __shared__ alignas(128) uint32_t sadj[kListTile * QM];
  __shared__ alignas(8) uint64_t bar;
  if (!stage_adj_tile(a, sadj, &bar)) return;
  const int n = blockIdx.x * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;

  uint32_t e[QM];
  load_adj(sadj, threadIdx.x, e);

  double f[Q], o[Q];
#pragma unroll
  for (int i = 0; i < QM; ++i) f[i] = a.f[e[inv(i)]] + t.force[i];
  f[DC] = a.f[DC * a.nCells + n] + t.force[DC];

  trt_collide(t, f, o);

#pragma unroll
  for (int i = 0; i < QM; ++i) {
    const int j = inv(i);
    // A link that points back to the node itself is a bounce back: the PDF
    // becomes direction inv(i) of this node.
    const bool bounce = e[i] == static_cast<uint32_t>(j * a.nCells + n);
    a.f[e[i]] = o[i] + (bounce ? t.force[j] : t.force[i]);
  }
  a.f[DC * a.nCells + n] = o[DC] + t.force[DC];
}

__global__ void __launch_bounds__(kListTile) k_list_pull_fp64(const ListArgs a, const Trt<double> t) {
  __shared__ alignas(128) uint32_t sadj[kListTile * QM];
  __shared__ alignas(8) uint64_t bar;
  if (!stage_adj_tile(a, sadj, &bar)) return;
  const int n = blockIdx.x * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;

  uint32_t e[QM];
  load_adj(sadj, threadIdx.x, e);

  double f[Q], o[Q];
  f[DC] = a.f[DC * a.nCells + n];
#pragma unroll
  for (int d = 0; d < QM; ++d) f[d] = a.f[e[d]];
  trt_collide(t, f, o);
#pragma unroll
  for (int d = 0; d < Q; ++d) a.g[d * a.nCells + n] = o[d] + t.force[d];
}

static unsigned list_blocks(const ListArgs& a) { return (a.nFluid + kListTile - 1) / kListTile; }

void list_even_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  if (a.nFluid > 0) k_list_even_fp64<<<list_blocks(a), kListTile, 0, s>>>(a, t);
}
void list_odd_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  if (a.nFluid > 0) k_list_odd_fp64<<<list_blocks(a), kListTile, 0, s>>>(a, t);
}
void list_pull_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  if (a.nFluid > 0) k_list_pull_fp64<<<list_blocks(a), kListTile, 0, s>>>(a, t);
}

}  // namespace lbm
