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
#include <atomic>
#include <vector>

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
  // across a halo face the neighbour slab's cell is mirrored in the ghost plane
  nx = nx < 0 ? (a.haloLo ? -1 : a.nX - 1) : (nx >= a.nX ? (a.haloHi ? a.nX : 0) : nx);
  ny = ny < 0 ? a.nY - 1 : (ny >= a.nY ? 0 : ny);
  nz = nz < 0 ? a.nZ - 1 : (nz >= a.nZ ? 0 : nz);
  return aa_cell(a, nx, ny, nz);
}

// A reversed link (bit set) is open when x + c_d leaves the domain only
// through non-periodic faces: the PDF then goes to the ghost layer, as in the
// reference, instead of bouncing back.
__device__ __forceinline__ bool aa_open(const AaArgs& a, int x, int y, int z, int d) {
  int nx = x + cx(d), ny = y + cy(d), nz = z + cz(d);
  // crossing a halo face leaves the lattice only where it is the periodic x boundary
  bool ox = (nx < 0 && (!a.haloLo || a.crossLo)) || (nx >= a.nX && (!a.haloHi || a.crossHi));
  bool oy = ny < 0 || ny >= a.nY, oz = nz < 0 || nz >= a.nZ;
  bool crossesPeriodic = (ox && a.perX) || (oy && a.perY) || (oz && a.perZ);
  return (ox || oy || oz) && !crossesPeriodic;
}

// One block per 256 z-cells of a row (longer contiguous segments per plane),
// 4 resident blocks per SM (64 registers): 0.816 ms against 0.824 ms for
// 128-cell blocks and 0.850 ms for 32 x 4 blocks at 256^3 on B200.
constexpr int kAaEvenBlock = 256;
__global__ void __launch_bounds__(kAaEvenBlock, 1024 / kAaEvenBlock) k_aa_even_fp64(const AaArgs a, const Trt<double> t) {
  const int z = blockIdx.x * kAaEvenBlock + threadIdx.x;
  const int y = blockIdx.y;
  const int x = blockIdx.z + a.xBase;
  if (z >= a.nZ || y >= a.nY) return;
  const int c = aa_cell(a, x, y, z);
  if (!(__ldg(a.link + c) & kFluidBit)) return;
  double* const f = a.f + c;
  double* const fs = launder(f);
  const long long S = a.dstride;
  // local collide; the post-collision PDF of direction d goes to slot inv(d)
  trt_update(t, [&](int d) { return f[d * S]; }, [&](int d, double v) { fs[inv(d) * S] = v; });
}

// Odd step. Node x reads its incoming f_i from slot (x + c_j, j), j = inv(i)
// (the AA pattern: the slots a node reads are the slots it writes), plus the
// body-force increment of that post-even logical PDF; it writes f_i to slot
// (x + c_i, i) with the increment of i, or -- bounced back at a wall -- to
// its own slot (x, inv(i)) with the increment of inv(i).
//
// Two launches share the step. The interior launch takes every cell whose
// links leave the domain, if at all, only through periodic faces
// (aa_interior_range): the z faces when z is periodic, and the x and y faces
// too when every axis is periodic and no x face is a halo face (then the
// face launch has no cells left). A link through such a face moves by a
// fixed -/+ n cells along each crossed axis. (Taking the periodic x faces of
// a channel, periodic in x only, into the interior saves nothing: the face
// launch still runs for its wall faces, and the interior pays for the wrap
// tests of two more axes -- 256^3 channel odd step 0.873 + 0.029 ms against
// 0.862 + 0.029 ms; on the fully periodic box the face launch goes away,
// 0.813 + 0.039 -> 0.824 ms.) Interior cells are sorted on the
// host by their link words: a cell without reversed links is "direct" (every
// address is the neighbour's slot), the others are "general" (each address
// is a select between the neighbour's slot and the node's own slot). The
// launch runs a list of work items in x-plane order: for each plane, the
// blocks (128 z-cells of one row) that hold at least one direct cell --
// these skip the general cells in them -- then chunks of 128 of the plane's
// general cells, one thread per cell. So the select-free path covers every
// direct cell, also those next to a wall (in a 256^3 channel a split by
// whole blocks sends 27 % of the cells, every block with one wall-adjacent
// cell, down the general path; the general cells are 1.6 %), and a general
// cell runs while the direct blocks of its plane touch the same 32-byte
// sectors, so its scattered accesses (a column of wall-adjacent cells is
// `pitch` apart) hit L2 instead of DRAM. Blocks without fluid cells are not
// launched. In both paths the 19 loads are issued together. The face kernel
// takes the shell (x and y faces, and z faces unless z is periodic):
// links that leave the domain wrap periodically on every crossed axis, or,
// at a non-periodic face, go to the ghost layer (an "open" link), as in the
// reference.
//
// Cells of different nodes never share a slot in the odd step (each node
// reads and writes only its own links' slots), so the work items and the
// two launches may run in any order.

// Interior blocks of the odd step: kAaBZ z-cells x kAaBY rows of one x plane
// (128 threads). A 128-cell row segment per plane: interior 0.811 ms against
// 0.818 ms for 64 x 2 and 0.830 ms for 32 x 4 blocks (256^3 fluid box, B200).
constexpr int kAaBZ = 128, kAaBY = 1;

// Whether the interior launch takes the whole lattice (see above).
__host__ __device__ __forceinline__ bool aa_interior_all(const AaArgs& a) {
  return a.perX && a.perY && a.perZ && !a.haloLo && !a.haloHi;
}

// The interior ranges [lo, hi] of x, y and z (see above).
struct AaRange {
  int x0, x1, y0, y1, z0, z1;
};
__host__ __device__ __forceinline__ AaRange aa_interior_range(const AaArgs& a) {
  AaRange r;
  const bool all = aa_interior_all(a);
  r.x0 = all ? 0 : 1;
  r.x1 = all ? a.nX - 1 : a.nX - 2;
  r.y0 = all ? 0 : 1;
  r.y1 = all ? a.nY - 1 : a.nY - 2;
  r.z0 = a.perZ ? 0 : 1;
  r.z1 = a.perZ ? a.nZ - 1 : a.nZ - 2;
  return r;
}

// Interior blocks start at z = 0 whatever the interior's first z: row
// element kZOff + z then puts each warp's 32 cells on whole 32-byte sectors
// (with walls in z, a start at z = 1 made every warp's z-aligned accesses
// span one sector more); threads off the interior range return.
__host__ __device__ __forceinline__ int aa_interior_zblocks(const AaArgs& a) { return (a.nZ + kAaBZ - 1) / kAaBZ; }

// Interior block `id` of the list: (bz, by, bx) with bz fastest.
__device__ __forceinline__ void aa_interior_block(const AaArgs& a, const AaRange& r, int id, int& z, int& y,
                                                  int& x) {
  const int gz = aa_interior_zblocks(a), gy = (r.y1 - r.y0 + 1 + kAaBY - 1) / kAaBY;
  const int bz = id % gz, rest = id / gz;
  z = bz * kAaBZ + threadIdx.x;
  y = r.y0 + (rest % gy) * kAaBY + threadIdx.y;
  x = r.x0 + rest / gy;
}

// The periodic wraps of an interior cell, decided once per cell: a link with
// c_a = -1 leaving through the low face of axis a moves +n_a cells along a,
// one with c_a = +1 through the high face moves -n_a. ZWrap: only z faces
// are reached (interior cells are off the x and y faces, and off the z faces
// unless z is periodic); XyzWrap: the interior is the whole lattice.
struct ZWrap {
  int down, up;
  __device__ __forceinline__ ZWrap(const AaArgs& a, int z)
      : down(z == 0 ? a.nZ : 0), up(z == a.nZ - 1 ? -a.nZ : 0) {}
  __device__ __forceinline__ int operator()(int d) const { return cz(d) < 0 ? down : (cz(d) > 0 ? up : 0); }
};
struct XyzWrap {
  const AaArgs& a;
  unsigned m;  // bits 0-5: x == 0, x == nX - 1, y == 0, y == nY - 1, z == 0, z == nZ - 1
  __device__ __forceinline__ XyzWrap(const AaArgs& a_, int x, int y, int z)
      : a(a_),
        m((x == 0) | (x == a_.nX - 1) << 1 | (y == 0) << 2 | (y == a_.nY - 1) << 3 | (z == 0) << 4 |
          (z == a_.nZ - 1) << 5) {}
  __device__ __forceinline__ int operator()(int d) const {
    int o = 0;
    if (cx(d) < 0 && (m & 1u)) o += a.nX * a.xs;
    if (cx(d) > 0 && (m & 2u)) o -= a.nX * a.xs;
    if (cy(d) < 0 && (m & 4u)) o += a.nY * a.pitch;
    if (cy(d) > 0 && (m & 8u)) o -= a.nY * a.pitch;
    if (cz(d) < 0 && (m & 16u)) o += a.nZ;
    if (cz(d) > 0 && (m & 32u)) o -= a.nZ;
    return o;
  }
};
template <bool kXY>
__device__ __forceinline__ auto aa_wrap(const AaArgs& a, int x, int y, int z) {
  if constexpr (kXY)
    return XyzWrap(a, x, y, z);
  else
    return ZWrap(a, z);
}

// A general cell (interior, fluid, at least one reversed link).
template <bool kXY>
__device__ __noinline__ void aa_odd_general_cell(const AaArgs& a, const Trt<double>& t, int c) {
  // cell index -> (x, y, z): planes of xs cells, rows of pitch cells,
  // interior z = 0 at element kZOff (x and y only matter to XyzWrap)
  int x = 0, y = 0, z;
  if constexpr (kXY) {
    const int rem = c % a.xs;
    x = c / a.xs - 1;
    y = rem / a.pitch - 1;
    z = rem % a.pitch - kZOff;
  } else {
    z = c % a.pitch - kZOff;
  }
  const uint32_t w = __ldg(a.link + c);
  double* const fb = a.f + c;
  const auto wrap = aa_wrap<kXY>(a, x, y, z);
  const int S = (int)a.dstride;
  auto load = [&](int d) -> double {
    if (d == DC) return fb[a.ldOff[DC]] + t.force[DC];
    const int j = inv(d);
    const bool rev = (w >> j) & 1u;
    return fb[rev ? d * S : a.ldOff[d] + wrap(j)] + t.force[d];
  };
  auto store = [&](int d, double v) {
    double* const fs = launder(fb);
    if (d == DC) {
      fs[a.stOff[DC]] = v + t.force[DC];
      return;
    }
    const int j = inv(d);
    const bool rev = (w >> d) & 1u;
    fs[rev ? j * S : a.stOff[d] + wrap(d)] = v + (rev ? t.force[j] : t.force[d]);
  };
  trt_update(t, load, store);
}

// Work item `items[blockIdx.x]`: >= 0 a block id (direct cells), < 0 the
// general-cell chunk ~item (cells[128 * chunk + thread], -1 = none).
// Launch bounds: 7 resident blocks of 128 threads per SM (measured fastest
// among 1-8 on B200; the general path spills a few values into L1 under that
// cap). Direct addresses are the cell's base pointer plus a per-direction
// offset from the parameter bank (and the periodic wraps), so no
// per-direction address stays live in registers; store addresses come from a
// laundered base pointer, apart from the load addresses, so those need not
// stay live across the collision.
template <bool kXY>
__global__ void __launch_bounds__(128, 7)
    k_aa_odd_interior_fp64(const __grid_constant__ AaArgs a, const __grid_constant__ Trt<double> t, const int* items,
                           const int* cells) {
  const int item = __ldg(items + blockIdx.x);
  if (item < 0) {
    const int c = __ldg(cells + (size_t)(~item) * 128 + threadIdx.y * kAaBZ + threadIdx.x);
    if (c >= 0) aa_odd_general_cell<kXY>(a, t, c);
    return;
  }
  const AaRange r = aa_interior_range(a);
  int x, y, z;
  aa_interior_block(a, r, item, z, y, x);
  if (z < r.z0 || z > r.z1 || y > r.y1) return;
  const int c = aa_cell(a, x, y, z);
  const uint32_t w = __ldg(a.link + c);
  if ((w & (kFluidBit | kLinkBits)) != kFluidBit) return;  // solid, or a general cell (own item)
  double* const fb = a.f + c;
  const auto wrap = aa_wrap<kXY>(a, x, y, z);
  trt_update(t, [&](int d) -> double { return fb[a.ldOff[d] + wrap(inv(d))] + t.force[d]; },
             [&](int d, double v) { launder(fb)[a.stOff[d] + wrap(d)] = v + t.force[d]; });
}

// Cell of shell index i: the x faces (all y, z), then the y faces (inner x,
// all z), then -- when z is not periodic -- the z faces (inner x and y). A
// one-cell-thin axis has a single face. The arithmetic is 32-bit unsigned:
// the layout holds fewer than 2^31 PDFs, so every product and index here is
// below 2^31.
__device__ __forceinline__ void aa_shell_cell(const AaArgs& a, long long i64, int& x, int& y, int& z) {
  const unsigned i = static_cast<unsigned>(i64);
  const unsigned nY = a.nY, nZ = a.nZ;
  const unsigned sx = a.nX > 1 ? 2 : 1, sy = a.nY > 1 ? 2 : 1;
  const unsigned mx = a.nX > 2 ? a.nX - 2 : 0, my = a.nY > 2 ? a.nY - 2 : 0;
  const unsigned nA = sx * nY * nZ, nB = sy * mx * nZ;
  if (i < nA) {
    x = (i / (nY * nZ)) == 0 ? 0 : a.nX - 1;
    const unsigned r = i % (nY * nZ);
    y = (int)(r / nZ);
    z = (int)(r % nZ);
  } else if (i < nA + nB) {
    const unsigned j = i - nA;
    y = (j / (mx * nZ)) == 0 ? 0 : a.nY - 1;
    const unsigned r = j % (mx * nZ);
    x = 1 + (int)(r / nZ);
    z = (int)(r % nZ);
  } else {
    const unsigned k = i - nA - nB;
    z = (k / (mx * my)) == 0 ? 0 : a.nZ - 1;
    const unsigned r = k % (mx * my);
    x = 1 + (int)(r / my);
    y = 1 + (int)(r % my);
  }
}

__global__ void __launch_bounds__(128) k_aa_odd_face_fp64(const AaArgs a, const Trt<double> t, long long nShell) {
  const long long i = static_cast<long long>(blockIdx.x) * 128 + threadIdx.x;
  if (i >= nShell) return;
  int x, y, z;
  aa_shell_cell(a, i, x, y, z);
  const int c = aa_cell(a, x, y, z);
  const uint32_t w = __ldg(a.link + c);
  if (!(w & kFluidBit)) return;
  const long long S = a.dstride;
  double* const f = a.f;
  auto load = [&](int d) -> double {
    if (d == DC) return f[DC * S + c] + t.force[DC];
    const int j = inv(d);
    const bool rev = (w >> j) & 1u;
    const bool open = rev && aa_open(a, x, y, z, j);
    const int nb = rev ? c + aa_off(a, j) : aa_wrapped(a, x, y, z, j);
    return f[(rev && !open) ? d * S + c : j * S + nb] + t.force[d];
  };
  auto store = [&](int d, double v) {
    if (d == DC) {
      f[DC * S + c] = v + t.force[DC];
      return;
    }
    const int j = inv(d);
    const bool rev = (w >> d) & 1u;
    if (!rev) {
      f[d * S + aa_wrapped(a, x, y, z, d)] = v + t.force[d];
    } else if (aa_open(a, x, y, z, d)) {
      // open face: the PDF leaves into the ghost layer; the node's own slot
      // of direction inv(d) keeps its even-step value and gets its increment
      f[d * S + c + aa_off(a, d)] = v;
      f[j * S + c] = f[j * S + c] + t.force[j];
    } else {
      f[j * S + c] = v + t.force[j];
    }
  };
  trt_update(t, load, store);
}

// ---------------------------------------------------------------------------
// x-slab halo messages.

// The 5 directions with c_x = +1 (E, NE, SE, TE, BE) and c_x = -1 (W, NW, SW,
// TW, BW), in the order of a message.
__device__ __forceinline__ int halo_dir(int k, bool plusX) {
  return plusX ? (k == 0 ? E : k == 1 ? NE : k == 2 ? SE : k == 3 ? TE : BE)
               : (k == 0 ? W : k == 1 ? NW : k == 2 ? SW : k == 3 ? TW : BW);
}

// plane: local x of the plane (-1 and nX are the ghost planes); plusX: which
// five directions; mode: 0 copy the slots into buf; 1 (phase-0 unpack into a
// ghost plane) and 2 (phase-1 unpack into a face plane) copy out of buf, but
// only into the slots the odd step exchanges through the face:
//  1: a ghost slot (g, y, z, d) is read and written by the face cell whose
//     direct link d lands on it, (y - c_dy, z - c_dz) wrapped on the face;
//     other ghost slots keep what they hold (open-face values);
//  2: a face slot (y, z, d) was written by the neighbour only if this slab's
//     cell reaches the neighbour's cell through the direct link inv(d); where
//     that link is reversed (a wall or an open face behind the halo face),
//     this slab's own odd step wrote the slot (bounce back) and keeps it.
__global__ void k_aa_halo(const AaArgs a, int plane, bool plusX, int mode, double* buf) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long face = (long long)a.nY * a.nZ;
  if (i >= 5 * face) return;
  const int k = (int)(i / face);
  const int y = (int)(i % face / a.nZ), z = (int)(i % a.nZ);
  const int d = halo_dir(k, plusX);
  const long long cell = (long long)(plane + 1) * a.xs + (long long)(y + 1) * a.pitch + z + kZOff;
  const long long slot = d * a.dstride + cell;
  if (mode == 0) {
    buf[i] = a.f[slot];
    return;
  }
  bool take;
  if (mode == 1) {
    const int rx = plane < 0 ? 0 : a.nX - 1;
    int ry = (y - cy(d)) % a.nY, rz = (z - cz(d)) % a.nZ;
    ry += ry < 0 ? a.nY : 0;
    rz += rz < 0 ? a.nZ : 0;
    const uint32_t w = a.link[(long long)(rx + 1) * a.xs + (long long)(ry + 1) * a.pitch + rz + kZOff];
    take = (w & kFluidBit) && !((w >> d) & 1u);
  } else {
    const uint32_t w = a.link[cell];
    take = (w & kFluidBit) && !((w >> inv(d)) & 1u);
  }
  if (take) a.f[slot] = buf[i];
}

// Side 1 (x = nX-1 face): the cells of this slab cross it with c_x = +1, the
// neighbour's with c_x = -1; side 0 the other way round.
void aa_halo_pack(const AaArgs& a, int side, int phase, double* buf, cudaStream_t s) {
  const long long n = 5LL * a.nY * a.nZ;
  const int plane = phase == 0 ? (side == 0 ? 0 : a.nX - 1) : (side == 0 ? -1 : a.nX);
  // phase 0: the face plane's slots the neighbour streams through (pointing
  // into this slab); phase 1: the ghost plane's slots this slab streamed into
  const bool plusX = phase == 0 ? side == 0 : side == 1;
  if (n > 0) k_aa_halo<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, plane, plusX, 0, buf);
}

void aa_halo_unpack(const AaArgs& a, int side, int phase, const double* buf, cudaStream_t s) {
  const long long n = 5LL * a.nY * a.nZ;
  const int plane = phase == 0 ? (side == 0 ? -1 : a.nX) : (side == 0 ? 0 : a.nX - 1);
  const bool plusX = phase == 0 ? side == 1 : side == 0;
  if (n > 0)
    k_aa_halo<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, plane, plusX, phase == 0 ? 1 : 2,
                                                           const_cast<double*>(buf));
}

// ---------------------------------------------------------------------------
// Two-grid full array (src/BenchKernelD3Q19.c:114-344) on the AA layout and
// link words, one thread per cell, obstacles skipped. The reference's
// bounce-back and periodic fix-up lists (src/BenchKernelD3Q19Common.c:
// 531-660), which copy slots after each step, and its body-force pass, which
// adds 3 w_i c_ix F through the logical node view, are folded into the
// stores; the result in every slot some fluid node views is the reference's
// bit for bit (tests against the oracle and the reference).

// Blocks of the two-grid steps: kFaBZ z-cells x kFaBY rows of one x plane.
// 32 x 4: push 0.860 / pull 0.897 ms at 256^3 (fluid box) against 0.867 /
// 0.925 for 64 x 2 and 0.887 / 0.986 for 128 x 1 (unlike the AA steps, whose
// longer row segments won).
constexpr int kFaBZ = 32, kFaBY = 4;

// Push: node x's own PDFs in from grid f; PDF d out to (x + c_d, d) of grid g
// (across a periodic face: the wrapped cell). A wall sends it back to the
// node's own slot inv(d); an open face leaves that slot untouched by the step,
// so only the force increment is added to what the grid held.
__global__ void __launch_bounds__(128) k_fa_push_fp64(const AaArgs a, const Trt<double> t) {
  const int z = blockIdx.x * kFaBZ + threadIdx.x;
  const int y = blockIdx.y * kFaBY + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= a.nZ || y >= a.nY) return;
  const int c = aa_cell(a, x, y, z);
  const uint32_t w = __ldg(a.link + c);
  if (!(w & kFluidBit)) return;
  const long long S = a.dstride;
  const double* const f = a.f + c;
  double* const g = launder(a.g);
  // a cell off every face with all links direct writes each PDF to x + c_d
  // without wrap or bounce logic (a warp-uniform branch for most warps)
  const bool inner = !(w & kLinkBits) && x > 0 && x < a.nX - 1 && y > 0 && y < a.nY - 1 && z > 0 && z < a.nZ - 1;
  if (inner) {
    trt_update(t, [&](int d) { return f[d * S]; },
               [&](int d, double v) { g[d * S + c + aa_off(a, d)] = v + t.force[d]; });
    return;
  }
  auto store = [&](int d, double v) {
    if (d == DC) {
      g[DC * S + c] = v + t.force[DC];
      return;
    }
    const int j = inv(d);
    if (!((w >> d) & 1u))
      g[d * S + aa_wrapped(a, x, y, z, d)] = v + t.force[d];
    else if (aa_open(a, x, y, z, d))
      g[j * S + c] = g[j * S + c] + t.force[j];
    else
      g[j * S + c] = v + t.force[j];
  };
  trt_update(t, [&](int d) { return f[d * S]; }, store);
}

// Pull: PDF d in from (x - c_d, d) of grid f (the slot the previous step
// filled for this node, ghost cells included); own PDFs out to grid g. For a
// link e that the next step pulls through a ghost or wall slot, the copy the
// reference's fix-up list makes is written directly: a wall slot (x + c_e,
// inv(e)) gets this node's PDF e (bounce back), the ghost slot of the periodic
// image q = wrap(x + c_e) gets it at (q - c_e, e), and an open slot only gets
// the force increment.
__global__ void __launch_bounds__(128) k_fa_pull_fp64(const AaArgs a, const Trt<double> t) {
  const int z = blockIdx.x * kFaBZ + threadIdx.x;
  const int y = blockIdx.y * kFaBY + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= a.nZ || y >= a.nY) return;
  const int c = aa_cell(a, x, y, z);
  const uint32_t w = __ldg(a.link + c);
  if (!(w & kFluidBit)) return;
  const long long S = a.dstride;
  const double* const f = a.f;
  double* const g = launder(a.g);
  auto load = [&](int d) -> double { return f[d * S + c - aa_off(a, d)]; };
  // a cell off every face with all links direct has no periodic image, wall
  // or open-face slot to write: its 19 stores are its own slots (the check is
  // uniform across most warps; 0.946 -> 0.896 ms per step at 256^3)
  const bool inner = !(w & kLinkBits) && x > 0 && x < a.nX - 1 && y > 0 && y < a.nY - 1 && z > 0 && z < a.nZ - 1;
  if (inner) {
    trt_update(t, load, [&](int e, double v) { g[e * S + c] = v + t.force[e]; });
    return;
  }
  auto store = [&](int e, double v) {
    g[e * S + c] = v + t.force[e];
    if (e == DC) return;
    const int j = inv(e);
    if (!((w >> e) & 1u)) {
      const int q = aa_wrapped(a, x, y, z, e);
      const int n = c + aa_off(a, e);
      if (q != n) g[e * S + q - aa_off(a, e)] = v + t.force[e];  // periodic image's ghost slot
    } else if (aa_open(a, x, y, z, e)) {
      g[j * S + c + aa_off(a, e)] = g[j * S + c + aa_off(a, e)] + t.force[j];
    } else {
      g[j * S + c + aa_off(a, e)] = v + t.force[j];
    }
  };
  trt_update(t, load, store);
}

void fa_push_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s) {
  k_fa_push_fp64<<<dim3((a.nZ + kFaBZ - 1) / kFaBZ, (a.nY + kFaBY - 1) / kFaBY, a.nX), dim3(kFaBZ, kFaBY), 0, s>>>(a, t);
}
void fa_pull_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s) {
  k_fa_pull_fp64<<<dim3((a.nZ + kFaBZ - 1) / kFaBZ, (a.nY + kFaBY - 1) / kFaBY, a.nX), dim3(kFaBZ, kFaBY), 0, s>>>(a, t);
}

long long aa_shell_cells(const AaArgs& a) {
  const long long sx = a.nX > 1 ? 2 : 1, sy = a.nY > 1 ? 2 : 1, sz = a.nZ > 1 ? 2 : 1;
  const long long mx = a.nX > 2 ? a.nX - 2 : 0, my = a.nY > 2 ? a.nY - 2 : 0;
  return sx * a.nY * a.nZ + sy * mx * a.nZ + (a.perZ ? 0 : sz * mx * my);
}

bool aa_has_interior(const AaArgs& a) {
  const AaRange r = aa_interior_range(a);
  return r.x1 >= r.x0 && r.y1 >= r.y0 && r.z1 >= r.z0;
}

long long aa_interior_block_count(const AaArgs& a) {
  if (!aa_has_interior(a)) return 0;
  const AaRange r = aa_interior_range(a);
  return (long long)aa_interior_zblocks(a) * ((r.y1 - r.y0 + 1 + kAaBY - 1) / kAaBY) * (r.x1 - r.x0 + 1);
}

// Whether the face kernel has work: the shell (x and y faces, z faces unless
// z is periodic) lies outside the interior range unless the interior is the
// whole lattice.
bool aa_shell_needed(const AaArgs& a) { return !aa_interior_all(a) && aa_shell_cells(a) > 0; }

void aa_interior_items(const AaArgs& a, const uint32_t* link, std::vector<int>& items, std::vector<int>& cells) {
  items.clear();
  cells.clear();
  const long long n = aa_interior_block_count(a);
  if (n == 0) return;
  const AaRange r = aa_interior_range(a);
  const int gz = aa_interior_zblocks(a), gy = (r.y1 - r.y0 + 1 + kAaBY - 1) / kAaBY;
  const long long perPlane = (long long)gz * gy;
  auto word = [&](int x, int y, int z) { return link[(long long)(x + 1) * a.xs + (long long)(y + 1) * a.pitch + z + kZOff]; };
  for (int x = r.x0; x <= r.x1; ++x) {
    // the plane's blocks holding direct cells (block ids: bz fastest, then by, then x)
    for (long long k = 0; k < perPlane; ++k) {
      const int bz = (int)(k % gz), by = (int)(k / gz);
      bool direct = false;
      for (int ty = 0; ty < kAaBY && !direct; ++ty) {
        const int y = r.y0 + by * kAaBY + ty;
        if (y > r.y1) break;
        for (int tz = 0; tz < kAaBZ; ++tz) {
          const int z = bz * kAaBZ + tz;
          if (z < r.z0) continue;
          if (z > r.z1) break;
          if ((word(x, y, z) & (kFluidBit | kLinkBits)) == kFluidBit) { direct = true; break; }
        }
      }
      if (direct) items.push_back((int)((x - r.x0) * perPlane + k));
    }
    // then the plane's general cells in chunks of 128
    const size_t first = cells.size();
    for (int y = r.y0; y <= r.y1; ++y)
      for (int z = r.z0; z <= r.z1; ++z) {
        const uint32_t w = word(x, y, z);
        if ((w & kFluidBit) && (w & kLinkBits)) cells.push_back((x + 1) * a.xs + (y + 1) * a.pitch + z + kZOff);
      }
    while ((cells.size() - first) % 128) cells.push_back(-1);
    for (size_t c = first; c < cells.size(); c += 128) items.push_back(~(int)(c / 128));
  }
}

void aa_even_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s) {
  AaArgs b = a;
  b.xBase = 0;
  k_aa_even_fp64<<<dim3((a.nZ + kAaEvenBlock - 1) / kAaEvenBlock, a.nY, a.nX), kAaEvenBlock, 0, s>>>(b, t);
}

void aa_even_fp64_planes(const AaArgs& a, const Trt<double>& t, int x0, int x1, cudaStream_t s) {
  if (x1 <= x0) return;
  AaArgs b = a;
  b.xBase = x0;
  k_aa_even_fp64<<<dim3((a.nZ + kAaEvenBlock - 1) / kAaEvenBlock, a.nY, x1 - x0), kAaEvenBlock, 0, s>>>(b, t);
}

void aa_odd_interior_fp64(const AaArgs& a, const Trt<double>& t, const int* items, int nItems, const int* cells,
                          cudaStream_t s) {
  if (nItems <= 0) return;
  if (aa_interior_all(a))
    k_aa_odd_interior_fp64<true><<<nItems, dim3(kAaBZ, kAaBY), 0, s>>>(a, t, items, cells);
  else
    k_aa_odd_interior_fp64<false><<<nItems, dim3(kAaBZ, kAaBY), 0, s>>>(a, t, items, cells);
}

void aa_odd_face_fp64(const AaArgs& a, const Trt<double>& t, cudaStream_t s) {
  const long long n = aa_shell_cells(a);
  if (n > 0) k_aa_odd_face_fp64<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, t, n);
}

// ---------------------------------------------------------------------------
// Fluid-node lists.

// 4 blocks of 256 threads per SM (64 registers, no spills)
__global__ void __launch_bounds__(kListTile, 4) k_list_even_fp64(const ListArgs a, const Trt<double> t) {
  const int n = (blockIdx.x + a.tileBase) * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  double* const f = a.f + n;
  double* const fs = launder(f);
  const long long S = a.nCells;
  trt_update(t, [&](int d) { return f[d * S]; }, [&](int d, double v) { fs[inv(d) * S] = v; });
}

// L2 prefetch of the PDF regions that the block of tile u will touch: for
// each of the 18 links, the 256 slots from the link of the tile's first node
// on (consecutive nodes mostly reach consecutive slots), and the tile's own
// rest-direction slots; one lane per region, clamped to the PDF array. The
// tile's run record was prefetched into L2 half a resident wave earlier.
__device__ __forceinline__ void prefetch_tile_pdfs(const ListArgs& a, unsigned u, int lane) {
  if (lane >= Q) return;
  const unsigned long long first =
      lane == DC ? (unsigned long long)DC * a.nCells + (unsigned long long)u * kListTile
                 : a.runs[(size_t)a.runOff[u] * 4 + kRunHdrWords + lane];
  const unsigned long long endB = (unsigned long long)Q * a.nCells * 8ull / 16ull * 16ull;
  const unsigned long long b0 = first * 8ull / 16ull * 16ull;
  if (b0 >= endB) return;
  unsigned long long len = kListTile * 8ull + 16ull;
  if (b0 + len > endB) len = endB - b0;
  if (len >= 16) bulk_prefetch_l2(reinterpret_cast<const char*>(a.f) + b0, static_cast<uint32_t>(len / 16 * 16));
}

// 3 blocks of 256 threads per SM. The adjacency comes run-compressed (one
// row per run of consecutive nodes, see kRunHdrWords): at the 256^3 sphere
// packing 0.49 rows per node, 35 instead of 72 bytes per node. The block's
// gathers are latency-bound at this occupancy (80 registers; a 64-register
// build spills and is slower), so warp 2 prefetches into L2 the PDF regions
// of the tile half a resident wave ahead (the run records are one wave
// ahead): 0.395 -> 0.371 ms at the 256^3 packing. Measured distances: one
// wave 0.386 ms, two waves 0.435, a quarter wave 0.377.
__global__ void __launch_bounds__(kListTile, 3) k_list_odd_fp64(const ListArgs a, const Trt<double> t) {
  __shared__ alignas(128) uint32_t srun[kRunTileWords];
  __shared__ alignas(8) uint64_t bar;
  __shared__ int ok;
  if (!stage_run_tile(a, srun, &bar, &ok)) return;
  const unsigned tile = blockIdx.x + static_cast<unsigned>(a.tileBase);
  const unsigned pdfAhead = static_cast<unsigned>(a.prefetch) / 2;
  if (threadIdx.x >= 64 && threadIdx.x < 96 && pdfAhead > 0 &&
      tile + pdfAhead < static_cast<unsigned>((a.nFluid + kListTile - 1) / kListTile))
    prefetch_tile_pdfs(a, tile + pdfAhead, threadIdx.x - 64);
  const int n = static_cast<int>(tile) * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  uint32_t off;
  const uint32_t* e = run_row(srun, threadIdx.x, off);  // link d = e[d] + off
  double* const f = a.f;
  const long long S = a.nCells;

  // incoming f_d (the post-even logical PDF) through link inv(d), plus its
  // body-force increment
  auto load = [&](int d) -> double {
    return (d == DC ? f[DC * S + n] : f[e[inv(d)] + off]) + t.force[d];
  };
  // outgoing f_d through link d; a link that points back to the node itself
  // is a bounce back: the PDF becomes direction inv(d) of this node and gets
  // the increment of inv(d)
  auto store = [&](int d, double v) {
    if (d == DC) { f[DC * S + n] = v + t.force[DC]; return; }
    const uint32_t dst = reinterpret_cast<const volatile uint32_t*>(e)[d] + off;  // re-read: keeps no 64-bit addresses live across the collision
    const int j = inv(d);
    const bool bounce = dst == static_cast<uint32_t>(j * S + n);
    f[dst] = v + (bounce ? t.force[j] : t.force[d]);
  };
  trt_update(t, load, store);
}

__global__ void __launch_bounds__(kListTile) k_list_pull_fp64(const ListArgs a, const Trt<double> t) {
  __shared__ alignas(128) uint32_t srun[kRunTileWords];
  __shared__ alignas(8) uint64_t bar;
  __shared__ int ok;
  if (!stage_run_tile(a, srun, &bar, &ok)) return;
  const int n = (blockIdx.x + a.tileBase) * kListTile + threadIdx.x;
  if (n >= a.nFluid) return;
  uint32_t off;
  const uint32_t* e = run_row(srun, threadIdx.x, off);  // link d = e[d] + off (run-compressed pull adjacency)
  const long long S = a.nCells;
  // one pass: the gathers are issued together and the 19 outputs are
  // contiguous stores to the second grid
  double f[Q], o[Q];
  f[DC] = a.f[DC * S + n];
#pragma unroll
  for (int d = 0; d < QM; ++d) f[d] = a.f[e[d] + off];
  trt_collide(t, f, o);
#pragma unroll
  for (int d = 0; d < Q; ++d) a.g[d * S + n] = o[d] + t.force[d];
}

// Two-grid list push (src/BenchKernelD3Q19List.c:114-320, PROP_MODEL_PUSH):
// the node's own 19 PDFs from the source grid, each post-collision PDF
// written through the push adjacency into the destination grid with the
// body-force increment of the slot's direction (a bounce back lands in the
// node's own slot inv(d) and gets the increment of inv(d)). The own PDFs do
// not depend on the adjacency: their loads are issued before the wait for
// the tile's run record, so the two latencies overlap.
__global__ void __launch_bounds__(kListTile, 3) k_list_push_fp64(const ListArgs a, const Trt<double> t) {
  __shared__ alignas(128) uint32_t srun[kRunTileWords];
  __shared__ alignas(8) uint64_t bar;
  __shared__ int ok;
  if (!stage_run_tile_issue(a, srun, &bar, &ok)) return;
  const int n = (blockIdx.x + a.tileBase) * kListTile + threadIdx.x;
  const long long S = a.nCells;
  double x[Q];
  if (n < a.nFluid) {
    const double* const f = a.f + n;
#pragma unroll
    for (int d = 0; d < Q; ++d) x[d] = f[d * S];
  }
  if (!stage_run_tile_wait(a, &bar) || n >= a.nFluid) return;
  uint32_t off;
  const uint32_t* e = run_row(srun, threadIdx.x, off);
  double* const g = a.g;
  auto store = [&](int d, double v) {
    if (d == DC) { g[DC * S + n] = v + t.force[DC]; return; }
    const uint32_t dst = reinterpret_cast<const volatile uint32_t*>(e)[d] + off;
    const int j = inv(d);
    const bool bounce = dst == static_cast<uint32_t>(j * S + n);
    g[dst] = v + (bounce ? t.force[j] : t.force[d]);
  };
  trt_update(t, [&](int d) { return x[d]; }, store);
}

template <typename E>
__global__ void k_slot_gather(const E* __restrict__ f, const uint32_t* __restrict__ idx, long long n,
                              E* __restrict__ buf) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < n) buf[k] = f[idx[k]];
}

template <typename E>
__global__ void k_slot_scatter(E* __restrict__ f, const uint32_t* __restrict__ idx, long long n,
                               const E* __restrict__ buf) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < n) f[idx[k]] = buf[k];
}

template <typename E>
static void slot_move(bool gather, void* f, const uint32_t* idx, long long n, void* buf, cudaStream_t s) {
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (gather)
    k_slot_gather<E><<<blocks, 256, 0, s>>>(static_cast<const E*>(f), idx, n, static_cast<E*>(buf));
  else
    k_slot_scatter<E><<<blocks, 256, 0, s>>>(static_cast<E*>(f), idx, n, static_cast<const E*>(buf));
}

static void slot_move_bytes(bool gather, void* f, const uint32_t* idx, long long n, void* buf, int elemBytes,
                            cudaStream_t s) {
  if (n <= 0) return;
  if (elemBytes == 8)
    slot_move<unsigned long long>(gather, f, idx, n, buf, s);
  else if (elemBytes == 4)
    slot_move<unsigned int>(gather, f, idx, n, buf, s);
  else if (elemBytes == 2)
    slot_move<unsigned short>(gather, f, idx, n, buf, s);
}

void slot_gather(const void* f, const uint32_t* idx, long long n, void* buf, int elemBytes, cudaStream_t s) {
  slot_move_bytes(true, const_cast<void*>(f), idx, n, buf, elemBytes, s);
}

void slot_scatter(void* f, const uint32_t* idx, long long n, const void* buf, int elemBytes, cudaStream_t s) {
  slot_move_bytes(false, f, idx, n, const_cast<void*>(buf), elemBytes, s);
}

static unsigned list_blocks(const ListArgs& a) { return (a.nFluid + kListTile - 1) / kListTile; }

void list_even_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  ListArgs b = a;
  b.tileBase = 0;
  if (a.nFluid > 0) k_list_even_fp64<<<list_blocks(b), kListTile, 0, s>>>(b, t);
}

void list_even_fp64_tiles(const ListArgs& a, const Trt<double>& t, int t0, int t1, cudaStream_t s) {
  if (a.nFluid <= 0 || t1 <= t0) return;
  ListArgs b = a;
  b.tileBase = t0;
  k_list_even_fp64<<<(unsigned)(t1 - t0), kListTile, 0, s>>>(b, t);
}
static std::atomic<int> g_oddAhead{0};

void list_odd_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  if (a.nFluid <= 0) return;
  ListArgs b = a;
  b.tileBase = 0;
  b.prefetch = prefetch_distance(g_oddAhead, k_list_odd_fp64, kListTile, a.prefetch != 0);
  k_list_odd_fp64<<<list_blocks(b), kListTile, 0, s>>>(b, t);
}

void list_odd_fp64_tiles(const ListArgs& a, const Trt<double>& t, int t0, int t1, cudaStream_t s) {
  if (a.nFluid <= 0 || t1 <= t0) return;
  ListArgs b = a;
  b.tileBase = t0;
  b.prefetch = prefetch_distance(g_oddAhead, k_list_odd_fp64, kListTile, a.prefetch != 0);
  k_list_odd_fp64<<<(unsigned)(t1 - t0), kListTile, 0, s>>>(b, t);
}
void list_pull_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  // no adjacency prefetch: with the full adjacency it slowed this kernel by
  // 8 % on a 256^3 sphere packing
  if (a.nFluid <= 0) return;
  ListArgs b = a;
  b.prefetch = 0;
  k_list_pull_fp64<<<list_blocks(b), kListTile, 0, s>>>(b, t);
}
void list_push_fp64(const ListArgs& a, const Trt<double>& t, cudaStream_t s) {
  static std::atomic<int> ahead{0};
  if (a.nFluid <= 0) return;
  ListArgs b = a;
  b.prefetch = prefetch_distance(ahead, k_list_push_fp64, kListTile, a.prefetch != 0);
  k_list_push_fp64<<<list_blocks(b), kListTile, 0, s>>>(b, t);
}

}  // namespace lbm
