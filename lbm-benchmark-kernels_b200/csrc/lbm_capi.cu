// lbm_capi.cu -- the C ABI of the B200 kernels: Init/Deinit pairs with the
// reference's KernelFunctions signatures, the KernelData callbacks they
// install, and a few flat helpers (include/lbm_b200.h).
//
// Device state per kernel instance:
//   AA full array   one PDF array (19 planes of the padded ghost-layer grid) and
//                   one uint32 link word per cell;
//   list AA         one PDF array (19 planes of nCells) and the push adjacency;
//   list pull       two PDF arrays and the pull adjacency.
// The host keeps a pinned mirror of the current PDF array for
// GetNode/SetNode; Kernel uploads it when SetNode has touched it, runs the time
// steps back to back on the instance's stream, and downloads it afterwards.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <strings.h>

#include "../../include/lbm_b200.h"
#include "lbm_host.h"
#include "lbm_kernels.cuh"

namespace {

using lbm::Q;
using lbm::QM;

// kListPull: pull-split layout (with its cache-line pad); kListPullPlain and
// kListPush: the two-grid list kernels list-pull-soa / list-push-soa
// kFaPush / kFaPull: the two-grid full-array kernels push-soa / pull-soa
enum Kind { kAa = 0, kListAa = 1, kListPull = 2, kListPullPlain = 3, kListPush = 4, kFaPush = 5, kFaPull = 6 };

bool full_array(int kind) { return kind == kAa || kind == kFaPush || kind == kFaPull; }
bool two_grid(int kind) {
  return kind == kListPull || kind == kListPullPlain || kind == kListPush || kind == kFaPush || kind == kFaPull;
}

thread_local std::string g_lastError;

struct Gpu {
  KernelData kd;  // first member: the reference's KernelData layout
  Kind kind;
  int dims[3];
  int per[3];
  double lambda;
  int iteration;  // logical view: -1 before the first step, then the last step done

  // pinned host mirror of the current PDF array (FP64 whatever the storage)
  double* mirror;
  size_t mirrorElems;
  bool dirty;
  int storage;       // lbm::kStoreF64 / F32 / F16
  size_t elemBytes;  // bytes per stored PDF
  void* rawStage;    // pinned staging buffer of the device format (reduced storage)

  // device memory
  double* dF;
  double* dG;
  uint32_t* dLink;
  uint32_t* dAdj;
  int* dErr;
  // Set once the device error word was found non-zero: a bounded wait gave up
  // (bit 1; a bulk copy may still have landed in another block's shared
  // memory) or a tile was skipped (bit 4), so the device PDFs are not a state
  // of the update. Steps are refused until the host state is uploaded again
  // (set_field / SetNode, or a checkpoint restore), which clears it.
  bool stateLost;
  uint64_t maskHash;       // FNV-1a of the instance's lattice mask (checkpoint check)
  double* dVerify;         // device -verify: x-velocity slice (nY*nZ) + the error
  long long* dVerifyBase;  // device -verify: element base of each slice cell
  cudaStream_t stream;
  cudaEvent_t ev0, ev1;

  // AA layout
  int xs, pitch;
  long long dstride;
  int* dOddItems;          // odd step: nOddItems interior work items (aa_interior_items)
  int* dOddCells;          // odd step: the general cells of the items, in chunks of 128
  int nOddItems;
  // x-slab of a larger lattice (lbm_aa_slab_init): halo/cross flags of the two x faces
  int halo[2], cross[2];
  int* sliceMask;          // the slab's own mask (owned)
  // x-slab of a list-AA lattice (lbm_aa_list_slab_init): halo slot lists per
  // side, [side][0] = own slots the neighbour reaches, [side][1] = ghost slots
  uint32_t* dHalo[2][2];
  long long nHalo[2][2];
  bool listSlab;
  int innerT0, innerT1;  // list slab: tiles whose odd step touches no halo slot

  // list layout
  uint32_t* grid;
  uint32_t* adjHost;
  uint32_t* dRuns;    // run-compressed adjacency (list AA and list push kernels)
  uint32_t* dRunOff;
  size_t runBytes;
  int nFluid, nCells;
  int cur;  // pull: index of the current grid (0 = dF, 1 = dG)

  double* dMomOut;  // 4 doubles for lbm_b200_instance_moments (allocated on first use)
  double* dMomPartials;  // its per-block partial sums for reduced storage (first use)

  // last Kernel call
  double lastDeviceMs;
  long lastLaunches;
  size_t lastH2D, lastD2H;
};

#define LBM_CK(call)                                                                                 \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) {                                                                         \
      g_lastError = std::string(#call) + ": " + cudaGetErrorString(e_);                              \
      std::printf("ERROR: CUDA: %s (%s:%d)\n", g_lastError.c_str(), __FILE__, __LINE__);            \
      std::exit(1);                                                                                  \
    }                                                                                                \
  } while (0)

void usage() {
  std::printf("Kernel parameters:\n");
  std::printf("  [-lambda <v|a/b>] [-blk <n>] [-blk-[xyz] <n>] [-pad auto|no|m+o(,m+o)*] [-bs <n>]\n");
  std::printf("  [-precision fp64|fp32|fp16]   (cuda-list-aa-pv-soa: PDF storage; fp32/fp16 relax in FP32)\n");
}

struct Args {
  double lambda = 1.0 / 12.0;
  int blk[3] = {0, 0, 0};
  const char* pad = nullptr;
  int storage = lbm::kStoreF64;
};

Args parse_args(Parameters* p) {
  Args a;
  if (p == nullptr) return a;
  for (int i = 0; i < p->nKernelArgs; ++i) {
    const char* s = p->KernelArgs[i];
    auto need = [&]() -> const char* {
      if (i + 1 >= p->nKernelArgs) {
        std::printf("ERROR: argument %s requires a parameter.\n", s);
        std::exit(1);
      }
      return p->KernelArgs[++i];
    };
    if (!std::strcmp(s, "-lambda") || !std::strcmp(s, "--lambda")) {
      const char* v = need();
      if (lbmh_parse_fraction(v, &a.lambda) || !(a.lambda > 0.0)) {
        std::printf("ERROR: -lambda needs a positive number or fraction, got \"%s\".\n", v);
        std::exit(1);
      }
    } else if (!std::strcmp(s, "-blk") || !std::strcmp(s, "--blk")) {
      int v = (int)std::strtol(need(), nullptr, 0);
      if (v < 0) { std::printf("ERROR: blocking parameter must be >= 0.\n"); std::exit(1); }
      a.blk[0] = a.blk[1] = a.blk[2] = v;
    } else if (!std::strncmp(s, "-blk-", 5) || !std::strncmp(s, "--blk-", 6)) {
      char axis = s[std::strlen(s) - 1];
      int v = (int)std::strtol(need(), nullptr, 0);
      if (v < 0 || axis < 'x' || axis > 'z') { std::printf("ERROR: blocking parameter must be >= 0.\n"); std::exit(1); }
      a.blk[axis - 'x'] = v;
    } else if (!std::strcmp(s, "-pad") || !std::strcmp(s, "--pad")) {
      a.pad = need();
    } else if (!std::strcmp(s, "-precision") || !std::strcmp(s, "--precision")) {
      const char* v = need();
      if (!std::strcmp(v, "fp64")) a.storage = lbm::kStoreF64;
      else if (!std::strcmp(v, "fp32")) a.storage = lbm::kStoreF32;
      else if (!std::strcmp(v, "fp16")) a.storage = lbm::kStoreF16;
      else {
        std::printf("ERROR: -precision must be fp64, fp32 or fp16, got \"%s\".\n", v);
        std::exit(1);
      }
    } else if (!std::strcmp(s, "-bs") || !std::strcmp(s, "--bs")) {
      (void)need();  // accepted for command-line compatibility; tiles are fixed per kernel
    } else if (!std::strcmp(s, "-h") || !std::strcmp(s, "-help") || !std::strcmp(s, "--help")) {
      usage();
      std::exit(1);
    } else {
      std::printf("ERROR: unknown kernel parameter.\n");
      usage();
      std::exit(1);
    }
  }
  return a;
}

lbm::Trt<double> make_trt(double omega, double lambda, double xforce) {
  // evaluated as the reference does at the top of its kernels
  // (src/BenchKernelD3Q19Aa.c:69-88, src/Kernel.c:769-795)
  lbm::Trt<double> t;
  t.omegaEven = omega;
  t.omegaOdd = 1.0 / (0.5 + lambda / (1.0 / omega - 0.5));
  t.w0 = 1.0 / 3.0;
  t.w1 = 1.0 / 18.0;
  t.w2 = 1.0 / 36.0;
  t.w1x3 = t.w1 * 3.0;
  t.w1nh = t.w1 * 9.0 / 2.0;
  t.w2x3 = t.w2 * 3.0;
  t.w2nh = t.w2 * 9.0 / 2.0;
  const double w[Q] = {t.w1, t.w1, t.w1, t.w1, t.w2, t.w2, t.w2, t.w2, t.w1, t.w2,
                       t.w2, t.w2, t.w2, t.w1, t.w2, t.w2, t.w2, t.w2, t.w0};
  for (int d = 0; d < Q; ++d) t.force[d] = 3.0 * w[d] * lbm::cx(d) * xforce;
  return t;
}

// The reduced-storage kernels' constants: the two rates and the x body force
// as its two class increments (the FP32 values of the FP64 table's E and NE
// entries).
lbm::TrtW to_trtw(const lbm::Trt<double>& d) {
  lbm::TrtW t;
  t.omegaEven = (float)d.omegaEven;
  t.omegaOdd = (float)d.omegaOdd;
  t.fx1 = (float)d.force[lbm::E];
  t.fx2 = (float)d.force[lbm::NE];
  return t;
}

// Weights and FP16 scales per direction (the device's StoreF16 uses the same
// powers of two).
double weight_of(int d) { return d == lbm::DC ? 1.0 / 3.0 : (lbm::cx(d) * lbm::cx(d) + lbm::cy(d) * lbm::cy(d) + lbm::cz(d) * lbm::cz(d) == 1 ? 1.0 / 18.0 : 1.0 / 36.0); }
double f16_scale_of(int d) { return d == lbm::DC ? 32768.0 : (weight_of(d) > 0.05 ? 262144.0 : 524288.0); }

// --- logical node view on the mirror ---------------------------------------

inline double* slot(Gpu* g, int x, int y, int z, int d) {
  if (full_array(g->kind)) {
    // pull-soa keeps node x's PDF d at x - c_d (src/BenchKernelD3Q19Common.c:120-196)
    if (g->kind == kFaPull) {
      x -= lbm::cx(d);
      y -= lbm::cy(d);
      z -= lbm::cz(d);
    }
    long c = (long)(x + 1) * g->xs + (long)(y + 1) * g->pitch + z + lbm::kZOff;
    return g->mirror + d * g->dstride + c;
  }
  uint32_t node = g->grid[lbmh_lidx(g->dims, x, y, z)];
  return g->mirror + (size_t)d * g->nCells + node;
}

void check_node(Gpu* g, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= g->dims[0] || y >= g->dims[1] || z >= g->dims[2]) {
    std::printf("ERROR: node (%d, %d, %d) outside the lattice.\n", x, y, z);
    std::exit(1);
  }
  if (!full_array(g->kind) && g->grid[lbmh_lidx(g->dims, x, y, z)] == 0xffffffffu) {
    std::printf("ERROR: node (%d, %d, %d) is an obstacle and has no PDFs in a list layout.\n", x, y, z);
    std::exit(1);
  }
}

// The device state is kept in the reference's natural layout between Kernel
// calls: the AA kernels always finish an even/odd pair and the pull kernel
// writes the natural layout every step, so GetNode/SetNode read slot (x, d).
void cb_get_node(KernelData* kd, int x, int y, int z, PdfT* pdfs) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  check_node(g, x, y, z);
  for (int d = 0; d < Q; ++d) pdfs[d] = *slot(g, x, y, z, d);
}

void cb_set_node(KernelData* kd, int x, int y, int z, PdfT* pdfs) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  check_node(g, x, y, z);
  for (int d = 0; d < Q; ++d) *slot(g, x, y, z, d) = pdfs[d];
  g->dirty = true;
}

void cb_bc_get(KernelData* kd, int x, int y, int z, int dir, PdfT* pdf) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  check_node(g, x, y, z);
  *pdf = *slot(g, x, y, z, dir);
}

void cb_bc_set(KernelData* kd, int x, int y, int z, int dir, PdfT pdf) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  check_node(g, x, y, z);
  *slot(g, x, y, z, dir) = pdf;
  g->dirty = true;
}

// --- device steps -------------------------------------------------------------

lbm::AaArgs aa_args(Gpu* g) {
  lbm::AaArgs a;
  a.f = g->cur == 0 ? g->dF : g->dG;  // two-grid kinds: source grid, then
  a.g = g->cur == 0 ? g->dG : g->dF;  // destination grid (null for AA)
  a.dstride = g->dstride;
  a.link = g->dLink;
  a.nX = g->dims[0];
  a.nY = g->dims[1];
  a.nZ = g->dims[2];
  a.xs = g->xs;
  a.pitch = g->pitch;
  a.perX = g->per[0];
  a.perY = g->per[1];
  a.perZ = g->per[2];
  a.haloLo = g->halo[0];
  a.haloHi = g->halo[1];
  a.crossLo = g->cross[0];
  a.crossHi = g->cross[1];
  a.xBase = 0;
  const int S = (int)g->dstride;
  for (int d = 0; d < Q; ++d) {
    const int j = lbm::inv(d);
    a.ldOff[d] = d == lbm::DC ? lbm::DC * S : j * S + lbm::cx(j) * g->xs + lbm::cy(j) * g->pitch + lbm::cz(j);
    a.stOff[d] = d == lbm::DC ? lbm::DC * S : d * S + lbm::cx(d) * g->xs + lbm::cy(d) * g->pitch + lbm::cz(d);
  }
  return a;
}

// Whether list steps prefetch the adjacency of later tiles into L2
// (LBM_ADJ_PREFETCH=0 turns it off; the launchers pick the distance).
int list_prefetch_enabled() {
  static std::atomic<int> on{-1};
  int v = on.load(std::memory_order_acquire);
  if (v < 0) {
    const char* env = std::getenv("LBM_ADJ_PREFETCH");
    v = (env && *env && std::atoi(env) == 0) ? 0 : 1;
    on.store(v, std::memory_order_release);
  }
  return v;
}

lbm::ListArgs list_args(Gpu* g) {
  lbm::ListArgs a;
  a.prefetch = list_prefetch_enabled();
  a.f = g->cur == 0 ? g->dF : g->dG;
  a.g = g->cur == 0 ? g->dG : g->dF;
  a.adj = g->dAdj;
  a.runs = g->dRuns;
  a.runOff = g->dRunOff;
  a.tileBase = 0;
  a.nCells = g->nCells;
  a.nFluid = g->nFluid;
  a.err = g->dErr;
  return a;
}

lbm::ListArgsLp list_args_lp(Gpu* g) {
  lbm::ListArgsLp a;
  a.prefetch = list_prefetch_enabled();
  a.f = g->dF;
  a.adj = g->dAdj;
  a.runs = g->dRuns;
  a.runOff = g->dRunOff;
  a.tileBase = 0;
  a.nCells = g->nCells;
  a.nFluid = g->nFluid;
  a.err = g->dErr;
  return a;
}

double* current_grid(Gpu* g) { return (two_grid(g->kind) && g->cur == 1) ? g->dG : g->dF; }

// Enqueues n time steps (AA kernels: rounded up to whole even/odd pairs, as
// the reference's loop `for (iter = 0; iter < n; iter += 2)`); returns the
// number of launches. With `ev`, event k is recorded before launch k and one
// more after the last launch.
long enqueue_steps(Gpu* g, const lbm::Trt<double>& t, int n, cudaEvent_t* ev = nullptr) {
  long k = 0;
  auto mark = [&]() {
    if (ev) cudaEventRecord(ev[k], g->stream);
  };
  if (g->kind == kAa) {
    lbm::AaArgs a = aa_args(g);
    const bool shell = lbm::aa_shell_needed(a);
    for (int it = 0; it < n; it += 2) {
      mark();
      lbm::aa_even_fp64(a, t, g->stream);
      ++k;
      if (g->nOddItems > 0) {
        mark();
        lbm::aa_odd_interior_fp64(a, t, g->dOddItems, g->nOddItems, g->dOddCells, g->stream);
        ++k;
      }
      if (shell) {
        mark();
        lbm::aa_odd_face_fp64(a, t, g->stream);
        ++k;
      }
      g->iteration = it + 1;
    }
  } else if (g->kind == kListAa && g->storage != lbm::kStoreF64) {
    const lbm::ListArgsLp a = list_args_lp(g);
    const lbm::TrtW tf = to_trtw(t);
    for (int it = 0; it < n; it += 2) {
      mark();
      lbm::list_even_lp(a, tf, g->storage, g->stream);
      ++k;
      mark();
      lbm::list_odd_lp(a, tf, g->storage, g->stream);
      ++k;
      g->iteration = it + 1;
    }
  } else if (g->kind == kListAa) {
    lbm::ListArgs a = list_args(g);
    for (int it = 0; it < n; it += 2) {
      mark();
      lbm::list_even_fp64(a, t, g->stream);
      ++k;
      mark();
      lbm::list_odd_fp64(a, t, g->stream);
      ++k;
      g->iteration = it + 1;
    }
  } else if (g->kind == kFaPush || g->kind == kFaPull) {
    for (int it = 0; it < n; ++it) {
      const lbm::AaArgs a = aa_args(g);
      mark();
      if (g->kind == kFaPush)
        lbm::fa_push_fp64(a, t, g->stream);
      else
        lbm::fa_pull_fp64(a, t, g->stream);
      ++k;
      g->cur ^= 1;
      g->iteration = it;
    }
  } else {
    for (int it = 0; it < n; ++it) {
      lbm::ListArgs a = list_args(g);
      mark();
      if (g->kind == kListPush)
        lbm::list_push_fp64(a, t, g->stream);
      else
        lbm::list_pull_fp64(a, t, g->stream);
      ++k;
      g->cur ^= 1;
      g->iteration = it;
    }
  }
  mark();
  return k;
}

long launches_for(Gpu* g, int n) {
  if (two_grid(g->kind)) return n;
  long perPair = 2;
  if (g->kind == kAa) {
    const lbm::AaArgs a = aa_args(g);
    perPair = 1 + (g->nOddItems > 0) + (lbm::aa_shell_needed(a) ? 1 : 0);
  }
  return perPair * ((n + 1) / 2);
}

// Elements of each direction's plane that hold state. A list layout keeps its
// nodes in [0, nFluid) of a plane of nCells elements; the padding behind them
// is read by no step, so the field copies and conversions skip it (22 % of
// the FP64 field of a 256^3 sphere packing at porosity 0.40). Full-array
// layouts and list slabs (whose ghost slots follow the nodes) use whole
// planes.
size_t plane_elems(const Gpu* g) { return g->mirrorElems / Q; }
size_t live_per_plane(const Gpu* g) {
  return (!full_array(g->kind) && !g->listSlab) ? static_cast<size_t>(g->nFluid) : plane_elems(g);
}

// Copies the live part of the field between host and device on the
// instance's stream (one 2D copy over the 19 planes, or one flat copy when
// no padding is skipped); returns the bytes moved.
size_t field_copy(Gpu* g, void* dst, const void* src, cudaMemcpyKind dir) {
  const size_t plane = plane_elems(g), live = live_per_plane(g), eb = g->elemBytes;
  if (live == plane || plane * eb > static_cast<size_t>(INT32_MAX)) {
    LBM_CK(cudaMemcpyAsync(dst, src, g->mirrorElems * eb, dir, g->stream));
    return g->mirrorElems * eb;
  }
  if (live > 0) LBM_CK(cudaMemcpy2DAsync(dst, plane * eb, src, plane * eb, live * eb, Q, dir, g->stream));
  return Q * live * eb;
}

// Host-side conversion between the FP64 mirror and the device storage format
// (element k of plane d belongs to direction d), over the live elements.
void mirror_to_raw(Gpu* g) {
  const size_t nc = plane_elems(g), live = live_per_plane(g);
  for (int d = 0; d < Q; ++d) {
    const double* m = g->mirror + d * nc;
    const double w = weight_of(d);
    if (g->storage == lbm::kStoreF32) {
      float* r = static_cast<float*>(g->rawStage) + d * nc;
      for (size_t k = 0; k < live; ++k) r[k] = (float)(m[k] - w);
    } else {
      uint16_t* r = static_cast<uint16_t*>(g->rawStage) + d * nc;
      const double sc = f16_scale_of(d);
      for (size_t k = 0; k < live; ++k) r[k] = lbmh_f32_to_f16((float)((m[k] - w) * sc));
    }
  }
}

void raw_to_mirror(Gpu* g) {
  const size_t nc = plane_elems(g), live = live_per_plane(g);
  for (int d = 0; d < Q; ++d) {
    double* m = g->mirror + d * nc;
    const double w = weight_of(d);
    if (g->storage == lbm::kStoreF32) {
      const float* r = static_cast<const float*>(g->rawStage) + d * nc;
      for (size_t k = 0; k < live; ++k) m[k] = w + (double)r[k];
    } else {
      const uint16_t* r = static_cast<const uint16_t*>(g->rawStage) + d * nc;
      const double sc = f16_scale_of(d);
      for (size_t k = 0; k < live; ++k) m[k] = w + (double)lbmh_f16_to_f32(r[k]) / sc;
    }
  }
}

// A fresh host state is on its way to the device: the error word and the
// lost flag start over (stream-ordered after the upload).
void clear_lost(Gpu* g) {
  if (!g->stateLost) return;
  LBM_CK(cudaMemsetAsync(g->dErr, 0, sizeof(int), g->stream));
  g->stateLost = false;
}

void upload_if_dirty(Gpu* g) {
  g->lastH2D = 0;
  if (!g->dirty) return;
  const void* src = g->mirror;
  if (g->storage != lbm::kStoreF64) {
    LBM_CK(cudaStreamSynchronize(g->stream));
    mirror_to_raw(g);
    src = g->rawStage;
  }
  g->lastH2D = field_copy(g, current_grid(g), src, cudaMemcpyHostToDevice);
  g->dirty = false;
  clear_lost(g);
}

void download(Gpu* g) {
  void* dst = g->storage == lbm::kStoreF64 ? static_cast<void*>(g->mirror) : g->rawStage;
  g->lastD2H = field_copy(g, dst, current_grid(g), cudaMemcpyDeviceToHost);
  LBM_CK(cudaStreamSynchronize(g->stream));
  if (g->storage != lbm::kStoreF64) raw_to_mirror(g);
}

// Reads the device error word (synchronous); a non-zero word marks the
// device state as lost. Returns the word.
int read_device_error(Gpu* g) {
  int err = 0;
  LBM_CK(cudaMemcpy(&err, g->dErr, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    g->stateLost = true;
    g_lastError = "a device wait exceeded its limit or a tile was skipped (error word " + std::to_string(err) +
                  "); the device state is lost until the host state is uploaded again";
  }
  return err;
}

void check_device_error(Gpu* g) {
  if (read_device_error(g)) {
    std::printf("ERROR: %s\n", g_lastError.c_str());
    std::exit(1);
  }
}

// Steps refuse to run on a lost device state (see Gpu::stateLost).
bool refuse_lost(Gpu* g) {
  if (!g->stateLost) return false;
  g_lastError = "the device state was lost to an earlier device error; upload a state (set_field, SetNode or a "
                "checkpoint restore) before stepping";
  return true;
}

void vtk_or_exit(LatticeDesc* ld, KernelData* kd, CaseData* cd, int label) {
  if (lbm_vtk_write(ld, kd, cd, label) != 0) std::exit(1);
}

// The step loop with VTK output (cd->VtkOutput), as the reference's kernels
// interleave it (src/BenchKernelD3Q19ListAaPv.c:67-150,
// src/BenchKernelD3Q19ListPullSplitNt.c:110-254): the state before the first
// step, after each step pair (AA forms; pull: each step) whose first step
// index is a multiple of VtkModulus, and after the last step. Each dump
// synchronises and downloads the mirror; the final dump follows the timed
// region.
long enqueue_steps_vtk(LatticeDesc* ld, Gpu* g, CaseData* cd, const lbm::Trt<double>& t) {
  const int n = cd->MaxIterations, stride = two_grid(g->kind) ? 1 : 2;
  const int modulus = cd->VtkModulus > 0 ? cd->VtkModulus : 1;
  long k = 0;
  for (int it = 0; it < n; it += stride) {
    k += enqueue_steps(g, t, stride);
    if (it % modulus == 0) {
      LBM_CK(cudaGetLastError());
      download(g);
      vtk_or_exit(ld, &g->kd, cd, it);
    }
  }
  return k;
}

void cb_kernel(LatticeDesc* ld, KernelData* kd, CaseData* cd) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (!(cd->Omega > 0.0 && cd->Omega < 2.0)) {
    std::printf("ERROR: omega must lie in (0, 2).\n");
    std::exit(1);
  }
  // the two-grid full-array kernels label their first file 0 (src/BenchKernelD3Q19.c:98-101)
  if (cd->VtkOutput) vtk_or_exit(ld, kd, cd, (g->kind == kFaPush || g->kind == kFaPull) ? 0 : -1);
  upload_if_dirty(g);
  if (refuse_lost(g)) {
    std::printf("ERROR: %s\n", g_lastError.c_str());
    std::exit(1);
  }
  const lbm::Trt<double> t = make_trt(cd->Omega, g->lambda, cd->XForce);

  LBM_CK(cudaStreamSynchronize(g->stream));
  auto w0 = std::chrono::steady_clock::now();
  LBM_CK(cudaEventRecord(g->ev0, g->stream));
  g->lastLaunches = cd->VtkOutput ? enqueue_steps_vtk(ld, g, cd, t) : enqueue_steps(g, t, cd->MaxIterations);
  LBM_CK(cudaGetLastError());
  LBM_CK(cudaEventRecord(g->ev1, g->stream));
  LBM_CK(cudaStreamSynchronize(g->stream));
  auto w1 = std::chrono::steady_clock::now();
  float ms = 0.f;
  LBM_CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
  g->lastDeviceMs = ms;
  kd->Duration = std::chrono::duration<double>(w1 - w0).count();
  check_device_error(g);
  download(g);
  if (cd->VtkOutput) vtk_or_exit(ld, kd, cd, cd->MaxIterations);
}

// --- Init / Deinit ----------------------------------------------------------------

// The x range [x0, x1) of a larger lattice that an AA instance covers.
struct SlabSpec {
  const LatticeDesc* global;
  int x0, x1;
  int halo[2];
  LbmhListSlab* list;  // list layout of a list-AA slab (ownership moves to the instance)
};

uint64_t fnv1a64(const void* data, size_t n);

Gpu* gpu_new(Kind kind, LatticeDesc* ld, Parameters* params, const SlabSpec* slab = nullptr) {
  Gpu* g = static_cast<Gpu*>(std::calloc(1, sizeof(Gpu)));
  if (!g) { std::printf("ERROR: allocation failed.\n"); std::exit(1); }
  Args a = parse_args(params);
  g->kind = kind;
  g->lambda = a.lambda;
  g->storage = a.storage;
  g->elemBytes = a.storage == lbm::kStoreF64 ? 8 : (a.storage == lbm::kStoreF32 ? 4 : 2);
  if (a.storage != lbm::kStoreF64 && kind != kListAa) {
    std::printf("ERROR: -precision fp32/fp16 is available for cuda-list-aa-pv-soa only.\n");
    std::exit(1);
  }
  g->iteration = -1;
  g->maskHash = fnv1a64(ld->Lattice, sizeof(int) * (size_t)ld->Dims[0] * ld->Dims[1] * ld->Dims[2]);
  for (int i = 0; i < 3; ++i) g->dims[i] = ld->Dims[i];
  g->per[0] = ld->PeriodicX;
  g->per[1] = ld->PeriodicY;
  g->per[2] = ld->PeriodicZ;
  LBM_CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  LBM_CK(cudaEventCreate(&g->ev0));
  LBM_CK(cudaEventCreate(&g->ev1));
  LBM_CK(cudaMalloc(&g->dErr, sizeof(int)));
  LBM_CK(cudaMemset(g->dErr, 0, sizeof(int)));

  KernelData* kd = &g->kd;
  kd->Dims[0] = ld->Dims[0];
  kd->Dims[1] = ld->Dims[1];
  kd->Dims[2] = ld->Dims[2];
  kd->GetNode = cb_get_node;
  kd->SetNode = cb_set_node;
  kd->BoundaryConditionsGetPdf = cb_bc_get;
  kd->BoundaryConditionsSetPdf = cb_bc_set;
  kd->Kernel = cb_kernel;

  const uint64_t nPdfs = 19ull * ld->Dims[0] * ld->Dims[1] * ld->Dims[2];
  if (nPdfs >= (1ull << 32)) {
    std::printf("ERROR: number of PDFs exceeds the 32-bit indices of this layout.\n");
    std::exit(1);
  }

  if (full_array(kind)) {
    const int gx = ld->Dims[0] + 2, gy = ld->Dims[1] + 2;
    g->pitch = (ld->Dims[2] + lbm::kZOff + 1 + 3) / 4 * 4;
    g->xs = gy * g->pitch;
    g->dstride = (long long)gx * g->xs;
    if (ld->Dims[0] > 65535 || ld->Dims[1] > 65535) {
      // the full-array kernels put x and y on the grid's y/z dimensions
      std::printf("ERROR: the full-array kernels take at most 65535 cells along x and y.\n");
      std::exit(1);
    }
    if ((unsigned long long)Q * g->dstride >= (1ull << 31)) {
      // the odd step addresses all 19 planes with 32-bit offsets (the
      // reference bounds its PDF count by 2^31 too, src/Main.c:399-406)
      std::printf("ERROR: the full-array layout of this lattice exceeds 2^31 PDFs; use a list kernel.\n");
      std::exit(1);
    }
    g->mirrorElems = (size_t)Q * g->dstride;
    kd->GlobalDims[0] = gx;
    kd->GlobalDims[1] = gy;
    kd->GlobalDims[2] = ld->Dims[2] + 2;
    kd->Offsets[0] = kd->Offsets[1] = kd->Offsets[2] = 1;
    kd->LoopBalance = 2.0 * 19 * sizeof(double);

    uint32_t* link = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (size_t)g->dstride));
    if (!link) { std::printf("ERROR: allocation failed.\n"); std::exit(1); }
    if (slab) {
      lbmh_aa_links_range(slab->global, slab->x0, slab->x1, g->xs, g->pitch, lbm::kZOff, link);
      for (int s2 = 0; s2 < 2; ++s2) g->halo[s2] = slab->halo[s2];
      // a halo face on the lattice's own x boundary is its periodic wrap
      g->cross[0] = slab->halo[0] && slab->x0 == 0;
      g->cross[1] = slab->halo[1] && slab->x1 == slab->global->Dims[0];
    } else {
      lbmh_aa_links(ld, g->xs, g->pitch, lbm::kZOff, link);
    }
    LBM_CK(cudaMalloc(&g->dLink, sizeof(uint32_t) * (size_t)g->dstride));
    LBM_CK(cudaMemcpy(g->dLink, link, sizeof(uint32_t) * (size_t)g->dstride, cudaMemcpyHostToDevice));
    LBM_CK(cudaMalloc(&g->dF, sizeof(double) * g->mirrorElems));
    LBM_CK(cudaMemset(g->dF, 0, sizeof(double) * g->mirrorElems));
    if (kind != kAa) {
      LBM_CK(cudaMalloc(&g->dG, sizeof(double) * g->mirrorElems));
      LBM_CK(cudaMemset(g->dG, 0, sizeof(double) * g->mirrorElems));
    }
    // the AA odd step's interior work items
    const lbm::AaArgs aa = aa_args(g);
    if (kind == kAa && lbm::aa_interior_block_count(aa) > 0) {
      std::vector<int> items, cells;
      lbm::aa_interior_items(aa, link, items, cells);
      g->nOddItems = (int)items.size();
      if (!items.empty()) {
        LBM_CK(cudaMalloc(&g->dOddItems, sizeof(int) * items.size()));
        LBM_CK(cudaMemcpy(g->dOddItems, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice));
      }
      if (!cells.empty()) {
        LBM_CK(cudaMalloc(&g->dOddCells, sizeof(int) * cells.size()));
        LBM_CK(cudaMemcpy(g->dOddCells, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice));
      }
    }
    std::free(link);
  } else {
    const bool pull = kind == kListPull || kind == kListPullPlain;
    int nCells = lbmh_pad_cells(ld->nFluid, (int)sizeof(double), a.pad);
    if (nCells < 0) std::exit(1);
    if (kind == kListPull) nCells = nCells + (8 - nCells % 8);  // cache-line pad (src/BenchKernelD3Q19ListPullSplitNtCommon.c:494-496)
    if (a.storage != lbm::kStoreF64)
      // reduced storage: planes padded to whole staging tiles (-pad does not apply)
      nCells = (std::max(ld->nFluid, 1) + lbm::kLpTileNodes - 1) / lbm::kLpTileNodes * lbm::kLpTileNodes;
    g->nCells = nCells;
    g->nFluid = ld->nFluid;
    const long ncell = (long)ld->Dims[0] * ld->Dims[1] * ld->Dims[2];
    g->grid = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * ncell));
    if (!g->grid) { std::printf("ERROR: allocation failed.\n"); std::exit(1); }
    const long nTiles = (g->nFluid + lbm::kListTile - 1) / lbm::kListTile;
    const size_t adjElems = (size_t)(nTiles > 0 ? nTiles : 1) * lbm::kListTile * QM;
    // numbering and adjacency built on the device (lbm_build.cu); the host
    // keeps the numbering for GetNode/SetNode
    LBM_CK(cudaMalloc(&g->dAdj, sizeof(uint32_t) * adjElems));
    LBM_CK(cudaMemset(g->dAdj, 0, sizeof(uint32_t) * adjElems));
    if (slab && slab->list) {
      // a list-AA slab: the host-built layout with ghost nodes after the owned ones
      LbmhListSlab* ls = slab->list;
      g->nCells = nCells = ls->nCells;
      std::free(g->grid);
      g->grid = ls->grid;
      ls->grid = nullptr;
      if (ls->nOwned > 0)
        LBM_CK(cudaMemcpy(g->dAdj, ls->adj, sizeof(uint32_t) * QM * (size_t)ls->nOwned, cudaMemcpyHostToDevice));
      for (int side = 0; side < 2; ++side)
        for (int list = 0; list < 2; ++list) {
          const uint32_t* h = list == 0 ? ls->own[side] : ls->ghost[side];
          const long n = list == 0 ? ls->nOwnSlots[side] : ls->nGhostSlots[side];
          g->nHalo[side][list] = h ? n : -1;
          if (h && n > 0) {
            LBM_CK(cudaMalloc(&g->dHalo[side][list], sizeof(uint32_t) * (size_t)n));
            LBM_CK(cudaMemcpy(g->dHalo[side][list], h, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice));
          }
        }
      g->listSlab = true;
      lbmh_list_slab_inner_tiles(ls, lbm::kListTile, &g->innerT0, &g->innerT1);
    }
    if (!g->listSlab) {
      // a slab's layout came from the host builder above
      int* dMask = nullptr;
      uint32_t* dGrid = nullptr;
      LBM_CK(cudaMalloc(&dMask, sizeof(int) * ncell));
      LBM_CK(cudaMalloc(&dGrid, sizeof(uint32_t) * ncell));
      LBM_CK(cudaMemcpy(dMask, ld->Lattice, sizeof(int) * ncell, cudaMemcpyHostToDevice));
      const int per3[3] = {ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ};
      const char* berr = "";
      const long long nf = lbm::list_build_device(dMask, ld->Dims, per3, pull ? 1 : 0, a.blk, nCells, dGrid, g->dAdj,
                                                  nTiles * lbm::kListTile, g->stream, &berr);
      if (nf != g->nFluid) {
        std::printf("ERROR: list build: %s (fluid nodes %lld, expected %d).\n", berr, nf, g->nFluid);
        std::exit(1);
      }
      LBM_CK(cudaMemcpy(g->grid, dGrid, sizeof(uint32_t) * ncell, cudaMemcpyDeviceToHost));
      LBM_CK(cudaFree(dGrid));
      LBM_CK(cudaFree(dMask));
    }
    {
      // the adjacency-driven steps read the run-compressed form (the full
      // adjacency stays for the host layout queries)
      const int rc = lbm::list_runs_device(g->dAdj, g->nFluid, g->stream, &g->dRuns, &g->dRunOff, &g->runBytes);
      if (rc) {
        std::printf("ERROR: CUDA: run-compressed adjacency: %s\n", cudaGetErrorString((cudaError_t)rc));
        std::exit(1);
      }
    }
    g->mirrorElems = (size_t)Q * nCells;
    LBM_CK(cudaMalloc(&g->dF, g->elemBytes * g->mirrorElems));
    LBM_CK(cudaMemset(g->dF, 0, g->elemBytes * g->mirrorElems));
    if (two_grid(kind)) {
      LBM_CK(cudaMalloc(&g->dG, sizeof(double) * g->mirrorElems));
      LBM_CK(cudaMemset(g->dG, 0, sizeof(double) * g->mirrorElems));
    }
    kd->GlobalDims[0] = ld->Dims[0];
    kd->GlobalDims[1] = ld->Dims[1];
    kd->GlobalDims[2] = ld->Dims[2];
    // bytes per node update: the PDFs plus the adjacency the step reads
    // (run-compressed for the list AA odd and list push steps)
    const double pb = 2.0 * 19 * (double)g->elemBytes;
    const double ab = g->dRuns && g->nFluid > 0 ? (double)g->runBytes / g->nFluid : 18 * 4.0;
    kd->LoopBalance = two_grid(kind) ? pb + ab : (pb + (pb + ab)) / 2.0;
  }

  LBM_CK(cudaMallocHost(&g->mirror, sizeof(double) * g->mirrorElems));
  std::memset(g->mirror, 0, sizeof(double) * g->mirrorElems);
  g->dirty = false;  // device and mirror both hold zeros
  if (g->storage != lbm::kStoreF64) {
    LBM_CK(cudaMallocHost(&g->rawStage, g->elemBytes * g->mirrorElems));
    // the device holds raw zeros; keep the mirror consistent with them
    LBM_CK(cudaMemcpy(g->rawStage, g->dF, g->elemBytes * g->mirrorElems, cudaMemcpyDeviceToHost));
    raw_to_mirror(g);
  }
  kd->Pdfs[0] = g->mirror;
  kd->Pdfs[1] = nullptr;
  kd->PdfsActive = g->mirror;
  return g;
}

void gpu_free(KernelData** kernelData) {
  if (kernelData == nullptr || *kernelData == nullptr) return;
  Gpu* g = reinterpret_cast<Gpu*>(*kernelData);
  cudaStreamSynchronize(g->stream);
  cudaFree(g->dF);
  cudaFree(g->dG);
  cudaFree(g->dLink);
  cudaFree(g->dOddItems);
  cudaFree(g->dVerify);
  cudaFree(g->dVerifyBase);
  cudaFree(g->dOddCells);
  std::free(g->sliceMask);
  cudaFree(g->dAdj);
  cudaFree(g->dRuns);
  cudaFree(g->dRunOff);
  for (int side = 0; side < 2; ++side)
    for (int list = 0; list < 2; ++list) cudaFree(g->dHalo[side][list]);
  cudaFree(g->dErr);
  cudaFree(g->dMomOut);
  cudaFree(g->dMomPartials);
  cudaFreeHost(g->mirror);
  cudaFreeHost(g->rawStage);
  cudaEventDestroy(g->ev0);
  cudaEventDestroy(g->ev1);
  cudaStreamDestroy(g->stream);
  std::free(g->grid);
  std::free(g->adjHost);
  std::free(g);
  *kernelData = nullptr;
}

// --- checkpoints ------------------------------------------------------------------

// FNV-1a (64 bit) of a byte range: the payload check of checkpoint files.
uint64_t fnv1a64(const void* data, size_t n) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint64_t h = 1469598103934665603ull;
  for (size_t k = 0; k < n; ++k) {
    h ^= p[k];
    h *= 1099511628211ull;
  }
  return h;
}

// Instance checkpoint: this header (host byte order), then the current PDF
// array exactly as the device holds it (storage format, padding included).
struct CkptHeader {
  char magic[8];  // "LBMCKPT2"
  int32_t kind, storage;
  int32_t dims[3], per[3];
  int32_t iteration, nFluid;
  int64_t elems;
  int32_t elemBytes, reserved;
  double lambda;
  uint64_t maskHash;  // FNV-1a of the lattice mask: the same geometry, not only the same counts
  uint64_t checksum;
};

const char kCkptMagic[8] = {'L', 'B', 'M', 'C', 'K', 'P', 'T', '2'};

CkptHeader ckpt_header_of(const Gpu* g) {
  CkptHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kCkptMagic, 8);
  h.kind = (int32_t)g->kind;
  h.storage = g->storage;
  for (int i = 0; i < 3; ++i) {
    h.dims[i] = g->dims[i];
    h.per[i] = g->per[i];
  }
  h.iteration = g->iteration;
  h.nFluid = g->nFluid;
  h.elems = (int64_t)g->mirrorElems;
  h.elemBytes = (int32_t)g->elemBytes;
  h.lambda = g->lambda;
  h.maskHash = g->maskHash;
  return h;
}

void* ckpt_payload(Gpu* g) { return g->storage == lbm::kStoreF64 ? static_cast<void*>(g->mirror) : g->rawStage; }

}  // namespace

extern "C" {

void D3Q19CudaAaInit_AaSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kAa, ld, params)->kd;
}
void D3Q19CudaAaDeinit_AaSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}

void D3Q19CudaListAaPvInit_PushSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListAa, ld, params)->kd;
}
void D3Q19CudaListAaPvDeinit_PushSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}

void D3Q19CudaListPullSplitNt1SInit_PullSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListPull, ld, params)->kd;
}
void D3Q19CudaListPullSplitNt2SInit_PullSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListPull, ld, params)->kd;
}
void D3Q19CudaListPullSplitNtDeinit_PullSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}

void D3Q19CudaListAaInit_PushSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListAa, ld, params)->kd;
}
void D3Q19CudaListAaDeinit_PushSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}
void D3Q19CudaListAaRiaInit_PushSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListAa, ld, params)->kd;
}
void D3Q19CudaListAaRiaDeinit_PushSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}
void D3Q19CudaListInit_PushSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListPush, ld, params)->kd;
}
void D3Q19CudaListDeinit_PushSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}
void D3Q19CudaListInit_PullSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kListPullPlain, ld, params)->kd;
}
void D3Q19CudaListDeinit_PullSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}

void D3Q19CudaInit_PushSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kFaPush, ld, params)->kd;
}
void D3Q19CudaDeinit_PushSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}
void D3Q19CudaInit_PullSoA(LatticeDesc* ld, KernelData** kernelData, Parameters* params) {
  *kernelData = &gpu_new(kFaPull, ld, params)->kd;
}
void D3Q19CudaDeinit_PullSoA(LatticeDesc* ld, KernelData** kernelData) {
  (void)ld;
  gpu_free(kernelData);
}

static const LbmB200KernelFunctions kTable[] = {
    {"cuda-aa-soa", D3Q19CudaAaInit_AaSoA, D3Q19CudaAaDeinit_AaSoA},
    {"cuda-list-aa-pv-soa", D3Q19CudaListAaPvInit_PushSoA, D3Q19CudaListAaPvDeinit_PushSoA},
    {"cuda-list-pull-split-nt-1s-soa", D3Q19CudaListPullSplitNt1SInit_PullSoA, D3Q19CudaListPullSplitNtDeinit_PullSoA},
    {"cuda-list-pull-split-nt-2s-soa", D3Q19CudaListPullSplitNt2SInit_PullSoA, D3Q19CudaListPullSplitNtDeinit_PullSoA},
    {"cuda-list-aa-soa", D3Q19CudaListAaInit_PushSoA, D3Q19CudaListAaDeinit_PushSoA},
    {"cuda-list-aa-ria-soa", D3Q19CudaListAaRiaInit_PushSoA, D3Q19CudaListAaRiaDeinit_PushSoA},
    {"cuda-list-push-soa", D3Q19CudaListInit_PushSoA, D3Q19CudaListDeinit_PushSoA},
    {"cuda-list-pull-soa", D3Q19CudaListInit_PullSoA, D3Q19CudaListDeinit_PullSoA},
    {"cuda-push-soa", D3Q19CudaInit_PushSoA, D3Q19CudaDeinit_PushSoA},
    {"cuda-pull-soa", D3Q19CudaInit_PullSoA, D3Q19CudaDeinit_PullSoA},
};

const LbmB200KernelFunctions* lbm_b200_kernels(int* count) {
  if (count) *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
  return kTable;
}

double lbm_b200_last_device_ms(KernelData* kd) { return reinterpret_cast<Gpu*>(kd)->lastDeviceMs; }

long lbm_b200_last_launches(KernelData* kd) { return reinterpret_cast<Gpu*>(kd)->lastLaunches; }

void lbm_b200_last_copy_bytes(KernelData* kd, size_t* h2d, size_t* d2h) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (h2d) *h2d = g->lastH2D;
  if (d2h) *d2h = g->lastD2H;
}

int lbm_b200_step_device(KernelData* kd, CaseData* cd, int n) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (g->dirty) upload_if_dirty(g);
  if (refuse_lost(g)) return -4;
  const lbm::Trt<double> t = make_trt(cd->Omega, g->lambda, cd->XForce);
  g->lastLaunches = enqueue_steps(g, t, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) g_lastError = cudaGetErrorString(e);
  return (int)e;
}

int lbm_b200_verify_device(LatticeDesc* ld, KernelData* kd, CaseData* cd, int write_file, double* err) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  const int nx = g->dims[0], ny = g->dims[1], nz = g->dims[2];
  if (ld->Dims[0] != nx || ld->Dims[1] != ny || ld->Dims[2] != nz || !err) return -1;
  if (g->dirty) upload_if_dirty(g);
  if (refuse_lost(g)) return -4;
  const size_t n = (size_t)ny * nz;
  // element base of each slice cell (x = nX/2) in the instance's layout
  std::vector<long long> base(n);
  const int xs = nx / 2;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y) {
      long long b = -1;
      if (ld->Lattice[lbmh_lidx(ld->Dims, xs, y, z)] != LAT_CELL_OBSTACLE)
        b = full_array(g->kind) ? (long long)(xs + 1) * g->xs + (long long)(y + 1) * g->pitch + z + lbm::kZOff
                                : (long long)g->grid[lbmh_lidx(ld->Dims, xs, y, z)];
      base[(size_t)y * nz + z] = b;
    }
  lbm::VerifyArgs a;
  a.f = current_grid(g);
  a.storage = g->storage;
  a.nY = ny;
  a.nZ = nz;
  a.xforce = cd->XForce;
  a.visc = (1.0 / cd->Omega - 0.5) / 3.0;
  for (int d = 0; d < Q; ++d) {
    if (full_array(g->kind)) {
      a.off[d] = (long long)d * g->dstride;
      // pull-soa keeps node x's PDF d at x - c_d (as GetNode)
      if (g->kind == kFaPull) a.off[d] -= (long long)lbm::cx(d) * g->xs + (long long)lbm::cy(d) * g->pitch + lbm::cz(d);
    } else {
      a.off[d] = (long long)d * g->nCells;
    }
  }
  cudaError_t e = cudaSuccess;
  if (!g->dVerify) e = cudaMalloc(&g->dVerify, sizeof(double) * (n + 1));
  if (e == cudaSuccess && !g->dVerifyBase) e = cudaMalloc(&g->dVerifyBase, sizeof(long long) * n);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->dVerifyBase, base.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) {
    a.base = g->dVerifyBase;
    lbm::verify_device(a, g->dVerify, g->dVerify + n, g->stream);
    e = cudaGetLastError();
  }
  // only the slice and the error come back
  std::vector<double> slice(n + 1);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(slice.data(), g->dVerify, sizeof(double) * (n + 1), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
  if (read_device_error(g)) return -4;
  g->lastD2H = sizeof(double) * (n + 1);
  *err = slice[n];
  if (write_file) lbmh_verify_profile(ny, nz, cd->Omega, cd->XForce, slice.data(), 1);
  return 0;
}

int lbm_b200_inject_device_error(KernelData* kd, int word) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) e = cudaMemcpy(g->dErr, &word, sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) g_lastError = cudaGetErrorString(e);
  return (int)e;
}

int lbm_b200_sync_mirror(KernelData* kd) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
  // a lost device state is not downloaded: the mirror keeps the last good one
  if (g->stateLost || read_device_error(g)) return -4;
  download(g);
  return 0;
}

const char* lbm_b200_last_error(void) { return g_lastError.c_str(); }

long lbm_b200_launches_for(KernelData* kd, int n) { return launches_for(reinterpret_cast<Gpu*>(kd), n); }

int lbm_b200_run_records(KernelData* kd, uint32_t* tileOffsets, uint32_t* records) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (full_array(g->kind) || !g->dRuns) return -1;
  cudaError_t e = cudaStreamSynchronize(g->stream);
  const long long tiles = (g->nFluid + lbm::kListTile - 1) / lbm::kListTile;
  if (e == cudaSuccess && tileOffsets)
    e = cudaMemcpy(tileOffsets, g->dRunOff, sizeof(uint32_t) * (size_t)(tiles + 1), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && records) e = cudaMemcpy(records, g->dRuns, g->runBytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) g_lastError = cudaGetErrorString(e);
  return (int)e;
}

long long lbm_b200_adjacency_bytes(KernelData* kd) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (full_array(g->kind)) return 0;
  return (long long)g->runBytes;
}

// --- x-slabs of an AA-pattern lattice (full-array and list layouts) -------------

// The slab's own cells of `global` as a lattice of its own (mask owned by the
// caller): x range [x0, x1), the other axes whole.
static int* slab_mask(const LatticeDesc* global, int x0, int x1, LatticeDesc* local) {
  const int nx = global->Dims[0], ny = global->Dims[1], nz = global->Dims[2];
  const int L = x1 - x0;
  int* mask = static_cast<int*>(std::malloc(sizeof(int) * (size_t)L * ny * nz));
  if (!mask) return nullptr;
  int nFluid = 0;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < L; ++x) {
        const int v = global->Lattice[((long)z * ny + y) * nx + x0 + x];
        mask[((long)z * ny + y) * L + x] = v;
        nFluid += v != LAT_CELL_OBSTACLE;
      }
  *local = *global;
  local->Dims[0] = L;
  local->Lattice = mask;
  local->nCells = L * ny * nz;
  local->nFluid = nFluid;
  local->nObst = local->nCells - nFluid;
  return mask;
}

KernelData* lbm_aa_slab_init(LatticeDesc* global, int x0, int x1, int haloLo, int haloHi, Parameters* params) {
  const int nx = global->Dims[0];
  if (x0 < 0 || x1 > nx || x1 - x0 < 1) {
    g_lastError = "slab range outside the lattice";
    return nullptr;
  }
  // halo faces on the lattice's own x boundary close a ring: with periodic x,
  // and also when only y or z is periodic, because a link that leaves through
  // the x boundary and a periodic y/z face at once wraps every crossed axis
  // (src/BenchKernelD3Q19AaCommon.c:522-578) and reaches the other x end
  const bool anyPeriodic = global->PeriodicX || global->PeriodicY || global->PeriodicZ;
  if (!anyPeriodic && ((haloLo && x0 == 0) || (haloHi && x1 == nx))) {
    g_lastError = "a halo face on the lattice's x boundary needs a periodic axis";
    return nullptr;
  }
  LatticeDesc local;
  int* mask = slab_mask(global, x0, x1, &local);
  if (!mask) return nullptr;
  SlabSpec spec{global, x0, x1, {haloLo != 0, haloHi != 0}, nullptr};
  Gpu* g = gpu_new(kAa, &local, params, &spec);
  g->sliceMask = mask;
  return &g->kd;
}

static const char* list_slab_error(int rc) {
  switch (rc) {
    case -1: return "slab range outside the lattice, or a halo on a slab that spans it";
    case -2: return "a link leaves the slab through an x face without a halo";
    case -3: return "allocation failed";
    case -4: return "malformed -pad string";
    case -5: return "the slab's PDFs exceed 32-bit indices";
    default: return "list slab build failed";
  }
}

KernelData* lbm_aa_list_slab_init(LatticeDesc* global, int x0, int x1, int haloLo, int haloHi, Parameters* params) {
  const Args a = parse_args(params);
  LbmhListSlab ls;
  const int halo[2] = {haloLo != 0, haloHi != 0};
  // reduced storage: planes padded to whole staging tiles, as for an instance
  const int quantum = a.storage == lbm::kStoreF64 ? 0 : lbm::kLpTileNodes;
  const int rc = lbmh_list_slab_build(global, x0, x1, halo, a.blk, a.pad, quantum, &ls);
  if (rc) {
    g_lastError = list_slab_error(rc);
    return nullptr;
  }
  LatticeDesc local;
  int* mask = slab_mask(global, x0, x1, &local);
  if (!mask) {
    lbmh_list_slab_free(&ls);
    g_lastError = "allocation failed";
    return nullptr;
  }
  SlabSpec spec{global, x0, x1, {halo[0], halo[1]}, &ls};
  Gpu* g = gpu_new(kListAa, &local, params, &spec);
  g->sliceMask = mask;
  lbmh_list_slab_free(&ls);
  return &g->kd;
}

int lbm_aa_list_slab_layout(const LatticeDesc* global, int x0, int x1, int haloLo, int haloHi, Parameters* params,
                            long long* counts, uint32_t* grid, uint32_t* adj, uint32_t* ownLo, uint32_t* ghostLo,
                            uint32_t* ownHi, uint32_t* ghostHi) {
  const Args a = parse_args(params);
  LbmhListSlab ls;
  const int halo[2] = {haloLo != 0, haloHi != 0};
  const int quantum = a.storage == lbm::kStoreF64 ? 0 : lbm::kLpTileNodes;
  const int rc = lbmh_list_slab_build(global, x0, x1, halo, a.blk, a.pad, quantum, &ls);
  if (rc) {
    g_lastError = list_slab_error(rc);
    return rc;
  }
  counts[0] = ls.nOwned;
  counts[1] = ls.nGhost;
  counts[2] = ls.nCells;
  counts[3] = ls.own[0] ? ls.nOwnSlots[0] : -1;
  counts[4] = ls.ghost[0] ? ls.nGhostSlots[0] : -1;
  counts[5] = ls.own[1] ? ls.nOwnSlots[1] : -1;
  counts[6] = ls.ghost[1] ? ls.nGhostSlots[1] : -1;
  int t0 = 0, t1 = 0;
  lbmh_list_slab_inner_tiles(&ls, lbm::kListTile, &t0, &t1);
  counts[7] = t0;
  counts[8] = t1;
  const size_t cells = (size_t)ls.L * global->Dims[1] * global->Dims[2];
  if (grid) std::memcpy(grid, ls.grid, sizeof(uint32_t) * cells);
  if (adj && ls.nOwned > 0) std::memcpy(adj, ls.adj, sizeof(uint32_t) * QM * (size_t)ls.nOwned);
  uint32_t* outs[4] = {ownLo, ghostLo, ownHi, ghostHi};
  const uint32_t* ins[4] = {ls.own[0], ls.ghost[0], ls.own[1], ls.ghost[1]};
  for (int k = 0; k < 4; ++k)
    if (outs[k] && ins[k] && counts[3 + k] > 0) std::memcpy(outs[k], ins[k], sizeof(uint32_t) * (size_t)counts[3 + k]);
  lbmh_list_slab_free(&ls);
  return 0;
}

void lbm_aa_slab_deinit(KernelData* kd) {
  KernelData* k = kd;
  gpu_free(&k);
}

long long lbm_aa_halo_message(KernelData* kd, int side, int phase, int send) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (side < 0 || side > 1 || phase < 0 || phase > 1) return -1;
  if (!g->listSlab) return g->kind == kAa ? 5LL * g->dims[1] * g->dims[2] : -1;
  // phase 0 sends the own slots and receives the ghosts; phase 1 the reverse
  const int list = (phase == 0) == (send != 0) ? 0 : 1;
  return g->nHalo[side][list];
}

long long lbm_aa_halo_count(KernelData* kd) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (!g->listSlab) return 5LL * g->dims[1] * g->dims[2];
  long long m = 0;
  for (int side = 0; side < 2; ++side)
    for (int list = 0; list < 2; ++list) m = std::max(m, g->nHalo[side][list]);
  return m;
}

// Pending SetNode edits go up on the instance's stream, which is then
// drained: the caller's stream may be another one.
static void sync_upload(Gpu* g) {
  if (!g->dirty) return;
  upload_if_dirty(g);
  LBM_CK(cudaStreamSynchronize(g->stream));
}

static cudaStream_t stream_or(Gpu* g, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : g->stream;
}

// The halo slot list a list slab packs (pack = true) or unpacks through
// `side` in `phase`, or -1 if that face has no halo.
static int list_halo_list(Gpu* g, int side, int phase, bool pack) {
  const int list = (phase == 0) == pack ? 0 : 1;
  return g->nHalo[side][list] < 0 ? -1 : list;
}

int lbm_aa_halo_elem_bytes(KernelData* kd) { return (int)reinterpret_cast<Gpu*>(kd)->elemBytes; }

int lbm_aa_halo_pack(KernelData* kd, int side, int phase, void* buf, void* stream) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (side < 0 || side > 1 || phase < 0 || phase > 1) return -1;
  if (g->listSlab) {
    const int list = list_halo_list(g, side, phase, true);
    if (list < 0) return -1;
    sync_upload(g);
    lbm::slot_gather(g->dF, g->dHalo[side][list], g->nHalo[side][list], buf, (int)g->elemBytes,
                     stream_or(g, stream));
    return (int)cudaGetLastError();
  }
  if (g->kind != kAa) return -1;
  sync_upload(g);
  lbm::aa_halo_pack(aa_args(g), side, phase, static_cast<double*>(buf), stream_or(g, stream));
  return (int)cudaGetLastError();
}

int lbm_aa_halo_unpack(KernelData* kd, int side, int phase, const void* buf, void* stream) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (side < 0 || side > 1 || phase < 0 || phase > 1) return -1;
  if (g->listSlab) {
    const int list = list_halo_list(g, side, phase, false);
    if (list < 0) return -1;
    sync_upload(g);
    lbm::slot_scatter(g->dF, g->dHalo[side][list], g->nHalo[side][list], buf, (int)g->elemBytes,
                      stream_or(g, stream));
    return (int)cudaGetLastError();
  }
  if (g->kind != kAa) return -1;
  sync_upload(g);
  lbm::aa_halo_unpack(aa_args(g), side, phase, static_cast<const double*>(buf), stream_or(g, stream));
  return (int)cudaGetLastError();
}

int lbm_aa_slab_step(KernelData* kd, CaseData* cd, int half, void* stream) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (half < 0 || half > 1 || (g->kind != kAa && !g->listSlab)) return -1;
  sync_upload(g);
  if (refuse_lost(g)) return -4;
  const lbm::Trt<double> t = make_trt(cd->Omega, g->lambda, cd->XForce);
  const cudaStream_t s = stream_or(g, stream);
  if (g->listSlab && g->storage != lbm::kStoreF64) {
    const lbm::ListArgsLp la = list_args_lp(g);
    const lbm::TrtW tf = to_trtw(t);
    if (half == 0) {
      lbm::list_even_lp(la, tf, g->storage, s);
    } else {
      lbm::list_odd_lp(la, tf, g->storage, s);
      g->iteration += 2;
    }
    return (int)cudaGetLastError();
  }
  if (g->listSlab) {
    const lbm::ListArgs la = list_args(g);
    if (half == 0) {
      lbm::list_even_fp64(la, t, s);
    } else {
      lbm::list_odd_fp64(la, t, s);
      g->iteration += 2;
    }
    return (int)cudaGetLastError();
  }
  const lbm::AaArgs a = aa_args(g);
  if (half == 0) {
    lbm::aa_even_fp64(a, t, s);
  } else {
    if (g->nOddItems > 0) lbm::aa_odd_interior_fp64(a, t, g->dOddItems, g->nOddItems, g->dOddCells, s);
    if (lbm::aa_shell_needed(a)) lbm::aa_odd_face_fp64(a, t, s);
    g->iteration += 2;
  }
  return (int)cudaGetLastError();
}

int lbm_aa_slab_even_part(KernelData* kd, CaseData* cd, int part, void* stream) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (part < 0 || part > 1 || (g->kind != kAa && !g->listSlab)) return -1;
  sync_upload(g);
  if (refuse_lost(g)) return -4;
  const lbm::Trt<double> t = make_trt(cd->Omega, g->lambda, cd->XForce);
  const cudaStream_t s = stream_or(g, stream);
  if (g->listSlab) {
    const int nTiles = (g->nFluid + lbm::kListTile - 1) / lbm::kListTile;
    const bool split = g->innerT1 > g->innerT0;
    if (!split) {
      if (part == 1) {
        if (g->storage != lbm::kStoreF64)
          lbm::list_even_lp(list_args_lp(g), to_trtw(t), g->storage, s);
        else
          lbm::list_even_fp64(list_args(g), t, s);
      }
      return (int)cudaGetLastError();
    }
    const int r[2][2] = {{part == 0 ? g->innerT0 : 0, part == 0 ? g->innerT1 : g->innerT0},
                         {part == 0 ? 0 : g->innerT1, part == 0 ? 0 : nTiles}};
    for (int k = 0; k < 2; ++k) {
      if (r[k][1] <= r[k][0]) continue;
      if (g->storage != lbm::kStoreF64)
        lbm::list_even_lp_tiles(list_args_lp(g), to_trtw(t), g->storage, r[k][0], r[k][1], s);
      else
        lbm::list_even_fp64_tiles(list_args(g), t, r[k][0], r[k][1], s);
    }
  } else {
    const lbm::AaArgs a = aa_args(g);
    const int nx = g->dims[0];
    if (nx <= 2) {
      if (part == 1) lbm::aa_even_fp64(a, t, s);
    } else if (part == 0) {
      lbm::aa_even_fp64_planes(a, t, 1, nx - 1, s);
    } else {
      lbm::aa_even_fp64_planes(a, t, 0, 1, s);
      lbm::aa_even_fp64_planes(a, t, nx - 1, nx, s);
    }
  }
  return (int)cudaGetLastError();
}

int lbm_aa_slab_odd_part(KernelData* kd, CaseData* cd, int part, void* stream) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (part < 0 || part > 1 || (g->kind != kAa && !g->listSlab)) return -1;
  sync_upload(g);
  if (refuse_lost(g)) return -4;
  const lbm::Trt<double> t = make_trt(cd->Omega, g->lambda, cd->XForce);
  const cudaStream_t s = stream_or(g, stream);
  if (g->listSlab) {
    const int nTiles = (g->nFluid + lbm::kListTile - 1) / lbm::kListTile;
    // part 0: the inner tiles; part 1: the tiles before and after them (all
    // tiles when the slab has no inner range)
    int r[2][2] = {{0, 0}, {0, 0}};
    if (g->innerT1 > g->innerT0) {
      if (part == 0) {
        r[0][0] = g->innerT0;
        r[0][1] = g->innerT1;
      } else {
        r[0][1] = g->innerT0;
        r[1][0] = g->innerT1;
        r[1][1] = nTiles;
      }
    } else if (part == 1) {
      r[0][1] = nTiles;
    }
    for (int k = 0; k < 2; ++k) {
      const int t0 = r[k][0], t1 = r[k][1];
      if (t1 <= t0) continue;
      if (g->storage != lbm::kStoreF64)
        lbm::list_odd_lp_tiles(list_args_lp(g), to_trtw(t), g->storage, t0, t1, s);
      else
        lbm::list_odd_fp64_tiles(list_args(g), t, t0, t1, s);
    }
  } else {
    const lbm::AaArgs a = aa_args(g);
    if (part == 0) {
      // the interior blocks read and write only the slab's own planes
      if (g->nOddItems > 0) lbm::aa_odd_interior_fp64(a, t, g->dOddItems, g->nOddItems, g->dOddCells, s);
    } else if (lbm::aa_shell_needed(a)) {
      lbm::aa_odd_face_fp64(a, t, s);
    }
  }
  if (part == 1) g->iteration += 2;
  return (int)cudaGetLastError();
}

int lbm_b200_checkpoint_save(KernelData* kd, const char* path) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (g->dirty) {
    upload_if_dirty(g);  // the mirror holds SetNode edits: they are the state
  }
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
  if (g->stateLost || read_device_error(g)) return -4;
  download(g);
  CkptHeader h = ckpt_header_of(g);
  const size_t bytes = g->mirrorElems * g->elemBytes;
  h.checksum = fnv1a64(ckpt_payload(g), bytes);
  FILE* fh = std::fopen(path, "wb");
  if (!fh) { g_lastError = std::string("cannot open ") + path; return -1; }
  const bool ok = std::fwrite(&h, sizeof(h), 1, fh) == 1 && std::fwrite(ckpt_payload(g), 1, bytes, fh) == bytes;
  if (std::fclose(fh) != 0 || !ok) { g_lastError = std::string("writing ") + path + " failed"; return -1; }
  return 0;
}

int lbm_b200_checkpoint_load(KernelData* kd, const char* path) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  FILE* fh = std::fopen(path, "rb");
  if (!fh) { g_lastError = std::string("cannot open ") + path; return -1; }
  CkptHeader h;
  const CkptHeader want = ckpt_header_of(g);
  if (std::fread(&h, sizeof(h), 1, fh) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0) {
    std::fclose(fh);
    g_lastError = std::string(path) + " is not an instance checkpoint";
    return -2;
  }
  bool same = h.kind == want.kind && h.storage == want.storage && h.nFluid == want.nFluid && h.elems == want.elems &&
              h.elemBytes == want.elemBytes && h.lambda == want.lambda && h.maskHash == want.maskHash;
  for (int i = 0; i < 3; ++i) same = same && h.dims[i] == want.dims[i] && h.per[i] == want.per[i];
  if (!same) {
    std::fclose(fh);
    g_lastError = std::string(path) + " was written by an instance of another kernel, lattice (geometry), storage or Lambda";
    return -2;
  }
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) { std::fclose(fh); g_lastError = cudaGetErrorString(e); return (int)e; }
  const size_t bytes = g->mirrorElems * g->elemBytes;
  const bool ok = std::fread(ckpt_payload(g), 1, bytes, fh) == bytes;
  std::fclose(fh);
  if (!ok) {
    g_lastError = std::string(path) + " is truncated";
    download(g);  // the mirror stays the device state
    return -1;
  }
  if (fnv1a64(ckpt_payload(g), bytes) != h.checksum) {
    g_lastError = std::string(path) + ": checksum mismatch";
    download(g);  // the mirror stays the device state
    return -3;
  }
  e = cudaMemcpyAsync(current_grid(g), ckpt_payload(g), bytes, cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
  if (g->storage != lbm::kStoreF64) raw_to_mirror(g);
  g->dirty = false;
  g->iteration = h.iteration;
  clear_lost(g);
  return 0;
}

void lbm_b200_mark_mirror_dirty(KernelData* kd) { reinterpret_cast<Gpu*>(kd)->dirty = true; }

int lbm_b200_time_steps(KernelData* kd, CaseData* cd, int n, double* total_ms, double* per_launch_ms) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (g->dirty) upload_if_dirty(g);
  if (refuse_lost(g)) return -4;
  const lbm::Trt<double> t = make_trt(cd->Omega, g->lambda, cd->XForce);
  const long nl = launches_for(g, n);
  cudaEvent_t* ev = static_cast<cudaEvent_t*>(std::malloc(sizeof(cudaEvent_t) * (nl + 1)));
  for (long k = 0; k <= nl; ++k) cudaEventCreate(&ev[k]);
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) {
    g->lastLaunches = enqueue_steps(g, t, n, ev);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[nl]);
    if (total_ms) *total_ms = ms;
    if (per_launch_ms)
      for (long k = 0; k < nl; ++k) {
        cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
        per_launch_ms[k] = ms;
      }
  }
  for (long k = 0; k <= nl; ++k) cudaEventDestroy(ev[k]);
  std::free(ev);
  if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
  if (read_device_error(g)) return -1;
  return 0;
}

int lbm_b200_device_state(KernelData* kd, double** pdfs, long long* nCells, int* nFluid, void** stream) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (full_array(g->kind)) return -1;
  if (pdfs) *pdfs = current_grid(g);
  if (nCells) *nCells = g->nCells;
  if (nFluid) *nFluid = g->nFluid;
  if (stream) *stream = g->stream;
  return 0;
}

int lbm_b200_moments_device(const double* pdfs, long long nCells, int nFluid, double* out_device, void* stream);

int lbm_b200_instance_moments(KernelData* kd, double* out) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (full_array(g->kind)) return -1;
  if (g->dirty) upload_if_dirty(g);
  if (g->dMomOut == nullptr) {
    cudaError_t e = cudaMalloc(&g->dMomOut, 4 * sizeof(double));
    if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
  }
  if (g->storage != lbm::kStoreF64) {
    // reduced storage: FP64 sums of the stored deviations (scratch kept by
    // the instance)
    if (g->dMomPartials == nullptr) {
      cudaError_t e = cudaMalloc(&g->dMomPartials, sizeof(double) * 4 * lbm::moment_blocks(g->nFluid));
      if (e != cudaSuccess) { g_lastError = cudaGetErrorString(e); return (int)e; }
    }
    lbm::moments_enqueue_lp(g->dF, g->storage, g->nCells, g->nFluid, g->dMomPartials, g->dMomOut, g->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e == cudaSuccess) e = cudaMemcpy(out, g->dMomOut, 4 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) g_lastError = cudaGetErrorString(e);
    if (e == cudaSuccess && (g->stateLost || read_device_error(g))) return -4;  // sums of a lost state
    return (int)e;
  }
  int rc = lbm_b200_moments_device(current_grid(g), g->nCells, g->nFluid, g->dMomOut, g->stream);
  if (rc) return rc;
  cudaError_t e = cudaMemcpy(out, g->dMomOut, 4 * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && (g->stateLost || read_device_error(g))) return -4;  // sums of a lost state
  return (int)e;
}

int lbm_b200_set_device(int device) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) g_lastError = cudaGetErrorString(e);
  return (int)e;
}

// Bulk access to the logical PDFs of every fluid cell (19 doubles per cell,
// cells x fastest, obstacle cells skipped), through GetNode/SetNode.
void lbm_b200_get_field(KernelData* kd, LatticeDesc* ld, double* out) {
  const int* dims = ld->Dims;
  for (int z = 0; z < dims[2]; ++z)
    for (int y = 0; y < dims[1]; ++y)
      for (int x = 0; x < dims[0]; ++x) {
        const long c = lbmh_lidx(dims, x, y, z);
        if (ld->Lattice[c] == LAT_CELL_OBSTACLE) continue;
        kd->GetNode(kd, x, y, z, out + c * Q);
      }
}

void lbm_b200_set_field(KernelData* kd, LatticeDesc* ld, const double* in) {
  const int* dims = ld->Dims;
  for (int z = 0; z < dims[2]; ++z)
    for (int y = 0; y < dims[1]; ++y)
      for (int x = 0; x < dims[0]; ++x) {
        const long c = lbmh_lidx(dims, x, y, z);
        if (ld->Lattice[c] == LAT_CELL_OBSTACLE) continue;
        kd->SetNode(kd, x, y, z, const_cast<double*>(in + c * Q));
      }
}

// The host-built list layout of a list kernel instance (for parity checks):
// grid (nX*nY*nZ), adjacency (nFluid*18, the reference's order), counts.
int lbm_b200_list_layout(KernelData* kd, const uint32_t** grid, const uint32_t** adj, int* nFluid, int* nCells) {
  Gpu* g = reinterpret_cast<Gpu*>(kd);
  if (full_array(g->kind)) return -1;
  if (adj && !g->adjHost && g->nFluid > 0) {
    // the adjacency lives on the device; a host copy is made on first request
    g->adjHost = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (size_t)g->nFluid * QM));
    if (!g->adjHost ||
        cudaMemcpy(g->adjHost, g->dAdj, sizeof(uint32_t) * (size_t)g->nFluid * QM, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
      std::free(g->adjHost);
      g->adjHost = nullptr;
      return -2;
    }
  }
  if (grid) *grid = g->grid;
  if (adj) *adj = g->adjHost;
  if (nFluid) *nFluid = g->nFluid;
  if (nCells) *nCells = g->nCells;
  return 0;
}

}  // extern "C"
