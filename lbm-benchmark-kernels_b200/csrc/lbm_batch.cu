// lbm_batch.cu -- host side of the batched list AA form (include/lbm_b200.h,
// "Batched domains"): admission of domains under an HBM budget, the device
// tile/domain tables, CUDA-graph replay of whole step sequences, the FP64
// per-domain sums, and the launch autotuner.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_batch.cuh"
#include "lbm_host.h"

namespace {

using lbm::Q;
using lbm::QM;

const char* g_batchError = "";

#define BCK(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      g_batchError = cudaGetErrorString(e_);                               \
      std::fprintf(stderr, "lbm batch: %s: %s\n", #call, g_batchError);   \
      return -(int)e_ - 1000;                                              \
    }                                                                      \
  } while (0)

double weight_of(int d) {
  const int c2 = lbm::cx(d) * lbm::cx(d) + lbm::cy(d) * lbm::cy(d) + lbm::cz(d) * lbm::cz(d);
  return c2 == 0 ? 1.0 / 3.0 : (c2 == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
}
double f16_scale_of(int d) { return d == lbm::DC ? 32768.0 : (weight_of(d) > 0.05 ? 262144.0 : 524288.0); }

struct DomainSlot {
  bool active = false;
  lbm::BatchDomain dev{};  // as uploaded to the device table
  void* pdfs = nullptr;
  uint32_t* runs = nullptr;    // run-compressed adjacency
  uint32_t* runOff = nullptr;
  int nTiles = 0;
  size_t bytes = 0;
  int dims[3] = {0, 0, 0};
  std::vector<uint32_t> grid;  // lattice cell -> node (for field access)
  double omega = 1.0, lambda = 1.0 / 12.0, xforce = 0.0;
};

struct Batch {
  int storage;
  size_t elemBytes;
  size_t budget, used = 0;
  int maxSlots, maxTiles;
  std::vector<DomainSlot> slots;
  std::vector<int> tileDomHost;
  int nTiles = 0;
  cudaStream_t stream = nullptr;
  lbm::BatchDomain* dDoms = nullptr;
  int* dTileDom = nullptr;
  lbm::BatchTile* dTiles = nullptr;  // tile records, capacity tileCap
  int tileCap = 0;
  int gridTiles = 0;  // grid of the one-block-per-tile launches (>= nTiles)
  int* dNTiles = nullptr;
  int* dErr = nullptr;
  double* dPartials = nullptr;
  int* dDomTileStart = nullptr;
  int* dDomTileCount = nullptr;
  double* dMoments = nullptr;
  lbm::BatchLaunch evenL{256, 1, 0}, oddL{256, 1, 0};
  std::map<int, cudaGraphExec_t> graphs;  // steps -> instantiated graph
  long long launches = 0;
  int numSMs = 148;
};

lbm::BatchArgs args_of(const Batch* b, const lbm::BatchLaunch& l) {
  lbm::BatchArgs a;
  a.doms = b->dDoms;
  a.tileDom = b->dTileDom;
  a.tiles = b->dTiles;
  a.nTiles = b->dNTiles;
  a.err = b->dErr;
  a.storage = b->storage;
  a.nodesPerThread = l.nodesPerThread;
  a.blockNodes = l.threads * l.nodesPerThread;
  return a;
}

void drop_graphs(Batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
}

// Rebuilds the tile table, the per-domain tile ranges and the tile records
// after a change of membership (stream-ordered uploads, then a device pass
// that fills the records).
int publish(Batch* b) {
  b->tileDomHost.clear();
  std::vector<int> start(b->maxSlots, 0), count(b->maxSlots, 0);
  for (int s = 0; s < b->maxSlots; ++s) {
    DomainSlot& d = b->slots[s];
    if (!d.active) continue;
    d.dev.tileStart = (int)b->tileDomHost.size();
    start[s] = d.dev.tileStart;
    count[s] = d.nTiles;
    for (int t = 0; t < d.nTiles; ++t) b->tileDomHost.push_back(s);
    BCK(cudaMemcpyAsync(b->dDoms + s, &d.dev, sizeof(lbm::BatchDomain), cudaMemcpyHostToDevice, b->stream));
  }
  b->nTiles = (int)b->tileDomHost.size();
  if (b->nTiles > b->maxTiles) return -3;
  if (b->nTiles)
    BCK(cudaMemcpyAsync(b->dTileDom, b->tileDomHost.data(), sizeof(int) * b->nTiles, cudaMemcpyHostToDevice,
                        b->stream));
  if (b->nTiles > b->tileCap) {
    // records are reallocated: graphs captured with the old table go
    BCK(cudaStreamSynchronize(b->stream));
    drop_graphs(b);
    cudaFree(b->dTiles);
    b->dTiles = nullptr;
    b->tileCap = 0;
    const int cap = std::min(b->maxTiles, std::max(b->nTiles + b->nTiles / 2, 1024));
    BCK(cudaMalloc(&b->dTiles, sizeof(lbm::BatchTile) * (size_t)cap));
    b->tileCap = cap;
  }
  // the grid of one-block-per-tile launches keeps some headroom, so that
  // graphs survive admissions; it is resized (and graphs dropped) when the
  // table outgrows it or shrinks below half of it
  if (b->nTiles > b->gridTiles || b->nTiles < b->gridTiles / 2) {
    const int g = std::max(b->nTiles + b->nTiles / 8, 64);
    if (g != b->gridTiles) {
      drop_graphs(b);
      b->gridTiles = g;
    }
  }
  BCK(cudaMemcpyAsync(b->dNTiles, &b->nTiles, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->dDomTileStart, start.data(), sizeof(int) * b->maxSlots, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->dDomTileCount, count.data(), sizeof(int) * b->maxSlots, cudaMemcpyHostToDevice, b->stream));
  lbm::batch_build_tiles(b->dDoms, b->dTileDom, b->nTiles, b->dTiles, b->stream);
  BCK(cudaGetLastError());
  // the host vectors above are read by the copies: wait before they go away
  BCK(cudaStreamSynchronize(b->stream));
  return 0;
}

int enqueue(Batch* b, int nsteps) {
  if (b->nTiles == 0) return 0;
  const lbm::BatchArgs ae = args_of(b, b->evenL), ao = args_of(b, b->oddL);
  for (int it = 0; it < nsteps; it += 2) {
    lbm::batch_even_lp(ae, b->evenL, b->evenL.blocks ? b->evenL.blocks : b->gridTiles, b->stream);
    lbm::batch_odd_lp(ao, b->oddL, b->oddL.blocks ? b->oddL.blocks : b->gridTiles, b->stream);
    b->launches += 2;
  }
  BCK(cudaGetLastError());
  return 0;
}

// Bound on a domain's device bytes: PDFs plus the adjacency (full rows
// while the run-compressed form is built from them; the runs never exceed
// the full rows plus a 48-byte header per tile).
size_t domain_bytes(const Batch* b, long long nCells) {
  return (size_t)nCells * Q * b->elemBytes + (size_t)nCells * QM * 4 +
         (size_t)(nCells / lbm::kBatchTileNodes) * lbm::kRunHdrWords * 4;
}

lbm::TrtW trt_of(double omega, double lambda, double xforce) {
  lbm::TrtW t;
  t.omegaEven = (float)omega;
  t.omegaOdd = (float)(1.0 / (0.5 + lambda / (1.0 / omega - 0.5)));
  t.fx1 = (float)(3.0 * (1.0 / 18.0) * xforce);
  t.fx2 = (float)(3.0 * (1.0 / 36.0) * xforce);
  return t;
}

// Domain checkpoint: header (host byte order), then the slot's PDF array as
// the device holds it (storage format, tile padding included).
struct DomCkpt {
  char magic[8];  // "LBMBDOM1"
  int32_t storage, nFluid;
  int32_t dims[3], reserved;
  int64_t nCells;
  double omega, lambda, xforce;
  uint64_t checksum;
};
const char kDomMagic[8] = {'L', 'B', 'M', 'B', 'D', 'O', 'M', '1'};

uint64_t dom_fnv1a64(const void* data, size_t n) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint64_t h = 1469598103934665603ull;
  for (size_t k = 0; k < n; ++k) {
    h ^= p[k];
    h *= 1099511628211ull;
  }
  return h;
}

DomCkpt dom_header_of(const Batch* b, const DomainSlot& d) {
  DomCkpt c;
  std::memset(&c, 0, sizeof(c));
  std::memcpy(c.magic, kDomMagic, 8);
  c.storage = b->storage;
  c.nFluid = d.dev.nFluid;
  for (int i = 0; i < 3; ++i) c.dims[i] = d.dims[i];
  c.nCells = d.dev.nCells;
  c.omega = d.omega;
  c.lambda = d.lambda;
  c.xforce = d.xforce;
  return c;
}
}  // namespace

extern "C" {

const char* lbm_batch_last_error(void) { return g_batchError; }

int lbm_batch_reset(void* h, int slot);

void* lbm_batch_create(int storage, double budgetGB, int maxDomains) {
  if (storage != lbm::kStoreF32 && storage != lbm::kStoreF16) {
    g_batchError = "batched domains support storage fp32 (1) and fp16 (2)";
    return nullptr;
  }
  Batch* b = new Batch();
  b->storage = storage;
  b->elemBytes = storage == lbm::kStoreF32 ? 4 : 2;
  b->budget = (size_t)(budgetGB * 1e9);
  b->maxSlots = maxDomains > 0 ? maxDomains : 1024;
  b->slots.resize(b->maxSlots);
  const size_t perTile = domain_bytes(b, lbm::kBatchTileNodes);
  b->maxTiles = (int)std::min<size_t>(b->budget / perTile + (size_t)b->maxSlots, (size_t)1 << 26);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, dev);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&b->dDoms, sizeof(lbm::BatchDomain) * b->maxSlots) == cudaSuccess &&
            cudaMalloc(&b->dTileDom, sizeof(int) * b->maxTiles) == cudaSuccess &&
            cudaMalloc(&b->dNTiles, sizeof(int)) == cudaSuccess && cudaMalloc(&b->dErr, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&b->dPartials, sizeof(double) * 4 * (size_t)b->maxTiles) == cudaSuccess &&
            cudaMalloc(&b->dDomTileStart, sizeof(int) * b->maxSlots) == cudaSuccess &&
            cudaMalloc(&b->dDomTileCount, sizeof(int) * b->maxSlots) == cudaSuccess &&
            cudaMalloc(&b->dMoments, sizeof(double) * 4 * b->maxSlots) == cudaSuccess &&
            cudaMemset(b->dErr, 0, sizeof(int)) == cudaSuccess && cudaMemset(b->dNTiles, 0, sizeof(int)) == cudaSuccess;
  if (!ok) {
    g_batchError = "device allocation of the batch tables failed";
    delete b;
    return nullptr;
  }
  b->evenL.blocks = b->oddL.blocks = 0;  // one block per tile until tuned
  return b;
}

void lbm_batch_destroy(void* h) {
  Batch* b = static_cast<Batch*>(h);
  if (!b) return;
  cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  for (auto& s : b->slots) {
    cudaFree(s.pdfs);
    cudaFree(s.runs);
    cudaFree(s.runOff);
  }
  cudaFree(b->dDoms);
  cudaFree(b->dTileDom);
  cudaFree(b->dTiles);
  cudaFree(b->dNTiles);
  cudaFree(b->dErr);
  cudaFree(b->dPartials);
  cudaFree(b->dDomTileStart);
  cudaFree(b->dDomTileCount);
  cudaFree(b->dMoments);
  cudaStreamDestroy(b->stream);
  delete b;
}

// Admits a domain; returns its slot, -1 when the HBM budget is exhausted,
// -2 when every slot is taken, or another negative code on errors. The PDFs
// start at rest (f = w, rho = 1, u = 0).
int lbm_batch_add(void* h, const LatticeDesc* ld, double omega, double lambda, double xforce) {
  Batch* b = static_cast<Batch*>(h);
  if (!(omega > 0.0 && omega < 2.0) || !(lambda > 0.0)) return -4;
  int slot = -1;
  for (int s = 0; s < b->maxSlots; ++s)
    if (!b->slots[s].active) { slot = s; break; }
  if (slot < 0) return -2;
  const int nFluid = ld->nFluid;
  const long long nCells = ((long long)std::max(nFluid, 1) + lbm::kBatchTileNodes - 1) / lbm::kBatchTileNodes *
                           lbm::kBatchTileNodes;
  const size_t bytes = domain_bytes(b, nCells);
  if (b->used + bytes > b->budget) return -1;
  if ((uint64_t)nCells * Q >= (1ull << 32)) return -5;

  DomainSlot& d = b->slots[slot];
  d = DomainSlot();
  const long ncell = (long)ld->Dims[0] * ld->Dims[1] * ld->Dims[2];
  d.grid.resize(ncell);
  BCK(cudaMalloc(&d.pdfs, (size_t)nCells * Q * b->elemBytes));
  uint32_t* adj = nullptr;
  BCK(cudaMalloc(&adj, (size_t)nCells * QM * 4));
  // numbering and adjacency built on the device (lbm_build.cu); padding
  // nodes then point at their own slots so that every entry is in range;
  // the steps read the run-compressed form, built from it
  int* dMask = nullptr;
  uint32_t* dGrid = nullptr;
  BCK(cudaMallocAsync(&dMask, sizeof(int) * ncell, b->stream));
  BCK(cudaMallocAsync(&dGrid, sizeof(uint32_t) * ncell, b->stream));
  BCK(cudaMemcpyAsync(dMask, ld->Lattice, sizeof(int) * ncell, cudaMemcpyHostToDevice, b->stream));
  const int blk[3] = {0, 0, 0}, per[3] = {ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ};
  const char* berr = "";
  const long long nf = lbm::list_build_device(dMask, ld->Dims, per, 0, blk, (int)nCells, dGrid, adj, nCells,
                                              b->stream, &berr);
  if (nf == nFluid) {
    lbm::batch_pad_adjacency(adj, nFluid, nCells, b->stream);
    BCK(cudaMemcpyAsync(d.grid.data(), dGrid, sizeof(uint32_t) * ncell, cudaMemcpyDeviceToHost, b->stream));
  }
  cudaFreeAsync(dGrid, b->stream);
  cudaFreeAsync(dMask, b->stream);
  BCK(cudaStreamSynchronize(b->stream));
  int rrc = 0;
  size_t runBytes = 0;
  if (nf == nFluid) rrc = lbm::list_runs_device(adj, (int)nCells, b->stream, &d.runs, &d.runOff, &runBytes);
  cudaFree(adj);
  if (nf != nFluid || rrc) {
    g_batchError = rrc ? "building the run-compressed adjacency failed"
                       : (nf < 0 ? berr : "the mask's fluid cell count differs from the lattice's");
    cudaFree(d.pdfs);
    d = DomainSlot();
    return -6;
  }
  d.active = true;
  d.bytes = bytes;
  d.nTiles = (int)(nCells / lbm::kBatchTileNodes);
  for (int i = 0; i < 3; ++i) d.dims[i] = ld->Dims[i];
  d.omega = omega;
  d.lambda = lambda;
  d.xforce = xforce;
  d.dev.f = d.pdfs;
  d.dev.runs = d.runs;
  d.dev.runOff = d.runOff;
  d.dev.nCells = nCells;
  d.dev.nFluid = nFluid;
  d.dev.trt = trt_of(omega, lambda, xforce);
  b->used += bytes;
  int rc = lbm_batch_reset(h, slot);
  if (rc) return rc;
  rc = publish(b);  // synchronises: the host adjacency may go
  return rc ? rc : slot;
}

int lbm_batch_remove(void* h, int slot) {
  Batch* b = static_cast<Batch*>(h);
  if (slot < 0 || slot >= b->maxSlots || !b->slots[slot].active) return -1;
  BCK(cudaStreamSynchronize(b->stream));
  DomainSlot& d = b->slots[slot];
  cudaFree(d.pdfs);
  cudaFree(d.runs);
  cudaFree(d.runOff);
  b->used -= d.bytes;
  d = DomainSlot();
  return publish(b);
}

// PDFs of a slot back to rest, f = w (stream-ordered).
int lbm_batch_reset(void* h, int slot) {
  Batch* b = static_cast<Batch*>(h);
  DomainSlot& d = b->slots[slot];
  const size_t nc = (size_t)d.dev.nCells;
  // both storage formats hold deviations from w: rest is all zero bits
  BCK(cudaMemsetAsync(d.pdfs, 0, nc * Q * b->elemBytes, b->stream));
  return 0;
}

// Enqueues nsteps time steps (rounded up to even) of every active domain.
// With use_graph, sequences are captured once per length into a CUDA graph
// and replayed (the kernels read the tables from device memory, so the graph
// stays valid when domains come and go).
int lbm_batch_step(void* h, int nsteps, int use_graph) {
  Batch* b = static_cast<Batch*>(h);
  nsteps += nsteps & 1;
  if (nsteps <= 0) return 0;
  if (!use_graph) return enqueue(b, nsteps);
  auto it = b->graphs.find(nsteps);
  if (it == b->graphs.end()) {
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = b->launches;
    enqueue(b, nsteps);
    b->launches = before;
    BCK(cudaStreamEndCapture(b->stream, &g));
    cudaGraphExec_t ge;
    BCK(cudaGraphInstantiate(&ge, g, 0));
    cudaGraphDestroy(g);
    it = b->graphs.emplace(nsteps, ge).first;
  }
  BCK(cudaGraphLaunch(it->second, b->stream));
  b->launches += nsteps;
  return 0;
}

int lbm_batch_sync(void* h) {
  Batch* b = static_cast<Batch*>(h);
  BCK(cudaStreamSynchronize(b->stream));
  int err = 0;
  BCK(cudaMemcpy(&err, b->dErr, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    g_batchError = "a device wait exceeded its limit";
    return -7;
  }
  return 0;
}

// FP64 sums {rho, jx, jy, jz} of every slot into out (maxDomains x 4,
// inactive slots 0). Synchronises.
int lbm_batch_moments(void* h, double* out) {
  Batch* b = static_cast<Batch*>(h);
  const lbm::BatchArgs a = args_of(b, b->evenL);
  BCK(cudaMemsetAsync(b->dMoments, 0, sizeof(double) * 4 * b->maxSlots, b->stream));
  if (b->nTiles > 0)
    lbm::batch_moments(a, b->nTiles, b->dPartials, b->dDomTileStart, b->dDomTileCount, b->maxSlots, b->dMoments,
                       b->stream);
  BCK(cudaGetLastError());
  BCK(cudaMemcpyAsync(out, b->dMoments, sizeof(double) * 4 * b->maxSlots, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return 0;
}

// Logical PDFs of a slot (cells x fastest, 19 per cell, obstacles untouched)
// after the last completed even/odd pair.
int lbm_batch_get_field(void* h, int slot, double* out) {
  Batch* b = static_cast<Batch*>(h);
  DomainSlot& d = b->slots[slot];
  if (!d.active) return -1;
  const size_t nc = (size_t)d.dev.nCells;
  std::vector<unsigned char> raw(nc * Q * b->elemBytes);
  BCK(cudaMemcpyAsync(raw.data(), d.pdfs, raw.size(), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  const long ncell = (long)d.dims[0] * d.dims[1] * d.dims[2];
  for (long c = 0; c < ncell; ++c) {
    const uint32_t n = d.grid[c];
    if (n == 0xffffffffu) continue;
    for (int q = 0; q < Q; ++q) {
      const size_t k = (size_t)q * nc + n;
      double v;
      if (b->storage == lbm::kStoreF32)
        v = weight_of(q) + (double)reinterpret_cast<const float*>(raw.data())[k];
      else
        v = weight_of(q) + (double)lbmh_f16_to_f32(reinterpret_cast<const uint16_t*>(raw.data())[k]) / f16_scale_of(q);
      out[c * Q + q] = v;
    }
  }
  return 0;
}

int lbm_batch_set_field(void* h, int slot, const double* in) {
  Batch* b = static_cast<Batch*>(h);
  DomainSlot& d = b->slots[slot];
  if (!d.active) return -1;
  const size_t nc = (size_t)d.dev.nCells;
  std::vector<unsigned char> raw(nc * Q * b->elemBytes);
  BCK(cudaMemcpyAsync(raw.data(), d.pdfs, raw.size(), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  const long ncell = (long)d.dims[0] * d.dims[1] * d.dims[2];
  for (long c = 0; c < ncell; ++c) {
    const uint32_t n = d.grid[c];
    if (n == 0xffffffffu) continue;
    for (int q = 0; q < Q; ++q) {
      const size_t k = (size_t)q * nc + n;
      if (b->storage == lbm::kStoreF32)
        reinterpret_cast<float*>(raw.data())[k] = (float)(in[c * Q + q] - weight_of(q));
      else
        reinterpret_cast<uint16_t*>(raw.data())[k] =
            lbmh_f32_to_f16((float)((in[c * Q + q] - weight_of(q)) * f16_scale_of(q)));
    }
  }
  BCK(cudaMemcpyAsync(d.pdfs, raw.data(), raw.size(), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return 0;
}

int lbm_batch_set_launch(void* h, int which, int threads, int blocks) {
  Batch* b = static_cast<Batch*>(h);
  if (threads != 64 && threads != 128 && threads != 256) return -1;
  if (blocks < 0) return -1;
  lbm::BatchLaunch l{threads, lbm::kBatchTileNodes / threads, blocks};
  if (which == 0 || which == 2) b->evenL = l;
  if (which == 1 || which == 2) b->oddL = l;
  drop_graphs(b);
  return 0;
}

void lbm_batch_get_launch(void* h, int* out6) {
  Batch* b = static_cast<Batch*>(h);
  out6[0] = b->evenL.threads;
  out6[1] = b->evenL.nodesPerThread;
  out6[2] = b->evenL.blocks;
  out6[3] = b->oddL.threads;
  out6[4] = b->oddL.nodesPerThread;
  out6[5] = b->oddL.blocks;
}

// Device time (ms) of nsteps steps of the active domains (CUDA events on the
// batch stream, direct launches).
int lbm_batch_time_steps(void* h, int nsteps, double* ms) {
  Batch* b = static_cast<Batch*>(h);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  BCK(cudaStreamSynchronize(b->stream));
  cudaEventRecord(e0, b->stream);
  int rc = enqueue(b, nsteps);
  cudaEventRecord(e1, b->stream);
  cudaEventSynchronize(e1);
  float f = 0.f;
  cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = f;
  return rc;
}

// Autotuner: times each (block size, nodes per thread, grid) candidate --
// grids of 2..6 persistent blocks per SM, or one block per tile -- on the current batch for `trialSteps` steps, separately for the
// even and the odd kernel (each candidate runs whole even/odd pairs with the
// other kernel on its current setting), and keeps the fastest. Advances the
// domains by the trial steps. results (optional): rows of
// {which, threads, nodesPerThread, blocks, ms} for every candidate; returns the
// number of rows written (at most maxRows).
int lbm_batch_tune(void* h, int trialSteps, double* results, int maxRows) {
  Batch* b = static_cast<Batch*>(h);
  const int threadsC[3] = {256, 128, 64};
  const int perSM[6] = {0, 2, 3, 4, 5, 6};  // 0: one block per tile
  int rows = 0;
  for (int which = 0; which < 2; ++which) {
    double bestMs = 1e300;
    lbm::BatchLaunch best = which == 0 ? b->evenL : b->oddL;
    for (int ti = 0; ti < 3; ++ti)
      for (int pi = 0; pi < 6; ++pi) {
        lbm::BatchLaunch l{threadsC[ti], lbm::kBatchTileNodes / threadsC[ti], perSM[pi] * b->numSMs};
        if (which == 0) b->evenL = l; else b->oddL = l;
        double ms = 0.0;
        if (lbm_batch_time_steps(h, 2, &ms) != 0) continue;  // warm
        if (lbm_batch_time_steps(h, trialSteps, &ms) != 0) continue;
        if (results && rows < maxRows) {
          double* r = results + 5 * rows;
          r[0] = which; r[1] = l.threads; r[2] = l.nodesPerThread; r[3] = l.blocks; r[4] = ms;
        }
        ++rows;
        if (ms < bestMs) { bestMs = ms; best = l; }
      }
    if (which == 0) b->evenL = best; else b->oddL = best;
  }
  drop_graphs(b);
  return std::min(rows, maxRows);
}

int lbm_batch_checkpoint_save(void* h, int slot, const char* path) {
  Batch* b = static_cast<Batch*>(h);
  if (slot < 0 || slot >= b->maxSlots || !b->slots[slot].active) return -1;
  DomainSlot& d = b->slots[slot];
  std::vector<unsigned char> raw((size_t)d.dev.nCells * Q * b->elemBytes);
  BCK(cudaMemcpyAsync(raw.data(), d.pdfs, raw.size(), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  DomCkpt c = dom_header_of(b, d);
  c.checksum = dom_fnv1a64(raw.data(), raw.size());
  FILE* fh = std::fopen(path, "wb");
  if (!fh) { g_batchError = "cannot open the checkpoint file"; return -1; }
  const bool ok = std::fwrite(&c, sizeof(c), 1, fh) == 1 && std::fwrite(raw.data(), 1, raw.size(), fh) == raw.size();
  if (std::fclose(fh) != 0 || !ok) { g_batchError = "writing the checkpoint file failed"; return -1; }
  return 0;
}

int lbm_batch_checkpoint_load(void* h, int slot, const char* path) {
  Batch* b = static_cast<Batch*>(h);
  if (slot < 0 || slot >= b->maxSlots || !b->slots[slot].active) return -1;
  DomainSlot& d = b->slots[slot];
  FILE* fh = std::fopen(path, "rb");
  if (!fh) { g_batchError = "cannot open the checkpoint file"; return -1; }
  DomCkpt c;
  const DomCkpt want = dom_header_of(b, d);
  if (std::fread(&c, sizeof(c), 1, fh) != 1 || std::memcmp(c.magic, kDomMagic, 8) != 0) {
    std::fclose(fh);
    g_batchError = "not a domain checkpoint";
    return -2;
  }
  bool same = c.storage == want.storage && c.nFluid == want.nFluid && c.nCells == want.nCells &&
              c.omega == want.omega && c.lambda == want.lambda && c.xforce == want.xforce;
  for (int i = 0; i < 3; ++i) same = same && c.dims[i] == want.dims[i];
  if (!same) {
    std::fclose(fh);
    g_batchError = "the checkpoint belongs to a domain of another lattice, storage or relaxation";
    return -2;
  }
  std::vector<unsigned char> raw((size_t)d.dev.nCells * Q * b->elemBytes);
  const bool ok = std::fread(raw.data(), 1, raw.size(), fh) == raw.size();
  std::fclose(fh);
  if (!ok) { g_batchError = "the checkpoint file is truncated"; return -1; }
  if (dom_fnv1a64(raw.data(), raw.size()) != c.checksum) { g_batchError = "checkpoint checksum mismatch"; return -3; }
  BCK(cudaMemcpyAsync(d.pdfs, raw.data(), raw.size(), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return 0;
}

size_t lbm_batch_bytes_used(void* h) { return static_cast<Batch*>(h)->used; }
long long lbm_batch_launches(void* h) { return static_cast<Batch*>(h)->launches; }
int lbm_batch_active_domains(void* h) {
  Batch* b = static_cast<Batch*>(h);
  int n = 0;
  for (auto& s : b->slots) n += s.active ? 1 : 0;
  return n;
}
int lbm_batch_fluid_nodes(void* h, int slot) {
  Batch* b = static_cast<Batch*>(h);
  return (slot >= 0 && slot < b->maxSlots && b->slots[slot].active) ? b->slots[slot].dev.nFluid : -1;
}

}  // extern "C"
