// lbm_moments_noalloc.cu -- the FP64 conservation sums of lbm_moments.cu for
// callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code running while
// another component owns the device allocator (a memory pool that must not be
// fragmented, or an allocator that is not reentrant from this call site), and
// code that only receives device buffers from its host application and is not
// allowed to grow the process's device footprint behind its back. For them,
// lbm_b200_moments_noalloc keeps the reduction's scratch in a fixed array that
// is part of the library image instead of allocating it per call.
//
// The scratch (4 partial sums per block of 256 nodes) is the file-scope
// __device__ array below: 65,536 blocks x 4 doubles = 2 MiB, so at most
// 16,777,216 fluid nodes per call. Every GPU that loads the library holds this
// array until the process exits. Every call shares it and it keeps the last
// call's contents; each block overwrites all four of its partials before the
// final pass reads them, so nothing has to start at zero. Two calls whose work
// overlaps on the GPU (different streams, or different host threads on one
// device) race on the array.
//
// In host code `g_moment_scratch` names a host-side shadow, not device memory;
// a kernel given that name would fault or read the wrong memory. The device
// address is obtained with cudaGetSymbolAddress, once per device, with that
// device current, on the first call of the entry point on that device, and
// kept for the life of the process: the cache assumes the device's context is
// not reset (cudaDeviceReset) while the process uses this entry point.
#include <cstdio>
#include <mutex>

#include "lbm_kernels.cuh"

namespace lbm {

constexpr int kNoAllocMaxBlocks = 65536;
constexpr long long kNoAllocMaxNodes = static_cast<long long>(kNoAllocMaxBlocks) * kListTile;
static __device__ __align__(256) double g_moment_scratch[kNoAllocMaxBlocks * 4];

}  // namespace lbm

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratchLock;
double* g_scratchAddr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up on
// the first call per device). Returns a CUDA error code.
int scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) {
    std::fprintf(stderr, "lbm_b200_moments_noalloc: device ordinal %d out of range\n", dev);
    return -3;
  }
  std::lock_guard<std::mutex> lock(g_scratchLock);
  if (g_scratchAddr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, lbm::g_moment_scratch);
    if (e != cudaSuccess) {
      std::fprintf(stderr, "lbm_b200_moments_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return (int)e;
    }
    g_scratchAddr[dev] = static_cast<double*>(p);
  }
  *out = g_scratchAddr[dev];
  return 0;
}

}  // namespace

extern "C" {

// Declared in include/lbm_b200.h.
int lbm_b200_moments_noalloc(const double* pdfs, long long nCells, int nFluid, double* out_device, void* stream) {
  if (pdfs == nullptr || out_device == nullptr || nFluid < 0 || nCells < nFluid) {
    std::fprintf(stderr, "lbm_b200_moments_noalloc: invalid arguments\n");
    return -1;
  }
  if (nFluid > lbm::kNoAllocMaxNodes) {
    std::fprintf(stderr,
                 "lbm_b200_moments_noalloc: %d fluid nodes exceed the fixed scratch of this entry point "
                 "(at most %lld nodes); use lbm_b200_moments_device instead\n",
                 nFluid, lbm::kNoAllocMaxNodes);
    return -2;
  }
  // an error left by earlier, unrelated work is reported as such, not as
  // this call's: the call refuses to enqueue behind it
  cudaError_t before = cudaPeekAtLastError();
  if (before != cudaSuccess) {
    std::fprintf(stderr, "lbm_b200_moments_noalloc: an earlier CUDA error is pending (%s); nothing enqueued\n",
                 cudaGetErrorString(before));
    return (int)before;
  }
  double* scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc != 0) return rc;
  lbm::moments_enqueue(pdfs, nCells, nFluid, scratch, out_device, static_cast<cudaStream_t>(stream));
  return (int)cudaGetLastError();
}

}  // extern "C"
