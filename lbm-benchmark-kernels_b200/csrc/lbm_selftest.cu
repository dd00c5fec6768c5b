// lbm_selftest.cu -- exercises the bounded-wait error path of the library's
// device waits without faulting or hanging the GPU: a kernel waits on a flag
// that nothing sets, gives up after a fixed number of polls, records the
// failure in the error word and returns; the host reads the word back and the
// context stays usable.
#include <cuda_runtime.h>

namespace {

__global__ void k_wait_unset_flag(const volatile int* flag, int* err, unsigned polls) {
  for (unsigned i = 0; i < polls; ++i)
    if (*flag) return;
  if (threadIdx.x == 0) atomicOr(err, 2);
}

}  // namespace

extern "C" {

// Declared in include/lbm_b200.h.
int lbm_b200_selftest_bounded_wait(unsigned polls, int* status) {
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 2 * sizeof(int));
  if (e != cudaSuccess) return (int)e;
  e = cudaMemset(d, 0, 2 * sizeof(int));
  if (e == cudaSuccess) {
    k_wait_unset_flag<<<1, 32>>>(d, d + 1, polls);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(status, d + 1, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

}  // extern "C"
