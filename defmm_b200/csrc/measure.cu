// Measurement helper: the L2-to-SM read bandwidth that bounds the L2-bound
// kernels of the matvec (M2L streams every far pair's source and transfer
// spectra from L2).  No counterpart in the reference.
#include <cstdint>

#include "../../include/defmm_b200.h"

namespace {

// Every thread streams 16-byte words of a buffer small enough to stay in L2
// (loads cached in L2 only, not in L1), `reps` times; the folded words go to
// `sink` only in a case that cannot happen, so the loads are kept.
__global__ void __launch_bounds__(256) k_l2_read(const uint4* __restrict__ buf, int64_t n16, int reps,
                                                 unsigned* __restrict__ sink) {
  unsigned acc = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int r = 0; r < reps; r++)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride) {
      const uint4 v = __ldcg(buf + i);
      acc += v.x ^ v.y ^ v.z ^ v.w;
    }
  if (acc == 0x9e3779b9u) *sink = acc;
}

}  // namespace

extern "C" int defmm_probe_l2_read(int64_t bytes, int reps, double* gbs) {
  if (!gbs || bytes < (1 << 20) || bytes > ((int64_t)96 << 20) || reps < 1 || reps > 10000) return DEFMM_ERR_ARG;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return DEFMM_ERR_CUDA;
  }
  void* buf = nullptr;
  unsigned* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int st = DEFMM_OK;
  const int64_t n16 = bytes / 16;
  float ms = 0.f;
  if (cudaMalloc(&buf, (size_t)n16 * 16) != cudaSuccess || cudaMalloc(&sink, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(buf, 1, (size_t)n16 * 16) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    st = DEFMM_ERR_MEMORY;
  } else {
    const int grid = nsm * 8;
    k_l2_read<<<grid, 256>>>((const uint4*)buf, n16, 2, sink);  // warm the L2
    cudaEventRecord(e0);
    k_l2_read<<<grid, 256>>>((const uint4*)buf, n16, reps, sink);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.f)
      st = DEFMM_ERR_CUDA;
    else
      *gbs = (double)n16 * 16.0 * reps / (ms * 1e-3) / 1e9;
  }
  cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  if (buf) cudaFree(buf);
  return st;
}
