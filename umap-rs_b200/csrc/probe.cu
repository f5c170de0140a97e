// Peak rates of the SGD epoch's memory access pattern, for its L2 roofline: random 8-byte
// row reads (tail rows, negative samples) and random 8-byte red.add row moves (tail moves)
// on a table the caller sizes like the epoch's snapshot embedding.  Each thread issues
// independent accesses, eight at a time, at rows drawn by a SplitMix64 finaliser of its
// access counter, so the rate measured is the memory system's for this pattern, not a
// latency chain.
#include <cuda_runtime.h>

#include <cstdint>

#include "ub_internal.hpp"

namespace ub {
namespace {

__device__ __forceinline__ uint64_t probe_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// mode 0: reads (summed into out[thread] so that they are not dropped); mode 1: red.add of a
// small value to each row.
__global__ void __launch_bounds__(256) random_rows_probe_kernel(float2* table, uint32_t n_rows, uint32_t per_thread,
                                                               int mode, float* __restrict__ out) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float acc = 0.0f;
  for (uint32_t i = 0; i < per_thread; i += 8) {
    uint32_t row[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint64_t h = probe_mix(tid * 0x9E3779B97F4A7C15ull + (uint64_t)(i + u));
      row[u] = __umulhi((uint32_t)h, n_rows);
    }
    if (mode == 0) {
      float2 v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = table[row[u]];
#pragma unroll
      for (int u = 0; u < 8; ++u) acc += v[u].x + v[u].y;
    } else {
#pragma unroll
      for (int u = 0; u < 8; ++u) atomicAdd(table + row[u], make_float2(1e-7f, -1e-7f));
    }
  }
  if (mode == 0) out[tid] = acc;
}

}  // namespace

float random_rows_probe(float* table, uint64_t n_rows, uint64_t accesses, int mode, float* out, uint64_t* done,
                        cudaStream_t s) {
  if (n_rows == 0 || n_rows >= 0xFFFFFFFFull) throw Error(INVALID_ARGUMENT, "probe table rows must be 1..2^32-1");
  const unsigned blocks = 148 * 8, threads = 256;
  const uint64_t total = (uint64_t)blocks * threads;
  uint64_t per = (accesses + total - 1) / total;
  per = (per + 7) / 8 * 8;
  if (per > 0xFFFFFFFFull) throw Error(INVALID_ARGUMENT, "too many probe accesses");
  *done = per * total;
  cudaEvent_t e0, e1;
  UB_CUDA(cudaEventCreate(&e0));
  UB_CUDA(cudaEventCreate(&e1));
  // one untimed launch warms L2 with the table, then the timed one
  for (int it = 0; it < 2; ++it) {
    if (it == 1) UB_CUDA(cudaEventRecord(e0, s));
    random_rows_probe_kernel<<<blocks, threads, 0, s>>>(reinterpret_cast<float2*>(table), (uint32_t)n_rows,
                                                        (uint32_t)per, mode, out);
    UB_LAUNCH_CHECK();
  }
  UB_CUDA(cudaEventRecord(e1, s));
  UB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.0f;
  UB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  (void)cudaEventDestroy(e0);
  (void)cudaEventDestroy(e1);
  return ms;
}

}  // namespace ub
