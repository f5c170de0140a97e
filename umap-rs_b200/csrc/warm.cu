// Row helpers of the learned warm start (api.cpp: warm_start_impl): the network reads rows
// of a multiple of 64 features, trains on a subsample of them, and skips the subsample's
// rows that the plain fit returned as NaN (vertices with an empty graph row).
#include <cuda_runtime.h>

#include <cstdint>

#include "ub_internal.hpp"

namespace ub {
namespace {

// out[i][j] = x[row(i)][j] for j < d, 0 for d <= j < dp; row(i) = rows[i] or i.
__global__ void pad_gather_rows_kernel(const float* __restrict__ x, uint64_t d, uint64_t dp,
                                       const uint32_t* __restrict__ rows, uint64_t count, float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count * dp) return;
  const uint64_t r = i / dp, j = i - r * dp;
  const uint64_t src = rows ? rows[r] : r;
  out[i] = j < d ? x[src * d + j] : 0.0f;
}

__global__ void finite_rows_kernel(const float* __restrict__ y, uint64_t n, uint32_t dim, uint32_t* __restrict__ keep) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  uint32_t ok = 1;
  for (uint32_t d = 0; d < dim; ++d) ok &= isfinite(y[r * dim + d]) ? 1u : 0u;
  keep[r] = ok;
}

__global__ void compact_rows_kernel(const float* __restrict__ src, uint64_t n, uint64_t width,
                                    const uint32_t* __restrict__ keep, const uint64_t* __restrict__ pos,
                                    float* __restrict__ dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  const uint64_t r = i / width;
  if (keep[r]) dst[pos[r] * width + (i - r * width)] = src[i];
}

inline unsigned grid_for(uint64_t n, unsigned bt) { return (unsigned)((n + bt - 1) / bt); }

}  // namespace

void pad_gather_rows(const float* x, uint64_t d, uint64_t dp, const uint32_t* rows, uint64_t count, float* out,
                     cudaStream_t s) {
  if (count == 0 || dp == 0) return;
  pad_gather_rows_kernel<<<grid_for(count * dp, 256), 256, 0, s>>>(x, d, dp, rows, count, out);
  UB_LAUNCH_CHECK();
}

void finite_rows(const float* y, uint64_t n, uint32_t dim, uint32_t* keep, cudaStream_t s) {
  if (n == 0) return;
  finite_rows_kernel<<<grid_for(n, 256), 256, 0, s>>>(y, n, dim, keep);
  UB_LAUNCH_CHECK();
}

void compact_rows(const float* src, uint64_t n, uint64_t width, const uint32_t* keep, const uint64_t* pos,
                  float* dst, cudaStream_t s) {
  if (n == 0 || width == 0) return;
  compact_rows_kernel<<<grid_for(n * width, 256), 256, 0, s>>>(src, n, width, keep, pos, dst);
  UB_LAUNCH_CHECK();
}

}  // namespace ub
