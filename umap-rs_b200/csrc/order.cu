// Locality order of the vertices for DRAM-bound SGD layouts.
//
// When the embedding is far larger than L2, every random row access of the SGD epoch is a
// DRAM access.  A kNN graph links points that are close in the input space, but vertex ids
// usually carry no locality, so an edge's tail row lies anywhere in the embedding.  Renaming
// the vertices so that graph neighbours get nearby ids makes the tail reads and tail moves of
// the edges in flight fall into a window of the embedding that L2 holds.  The order is a
// multi-source breadth-first search of the kept-edge graph: one source per REGION vertices
// (evenly spaced ids), each vertex joins the region that reaches it first, and vertices are
// numbered by (region, BFS level, old id).  Vertices no source reaches (other components)
// come last in id order.  Negative samples stay uniform over all vertices, so renaming
// changes no distribution the reference's epoch draws from (optimize_layout_euclidean.rs:314).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "ub_internal.hpp"

namespace ub {
namespace {

constexpr uint32_t UNSEEN = 0xFFFFFFFFu;
// Vertices per BFS source.  30 epochs of a renamed 20M-point roll (tasks by length inside
// blocks of 4,096 rows): 4,096: 238.0 ms, 16,384: 236.9-237.1, 65,536: 237.5, 262,144: 238.0;
// UMAP_B200_BFS_REGION overrides it for such measurements.
constexpr uint64_t REGION = 16384;

__global__ void seed_kernel(uint64_t n, uint32_t n_seeds, uint32_t* __restrict__ label, uint32_t* __restrict__ queue) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_seeds) return;
  const uint32_t v = (uint32_t)((uint64_t)s * n / n_seeds);  // strictly increasing in s (n >= n_seeds)
  label[v] = s;
  queue[s] = v;
}

// One warp per frontier vertex: its lanes walk the row 32 edges at a time, claim unseen
// tails for the vertex's region (compare-and-swap, so each vertex joins exactly one region
// and one frontier), and append the claimed ones to the next frontier with one counter
// update per warp and step.
__global__ void expand_kernel(const uint64_t* __restrict__ kptr, const uint32_t* __restrict__ ktail,
                              const uint32_t* __restrict__ frontier, uint64_t count, uint32_t next_level,
                              uint32_t* label, uint32_t* __restrict__ level, uint32_t* __restrict__ next,
                              unsigned long long* __restrict__ next_count) {
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (w >= count) return;  // warp-uniform
  const uint32_t v = frontier[w];
  const uint32_t lab = label[v];
  const uint64_t b = kptr[v], e = kptr[v + 1];
  for (uint64_t j0 = b; j0 < e; j0 += 32) {
    const uint64_t j = j0 + lane;
    bool push = false;
    uint32_t t = 0;
    if (j < e) {
      t = ktail[j];
      push = label[t] == UNSEEN && atomicCAS(&label[t], UNSEEN, lab) == UNSEEN;
    }
    const unsigned m = __ballot_sync(0xFFFFFFFFu, push);
    if (m) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(next_count, (unsigned long long)__popc(m));
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (push) {
        level[t] = next_level;
        next[base + __popc(m & ((1u << lane) - 1u))] = t;
      }
    }
  }
}

__global__ void unreached_kernel(uint64_t n, uint32_t region, uint32_t* __restrict__ label) {
  const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n && label[v] == UNSEEN) label[v] = region;
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, uint64_t n,
                                  uint32_t* __restrict__ dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

__global__ void invert_kernel(const uint32_t* __restrict__ order, uint64_t n, uint32_t* __restrict__ rank) {
  const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) rank[order[u]] = (uint32_t)u;
}

// dst row u = src row order[u] (to_new) or dst row order[u] = src row u (from new).
__global__ void permute_rows_kernel(const float* __restrict__ src, const uint32_t* __restrict__ order, uint64_t n,
                                    uint32_t dim, bool to_new, float* __restrict__ dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * dim) return;
  const uint64_t u = i / dim;
  const uint32_t d = (uint32_t)(i - u * dim);
  const uint64_t v = order[u];
  if (to_new) dst[i] = src[v * dim + d];
  else dst[v * dim + d] = src[i];
}

inline unsigned grid_for(uint64_t n, unsigned bt) { return (unsigned)((n + bt - 1) / bt); }

}  // namespace

void locality_order(const uint64_t* kptr, const uint32_t* ktail, uint64_t n, uint32_t* order, uint32_t* rank,
                    cudaStream_t s) {
  if (n == 0) return;
  if (n >= 0xFFFFFFFFull) throw Error(UNSUPPORTED, "locality order: n must be < 2^32");
  uint64_t region = REGION;
  if (const char* e = getenv("UMAP_B200_BFS_REGION")) {
    const long v = atol(e);
    if (v >= 64 && v <= (1l << 30)) region = (uint64_t)v;
  }
  const uint32_t n_seeds = (uint32_t)std::max<uint64_t>(1, n / region);
  DevBuf<uint32_t> label(n, s), level(n, s), qa(n, s), qb(n, s);
  DevBuf<unsigned long long> cnt(1, s);
  UB_CUDA(cudaMemsetAsync(label.p, 0xFF, n * 4, s));
  UB_CUDA(cudaMemsetAsync(level.p, 0, n * 4, s));
  seed_kernel<<<grid_for(n_seeds, 256), 256, 0, s>>>(n, n_seeds, label.p, qa.p);
  UB_LAUNCH_CHECK();
  uint64_t count = n_seeds;
  uint32_t lev = 0;
  uint32_t* cur = qa.p;
  uint32_t* nxt = qb.p;
  while (count > 0) {
    if (lev == 0xFFFFFFFEu) throw Error(UNSUPPORTED, "locality order: too many BFS levels");
    UB_CUDA(cudaMemsetAsync(cnt.p, 0, 8, s));
    const uint64_t threads = count * 32;
    expand_kernel<<<grid_for(threads, 256), 256, 0, s>>>(kptr, ktail, cur, count, lev + 1, label.p, level.p, nxt,
                                                         cnt.p);
    UB_LAUNCH_CHECK();
    unsigned long long c = 0;
    UB_CUDA(cudaMemcpyAsync(&c, cnt.p, 8, cudaMemcpyDeviceToHost, s));
    UB_CUDA(cudaStreamSynchronize(s));
    count = c;
    ++lev;
    std::swap(cur, nxt);
  }
  unreached_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, n_seeds, label.p);
  UB_LAUNCH_CHECK();
  // (region, level, id): stable sort by level, then stable by region.
  DevBuf<uint32_t> k1(n, s), v1(n, s);
  radix_sort_pairs(level.p, nullptr, k1.p, v1.p, n, bits_for(lev), s);
  gather_u32_kernel<<<grid_for(n, 256), 256, 0, s>>>(label.p, v1.p, n, k1.p);
  UB_LAUNCH_CHECK();
  radix_sort_pairs(k1.p, v1.p, level.p, order, n, bits_for(n_seeds), s);
  invert_kernel<<<grid_for(n, 256), 256, 0, s>>>(order, n, rank);
  UB_LAUNCH_CHECK();
}

void permute_rows(const float* src, const uint32_t* order, uint64_t n, uint32_t dim, bool to_new, float* dst,
                  cudaStream_t s) {
  if (n == 0 || dim == 0) return;
  permute_rows_kernel<<<grid_for(n * dim, 256), 256, 0, s>>>(src, order, n, dim, to_new, dst);
  UB_LAUNCH_CHECK();
}

}  // namespace ub
