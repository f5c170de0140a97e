// Graph build kernels: smooth-kNN rho/sigma (K1), directed membership rows (K2), the
// transpose bookkeeping around the radix sort, and the per-row fuzzy-union merge-join (K4).
//
// Bit-exactness: every f32 operation that decides rho, sigma, a membership weight or a
// union weight is written with an explicit round-to-nearest intrinsic (__fadd_rn etc.), so
// it rounds exactly like the Rust source (which never contracts into an FMA).  exp is
// evaluated in double by CUDA's exp() and rounded once to f32.
#include <cuda_runtime.h>

#include <cstdint>

#include "ub_internal.hpp"

namespace ub {
namespace {

constexpr float SMOOTH_K_TOLERANCE = 1e-5f;  // umap/constants.rs:4
constexpr float MIN_K_DIST_SCALE = 1e-3f;    // umap/constants.rs:7
constexpr int BT = 128;

__device__ __forceinline__ float exp_f32(float x) { return (float)exp((double)x); }

// ndarray 0.17 mean of a contiguous f32 slice: unrolled 8-way fold, then / len as f32.
__device__ float nd_mean(const float* xs, uint64_t n, uint64_t stride_elems) {
  float p[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  uint64_t i = 0;
  for (; i + 8 <= n; i += 8)
#pragma unroll
    for (int j = 0; j < 8; ++j) p[j] = __fadd_rn(p[j], xs[(i + j) * stride_elems]);
  float acc = 0.0f;
  acc = __fadd_rn(acc, __fadd_rn(p[0], p[4]));
  acc = __fadd_rn(acc, __fadd_rn(p[1], p[5]));
  acc = __fadd_rn(acc, __fadd_rn(p[2], p[6]));
  acc = __fadd_rn(acc, __fadd_rn(p[3], p[7]));
  for (uint64_t t = 0; i + t < n && t < 7; ++t) acc = __fadd_rn(acc, xs[(i + t) * stride_elems]);
  return __fdiv_rn(acc, __ull2float_rn(n));
}

// Cooperative, coalesced staging of `rows` consecutive k-wide rows into shared memory with
// an odd row stride (conflict-free column access).
template <class T>
__device__ __forceinline__ void stage_rows(T* s, const T* __restrict__ g, uint64_t row0,
                                           uint32_t rows, uint32_t k, uint32_t stride) {
  const T* src = g + row0 * k;
  const uint32_t total = rows * k;
  for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
    uint32_t r = t / k, j = t - r * k;
    s[r * stride + j] = src[t];
  }
}

// ------------------------------------------------------------------------------ K1
// smooth_knn_dist.rs:78-186 for one row per thread.
template <bool SMEM>
__global__ void __launch_bounds__(BT) smooth_knn_kernel(const float* __restrict__ dist, uint64_t n,
                                                        uint32_t k, GraphParams gp,
                                                        float* __restrict__ sigmas,
                                                        float* __restrict__ rhos,
                                                        unsigned* __restrict__ need_global) {
  extern __shared__ float s_rows[];
  const uint32_t stride = k | 1u;
  const uint64_t row0 = (uint64_t)blockIdx.x * BT;
  const uint32_t rows = (uint32_t)min((uint64_t)BT, n - row0);
  if (SMEM) {
    stage_rows(s_rows, dist, row0, rows, k, stride);
    __syncthreads();
  }
  if (threadIdx.x >= rows) return;
  const uint64_t i = row0 + threadIdx.x;
  const float* row = SMEM ? s_rows + threadIdx.x * stride : dist + i * k;

  // :88-97
  uint64_t non_zero_count = 0;
  float max_non_zero = 0.0f;
  for (uint32_t j = 0; j < k; ++j) {
    float d = row[j];
    if (d > 0.0f) {
      ++non_zero_count;
      if (d > max_non_zero) max_non_zero = d;
    }
  }
  // :101-142
  float rho = 0.0f;
  if (non_zero_count >= gp.lc_usize) {
    const uint64_t index = gp.lc_index;
    float nth_minus_1 = 0.0f, nth = 0.0f;
    uint64_t count = 0;
    for (uint32_t j = 0; j < k; ++j) {
      float d = row[j];
      if (d > 0.0f) {
        if (count + 1 == index) nth_minus_1 = d;
        if (count + 1 == index + 1) nth = d;
        ++count;
        if (count > index + 1) break;
      }
    }
    if (index > 0) {
      rho = nth_minus_1;
      if (gp.interpolation > SMOOTH_K_TOLERANCE)
        rho = __fadd_rn(rho, __fmul_rn(gp.interpolation, __fsub_rn(nth, nth_minus_1)));
    } else {
      float first = 0.0f;
      for (uint32_t j = 0; j < k; ++j)
        if (row[j] > 0.0f) { first = row[j]; break; }
      rho = __fmul_rn(gp.interpolation, first);
    }
  } else if (non_zero_count > 0) {
    rho = max_non_zero;
  }
  // :145-171 bisection
  float lo = 0.0f, hi = INFINITY, mid = 1.0f;
  for (int it = 0; it < gp.n_iter; ++it) {
    float psum = 0.0f;
    for (uint32_t j = 1; j < k; ++j) {
      float d = __fsub_rn(row[j], rho);
      if (d > 0.0f) psum = __fadd_rn(psum, exp_f32(-__fdiv_rn(d, mid)));
      else psum = __fadd_rn(psum, 1.0f);
    }
    if (fabsf(__fsub_rn(psum, gp.target)) < SMOOTH_K_TOLERANCE) break;
    if (psum > gp.target) {
      hi = mid;
      mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
    } else {
      lo = mid;
      if (hi == INFINITY) mid = __fmul_rn(mid, 2.0f);
      else mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
    }
  }
  float sigma = mid;
  // :176-183.  Rows with rho <= 0 need the global mean: left unclamped and fixed up by
  // global_mean_fixup (rare: all-zero rows or local_connectivity < 1).
  if (rho > 0.0f) {
    float m = nd_mean(row, k, 1);
    float lim = __fmul_rn(MIN_K_DIST_SCALE, m);
    if (sigma < lim) sigma = lim;
  } else {
    atomicOr(need_global, 1u);
  }
  sigmas[i] = sigma;
  rhos[i] = rho;
}

// distances.mean() over a contiguous [rows, k] array (smooth_knn_dist.rs:74), in the exact
// order of ndarray's unrolled fold: 8 sequential partial sums.  One warp per segment (a
// batch instance; a plain fit is one segment), lanes 0-7 each own one partial sum; only
// runs when some row needs it.
__global__ void segment_mean_kernel(const float* __restrict__ dist, uint32_t k,
                                    const uint64_t* __restrict__ seg_off, uint64_t n,
                                    const unsigned* __restrict__ need, float* __restrict__ out) {
  if (*need == 0) return;
  const uint32_t sgm = blockIdx.x;
  const uint64_t r0 = seg_off ? seg_off[sgm] : 0, r1 = seg_off ? seg_off[sgm + 1] : n;
  const uint64_t total = (r1 - r0) * k;
  const float* x0 = dist + r0 * k;
  const int lane = threadIdx.x;
  __shared__ float s_p[8];
  const uint64_t chunks = total / 8;
  if (lane < 8) {
    float p = 0.0f;
    const float* x = x0 + lane;
    uint64_t c = 0;
    for (; c + 8 <= chunks; c += 8) {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = x[(c + u) * 8];
#pragma unroll
      for (int u = 0; u < 8; ++u) p = __fadd_rn(p, v[u]);
    }
    for (; c < chunks; ++c) p = __fadd_rn(p, x[c * 8]);
    s_p[lane] = p;
  }
  __syncwarp();
  if (lane == 0) {
    float acc = 0.0f;
    acc = __fadd_rn(acc, __fadd_rn(s_p[0], s_p[4]));
    acc = __fadd_rn(acc, __fadd_rn(s_p[1], s_p[5]));
    acc = __fadd_rn(acc, __fadd_rn(s_p[2], s_p[6]));
    acc = __fadd_rn(acc, __fadd_rn(s_p[3], s_p[7]));
    const uint64_t rem = total - chunks * 8;
    for (uint64_t t = 0; t < rem && t < 7; ++t) acc = __fadd_rn(acc, x0[chunks * 8 + t]);
    out[sgm] = total ? __fdiv_rn(acc, __ull2float_rn(total)) : 0.0f;
  }
}

__global__ void global_mean_fixup(float* __restrict__ sigmas, const float* __restrict__ rhos,
                                  uint64_t n, const unsigned* __restrict__ need,
                                  const float* __restrict__ gmean, const uint32_t* __restrict__ row_seg) {
  if (*need == 0) return;
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!(rhos[i] > 0.0f)) {
    float lim = __fmul_rn(MIN_K_DIST_SCALE, gmean[row_seg ? row_seg[i] : 0]);
    if (sigmas[i] < lim) sigmas[i] = lim;
  }
}

// Batched instances: local kNN ids (0..n_s-1 within instance s) -> global vertex ids; ids
// outside the instance become the sentinel 0xFFFFFFFF (skipped like the reference's
// `knn_idx >= n_samples`, fuzzy_simplicial_set.rs:192).
__global__ void localize_kernel(const uint32_t* __restrict__ idx, uint64_t n, uint32_t k,
                                const uint32_t* __restrict__ row_seg, const uint64_t* __restrict__ seg_off,
                                uint32_t* __restrict__ out) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n * k) return;
  const uint32_t sgm = row_seg[p / k];
  const uint64_t off = seg_off[sgm], ns = seg_off[sgm + 1] - off;
  const uint32_t v = idx[p];
  out[p] = (uint64_t)v < ns ? (uint32_t)(off + v) : 0xFFFFFFFFu;
}

__global__ void row_segment_kernel(const uint64_t* __restrict__ seg_off, uint32_t n_seg,
                                   uint32_t* __restrict__ row_seg) {
  const uint32_t sgm = blockIdx.x;
  if (sgm >= n_seg) return;
  for (uint64_t r = seg_off[sgm] + threadIdx.x; r < seg_off[sgm + 1]; r += blockDim.x) row_seg[r] = sgm;
}

// ------------------------------------------------------------------------------ K2
// fuzzy_simplicial_set.rs:182-255 + :294-306 for one row per thread: kept entries (not
// disconnected, not self, not a sentinel >= n, weight != 0) in j order, then a stable
// insertion sort by column (:264-282).  Rows are staged in shared memory; output rows are
// written back cooperatively (coalesced) into the padded [n][k] arrays.
// The reference hands each sorted row to sprs's CsMatI::new (:291), whose structure check
// wants strictly increasing column indices in a row, so a row that keeps the same neighbour
// twice makes it panic.  Such rows are reported through dup_row (the largest ~row, i.e. the
// smallest offending row, by atomicMax over ~row; 0 = none) for the host to refuse.
__global__ void __launch_bounds__(BT) membership_kernel(
    const uint32_t* __restrict__ idx, const float* __restrict__ dist, uint64_t n, uint32_t k,
    GraphParams gp, const float* __restrict__ sigmas, const float* __restrict__ rhos,
    uint32_t* __restrict__ pcol, float* __restrict__ pw, uint32_t* __restrict__ cnt,
    unsigned long long* __restrict__ edges_removed, unsigned long long* __restrict__ dup_row) {
  extern __shared__ unsigned char smem[];
  const uint32_t stride = k | 1u;
  uint32_t* s_col = (uint32_t*)smem;
  float* s_w = (float*)(s_col + BT * stride);
  const uint64_t row0 = (uint64_t)blockIdx.x * BT;
  const uint32_t rows = (uint32_t)min((uint64_t)BT, n - row0);
  // Stage inputs: s_col <- idx rows, s_w <- dist rows.
  stage_rows(s_col, idx, row0, rows, k, stride);
  stage_rows(s_w, dist, row0, rows, k, stride);
  __syncthreads();
  unsigned removed = 0;
  if (threadIdx.x < rows) {
    const uint64_t i = row0 + threadIdx.x;
    uint32_t* c = s_col + threadIdx.x * stride;
    float* w = s_w + threadIdx.x * stride;
    const float rho = rhos[i], sigma = sigmas[i];
    uint32_t o = 0;
    for (uint32_t j = 0; j < k; ++j) {
      const float d = w[j];
      const uint32_t col = c[j];
      if (d >= gp.disc_thr) { ++removed; continue; }
      if ((uint64_t)col == i || (uint64_t)col >= n) continue;
      const float t = __fsub_rn(d, rho);
      float v;
      if (t <= 0.0f || sigma == 0.0f) v = 1.0f;
      else v = exp_f32(__fdiv_rn(-t, sigma));
      if (v != 0.0f) {  // o <= j: in-place compaction is safe
        c[o] = col;
        w[o] = v;
        ++o;
      }
    }
    for (uint32_t q = 1; q < o; ++q) {  // stable insertion sort by column
      uint32_t m = q;
      while (m > 0 && c[m - 1] > c[m]) {
        uint32_t tc = c[m - 1]; c[m - 1] = c[m]; c[m] = tc;
        float tw = w[m - 1]; w[m - 1] = w[m]; w[m] = tw;
        --m;
      }
    }
    for (uint32_t q = 1; q < o; ++q)
      if (c[q - 1] == c[q]) {
        atomicMax(dup_row, (unsigned long long)~i);
        break;
      }
    for (uint32_t q = o; q < k; ++q) { c[q] = 0xFFFFFFFFu; w[q] = 0.0f; }
    cnt[i] = o;
  }
  __syncthreads();
  const uint32_t total = rows * k;
  for (uint32_t t = threadIdx.x; t < total; t += BT) {
    uint32_t r = t / k, j = t - r * k;
    pcol[row0 * k + t] = s_col[r * stride + j];
    pw[row0 * k + t] = s_w[r * stride + j];
  }
  // block-reduce the removed count
  unsigned v = removed;
  for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o2);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(edges_removed, (unsigned long long)v);
}

__global__ void compact_kernel(const uint32_t* __restrict__ pcol, const uint32_t* __restrict__ cnt,
                               const uint64_t* __restrict__ dptr, uint64_t n, uint32_t k,
                               uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n * k) return;
  const uint64_t r = p / k;
  const uint32_t e = (uint32_t)(p - r * k);
  if (e < cnt[r]) {
    const uint64_t q = dptr[r] + e;
    keys[q] = pcol[p];
    vals[q] = (uint32_t)p;
  }
}

__global__ void gather_kernel(const float* __restrict__ pw, const uint32_t* __restrict__ vals,
                              uint64_t nnz, float* __restrict__ data) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nnz) data[q] = pw[vals[q]];
}

__global__ void segment_starts_kernel(const uint32_t* __restrict__ keys, uint64_t nnz, uint64_t n,
                                      uint64_t* __restrict__ tptr) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nnz) return;
  // Column range whose first element is at position i: (prev, cur] with prev = key[i-1]
  // (or -1) and cur = key[i] (or n at i == nnz).
  const int64_t prev = i == 0 ? -1 : (int64_t)keys[i - 1];
  const int64_t cur = i == nnz ? (int64_t)n : (int64_t)keys[i];
  for (int64_t c = prev + 1; c <= cur; ++c) tptr[c] = i;
}

// ------------------------------------------------------------------------------ K4
// fuzzy_simplicial_set.rs:392-552 for one output row per thread: merge-join of the sorted
// directed row r (columns col, value A[r,col]) with the transposed row r (sources c in
// ascending order, value A[c,r]).  Emits mix*a + mix*b + (1-2mix)*a*b (:423/:488) for
// direct entries and mix*b (:506) for transpose-only entries, dropping zeros.
__global__ void __launch_bounds__(BT) union_kernel(
    const uint32_t* __restrict__ pcol, const float* __restrict__ pw, const uint32_t* __restrict__ cnt,
    uint32_t k, const uint64_t* __restrict__ tptr, const uint32_t* __restrict__ tvals, uint64_t n,
    float mix, float prod, uint32_t* __restrict__ out_cnt, const uint64_t* __restrict__ out_ptr,
    uint32_t* __restrict__ out_idx, float* __restrict__ out_w, bool fill) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const uint64_t abase = r * k;
  const uint32_t an = cnt[r];
  uint64_t j = tptr[r];
  const uint64_t jend = tptr[r + 1];
  uint32_t i = 0, count = 0;
  uint64_t o = fill ? out_ptr[r] : 0;
  uint32_t ca = i < an ? pcol[abase] : 0xFFFFFFFFu;
  uint32_t pb = 0, cb = 0xFFFFFFFFu;
  if (j < jend) { pb = tvals[j]; cb = pb / k; }
  while (ca != 0xFFFFFFFFu || cb != 0xFFFFFFFFu) {
    float v;
    uint32_t col;
    if (ca < cb) {
      const float a = pw[abase + i];
      v = __fadd_rn(__fadd_rn(__fmul_rn(mix, a), __fmul_rn(mix, 0.0f)), __fmul_rn(__fmul_rn(prod, a), 0.0f));
      col = ca;
      ++i;
      ca = i < an ? pcol[abase + i] : 0xFFFFFFFFu;
    } else if (ca == cb) {
      const float a = pw[abase + i], b = pw[pb];
      v = __fadd_rn(__fadd_rn(__fmul_rn(mix, a), __fmul_rn(mix, b)), __fmul_rn(__fmul_rn(prod, a), b));
      col = ca;
      ++i;
      ca = i < an ? pcol[abase + i] : 0xFFFFFFFFu;
      ++j;
      if (j < jend) { pb = tvals[j]; cb = pb / k; } else cb = 0xFFFFFFFFu;
    } else {
      const float b = pw[pb];
      v = __fmul_rn(mix, b);
      col = cb;
      ++j;
      if (j < jend) { pb = tvals[j]; cb = pb / k; } else cb = 0xFFFFFFFFu;
    }
    if (v != 0.0f) {
      if (fill) {
        out_idx[o] = col;
        out_w[o] = v;
        ++o;
      }
      ++count;
    }
  }
  if (!fill) out_cnt[r] = count;
}

__global__ void empty_rows_kernel(const uint64_t* __restrict__ indptr, const float* __restrict__ data,
                                  uint64_t n, unsigned long long* __restrict__ out) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned e = 0;
  if (r < n) {
    float s = -0.0f;
    for (uint64_t q = indptr[r]; q < indptr[r + 1]; ++q) s = __fadd_rn(s, data[q]);
    e = (s == 0.0f) ? 1u : 0u;
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0 && e) atomicAdd(out, (unsigned long long)e);
}

inline unsigned grid_for(uint64_t n, unsigned bt) { return (unsigned)((n + bt - 1) / bt); }

}  // namespace

void smooth_knn(const float* dist, uint64_t n, uint64_t k, const GraphParams& gp, float* sigmas,
                float* rhos, cudaStream_t s, const Segments* seg) {
  if (n == 0) return;
  const uint32_t n_seg = seg ? seg->n_seg : 1u;
  DevBuf<unsigned> need(1, s);
  DevBuf<float> gmean(n_seg, s);
  UB_CUDA(cudaMemsetAsync(need.p, 0, sizeof(unsigned), s));
  const uint32_t stride = (uint32_t)k | 1u;
  const size_t smem = (size_t)BT * stride * sizeof(float);
  const unsigned grid = grid_for(n, BT);
  if (smem <= 48 * 1024) {
    smooth_knn_kernel<true><<<grid, BT, smem, s>>>(dist, n, (uint32_t)k, gp, sigmas, rhos, need.p);
  } else {
    smooth_knn_kernel<false><<<grid, BT, 0, s>>>(dist, n, (uint32_t)k, gp, sigmas, rhos, need.p);
  }
  UB_LAUNCH_CHECK();
  segment_mean_kernel<<<n_seg, 32, 0, s>>>(dist, (uint32_t)k, seg ? seg->seg_off : nullptr, n, need.p, gmean.p);
  UB_LAUNCH_CHECK();
  global_mean_fixup<<<grid_for(n, 256), 256, 0, s>>>(sigmas, rhos, n, need.p, gmean.p,
                                                     seg ? seg->row_seg : nullptr);
  UB_LAUNCH_CHECK();
}

void membership(const uint32_t* idx, const float* dist, uint64_t n, uint64_t k,
                const GraphParams& gp, const float* sigmas, const float* rhos, uint32_t* pcol,
                float* pw, uint32_t* cnt, unsigned long long* edges_removed, unsigned long long* dup_row,
                cudaStream_t s) {
  if (n == 0) return;
  const uint32_t stride = (uint32_t)k | 1u;
  const size_t smem = (size_t)BT * stride * 8;
  if (smem > 200 * 1024) throw Error(UNSUPPORTED, "n_neighbors too large for the membership kernel");
  if (smem > 48 * 1024)
    UB_CUDA(cudaFuncSetAttribute(membership_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  membership_kernel<<<grid_for(n, BT), BT, smem, s>>>(idx, dist, n, (uint32_t)k, gp, sigmas, rhos,
                                                      pcol, pw, cnt, edges_removed, dup_row);
  UB_LAUNCH_CHECK();
}

void compact_directed(const uint32_t* pcol, const uint32_t* cnt, const uint64_t* dptr, uint64_t n,
                      uint64_t k, uint32_t* keys, uint32_t* vals, cudaStream_t s) {
  if (n * k == 0) return;
  compact_kernel<<<grid_for(n * k, 256), 256, 0, s>>>(pcol, cnt, dptr, n, (uint32_t)k, keys, vals);
  UB_LAUNCH_CHECK();
}

void gather_weights(const float* pw, const uint32_t* vals, uint64_t nnz, float* data, cudaStream_t s) {
  if (nnz == 0) return;
  gather_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(pw, vals, nnz, data);
  UB_LAUNCH_CHECK();
}

void segment_starts(const uint32_t* sorted_keys, uint64_t nnz, uint64_t n, uint64_t* tptr,
                    cudaStream_t s) {
  segment_starts_kernel<<<grid_for(nnz + 1, 256), 256, 0, s>>>(sorted_keys, nnz, n, tptr);
  UB_LAUNCH_CHECK();
}

void union_rows(const uint32_t* pcol, const float* pw, const uint32_t* cnt, uint64_t k,
                const uint64_t* tptr, const uint32_t* tvals, uint64_t n, const GraphParams& gp,
                uint32_t* out_cnt, const uint64_t* out_ptr, uint32_t* out_idx, float* out_w,
                bool fill, cudaStream_t s) {
  if (n == 0) return;
  union_kernel<<<grid_for(n, BT), BT, 0, s>>>(pcol, pw, cnt, (uint32_t)k, tptr, tvals, n, gp.mix,
                                              gp.prod_coeff, out_cnt, out_ptr, out_idx, out_w, fill);
  UB_LAUNCH_CHECK();
}

void localize_knn(const uint32_t* idx, uint64_t n, uint64_t k, const Segments& seg, uint32_t* out,
                  cudaStream_t s) {
  if (n * k == 0) return;
  localize_kernel<<<grid_for(n * k, 256), 256, 0, s>>>(idx, n, (uint32_t)k, seg.row_seg, seg.seg_off, out);
  UB_LAUNCH_CHECK();
}

void fill_row_segments(const uint64_t* seg_off, uint32_t n_seg, uint32_t* row_seg, cudaStream_t s) {
  if (n_seg == 0) return;
  row_segment_kernel<<<n_seg, 256, 0, s>>>(seg_off, n_seg, row_seg);
  UB_LAUNCH_CHECK();
}

void count_empty_rows(const uint64_t* indptr, const float* data, uint64_t n, unsigned long long* out,
                      cudaStream_t s) {
  UB_CUDA(cudaMemsetAsync(out, 0, sizeof(unsigned long long), s));
  if (n == 0) return;
  empty_rows_kernel<<<grid_for(n, 256), 256, 0, s>>>(indptr, data, n, out);
  UB_LAUNCH_CHECK();
}

}  // namespace ub
