// umap_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference UMAP fit path (wilsonzlin/umap-rs 0.4.5, Rust, Rayon).
// It is the checker for the CUDA library and the timed CPU baseline; nothing in the
// product links, loads or calls it.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference leg may use it.
//
// PARITY STATUS: parity unpinned.  The reference is Rust and cannot be built in this
// environment (no cargo/rustc), and its own tests (umap-rs/src/tests.rs) pin no numeric
// value on this path -- only shapes, nnz > 0, a,b > 0, epoch bookkeeping, the overstep
// panic text and serde round trips.  This file is checked against those smoke tests and
// against hand-derived known answers (tests/test_oracle.py), not against outputs of the
// reference itself.
//
// Floating-point fidelity: built with -ffp-contract=off and no fast-math, so f32/f64
// expressions round exactly as the Rust source writes them (Rust never contracts a*b+c).
// Rust's f32::exp / powf / ln / log2 lower to glibc expf / powf / logf / log2f on
// x86_64-unknown-linux-gnu; this file calls the same functions.  f32::max/min are
// fmaxf/fminf (NaN-ignoring); f32::clamp passes NaN through; `x as usize` saturates.
//
// Third-party arithmetic restated here (crate sources are not part of the reference tree):
//  * ndarray 0.17 `ArrayBase::mean()` = `sum() / (len as f32)`, where `sum()` over a
//    contiguous slice is `numeric_util::unrolled_fold`: eight running partial sums over
//    xs[8i+0..8i+7], combined as acc=((((0+(p0+p4))+(p1+p5))+(p2+p6))+(p3+p7)), then the
//    (< 8) leftover elements added in order.  Used by smooth_knn_dist.rs:74 and :177.
//  * rand 0.9 `random_range(0..n)` (optimize_layout_euclidean.rs:314) is unseeded in the
//    reference; here a seeded per-thread xoshiro256** with Lemire's unbiased bounded draw.
//  * rayon 1.10 `into_par_iter()` over a range: contiguous chunks processed sequentially
//    by worker threads; restated as a chunked parallel-for over std::thread.
//  * dashmap 6.1 DashSet of disconnected (row, col): a per-entry predicate here.
//  * sprs 0.11 CsMatI<f32,u32,usize>: plain indptr(u64)/indices(u32)/data(f32) arrays.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr float SMOOTH_K_TOLERANCE = 1e-5f;  // umap/constants.rs:4
constexpr float MIN_K_DIST_SCALE = 1e-3f;    // umap/constants.rs:7

thread_local std::string g_err;
int g_threads = 0;

int n_threads() {
  if (g_threads > 0) return g_threads;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// Contiguous-chunk parallel for (stand-in for rayon's range producer).  Chunks are
// handed out dynamically; each chunk runs sequentially on one thread.
template <class F>
void parallel_for(uint64_t n, F&& f, uint64_t min_chunk = 1024) {
  int nt = n_threads();
  if (nt <= 1 || n <= min_chunk) {
    f((uint64_t)0, n, 0);
    return;
  }
  uint64_t chunks = std::min<uint64_t>((uint64_t)nt * 8, (n + min_chunk - 1) / min_chunk);
  uint64_t csize = (n + chunks - 1) / chunks;
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 0; t < nt; ++t) {
    th.emplace_back([&, t]() {
      for (;;) {
        uint64_t c = next.fetch_add(1);
        if (c >= chunks) break;
        uint64_t b = c * csize, e = std::min(n, b + csize);
        if (b < e) f(b, e, t);
      }
    });
  }
  for (auto& x : th) x.join();
}

// Rust `f32::clamp`: NaN passes through.
inline float rust_clamp(float v, float lo, float hi) {
  float x = v;
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// Rust `f64 as usize`: saturating, NaN -> 0.
inline uint64_t rust_f64_to_usize(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 18446744073709551615.0) return UINT64_MAX;
  return (uint64_t)v;
}

// ndarray 0.17 unrolled_fold sum over a contiguous f32 slice (see header).
float ndarray_sum(const float* xs, uint64_t n) {
  float acc = 0.0f;
  float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f, p3 = 0.0f, p4 = 0.0f, p5 = 0.0f, p6 = 0.0f, p7 = 0.0f;
  while (n >= 8) {
    p0 = p0 + xs[0];
    p1 = p1 + xs[1];
    p2 = p2 + xs[2];
    p3 = p3 + xs[3];
    p4 = p4 + xs[4];
    p5 = p5 + xs[5];
    p6 = p6 + xs[6];
    p7 = p7 + xs[7];
    xs += 8;
    n -= 8;
  }
  acc = acc + (p0 + p4);
  acc = acc + (p1 + p5);
  acc = acc + (p2 + p6);
  acc = acc + (p3 + p7);
  for (uint64_t i = 0; i < n && i < 7; ++i) acc = acc + xs[i];
  return acc;
}

float ndarray_mean(const float* xs, uint64_t n) { return ndarray_sum(xs, n) / (float)n; }

// ---------------------------------------------------------------- find_ab_params
// umap/find_ab_params.rs:9-82 (custom f32 gradient descent, not scipy curve_fit).
void find_ab_params(float spread, float min_dist, float* a_out, float* b_out) {
  const int n_points = 300;
  std::vector<float> xv(n_points), yv(n_points);
  for (int i = 0; i < n_points; ++i)
    xv[i] = ((spread * 3.0f) * (float)i) / ((float)n_points - 1.0f);  // :13-15
  for (int i = 0; i < n_points; ++i) {                                  // :19-26
    float x = xv[i];
    if (x < min_dist) yv[i] = 1.0f;
    else yv[i] = expf((-(x - min_dist)) / spread);
  }
  float a = 1.5f, b = 0.9f;  // :31-32
  const float learning_rate = 0.01f;
  const int n_iterations = 1000;
  for (int it = 0; it < n_iterations; ++it) {  // :38-79
    float grad_a = 0.0f, grad_b = 0.0f, total_error = 0.0f;
    for (int i = 0; i < n_points; ++i) {
      float x = xv[i];
      float y_true = yv[i];
      float x_2b = powf(x, 2.0f * b);
      float denom = 1.0f + a * x_2b;
      float y_pred = 1.0f / denom;
      float error = y_pred - y_true;
      total_error = total_error + error * error;
      grad_a = grad_a + (2.0f * error) * ((-x_2b) / (denom * denom));
      if (x > 0.0f) {
        float ln_x = logf(x);
        grad_b = grad_b + (2.0f * error) * ((((-2.0f * a) * x_2b) * ln_x) / (denom * denom));
      }
    }
    a = a - (learning_rate * grad_a) / (float)n_points;
    b = b - (learning_rate * grad_b) / (float)n_points;
    a = rust_clamp(a, 0.001f, 10.0f);
    b = rust_clamp(b, 0.001f, 10.0f);
    if (total_error / (float)n_points < 1e-7f) break;
  }
  *a_out = a;
  *b_out = b;
}

// ---------------------------------------------------------------- smooth_knn_dist
// umap/smooth_knn_dist.rs:60-198.  Returns per-row sigma and rho.
void smooth_knn_dist(const float* distances, uint64_t n_samples, uint64_t n_neighbors,
                     uint64_t n_iter, float local_connectivity, float bandwidth,
                     float* sigmas, float* rhos) {
  const uint64_t k = n_neighbors;
  const float target = log2f((float)k) * bandwidth;                        // :71
  const float mean_distances = ndarray_mean(distances, n_samples * k);     // :74
  parallel_for(n_samples, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t i = b; i < e; ++i) {
      const float* row = distances + i * k;
      float lo = 0.0f, hi = INFINITY, mid = 1.0f;                          // :81-83
      uint64_t non_zero_count = 0;                                         // :88-97
      float max_non_zero = 0.0f;
      for (uint64_t j = 0; j < k; ++j) {
        float d = row[j];
        if (d > 0.0f) {
          non_zero_count++;
          if (d > max_non_zero) max_non_zero = d;
        }
      }
      float rho_i = 0.0f;                                                  // :101-142
      float lc_floor = floorf(local_connectivity);
      uint64_t local_conn_usize = rust_f64_to_usize((double)local_connectivity);
      if (non_zero_count >= local_conn_usize) {
        uint64_t index = rust_f64_to_usize((double)lc_floor);
        float interpolation = local_connectivity - lc_floor;
        float nth_minus_1 = 0.0f, nth = 0.0f;
        uint64_t count = 0;
        for (uint64_t j = 0; j < k; ++j) {
          float d = row[j];
          if (d > 0.0f) {
            if (count + 1 == index) nth_minus_1 = d;
            if (count + 1 == index + 1) nth = d;
            count++;
            if (count > index + 1) break;
          }
        }
        if (index > 0) {
          rho_i = nth_minus_1;
          if (interpolation > SMOOTH_K_TOLERANCE) rho_i = rho_i + interpolation * (nth - nth_minus_1);
        } else {
          float first_non_zero = 0.0f;
          for (uint64_t j = 0; j < k; ++j)
            if (row[j] > 0.0f) { first_non_zero = row[j]; break; }
          rho_i = interpolation * first_non_zero;
        }
      } else if (non_zero_count > 0) {
        rho_i = max_non_zero;
      }
      for (uint64_t it = 0; it < n_iter; ++it) {                           // :145-171
        float psum = 0.0f;
        for (uint64_t j = 1; j < k; ++j) {
          float d = row[j] - rho_i;
          if (d > 0.0f) psum = psum + expf(-(d / mid));
          else psum = psum + 1.0f;
        }
        if (fabsf(psum - target) < SMOOTH_K_TOLERANCE) break;
        if (psum > target) {
          hi = mid;
          mid = (lo + hi) / 2.0f;
        } else {
          lo = mid;
          if (hi == INFINITY) mid = mid * 2.0f;
          else mid = (lo + hi) / 2.0f;
        }
      }
      float sigma_i = mid;
      if (rho_i > 0.0f) {                                                  // :176-183
        float mean_ith = ndarray_mean(row, k);
        if (sigma_i < MIN_K_DIST_SCALE * mean_ith) sigma_i = MIN_K_DIST_SCALE * mean_ith;
      } else if (sigma_i < MIN_K_DIST_SCALE * mean_distances) {
        sigma_i = MIN_K_DIST_SCALE * mean_distances;
      }
      sigmas[i] = sigma_i;
      rhos[i] = rho_i;
    }
  }, 256);
}

// ---------------------------------------------------------------- CSR types
struct Csr {
  uint64_t n = 0;
  std::vector<uint64_t> indptr;
  std::vector<uint32_t> indices;
  std::vector<float> data;
  uint64_t nnz() const { return indices.size(); }
};

// umap/fuzzy_simplicial_set.rs:294-306
inline float membership_strength(float d, float rho, float sigma) {
  if (d - rho <= 0.0f || sigma == 0.0f) return 1.0f;
  return expf((-(d - rho)) / sigma);
}

// umap/fuzzy_simplicial_set.rs:171-292 (count -> prefix -> fill -> per-row insertion sort).
// `disconnected(i, j)` is the DashSet membership test of embedding.rs:177-186.
Csr build_membership_csr(uint64_t n, uint64_t k, const uint32_t* idx, const float* dist,
                         float disc_thr, const float* sigmas, const float* rhos) {
  Csr out;
  out.n = n;
  std::vector<uint32_t> row_counts(n);
  auto keep = [&](uint64_t i, uint64_t j, float* val) {
    if (dist[i * k + j] >= disc_thr) return false;                 // :187 / :237
    uint64_t knn_idx = idx[i * k + j];
    if (knn_idx == i || knn_idx >= n) return false;                // :192 / :242
    float v = membership_strength(dist[i * k + j], rhos[i], sigmas[i]);
    *val = v;
    return v != 0.0f;
  };
  parallel_for(n, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t i = b; i < e; ++i) {
      uint32_t c = 0;
      float v;
      for (uint64_t j = 0; j < k; ++j) c += keep(i, j, &v) ? 1 : 0;
      row_counts[i] = c;
    }
  });
  out.indptr.resize(n + 1);
  out.indptr[0] = 0;
  for (uint64_t i = 0; i < n; ++i) out.indptr[i + 1] = out.indptr[i] + row_counts[i];
  uint64_t nnz = out.indptr[n];
  out.indices.assign(nnz, 0);
  out.data.assign(nnz, 0.0f);
  parallel_for(n, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t i = b; i < e; ++i) {
      uint64_t o = out.indptr[i];
      float v;
      for (uint64_t j = 0; j < k; ++j) {
        if (keep(i, j, &v)) {
          out.indices[o] = idx[i * k + j];
          out.data[o] = v;
          ++o;
        }
      }
      uint64_t s = out.indptr[i], len = out.indptr[i + 1] - s;   // :264-282 insertion sort
      uint32_t* ri = out.indices.data() + s;
      float* rd = out.data.data() + s;
      for (uint64_t q = 1; q < len; ++q) {
        uint64_t m = q;
        while (m > 0 && ri[m - 1] > ri[m]) {
          std::swap(ri[m - 1], ri[m]);
          std::swap(rd[m - 1], rd[m]);
          --m;
        }
      }
    }
  });
  return out;
}

// fuzzy_simplicial_set.rs:291 passes the sorted rows to sprs 0.11's CsMatI::new, which
// unwraps its structure check; that check (a dependency, not in the reference tree) wants
// the column indices of every row strictly increasing, so a row that keeps one neighbour
// twice panics.  Returns the first such row, or n when there is none.
uint64_t first_repeated_column_row(const Csr& a) {
  for (uint64_t r = 0; r < a.n; ++r)
    for (uint64_t q = a.indptr[r] + 1; q < a.indptr[r + 1]; ++q)
      if (a.indices[q - 1] == a.indices[q]) return r;
  return a.n;
}

// umap/fuzzy_simplicial_set.rs:373-383 (binary search within the sorted row).
inline float csr_get(const Csr& a, uint64_t row, uint32_t col) {
  const uint32_t* b = a.indices.data() + a.indptr[row];
  const uint32_t* e = a.indices.data() + a.indptr[row + 1];
  const uint32_t* p = std::lower_bound(b, e, col);
  if (p != e && *p == col) return a.data[a.indptr[row] + (p - b)];
  return 0.0f;
}

// umap/fuzzy_simplicial_set.rs:310-370 (structure-only CSC; sequential fill keeps row order).
void build_csc_structure(const Csr& a, std::vector<uint64_t>& cptr, std::vector<uint32_t>& cind) {
  uint64_t n = a.n;
  std::vector<std::atomic<uint32_t>> counts(n);
  for (auto& c : counts) c.store(0, std::memory_order_relaxed);
  parallel_for(n, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t r = b; r < e; ++r)
      for (uint64_t q = a.indptr[r]; q < a.indptr[r + 1]; ++q)
        counts[a.indices[q]].fetch_add(1, std::memory_order_relaxed);
  });
  cptr.assign(n + 1, 0);
  for (uint64_t c = 0; c < n; ++c) cptr[c + 1] = cptr[c] + counts[c].load(std::memory_order_relaxed);
  cind.assign(a.nnz(), 0);
  std::vector<uint64_t> off(n, 0);
  for (uint64_t r = 0; r < n; ++r)
    for (uint64_t q = a.indptr[r]; q < a.indptr[r + 1]; ++q) {
      uint32_t c = a.indices[q];
      cind[cptr[c] + off[c]] = (uint32_t)r;
      off[c]++;
    }
}

// umap/fuzzy_simplicial_set.rs:392-552
Csr apply_set_operations(const Csr& in, float mix) {
  const uint64_t n = in.n;
  const float prod_coeff = 1.0f - 2.0f * mix;                              // :394
  std::vector<uint64_t> cptr;
  std::vector<uint32_t> cind;
  build_csc_structure(in, cptr, cind);
  auto combine = [&](float val_rc, float val_cr) {                         // :423 / :488
    return ((mix * val_rc) + (mix * val_cr)) + ((prod_coeff * val_rc) * val_cr);
  };
  std::vector<uint32_t> row_counts(n);
  parallel_for(n, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t row = b; row < e; ++row) {
      uint32_t count = 0;
      for (uint64_t q = in.indptr[row]; q < in.indptr[row + 1]; ++q) {
        float val_cr = csr_get(in, in.indices[q], (uint32_t)row);
        if (combine(in.data[q], val_cr) != 0.0f) count++;
      }
      for (uint64_t q = cptr[row]; q < cptr[row + 1]; ++q) {
        uint32_t c = cind[q];
        if (csr_get(in, row, c) != 0.0f) continue;
        float val_cr = csr_get(in, c, (uint32_t)row);
        if (mix * val_cr != 0.0f) count++;
      }
      row_counts[row] = count;
    }
  });
  Csr out;
  out.n = n;
  out.indptr.resize(n + 1);
  out.indptr[0] = 0;
  for (uint64_t i = 0; i < n; ++i) out.indptr[i + 1] = out.indptr[i] + row_counts[i];
  out.indices.assign(out.indptr[n], 0);
  out.data.assign(out.indptr[n], 0.0f);
  parallel_for(n, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t row = b; row < e; ++row) {
      uint64_t o = out.indptr[row];
      for (uint64_t q = in.indptr[row]; q < in.indptr[row + 1]; ++q) {
        uint32_t col = in.indices[q];
        float val_cr = csr_get(in, col, (uint32_t)row);
        float v = combine(in.data[q], val_cr);
        if (v != 0.0f) { out.indices[o] = col; out.data[o] = v; ++o; }
      }
      for (uint64_t q = cptr[row]; q < cptr[row + 1]; ++q) {
        uint32_t c = cind[q];
        if (csr_get(in, row, c) != 0.0f) continue;
        float val_cr = csr_get(in, c, (uint32_t)row);
        float v = mix * val_cr;
        if (v != 0.0f) { out.indices[o] = c; out.data[o] = v; ++o; }
      }
      uint64_t s = out.indptr[row], len = out.indptr[row + 1] - s;           // :524-542
      uint32_t* ri = out.indices.data() + s;
      float* rd = out.data.data() + s;
      for (uint64_t q = 1; q < len; ++q) {
        uint64_t m = q;
        while (m > 0 && ri[m - 1] > ri[m]) {
          std::swap(ri[m - 1], ri[m]);
          std::swap(rd[m - 1], rd[m]);
          --m;
        }
      }
    }
  });
  return out;
}

// ---------------------------------------------------------------- RNG (seeded stand-in)
inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
struct Xoshiro256ss {  // Blackman & Vigna, xoshiro256**
  uint64_t s[4];
  explicit Xoshiro256ss(uint64_t seed) {
    for (int i = 0; i < 4; ++i) s[i] = splitmix64(seed);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  inline uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  // Lemire's unbiased bounded integer in [0, n).
  inline uint64_t below(uint64_t n) {
    __uint128_t m = (__uint128_t)next() * n;
    uint64_t l = (uint64_t)m;
    if (l < n) {
      uint64_t t = (0 - n) % n;
      while (l < t) { m = (__uint128_t)next() * n; l = (uint64_t)m; }
    }
    return (uint64_t)(m >> 64);
  }
};

// Hogwild access to the shared embedding: relaxed atomic loads/stores compile to plain
// moves (racy like the reference's UnsafeSyncCell) without C++ data-race UB.
inline float ld(const float* p) { float v; __atomic_load(p, &v, __ATOMIC_RELAXED); return v; }
inline void st(float* p, float v) { __atomic_store(p, &v, __ATOMIC_RELAXED); }

}  // namespace

// ================================================================ C interface
struct OrcManifold {
  Csr graph;
  Csr directed;          // membership CSR before the fuzzy union (kept for kernel parity)
  std::vector<float> sigmas, rhos;
  uint64_t n_vertices = 0;
  float a = 0, b = 0;
  uint64_t edges_removed = 0, vertices_disconnected = 0;
};

struct OrcOptimizer {
  OrcManifold manifold;
  std::vector<uint32_t> head, tail;
  std::vector<double> epochs_per_sample;
  std::vector<float> embedding;
  uint64_t n = 0, dim = 0;
  std::vector<double> epoch_of_next_sample, epoch_of_next_negative_sample, epochs_per_negative_sample;
  uint64_t current_epoch = 0, total_epochs = 0;
  float gamma = 1, initial_alpha = 1;
  double negative_sample_rate = 5;
  float max_val = 0, threshold = 0;
  uint64_t seed = 0;
  int metric_type = 0;  // metric.rs:6-12: 0 Euclidean specialisation, 1 Generic
};

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads() { return n_threads(); }

void orc_find_ab_params(float spread, float min_dist, float* a, float* b) {
  find_ab_params(spread, min_dist, a, b);
}

float orc_ndarray_mean(const float* x, uint64_t n) { return ndarray_mean(x, n); }

void orc_smooth_knn_dist(const float* dists, uint64_t n, uint64_t k, uint64_t n_iter,
                         float local_connectivity, float bandwidth, float* sigmas, float* rhos) {
  smooth_knn_dist(dists, n, k, n_iter, local_connectivity, bandwidth, sigmas, rhos);
}

// embedding.rs:149-240 + fuzzy_simplicial_set.rs:110-166.  Validation mirrors
// embedding.rs:339-429 (returns NULL with the panic text instead of panicking).
OrcManifold* orc_learn_manifold(uint64_t n_samples, uint64_t knn_rows, uint64_t knn_cols,
                                const uint32_t* knn_idx, const float* knn_dist,
                                uint64_t n_neighbors, float min_dist, float spread,
                                int has_a, float a, int has_b, float b,
                                float local_connectivity, float set_op_mix_ratio,
                                int has_disc, float disc, int symmetrize,
                                float repulsion_strength, float learning_rate,
                                uint64_t n_components) {
  char buf[512];
  auto fail = [&](const char* m) { g_err = m; return (OrcManifold*)nullptr; };
  if (set_op_mix_ratio < 0.0f || set_op_mix_ratio > 1.0f) {
    snprintf(buf, sizeof buf, "set_op_mix_ratio must be between 0.0 and 1.0, got %g", set_op_mix_ratio);
    return fail(buf);
  }
  if (n_neighbors < 2) {
    snprintf(buf, sizeof buf, "n_neighbors must be >= 2, got %llu", (unsigned long long)n_neighbors);
    return fail(buf);
  }
  if (repulsion_strength < 0.0f) {
    snprintf(buf, sizeof buf, "repulsion_strength cannot be negative, got %g", repulsion_strength);
    return fail(buf);
  }
  if (min_dist > spread) {
    snprintf(buf, sizeof buf, "min_dist (%g) must be <= spread (%g)", min_dist, spread);
    return fail(buf);
  }
  if (min_dist < 0.0f) {
    snprintf(buf, sizeof buf, "min_dist cannot be negative, got %g", min_dist);
    return fail(buf);
  }
  if (learning_rate < 0.0f) {
    snprintf(buf, sizeof buf, "learning_rate must be positive, got %g", learning_rate);
    return fail(buf);
  }
  if (n_components < 1) {
    snprintf(buf, sizeof buf, "n_components must be >= 1, got %llu", (unsigned long long)n_components);
    return fail(buf);
  }
  if (knn_cols != n_neighbors) {
    snprintf(buf, sizeof buf, "knn_dists has %llu neighbors but n_neighbors is %llu",
             (unsigned long long)knn_cols, (unsigned long long)n_neighbors);
    return fail(buf);
  }
  if (knn_rows != n_samples) {
    snprintf(buf, sizeof buf, "knn_dists has %llu samples but data has %llu samples",
             (unsigned long long)knn_rows, (unsigned long long)n_samples);
    return fail(buf);
  }
  if (n_samples <= n_neighbors) {
    snprintf(buf, sizeof buf, "Number of samples (%llu) must be > n_neighbors (%llu)",
             (unsigned long long)n_samples, (unsigned long long)n_neighbors);
    return fail(buf);
  }
  if (n_samples >= 0xFFFFFFFFull) return fail("n_samples must be < 2^32 for u32 indices");

  auto* m = new OrcManifold();
  if (has_a && has_b) { m->a = a; m->b = b; }                        // embedding.rs:161-166
  else find_ab_params(spread, min_dist, &m->a, &m->b);
  float disc_thr = has_disc ? disc : INFINITY;                        // :169-173 (Euclidean: +inf)
  uint64_t removed = 0;
  for (uint64_t i = 0; i < n_samples * knn_cols; ++i) removed += (knn_dist[i] >= disc_thr) ? 1 : 0;
  m->edges_removed = removed;
  m->n_vertices = n_samples;
  m->sigmas.resize(n_samples);
  m->rhos.resize(n_samples);
  smooth_knn_dist(knn_dist, n_samples, n_neighbors, 64, local_connectivity, 1.0f,
                  m->sigmas.data(), m->rhos.data());
  m->directed = build_membership_csr(n_samples, n_neighbors, knn_idx, knn_dist, disc_thr,
                                     m->sigmas.data(), m->rhos.data());
  if (uint64_t r = first_repeated_column_row(m->directed); r < n_samples) {
    delete m;
    snprintf(buf, sizeof buf,
             "knn_indices row %llu keeps the same neighbour more than once: called `Result::unwrap()` on an "
             "`Err` value: Unsorted(\"Indices are not sorted\")", (unsigned long long)r);
    return fail(buf);
  }
  if (symmetrize) m->graph = apply_set_operations(m->directed, set_op_mix_ratio);
  else m->graph = m->directed;
  uint64_t disconnected = 0;                                          // embedding.rs:216-223
  for (uint64_t r = 0; r < n_samples; ++r) {
    float s = 0.0f;
    for (uint64_t q = m->graph.indptr[r]; q < m->graph.indptr[r + 1]; ++q) s = s + m->graph.data[q];
    if (s == 0.0f) disconnected++;
  }
  m->vertices_disconnected = disconnected;
  return m;
}

void orc_manifold_free(OrcManifold* m) { delete m; }
uint64_t orc_manifold_nnz(const OrcManifold* m) { return m->graph.nnz(); }
uint64_t orc_manifold_directed_nnz(const OrcManifold* m) { return m->directed.nnz(); }
void orc_manifold_graph(const OrcManifold* m, uint64_t* indptr, uint32_t* indices, float* data) {
  memcpy(indptr, m->graph.indptr.data(), (m->n_vertices + 1) * 8);
  memcpy(indices, m->graph.indices.data(), m->graph.nnz() * 4);
  memcpy(data, m->graph.data.data(), m->graph.nnz() * 4);
}
void orc_manifold_directed(const OrcManifold* m, uint64_t* indptr, uint32_t* indices, float* data) {
  memcpy(indptr, m->directed.indptr.data(), (m->n_vertices + 1) * 8);
  memcpy(indices, m->directed.indices.data(), m->directed.nnz() * 4);
  memcpy(data, m->directed.data.data(), m->directed.nnz() * 4);
}
void orc_manifold_sigmas_rhos(const OrcManifold* m, float* sigmas, float* rhos) {
  memcpy(sigmas, m->sigmas.data(), m->n_vertices * 4);
  memcpy(rhos, m->rhos.data(), m->n_vertices * 4);
}
void orc_manifold_info(const OrcManifold* m, uint64_t* n_vertices, float* a, float* b,
                       uint64_t* edges_removed, uint64_t* vertices_disconnected) {
  *n_vertices = m->n_vertices;
  *a = m->a;
  *b = m->b;
  *edges_removed = m->edges_removed;
  *vertices_disconnected = m->vertices_disconnected;
}

// optimizer.rs:74-290.  The manifold is copied (the reference moves it in).
OrcOptimizer* orc_optimizer_new(const OrcManifold* manifold, const float* init, uint64_t n,
                                uint64_t dim, uint64_t total_epochs, float gamma,
                                float learning_rate, uint64_t negative_sample_rate, uint64_t seed) {
  if (n != manifold->n_vertices) { g_err = "init rows != n_vertices"; return nullptr; }
  auto* o = new OrcOptimizer();
  o->manifold = *manifold;
  o->gamma = gamma;
  o->initial_alpha = learning_rate;
  o->negative_sample_rate = (double)negative_sample_rate;
  o->n = n;
  o->dim = dim;
  o->seed = seed;
  const Csr& g = o->manifold.graph;
  float max_val = 0.0f;                                                 // :90-94
  for (float v : g.data) max_val = fmaxf(max_val, v);
  uint64_t default_epochs = n <= 10000 ? 500 : 200;                     // :96-102
  uint64_t threshold_epochs = total_epochs > 10 ? total_epochs : default_epochs;
  float threshold = max_val / (float)threshold_epochs;
  o->max_val = max_val;
  o->threshold = threshold;
  std::vector<float> weights;                                           // :110-163
  for (uint64_t r = 0; r < n; ++r)
    for (uint64_t q = g.indptr[r]; q < g.indptr[r + 1]; ++q)
      if (g.data[q] >= threshold) {
        o->head.push_back((uint32_t)r);
        o->tail.push_back(g.indices[q]);
        weights.push_back(g.data[q]);
      }
  // make_epochs_per_sample.rs:21-52
  float max_weight = -INFINITY;
  for (float w : weights) max_weight = fmaxf(max_weight, w);
  if (max_weight <= 0.0f) max_weight = 1.0f;
  double n_epochs_f64 = (double)total_epochs, max_weight_f64 = (double)max_weight;
  o->epochs_per_sample.resize(weights.size());
  for (size_t i = 0; i < weights.size(); ++i) {
    double n_samples = n_epochs_f64 * ((double)weights[i] / max_weight_f64);
    o->epochs_per_sample[i] = n_samples > 0.0 ? n_epochs_f64 / n_samples : -1.0;
  }
  // :181-230 normalise init to [0, 10] per dimension
  o->embedding.assign(init, init + n * dim);
  std::vector<float> mins(dim, INFINITY), maxs(dim, -INFINITY), scales(dim);
  for (uint64_t i = 0; i < n; ++i)
    for (uint64_t d = 0; d < dim; ++d) {
      mins[d] = fminf(mins[d], o->embedding[i * dim + d]);
      maxs[d] = fmaxf(maxs[d], o->embedding[i * dim + d]);
    }
  for (uint64_t d = 0; d < dim; ++d) {
    float range = maxs[d] - mins[d];
    scales[d] = range > 0.0f ? 10.0f / range : 0.0f;
  }
  for (uint64_t idx = 0; idx < n * dim; ++idx) {
    uint64_t d = idx % dim;
    if (scales[d] > 0.0f) o->embedding[idx] = (o->embedding[idx] - mins[d]) * scales[d];
  }
  // :236-272 schedule arrays
  double neg_rate = (double)negative_sample_rate;
  o->epoch_of_next_sample = o->epochs_per_sample;
  o->epochs_per_negative_sample.resize(weights.size());
  for (size_t i = 0; i < weights.size(); ++i) o->epochs_per_negative_sample[i] = o->epochs_per_sample[i] / neg_rate;
  o->epoch_of_next_negative_sample = o->epochs_per_negative_sample;
  o->current_epoch = 0;
  o->total_epochs = total_epochs;
  return o;
}

void orc_optimizer_free(OrcOptimizer* o) { delete o; }
uint64_t orc_optimizer_n_edges(const OrcOptimizer* o) { return o->head.size(); }
uint64_t orc_optimizer_current_epoch(const OrcOptimizer* o) { return o->current_epoch; }
uint64_t orc_optimizer_total_epochs(const OrcOptimizer* o) { return o->total_epochs; }
void orc_optimizer_threshold(const OrcOptimizer* o, float* max_val, float* threshold) {
  *max_val = o->max_val;
  *threshold = o->threshold;
}
void orc_optimizer_edges(const OrcOptimizer* o, uint32_t* head, uint32_t* tail, double* eps) {
  memcpy(head, o->head.data(), o->head.size() * 4);
  memcpy(tail, o->tail.data(), o->tail.size() * 4);
  memcpy(eps, o->epochs_per_sample.data(), o->epochs_per_sample.size() * 8);
}
void orc_optimizer_state(const OrcOptimizer* o, double* eons, double* eonns, double* epns) {
  size_t e = o->head.size() * 8;
  memcpy(eons, o->epoch_of_next_sample.data(), e);
  memcpy(eonns, o->epoch_of_next_negative_sample.data(), e);
  memcpy(epns, o->epochs_per_negative_sample.data(), e);
}
void orc_optimizer_embedding(const OrcOptimizer* o, float* out) {
  memcpy(out, o->embedding.data(), o->embedding.size() * 4);
}
// MetricType of the optimizer (optimizer.rs:318-359 dispatch): 0 Euclidean, 1 Generic.
void orc_optimizer_set_metric_type(OrcOptimizer* o, int metric_type) { o->metric_type = metric_type; }
void orc_optimizer_set_embedding(OrcOptimizer* o, const float* in) {
  memcpy(o->embedding.data(), in, o->embedding.size() * 4);
}

// distances.rs:22-37 EuclideanMetric::distance: (sqrt(sum diff^2), (x - y) / (dist + 1e-6)).
static float euclidean_distance(const float* x, const float* y, uint64_t dim, float* grad) {
  float sum_sq = 0.0f;
  for (uint64_t i = 0; i < dim; ++i) {
    float diff = x[i] - y[i];
    sum_sq = sum_sq + diff * diff;
  }
  float dist = sqrtf(sum_sq);
  float denom = dist + 1e-6f;
  for (uint64_t i = 0; i < dim; ++i) grad[i] = (x[i] - y[i]) / denom;
  return dist;
}

// layout/optimize_layout_generic.rs:35-124 (move_other = true) with the built-in output
// metric EuclideanMetric, the only Metric the reference ships.  Sequential over the edges
// with one RNG, as the reference's generic loop is (it has no parallel variant).
static void generic_epoch(OrcOptimizer* o, float* headp, float* tailp, uint64_t epoch, float alpha,
                   uint64_t* fired, uint64_t* negs) {
  const uint64_t nv = o->manifold.n_vertices, dim = o->dim, E = o->head.size();
  const float a = o->manifold.a, b = o->manifold.b, gamma = o->gamma;
  const double nd = (double)epoch;
  Xoshiro256ss rng(o->seed ^ (0x9E3779B97F4A7C15ull * (epoch + 1)));
  std::vector<float> grad(dim), rev(dim);
  uint64_t lf = 0, ln = 0;
  for (uint64_t i = 0; i < E; ++i) {
    if (!(o->epoch_of_next_sample[i] <= nd)) continue;                 // :57
    const uint64_t j = o->head[i], k = o->tail[i];
    float* cur = headp + j * dim;
    float* oth = tailp + k * dim;
    float dist = euclidean_distance(cur, oth, dim, grad.data());        // :65
    euclidean_distance(oth, cur, dim, rev.data());                      // :66
    float w_l = dist > 0.0f ? 1.0f / (1.0f + a * powf(dist, 2.0f * b)) : 1.0f;   // :71-75
    float grad_coeff = ((2.0f * b) * (w_l - 1.0f)) / (dist + 1e-6f);   // :76
    for (uint64_t d = 0; d < dim; ++d) {                                // :78-86
      cur[d] += rust_clamp(grad_coeff * grad[d], -4.0f, 4.0f) * alpha;
      oth[d] += rust_clamp(grad_coeff * rev[d], -4.0f, 4.0f) * alpha;
    }
    o->epoch_of_next_sample[i] += o->epochs_per_sample[i];              // :88
    uint64_t n_neg = rust_f64_to_usize((nd - o->epoch_of_next_negative_sample[i]) /
                                       o->epochs_per_negative_sample[i]);   // :91-92
    lf++;
    ln += n_neg;
    for (uint64_t p = 0; p < n_neg; ++p) {                              // :94-119
      uint64_t kk = rng.below(nv);
      if (j == kk) continue;
      float* ob = tailp + kk * dim;
      float dn = euclidean_distance(cur, ob, dim, grad.data());
      float wn = dn > 0.0f ? 1.0f / (1.0f + a * powf(dn, 2.0f * b)) : 1.0f;
      float gc = (((gamma * 2.0f) * b) * wn) / (dn + 1e-6f);            // :113
      for (uint64_t d = 0; d < dim; ++d) cur[d] += rust_clamp(gc * grad[d], -4.0f, 4.0f) * alpha;
    }
    o->epoch_of_next_negative_sample[i] += (double)n_neg * o->epochs_per_negative_sample[i];  // :121
  }
  *fired = lf;
  *negs = ln;
}

// optimizer.rs:297-366 + layout/optimize_layout_euclidean.rs:236-347 (parallel=true,
// move_other=true).  Live buffer = head_embedding, per-call clone = tail_embedding.
// `fires` / `negs` (optional, length n) receive per-epoch counts of fired edges and of
// negative samples drawn (the j == k skips included, as in the reference's loop count).
int orc_optimizer_step_epochs(OrcOptimizer* o, uint64_t n_ep, uint64_t* fires, uint64_t* negs) {
  if (o->current_epoch + n_ep > o->total_epochs) {
    char buf[256];
    snprintf(buf, sizeof buf, "Cannot step %llu epochs: would exceed total_epochs %llu (current: %llu)",
             (unsigned long long)n_ep, (unsigned long long)o->total_epochs,
             (unsigned long long)o->current_epoch);
    g_err = buf;
    return 1;
  }
  const uint64_t start = o->current_epoch, end = start + n_ep;
  const uint64_t nv = o->manifold.n_vertices, dim = o->dim;
  const float a = o->manifold.a, b = o->manifold.b, gamma = o->gamma;
  std::vector<float> copy = o->embedding;                               // :314
  float* headp = o->embedding.data();
  float* tailp = copy.data();
  const uint64_t E = o->head.size();
  const int nt = n_threads();
  for (uint64_t epoch = start; epoch < end; ++epoch) {
    const float alpha = o->initial_alpha * (1.0f - ((float)epoch / (float)o->total_epochs));  // :317
    const double nd = (double)epoch;
    if (o->metric_type == 1) {                                          // optimizer.rs:340-358
      uint64_t F = 0, N = 0;
      generic_epoch(o, headp, tailp, epoch, alpha, &F, &N);
      if (fires) fires[epoch - start] = F;
      if (negs) negs[epoch - start] = N;
      continue;
    }
    std::vector<uint64_t> tf(nt + 1, 0), tn(nt + 1, 0);
    parallel_for(E, [&](uint64_t bgn, uint64_t e, int tid) {
      Xoshiro256ss rng(o->seed ^ (0x9E3779B97F4A7C15ull * (epoch + 1)) ^ (bgn * 0xD1B54A32D192ED03ull));
      uint64_t lf = 0, ln = 0;
      for (uint64_t i = bgn; i < e; ++i) {
        if (o->epoch_of_next_sample[i] <= nd) {                         // :277
          uint64_t j = o->head[i], k = o->tail[i];
          float* cur = headp + j * dim;
          float* oth = tailp + k * dim;
          float dist_squared = 0.0f;                                    // :284-288
          for (uint64_t d = 0; d < dim; ++d) {
            float diff = ld(&cur[d]) - ld(&oth[d]);
            dist_squared = dist_squared + diff * diff;
          }
          float grad_coeff = 0.0f;                                      // :290-297
          if (dist_squared > 0.0f) {
            float dist_pow_b = powf(dist_squared, b);
            float gc = (((-2.0f * a) * b) * dist_pow_b) / dist_squared;
            gc = gc / (((a * dist_pow_b) * dist_squared) + 1.0f);
            grad_coeff = gc;
          }
          for (uint64_t d = 0; d < dim; ++d) {                          // :299-306
            float cd = ld(&cur[d]);
            float od = ld(&oth[d]);
            float grad_d = rust_clamp(grad_coeff * (cd - od), -4.0f, 4.0f);
            st(&cur[d], cd + grad_d * alpha);
            st(&oth[d], od - grad_d * alpha);
          }
          o->epoch_of_next_sample[i] += o->epochs_per_sample[i];        // :308
          uint64_t n_neg = rust_f64_to_usize((nd - o->epoch_of_next_negative_sample[i]) /
                                             o->epochs_per_negative_sample[i]);   // :310-311
          lf++;
          ln += n_neg;
          for (uint64_t p = 0; p < n_neg; ++p) {                        // :313-341
            uint64_t kk = rng.below(nv);
            if (j == kk) continue;
            float* ob = tailp + kk * dim;
            float ds = 0.0f;
            for (uint64_t d = 0; d < dim; ++d) {
              float diff = ld(&cur[d]) - ld(&ob[d]);
              ds = ds + diff * diff;
            }
            float gc = 0.0f;
            if (ds > 0.0f) {
              float dist_pow_b = powf(ds, b);
              gc = ((2.0f * gamma) * b) / ((0.001f + ds) * (((a * dist_pow_b) * ds) + 1.0f));
            }
            if (gc > 0.0f) {
              for (uint64_t d = 0; d < dim; ++d) {
                float cd = ld(&cur[d]);
                float od = ld(&ob[d]);
                float grad_d = rust_clamp(gc * (cd - od), -4.0f, 4.0f);
                st(&cur[d], cd + grad_d * alpha);
              }
            }
          }
          o->epoch_of_next_negative_sample[i] += (double)n_neg * o->epochs_per_negative_sample[i];  // :343
        }
      }
      __atomic_fetch_add(&tf[tid], lf, __ATOMIC_RELAXED);
      __atomic_fetch_add(&tn[tid], ln, __ATOMIC_RELAXED);
    }, 4096);
    uint64_t F = 0, N = 0;
    for (int t = 0; t < nt + 1; ++t) { F += tf[t]; N += tn[t]; }
    if (fires) fires[epoch - start] = F;
    if (negs) negs[epoch - start] = N;
  }
  o->current_epoch = end;
  return 0;
}

// examples/src/bin/mnist_demo.rs:203-239 compute_knn: for each row, the distances to every
// other row (f32, (x - y)^2 summed in coordinate order, then sqrt), stably sorted by distance
// (ties in index order), the first k kept; slots beyond n - 1 stay 0 / 0.0.
// Rows [r0, r1) only (outputs [r1 - r0, k]): a sample of the workload for timing and spot checks.
void orc_knn_bruteforce_rows(const float* X, uint64_t n, uint64_t d, uint64_t k, uint64_t r0, uint64_t r1,
                             uint32_t* idx, float* dist) {
  memset(idx, 0, (r1 - r0) * k * 4);
  memset(dist, 0, (r1 - r0) * k * 4);
  parallel_for(r1 - r0, [&](uint64_t b, uint64_t e, int) {
    std::vector<std::pair<float, uint32_t>> cand;
    cand.reserve(n);
    for (uint64_t i = r0 + b; i < r0 + e; ++i) {
      cand.clear();
      const float* x = X + i * d;
      for (uint64_t j = 0; j < n; ++j) {
        if (j == i) continue;
        const float* y = X + j * d;
        float acc = -0.0f;
        for (uint64_t c = 0; c < d; ++c) {
          float df = x[c] - y[c];
          acc = acc + df * df;
        }
        cand.emplace_back(sqrtf(acc), (uint32_t)j);
      }
      const uint64_t m = std::min<uint64_t>(k, cand.size());
      std::partial_sort(cand.begin(), cand.begin() + m, cand.end());  // (distance, index) order
      for (uint64_t t = 0; t < m; ++t) {
        idx[(i - r0) * k + t] = cand[t].second;
        dist[(i - r0) * k + t] = cand[t].first;
      }
    }
  }, 16);
}

void orc_knn_bruteforce(const float* X, uint64_t n, uint64_t d, uint64_t k, uint32_t* idx, float* dist) {
  orc_knn_bruteforce_rows(X, n, d, k, 0, n, idx, dist);
}

}  // extern "C"
