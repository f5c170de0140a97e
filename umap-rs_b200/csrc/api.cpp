// C-ABI implementation: handle types, orchestration of the fit path on one CUDA stream per
// handle, and checkpoints.  Mirrors the reference's Rust API (see include/umap_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <chrono>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/umap_b200.h"
#include "host_math.hpp"
#include "ub_internal.hpp"

namespace ub {

thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
bool alloc_log_enabled() {
  static const bool on = getenv("UMAP_B200_LOG") != nullptr;
  return on;
}
void log_slow_alloc(uint64_t bytes, double ms) {
  fprintf(stderr, "[umap_b200] slow device allocation: %llu bytes took %.1f ms\n", (unsigned long long)bytes, ms);
}

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
  (void)cudaGetLastError();
  int code = e == cudaErrorMemoryAllocation ? OUT_OF_MEMORY : CUDA;
  const char* f = strrchr(file, '/');
  throw Error(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + (f ? f + 1 : file) +
                        ":" + std::to_string(line) + ")");
}

namespace {

// ------------------------------------------------------------------ stream ownership
// Keeps freed blocks in the device's default stream-ordered pool (process lifetime) so
// that repeated fits do not pay for fresh device allocations.
void keep_pool_warm(int device) {
  static std::atomic<uint64_t> done_mask{0};
  if (device < 0 || device >= 64 || (done_mask.load() >> device) & 1ull) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    (void)cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  (void)cudaGetLastError();
  done_mask.fetch_or(1ull << device);
}

struct Stream {
  cudaStream_t s = nullptr;
  int device = 0;
  Stream() {
    UB_CUDA(cudaGetDevice(&device));
    keep_pool_warm(device);
    UB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  }
  ~Stream() {
    if (s) {
      (void)cudaStreamSynchronize(s);
      (void)cudaStreamDestroy(s);
    }
  }
  Stream(const Stream&) = delete;
  Stream& operator=(const Stream&) = delete;
  void sync() const { UB_CUDA(cudaStreamSynchronize(s)); }
  void activate() const { UB_CUDA(cudaSetDevice(device)); }
};

// Phase timing with the reference's tracing phase names (fuzzy_simplicial_set.rs:133-162,
// optimizer.rs:103-272), measured by CUDA events on the handle's stream; printed to stderr
// when UMAP_B200_LOG is set.
struct PhaseLog {
  cudaStream_t s;
  bool on;
  cudaEvent_t last = nullptr;
  explicit PhaseLog(cudaStream_t st) : s(st), on(getenv("UMAP_B200_LOG") != nullptr) {
    if (on) {
      UB_CUDA(cudaEventCreate(&last));
      UB_CUDA(cudaEventRecord(last, s));
    }
  }
  void mark(const char* name) {
    if (!on) return;
    cudaEvent_t e;
    UB_CUDA(cudaEventCreate(&e));
    UB_CUDA(cudaEventRecord(e, s));
    UB_CUDA(cudaEventSynchronize(e));
    float ms = 0;
    UB_CUDA(cudaEventElapsedTime(&ms, last, e));
    fprintf(stderr, "[umap_b200] duration_ms=%.3f %s\n", ms, name);
    (void)cudaEventDestroy(last);
    last = e;
  }
  ~PhaseLog() {
    if (last) (void)cudaEventDestroy(last);
  }
};

template <class T>
void d2h(T* dst, const T* src, uint64_t n, cudaStream_t s) {
  if (n) UB_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, s));
}
template <class T>
void h2d(T* dst, const T* src, uint64_t n, cudaStream_t s) {
  if (n) UB_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
}
template <class T>
void d2d(T* dst, const T* src, uint64_t n, cudaStream_t s) {
  if (n) UB_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
}

}  // namespace
}  // namespace ub

// ------------------------------------------------------------------ handle types
struct umap_manifold {
  std::unique_ptr<ub::Stream> stream;  // declared first: destroyed last
  uint64_t n_vertices = 0, nnz = 0;
  float a = 0, b = 0;
  uint64_t edges_removed = 0, vertices_disconnected = 0;
  ub::DevBuf<uint64_t> indptr;
  ub::DevBuf<uint32_t> indices;
  ub::DevBuf<float> data;
  ub::DevBuf<float> sigmas, rhos;
  cudaStream_t s() const { return stream->s; }
};

namespace ub {
namespace {
void release_l2_window(umap_optimizer& o) noexcept;
}  // namespace
}  // namespace ub

struct umap_optimizer {
  std::unique_ptr<umap_manifold> manifold;  // declared first: owns the stream
  uint64_t n = 0, dim = 0;
  ub::DevBuf<float> emb2;  // [live | snapshot], each n*dim
  ub::SgdLayout layout;
  uint64_t current_epoch = 0, total_epochs = 0;
  float gamma = 1, initial_alpha = 1;
  uint64_t negative_sample_rate = 5;
  int metric_type = UMAP_METRIC_EUCLIDEAN;
  float max_val = 0, threshold = 0, max_w = 1;
  uint64_t seed = 0;
  float last_step_ms = 0;  // CUDA-event time of the last step_epochs epoch loop
  // Batched instances (n_seg > 0): instance s owns rows [seg_off[s], seg_off[s+1]).
  uint32_t n_seg = 0;
  ub::DevBuf<uint64_t> seg_off;
  ub::DevBuf<uint32_t> row_seg;
  ub::DevBuf<float> seg_thr, seg_maxw;
  bool l2_window = false;  // holds a persisting-L2 access-policy window (see set_l2_window)
  cudaStream_t s() const { return manifold->s(); }
  umap_optimizer() = default;
  umap_optimizer(const umap_optimizer&) = delete;
  umap_optimizer& operator=(const umap_optimizer&) = delete;
  ~umap_optimizer() { ub::release_l2_window(*this); }
};

struct umap_fitted {
  std::unique_ptr<umap_manifold> manifold;
  uint64_t n = 0, dim = 0;
  ub::DevBuf<float> embedding;
  umap_config config{};
  cudaStream_t s() const { return manifold->s(); }
};

struct umap_mlp {
  std::unique_ptr<ub::Stream> stream;  // declared first: destroyed last
  std::unique_ptr<ub::Mlp> net;
};

namespace ub {
namespace {

void set_error(const std::string& m) { g_last_error = m; }

#define API_BEGIN try {
#define API_END                                                  \
  }                                                              \
  catch (const ub::Error& e) {                                   \
    ub::set_error(e.what());                                     \
    return e.code;                                               \
  }                                                              \
  catch (const std::bad_alloc&) {                                \
    ub::set_error("host allocation failed");                     \
    return UMAP_ERR_OUT_OF_MEMORY;                               \
  }                                                              \
  catch (const std::exception& e) {                              \
    ub::set_error(e.what());                                     \
    return UMAP_ERR_CUDA;                                        \
  }                                                              \
  ub::set_error("");                                             \
  return UMAP_OK;

// Device inputs are produced by the caller on the legacy default stream (PyTorch's default):
// order after that work only, so calls on other handles (other streams) keep running.
void wait_for_inputs() { UB_CUDA(cudaStreamSynchronize(cudaStreamLegacy)); }

void need(const void* p, const char* what) {
  if (!p) throw Error(NULLPTR, std::string(what) + " is NULL");
}

GraphParams graph_params(const umap_config& c) {
  GraphParams gp{};
  gp.local_connectivity = c.local_connectivity;
  const float lcf = floorf(c.local_connectivity);
  gp.interpolation = c.local_connectivity - lcf;
  gp.lc_usize = rust_f32_as_usize(c.local_connectivity);
  gp.lc_index = rust_f32_as_usize(lcf);
  gp.target = log2f((float)c.n_neighbors) * 1.0f;  // smooth_knn_dist.rs:71, bandwidth 1
  gp.disc_thr = c.has_disconnection_distance ? c.disconnection_distance : INFINITY;
  gp.mix = c.set_op_mix_ratio;
  gp.prod_coeff = 1.0f - 2.0f * c.set_op_mix_ratio;  // fuzzy_simplicial_set.rs:394
  gp.n_iter = 64;
  return gp;
}

// ------------------------------------------------------------------ learn_manifold
// embedding.rs:149-240 on device arrays.
std::unique_ptr<umap_manifold> learn_manifold_impl(const umap_config& c, uint64_t n_samples,
                                                   const uint32_t* idx, const float* dist,
                                                   uint64_t rows, uint64_t cols,
                                                   const Segments* seg = nullptr) {
  std::string err = validate_parameters(c, n_samples, rows, cols);
  if (!err.empty()) throw Error(INVALID_ARGUMENT, err);
  const uint64_t n = n_samples, k = cols;
  if (n * k >= 0xFFFFFFFFull)
    throw Error(UNSUPPORTED, "n_samples * n_neighbors must be < 2^32 on this build");
  auto m = std::make_unique<umap_manifold>();
  m->stream = std::make_unique<Stream>();
  cudaStream_t s = m->s();
  m->n_vertices = n;
  if (c.has_a && c.has_b) {  // embedding.rs:161-166
    m->a = c.a;
    m->b = c.b;
  } else {
    find_ab_params(c.spread, c.min_dist, &m->a, &m->b);
  }
  const GraphParams gp = graph_params(c);
  PhaseLog log(s);

  m->sigmas.alloc(n, s);
  m->rhos.alloc(n, s);
  smooth_knn(dist, n, k, gp, m->sigmas.p, m->rhos.p, s, seg);
  log.mark("smooth_knn_dist complete");

  DevBuf<uint32_t> pcol(n * k, s), cnt(n, s);
  DevBuf<float> pw(n * k, s);
  DevBuf<unsigned long long> dcount(3, s);
  UB_CUDA(cudaMemsetAsync(dcount.p, 0, 24, s));
  membership(idx, dist, n, k, gp, m->sigmas.p, m->rhos.p, pcol.p, pw.p, cnt.p, dcount.p, dcount.p + 2, s);
  DevBuf<uint64_t> dptr(n + 1, s);
  scan_u32_to_u64(cnt.p, dptr.p, n, s);
  uint64_t nnz_dir = 0;
  unsigned long long dup = 0;
  d2h(&nnz_dir, dptr.p + n, 1, s);
  d2h(&dup, dcount.p + 2, 1, s);
  UB_CUDA(cudaStreamSynchronize(s));
  if (dup)  // fuzzy_simplicial_set.rs:291: sprs's CsMatI::new refuses a row with a repeated column
    throw Error(INVALID_ARGUMENT, "knn_indices row " + std::to_string(~dup) +
                                      " keeps the same neighbour more than once: called `Result::unwrap()` on an "
                                      "`Err` value: Unsorted(\"Indices are not sorted\")");
  DevBuf<uint32_t> keys(nnz_dir, s), vals(nnz_dir, s);
  compact_directed(pcol.p, cnt.p, dptr.p, n, k, keys.p, vals.p, s);
  log.mark("build_membership_csr complete");

  if (c.symmetrize) {
    // Transpose: stable radix sort of (column, position) -> per-column source rows ascending.
    DevBuf<uint32_t> tkeys(nnz_dir, s), tvals(nnz_dir, s);
    radix_sort_pairs(keys.p, vals.p, tkeys.p, tvals.p, nnz_dir, bits_for(n ? n - 1 : 0), s);
    keys.reset();
    vals.reset();
    DevBuf<uint64_t> tptr(n + 1, s);
    segment_starts(tkeys.p, nnz_dir, n, tptr.p, s);
    tkeys.reset();
    DevBuf<uint32_t> ucnt(n, s);
    union_rows(pcol.p, pw.p, cnt.p, k, tptr.p, tvals.p, n, gp, ucnt.p, nullptr, nullptr, nullptr,
               false, s);
    m->indptr.alloc(n + 1, s);
    scan_u32_to_u64(ucnt.p, m->indptr.p, n, s);
    d2h(&m->nnz, m->indptr.p + n, 1, s);
    UB_CUDA(cudaStreamSynchronize(s));
    m->indices.alloc(m->nnz, s);
    m->data.alloc(m->nnz, s);
    union_rows(pcol.p, pw.p, cnt.p, k, tptr.p, tvals.p, n, gp, nullptr, m->indptr.p, m->indices.p,
               m->data.p, true, s);
    log.mark("set_operations complete");
  } else {
    m->nnz = nnz_dir;
    m->indptr = std::move(dptr);
    m->indices = std::move(keys);
    m->data.alloc(nnz_dir, s);
    gather_weights(pw.p, vals.p, nnz_dir, m->data.p, s);
  }
  count_empty_rows(m->indptr.p, m->data.p, n, dcount.p + 1, s);
  unsigned long long counts[2];
  d2h(counts, dcount.p, 2, s);
  UB_CUDA(cudaStreamSynchronize(s));
  m->edges_removed = counts[0];
  m->vertices_disconnected = counts[1];
  log.mark("disconnected vertex count complete");
  if (getenv("UMAP_B200_LOG")) {  // raise_disconnected_warning.rs:4-26 (counts only)
    fprintf(stderr, "[umap_b200] learn_manifold: n=%llu nnz=%llu edges_removed=%llu vertices_disconnected=%llu\n",
            (unsigned long long)n, (unsigned long long)m->nnz, counts[0], counts[1]);
  }
  return m;
}

std::unique_ptr<umap_manifold> clone_manifold(const umap_manifold& src) {
  auto m = std::make_unique<umap_manifold>();
  m->stream = std::make_unique<Stream>();
  cudaStream_t s = m->s();
  UB_CUDA(cudaStreamSynchronize(src.s()));
  m->n_vertices = src.n_vertices;
  m->nnz = src.nnz;
  m->a = src.a;
  m->b = src.b;
  m->edges_removed = src.edges_removed;
  m->vertices_disconnected = src.vertices_disconnected;
  m->indptr.alloc(src.n_vertices + 1, s);
  m->indices.alloc(src.nnz, s);
  m->data.alloc(src.nnz, s);
  m->sigmas.alloc(src.n_vertices, s);
  m->rhos.alloc(src.n_vertices, s);
  d2d(m->indptr.p, src.indptr.p, src.n_vertices + 1, s);
  d2d(m->indices.p, src.indices.p, src.nnz, s);
  d2d(m->data.p, src.data.p, src.nnz, s);
  d2d(m->sigmas.p, src.sigmas.p, src.n_vertices, s);
  d2d(m->rhos.p, src.rhos.p, src.n_vertices, s);
  UB_CUDA(cudaStreamSynchronize(s));
  return m;
}

// ------------------------------------------------------------------ Optimizer
// Optimizers on each device that currently hold a persisting-L2 window.  The set-aside
// (cudaLimitPersistingL2CacheSize) is device-wide and outlives the stream, so it is handed
// back, and lines still marked persisting are reset to normal, when the last holder on the
// device is consumed (into_fitted) or freed: the host application's own kernels then get
// the whole L2 again.
std::mutex g_l2_mu;
std::map<int, int> g_l2_holders;

void release_l2_window(umap_optimizer& o) noexcept {
  if (!o.l2_window) return;
  o.l2_window = false;
  int prev = -1;
  (void)cudaGetDevice(&prev);
  const int dev = o.manifold->stream->device;
  (void)cudaSetDevice(dev);
  cudaStreamAttrValue attr;
  memset(&attr, 0, sizeof attr);
  (void)cudaStreamSetAttribute(o.s(), cudaStreamAttributeAccessPolicyWindow, &attr);
  std::lock_guard<std::mutex> lock(g_l2_mu);
  if (--g_l2_holders[dev] <= 0) {
    g_l2_holders.erase(dev);
    (void)cudaStreamSynchronize(o.s());
    (void)cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    (void)cudaCtxResetPersistingL2Cache();
  }
  (void)cudaGetLastError();
  if (prev >= 0 && prev != dev) (void)cudaSetDevice(prev);
}

void set_l2_window(umap_optimizer& o, bool enable) {
  static const bool disabled = [] {
    const char* e = getenv("UMAP_B200_L2_PERSIST");
    return e && e[0] == '0';
  }();
  if (!enable) {
    release_l2_window(o);
    return;
  }
  cudaStreamAttrValue attr;
  memset(&attr, 0, sizeof attr);
  if (!disabled && o.emb2.p) {
    int dev = o.manifold->stream->device, max_persist = 0, max_window = 0;
    UB_CUDA(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev));
    UB_CUDA(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev));
    if (max_persist <= 0 || max_window <= 0) return;
    const size_t bytes = o.emb2.bytes();
    // Only an embedding pair that can persist whole gets a window.  A larger one (the
    // DRAM-bound, renamed layouts) is read in another vertex order during the epochs, and the
    // lines its gather marks persisting would hold the set-aside unused: renamed 20M / 40M-point
    // rolls ran 7-9% faster without it (30 epochs 239.0-239.4 -> 222.3-223.7 ms; 24 epochs
    // 475.8-476.2 -> 431.5 ms), and a window moved onto the working snapshot changed nothing.
    if (bytes > (size_t)max_persist) return;
    const size_t lim = std::min(bytes, (size_t)max_persist);
    {
      std::lock_guard<std::mutex> lock(g_l2_mu);
      if (!o.l2_window) ++g_l2_holders[dev];
      o.l2_window = true;
    }
    UB_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, lim));
    attr.accessPolicyWindow.base_ptr = o.emb2.p;
    attr.accessPolicyWindow.num_bytes = std::min(bytes, (size_t)max_window);
    attr.accessPolicyWindow.hitRatio =
        (float)std::min(1.0, (double)lim / (double)attr.accessPolicyWindow.num_bytes);
    attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  }
  UB_CUDA(cudaStreamSetAttribute(o.s(), cudaStreamAttributeAccessPolicyWindow, &attr));
}

// Kept edges in the reference's order (optimizer.rs:85-172).
struct KeptEdges {
  uint64_t E = 0;
  DevBuf<uint64_t> ptr;
  DevBuf<uint32_t> tail;
  DevBuf<double> eps;
};

void compute_kept_edges(const umap_optimizer& o, KeptEdges& K, bool want_tail, bool want_eps) {
  const umap_manifold& m = *o.manifold;
  cudaStream_t s = o.s();
  SegmentPrune sp;
  if (o.n_seg) {
    sp.seg_thr = o.seg_thr.p;
    sp.seg_maxw = o.seg_maxw.p;
    sp.row_seg = o.row_seg.p;
  }
  const SegmentPrune* spp = o.n_seg ? &sp : nullptr;
  K.ptr.alloc(m.n_vertices + 1, s);
  prune_edges(m.indptr.p, m.data.p, m.n_vertices, o.threshold, K.ptr.p, &K.E, s, spp);
  if (want_tail) K.tail.alloc(K.E, s);
  if (want_eps) K.eps.alloc(K.E, s);
  export_edges(m.indptr.p, m.indices.p, m.data.p, m.n_vertices, o.threshold, o.max_w, o.total_epochs,
               K.ptr.p, nullptr, want_tail ? K.tail.p : nullptr, want_eps ? K.eps.p : nullptr, s, spp);
}

// optimizer.rs:90-102 (prune threshold) and make_epochs_per_sample.rs:26-32 (max over kept
// weights: max_val itself is kept) from the manifold's graph and total_epochs.
void compute_thresholds(umap_optimizer& o) {
  cudaStream_t s = o.s();
  const uint64_t n = o.manifold->n_vertices;
  DevBuf<float> dmax(1, s);
  reduce_max_f32(o.manifold->data.p, o.manifold->nnz, 0.0f, dmax.p, s);
  float max_val = 0.0f;
  d2h(&max_val, dmax.p, 1, s);
  UB_CUDA(cudaStreamSynchronize(s));
  const uint64_t default_epochs = n <= 10000 ? 500 : 200;
  const uint64_t threshold_epochs = o.total_epochs > 10 ? o.total_epochs : default_epochs;
  o.max_val = max_val;
  o.threshold = max_val / (float)threshold_epochs;
  o.max_w = (o.manifold->nnz > 0 && max_val > 0.0f) ? max_val : 1.0f;
}

// optimizer.rs:74-290.  `init` is a device array of n*dim floats on stream `s` (or host).
// Optimizer::new up to, not including, the initial embedding (optimizer.rs:74-180): nothing
// here depends on `init`, so a caller that computes init meanwhile can run this first.
std::unique_ptr<umap_optimizer> optimizer_prepare_impl(std::unique_ptr<umap_manifold> man, uint64_t rows,
                                                       uint64_t dims, uint64_t total_epochs, const umap_config& c,
                                                       int metric_type);
// optimizer.rs:181-230 on a prepared optimizer: the initial embedding, normalised.
void optimizer_set_init_impl(umap_optimizer& o, const float* init, bool init_on_host);

std::unique_ptr<umap_optimizer> optimizer_new_impl(std::unique_ptr<umap_manifold> man, const float* init,
                                                   bool init_on_host, uint64_t rows, uint64_t dims,
                                                   uint64_t total_epochs, const umap_config& c,
                                                   int metric_type) {
  auto o = optimizer_prepare_impl(std::move(man), rows, dims, total_epochs, c, metric_type);
  optimizer_set_init_impl(*o, init, init_on_host);
  return o;
}

std::unique_ptr<umap_optimizer> optimizer_prepare_impl(std::unique_ptr<umap_manifold> man, uint64_t rows,
                                                       uint64_t dims, uint64_t total_epochs, const umap_config& c,
                                                       int metric_type) {
  if (metric_type != UMAP_METRIC_EUCLIDEAN && metric_type != UMAP_METRIC_GENERIC)
    throw Error(INVALID_ARGUMENT, "unknown metric_type");
  if (rows != man->n_vertices)
    throw Error(INVALID_ARGUMENT, "init has " + std::to_string(rows) + " samples but data has " +
                                      std::to_string(man->n_vertices) + " samples");
  if (dims < 1) throw Error(INVALID_ARGUMENT, "n_components must be >= 1, got 0");
  if (man->n_vertices >= 0xFFFFFFFFull) throw Error(UNSUPPORTED, "n_vertices must be < 2^32");
  if ((total_epochs + 1) * (c.negative_sample_rate + 1) >= 0xFFFFFFFFull)
    throw Error(UNSUPPORTED, "total_epochs * negative_sample_rate must be < 2^32");
  if (total_epochs > MAX_EPOCHS)
    throw Error(UNSUPPORTED, "total_epochs must be at most " + std::to_string(MAX_EPOCHS) + " on this build");
  auto o = std::make_unique<umap_optimizer>();
  o->manifold = std::move(man);
  cudaStream_t s = o->s();
  o->gamma = c.repulsion_strength;
  o->initial_alpha = c.learning_rate;
  o->negative_sample_rate = c.negative_sample_rate;
  o->metric_type = metric_type;
  o->n = rows;
  o->dim = dims;
  o->total_epochs = total_epochs;
  o->current_epoch = 0;
  const uint64_t n = o->manifold->n_vertices;

  // :90-102 threshold
  PhaseLog log(s);
  compute_thresholds(*o);
  log.mark("optimizer threshold computed");

  {
    KeptEdges K;
    compute_kept_edges(*o, K, true, true);
    log.mark("optimizer edge filtering + epochs_per_sample complete");
    const bool generic = o->metric_type == UMAP_METRIC_GENERIC;
    build_sgd_layout(K.ptr.p, K.tail.p, K.eps.p, n, generic ? pick_chunk_generic(K.E) : 0, o->layout, s, nullptr,
                     !generic);
    log.mark("optimizer task layout complete");
  }
  if (log.on)
    fprintf(stderr, "[umap_b200] edges=%llu tasks=%llu split_tasks=%llu chunk=%u max_degree=%u entries=%llu\n",
            (unsigned long long)o->layout.n_edges, (unsigned long long)o->layout.n_tasks,
            (unsigned long long)o->layout.split_tasks, o->layout.chunk, o->layout.max_degree,
            (unsigned long long)o->layout.n_entries);
  UB_CUDA(cudaStreamSynchronize(s));
  return o;
}

void optimizer_set_init_impl(umap_optimizer& o, const float* init, bool init_on_host) {
  cudaStream_t s = o.s();
  const uint64_t n = o.n, dims = o.dim;
  PhaseLog log(s);
  o.emb2.alloc(2 * n * dims, s);
  if (init_on_host) h2d(o.emb2.p, init, n * dims, s);
  else d2d(o.emb2.p, init, n * dims, s);
  normalize_init(o.emb2.p, n, (uint32_t)dims, s);
  log.mark("optimizer embedding normalization complete");
  set_l2_window(o, true);
  UB_CUDA(cudaStreamSynchronize(s));
}

SgdParams sgd_params(const umap_optimizer& o) {
  SgdParams p{};
  p.a = o.manifold->a;
  p.b = o.manifold->b;
  p.gamma = o.gamma;
  p.neg_attr = (-2.0f * p.a) * p.b;     // optimize_layout_euclidean.rs:292
  p.pos_rep = (2.0f * p.gamma) * p.b;   // :329
  p.neg_rate = (uint32_t)o.negative_sample_rate;
  p.n_vertices = (uint32_t)o.manifold->n_vertices;
  p.dim = (uint32_t)o.dim;
  p.seed = o.seed;
  p.row_seg = o.n_seg ? o.row_seg.p : nullptr;
  p.seg_off = o.n_seg ? o.seg_off.p : nullptr;
  p.generic_metric = o.metric_type == UMAP_METRIC_GENERIC ? 1u : 0u;
  p.two_b = 2.0f * p.b;                 // optimize_layout_generic.rs:72, :76
  return p;
}

// optimizer.rs:297-366.  `output_metric` is the device id of the metric the reference passes
// to step_epochs; like the reference, the Euclidean specialisation ignores it, and the generic
// path needs one with a device implementation.
void step_epochs_impl(umap_optimizer& o, uint64_t n_ep, int output_metric = UMAP_OUTPUT_METRIC_EUCLIDEAN) {
  if (o.current_epoch + n_ep > o.total_epochs)
    throw Error(OVERSTEP, "Cannot step " + std::to_string(n_ep) + " epochs: would exceed total_epochs " +
                              std::to_string(o.total_epochs) + " (current: " +
                              std::to_string(o.current_epoch) + ")");
  if (o.metric_type == UMAP_METRIC_GENERIC && output_metric != UMAP_OUTPUT_METRIC_EUCLIDEAN)
    throw Error(UNSUPPORTED, "output metric " + std::to_string(output_metric) +
                                 " has no device implementation (built in: 0 = Euclidean)");
  cudaStream_t s = o.s();
  const uint64_t nd = o.n * o.dim;
  float* live = o.emb2.p;
  float* snap = o.emb2.p + nd;
  // A layout with renamed vertices runs the epochs on a working pair in its own vertex order
  // (gathered here, scattered back below); the optimizer's embedding keeps the caller's order.
  DevBuf<float> work;
  if (o.layout.order.p) {
    work.alloc(2 * nd, s);
    permute_rows(o.emb2.p, o.layout.order.p, o.n, (uint32_t)o.dim, true, work.p, s);
    live = work.p;
    snap = work.p + nd;
  }
  d2d(snap, live, nd, s);  // :314 embedding_copy
  const SgdParams p = sgd_params(o);
  cudaEvent_t ev[2];
  UB_CUDA(cudaEventCreate(&ev[0]));
  UB_CUDA(cudaEventCreate(&ev[1]));
  // The epoch loop is captured into a CUDA graph (one kernel node per epoch, each with its
  // own epoch and learning rate) and launched once.
  static const bool no_graph = [] {
    const char* e = getenv("UMAP_B200_GRAPH");
    return e && e[0] == '0';
  }();
  // Worth it where launches are a visible share of an epoch: batches and small graphs.
  const bool use_graph = !no_graph && n_ep >= 2 && o.layout.n_slices > 0 &&
                         (o.n_seg > 0 || o.layout.n_edges < (8ull << 20));
  cudaGraphExec_t exec = nullptr;
  if (use_graph) {
    cudaGraph_t graph = nullptr;
    UB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      for (uint64_t epoch = o.current_epoch; epoch < o.current_epoch + n_ep; ++epoch) {
        const float alpha = o.initial_alpha * (1.0f - ((float)epoch / (float)o.total_epochs));  // :317
        sgd_epoch(o.layout, live, snap, p, (uint32_t)epoch, alpha, s);
      }
    } catch (...) {
      cudaGraph_t g2 = nullptr;
      (void)cudaStreamEndCapture(s, &g2);
      if (g2) (void)cudaGraphDestroy(g2);
      (void)cudaGetLastError();
      throw;
    }
    UB_CUDA(cudaStreamEndCapture(s, &graph));
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    (void)cudaGraphDestroy(graph);
    UB_CUDA(ie);
  }
  UB_CUDA(cudaEventRecord(ev[0], s));
  if (use_graph) {
    cudaError_t le = cudaGraphLaunch(exec, s);
    if (le != cudaSuccess) (void)cudaGraphExecDestroy(exec);
    UB_CUDA(le);
  } else {
    for (uint64_t epoch = o.current_epoch; epoch < o.current_epoch + n_ep; ++epoch) {
      const float alpha = o.initial_alpha * (1.0f - ((float)epoch / (float)o.total_epochs));  // :317
      sgd_epoch(o.layout, live, snap, p, (uint32_t)epoch, alpha, s);
    }
  }
  UB_CUDA(cudaEventRecord(ev[1], s));
  if (work.p) permute_rows(live, o.layout.order.p, o.n, (uint32_t)o.dim, false, o.emb2.p, s);
  cudaError_t se = cudaStreamSynchronize(s);
  if (exec) (void)cudaGraphExecDestroy(exec);
  UB_CUDA(se);
  float ms = 0.0f;
  (void)cudaEventElapsedTime(&ms, ev[0], ev[1]);
  (void)cudaEventDestroy(ev[0]);
  (void)cudaEventDestroy(ev[1]);
  o.last_step_ms = ms;
  if (getenv("UMAP_B200_LOG"))
    fprintf(stderr, "[umap_b200] duration_ms=%.3f step_epochs %llu epochs (%.4f ms/epoch)\n", ms,
            (unsigned long long)n_ep, n_ep ? ms / n_ep : 0.0);
  o.current_epoch += n_ep;
}

std::unique_ptr<umap_fitted> into_fitted_impl(std::unique_ptr<umap_optimizer> o, const umap_config& c) {
  auto f = std::make_unique<umap_fitted>();
  cudaStream_t s = o->s();
  set_l2_window(*o, false);
  f->n = o->n;
  f->dim = o->dim;
  f->embedding.alloc(o->n * o->dim, s);
  d2d(f->embedding.p, o->emb2.p, o->n * o->dim, s);
  f->config = c;
  o->emb2.reset();
  o->layout = SgdLayout();
  f->manifold = std::move(o->manifold);
  UB_CUDA(cudaStreamSynchronize(f->s()));
  return f;
}

// embedding.rs:299-337: the rest of Umap::fit once the manifold is learned.
std::unique_ptr<umap_fitted> fit_manifold_impl(const umap_config& c, std::unique_ptr<umap_manifold> m,
                                               const float* init, uint64_t irows, uint64_t icols, bool host,
                                               int metric_type = UMAP_METRIC_EUCLIDEAN,
                                               int output_metric = UMAP_OUTPUT_METRIC_EUCLIDEAN) {
  const uint64_t n_samples = m->n_vertices;
  if (icols != c.n_components)
    throw Error(INVALID_ARGUMENT, "init has " + std::to_string(icols) + " components but n_components is " +
                                      std::to_string(c.n_components));
  if (irows != n_samples)
    throw Error(INVALID_ARGUMENT, "init has " + std::to_string(irows) + " samples but data has " +
                                      std::to_string(n_samples) + " samples");
  const uint64_t total = c.has_n_epochs ? c.n_epochs : (n_samples <= 10000 ? 500 : 200);  // :304-308
  if (metric_type == UMAP_METRIC_GENERIC && output_metric != UMAP_OUTPUT_METRIC_EUCLIDEAN)
    throw Error(UNSUPPORTED, "output metric " + std::to_string(output_metric) +
                                 " has no device implementation (built in: 0 = Euclidean)");
  auto o = optimizer_new_impl(std::move(m), init, host, irows, icols, total, c, metric_type);  // :311-319
  step_epochs_impl(*o, total, output_metric);  // :321
  auto f = into_fitted_impl(std::move(o), c);
  nan_empty_rows(f->manifold->indptr.p, f->n, (uint32_t)f->dim, f->embedding.p, f->s());  // :327-334
  UB_CUDA(cudaStreamSynchronize(f->s()));
  return f;
}

std::unique_ptr<umap_fitted> fit_impl(const umap_config& c, uint64_t n_samples, const uint32_t* idx,
                                      const float* dist, uint64_t rows, uint64_t cols, const float* init,
                                      uint64_t irows, uint64_t icols, bool host) {
  // embedding.rs:284-297
  if (icols != c.n_components)
    throw Error(INVALID_ARGUMENT, "init has " + std::to_string(icols) + " components but n_components is " +
                                      std::to_string(c.n_components));
  if (irows != n_samples)
    throw Error(INVALID_ARGUMENT, "init has " + std::to_string(irows) + " samples but data has " +
                                      std::to_string(n_samples) + " samples");
  std::unique_ptr<umap_manifold> m;
  if (host) {
    std::string err = validate_parameters(c, n_samples, rows, cols);
    if (!err.empty()) throw Error(INVALID_ARGUMENT, err);
    // Upload on a temporary stream-ordered allocation of the manifold's future stream.
    cudaStream_t s0;
    UB_CUDA(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
    struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s0};
    DevBuf<uint32_t> di(rows * cols, s0);
    DevBuf<float> dd(rows * cols, s0);
    h2d(di.p, idx, rows * cols, s0);
    h2d(dd.p, dist, rows * cols, s0);
    UB_CUDA(cudaStreamSynchronize(s0));
    m = learn_manifold_impl(c, n_samples, di.p, dd.p, rows, cols);
    UB_CUDA(cudaStreamSynchronize(m->s()));
  } else {
    m = learn_manifold_impl(c, n_samples, idx, dist, rows, cols);
  }
  return fit_manifold_impl(c, std::move(m), init, irows, icols, host);
}

// ------------------------------------------------------------------ autotuning
// Picks the SGD task length ("edges per thread") and the block shape by timing a few
// epochs of each candidate on a scratch copy of the embedding.  Choices are cached per
// problem size (vertices, edges in MiB units, dims) for the life of the process.
struct TuneKey {
  uint64_t n, e_mib, dim;
  bool operator<(const TuneKey& o) const {
    return n != o.n ? n < o.n : e_mib != o.e_mib ? e_mib < o.e_mib : dim < o.dim;
  }
};
std::mutex& g_tune_mu = *new std::mutex;
std::map<TuneKey, std::pair<uint32_t, uint32_t>>& g_tuned = *new std::map<TuneKey, std::pair<uint32_t, uint32_t>>;

void tune_layout(umap_optimizer& o, const KeptEdges& K) {
  cudaStream_t s = o.s();
  const uint64_t n = o.manifold->n_vertices;
  const TuneKey key{n, K.E >> 20, o.dim};
  Segments sgs{o.n_seg, o.seg_off.p, o.row_seg.p};
  const Segments* seg_ptr = o.n_seg ? &sgs : nullptr;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      build_sgd_layout(K.ptr.p, K.tail.p, K.eps.p, n, it->second.first, o.layout, s, seg_ptr);
      o.layout.block_threads = it->second.second;
      return;
    }
  }
  const uint32_t chunks[] = {32, 64, 128, 256};
  const uint32_t blocks[] = {128, 256};
  const uint32_t mid = (uint32_t)std::max<uint64_t>(1, o.total_epochs / 2);
  DevBuf<float> scratch(2 * n * o.dim, s);
  d2d(scratch.p, o.emb2.p, n * o.dim, s);
  d2d(scratch.p + n * o.dim, o.emb2.p, n * o.dim, s);
  const SgdParams p = sgd_params(o);
  cudaEvent_t e0, e1;
  UB_CUDA(cudaEventCreate(&e0));
  UB_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  uint32_t best_chunk = 0, best_bt = 256;
  for (uint32_t ch : chunks) {
    SgdLayout L;
    build_sgd_layout(K.ptr.p, K.tail.p, K.eps.p, n, ch, L, s, seg_ptr);
    for (uint32_t bt : blocks) {
      L.block_threads = bt;
      sgd_epoch(L, scratch.p, scratch.p + n * o.dim, p, mid, 0.5f, s);  // warm-up
      UB_CUDA(cudaEventRecord(e0, s));
      for (int r = 0; r < 2; ++r) sgd_epoch(L, scratch.p, scratch.p + n * o.dim, p, mid + r, 0.5f, s);
      UB_CUDA(cudaEventRecord(e1, s));
      UB_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      UB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        best_chunk = ch;
        best_bt = bt;
      }
    }
  }
  (void)cudaEventDestroy(e0);
  (void)cudaEventDestroy(e1);
  build_sgd_layout(K.ptr.p, K.tail.p, K.eps.p, n, best_chunk, o.layout, s, seg_ptr);
  o.layout.block_threads = best_bt;
  if (getenv("UMAP_B200_LOG"))
    fprintf(stderr, "[umap_b200] autotune: chunk=%u block=%u (%.3f ms / 2 epochs)\n", best_chunk, best_bt, best);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned[key] = {best_chunk, best_bt};
}

// ------------------------------------------------------------------ batched instances
// Many independent UMAP fits in one problem: instance s owns points [off[s], off[s+1]) and
// its kNN ids are local to it.  The graph of the batch is block diagonal, so every
// row-local step (smooth-kNN, membership, transpose, union) is the plain one on global
// ids; the per-instance steps (distance-mean fallback, prune threshold, max weight, init
// normalisation, negative-sample range) use the instance tables.  Each epoch is one kernel
// launch over all instances.
std::unique_ptr<umap_optimizer> batch_new_impl(const umap_config& c, uint64_t n_inst, const uint64_t* h_off,
                                               const uint32_t* idx, const float* dist, uint64_t k,
                                               const float* init, uint64_t dims, uint64_t total_epochs,
                                               bool host) {
  if (n_inst == 0) throw Error(INVALID_ARGUMENT, "n_instances must be >= 1");
  if (n_inst >= 0xFFFFFFFFull) throw Error(UNSUPPORTED, "too many instances");
  if (h_off[0] != 0) throw Error(INVALID_ARGUMENT, "instance offsets must start at 0");
  for (uint64_t i = 0; i < n_inst; ++i) {
    if (h_off[i + 1] < h_off[i]) throw Error(INVALID_ARGUMENT, "instance offsets must be non-decreasing");
    const uint64_t ns = h_off[i + 1] - h_off[i];
    std::string err = validate_parameters(c, ns, ns, k);
    if (!err.empty()) throw Error(INVALID_ARGUMENT, "instance " + std::to_string(i) + ": " + err);
  }
  if (dims < 1) throw Error(INVALID_ARGUMENT, "n_components must be >= 1, got 0");
  const uint64_t N = h_off[n_inst];
  if (N >= 0xFFFFFFFFull || N * k >= 0xFFFFFFFFull)
    throw Error(UNSUPPORTED, "total points * n_neighbors must be < 2^32 on this build");
  if ((total_epochs + 1) * (c.negative_sample_rate + 1) >= 0xFFFFFFFFull)
    throw Error(UNSUPPORTED, "total_epochs * negative_sample_rate must be < 2^32");
  if (total_epochs > MAX_EPOCHS)
    throw Error(UNSUPPORTED, "total_epochs must be at most " + std::to_string(MAX_EPOCHS) + " on this build");

  cudaStream_t s0;
  UB_CUDA(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } guard{s0};
  DevBuf<uint64_t> seg_off(n_inst + 1, s0);
  DevBuf<uint32_t> row_seg(N, s0);
  h2d(seg_off.p, h_off, n_inst + 1, s0);
  fill_row_segments(seg_off.p, (uint32_t)n_inst, row_seg.p, s0);
  Segments sg{(uint32_t)n_inst, seg_off.p, row_seg.p};
  DevBuf<uint32_t> gidx(N * k, s0), hidx;
  DevBuf<float> hdist;
  const float* ddist = dist;
  if (host) {
    hidx.alloc(N * k, s0);
    hdist.alloc(N * k, s0);
    h2d(hidx.p, idx, N * k, s0);
    h2d(hdist.p, dist, N * k, s0);
    ddist = hdist.p;
    localize_knn(hidx.p, N, k, sg, gidx.p, s0);
  } else {
    localize_knn(idx, N, k, sg, gidx.p, s0);
  }
  UB_CUDA(cudaStreamSynchronize(s0));
  auto man = learn_manifold_impl(c, N, gidx.p, ddist, N, k, &sg);
  UB_CUDA(cudaStreamSynchronize(man->s()));

  auto o = std::make_unique<umap_optimizer>();
  o->manifold = std::move(man);
  cudaStream_t s = o->s();
  o->n_seg = (uint32_t)n_inst;
  o->seg_off = std::move(seg_off);
  o->seg_off.set_stream(s);
  o->row_seg = std::move(row_seg);
  o->row_seg.set_stream(s);
  o->gamma = c.repulsion_strength;
  o->initial_alpha = c.learning_rate;
  o->negative_sample_rate = c.negative_sample_rate;
  o->metric_type = UMAP_METRIC_EUCLIDEAN;
  o->n = N;
  o->dim = dims;
  o->total_epochs = total_epochs;
  o->current_epoch = 0;

  // per-instance threshold and max weight (optimizer.rs:90-102, make_epochs_per_sample.rs:26-32)
  DevBuf<float> smax(n_inst, s);
  segment_max(o->manifold->indptr.p, o->manifold->data.p, o->seg_off.p, (uint32_t)n_inst, smax.p, s);
  std::vector<float> hmax(n_inst), hthr(n_inst), hmw(n_inst);
  d2h(hmax.data(), smax.p, n_inst, s);
  UB_CUDA(cudaStreamSynchronize(s));
  for (uint64_t i = 0; i < n_inst; ++i) {
    const uint64_t ns = h_off[i + 1] - h_off[i];
    const uint64_t default_epochs = ns <= 10000 ? 500 : 200;
    const uint64_t threshold_epochs = total_epochs > 10 ? total_epochs : default_epochs;
    hthr[i] = hmax[i] / (float)threshold_epochs;
    hmw[i] = hmax[i] > 0.0f ? hmax[i] : 1.0f;
    o->max_val = std::max(o->max_val, hmax[i]);
  }
  o->seg_thr.alloc(n_inst, s);
  o->seg_maxw.alloc(n_inst, s);
  h2d(o->seg_thr.p, hthr.data(), n_inst, s);
  h2d(o->seg_maxw.p, hmw.data(), n_inst, s);
  UB_CUDA(cudaStreamSynchronize(s));

  o->emb2.alloc(2 * N * dims, s);
  if (host) h2d(o->emb2.p, init, N * dims, s);
  else d2d(o->emb2.p, init, N * dims, s);
  Segments so{(uint32_t)n_inst, o->seg_off.p, o->row_seg.p};
  normalize_init(o->emb2.p, N, (uint32_t)dims, s, &so);
  {
    KeptEdges K;
    compute_kept_edges(*o, K, true, true);
    static const bool no_tune = [] {
      const char* e = getenv("UMAP_B200_AUTOTUNE");
      return e && e[0] == '0';
    }();
    if (no_tune || total_epochs < 2) build_sgd_layout(K.ptr.p, K.tail.p, K.eps.p, N, 0, o->layout, s, &so);
    else tune_layout(*o, K);
  }
  set_l2_window(*o, true);
  UB_CUDA(cudaStreamSynchronize(s));
  return o;
}

uint64_t batch_epochs(const umap_config& c, uint64_t n_inst, const uint64_t* h_off) {
  if (c.has_n_epochs) return c.n_epochs;
  uint64_t e = 0;
  for (uint64_t i = 0; i < n_inst; ++i) {
    const uint64_t ns = h_off[i + 1] - h_off[i];
    const uint64_t d = ns <= 10000 ? 500 : 200;  // embedding.rs:304-308
    if (e && d != e)
      throw Error(UNSUPPORTED, "instances straddle 10,000 points, so their default epoch counts differ; "
                               "set optimization.n_epochs for a batched fit");
    e = d;
  }
  return e;
}

void batch_fit_impl(const umap_config& c, uint64_t n_inst, const uint64_t* h_off, const uint32_t* idx,
                    const float* dist, uint64_t k, const float* init, uint64_t icols, float* out, bool host) {
  if (icols != c.n_components)
    throw Error(INVALID_ARGUMENT, "init has " + std::to_string(icols) + " components but n_components is " +
                                      std::to_string(c.n_components));
  const uint64_t total = batch_epochs(c, n_inst, h_off);
  auto o = batch_new_impl(c, n_inst, h_off, idx, dist, k, init, icols, total, host);
  step_epochs_impl(*o, total);
  cudaStream_t s = o->s();
  nan_empty_rows(o->manifold->indptr.p, o->n, (uint32_t)o->dim, o->emb2.p, s);  // embedding.rs:327-334
  if (host) d2h(out, o->emb2.p, o->n * o->dim, s);
  else d2d(out, o->emb2.p, o->n * o->dim, s);
  UB_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------------ serialization
constexpr char MAGIC[8] = {'U', 'M', 'A', 'P', 'B', '2', '0', '0'};
constexpr uint32_t FORMAT_VERSION = 1;
enum Kind : uint32_t { KIND_MANIFOLD = 1, KIND_OPTIMIZER = 2, KIND_FITTED = 3 };

struct Writer {
  std::vector<uint8_t> b;
  void raw(const void* p, size_t n) {
    const uint8_t* c = (const uint8_t*)p;
    b.insert(b.end(), c, c + n);
  }
  template <class T>
  void put(T v) { raw(&v, sizeof v); }
};

struct Reader {
  const uint8_t* p;
  uint64_t n, off = 0;
  void raw(void* dst, uint64_t len) {
    if (len > n - off) throw Error(FORMAT, "checkpoint truncated");
    memcpy(dst, p + off, len);
    off += len;
  }
  template <class T>
  T get() {
    T v;
    raw(&v, sizeof v);
    return v;
  }
  uint64_t count(uint64_t elem_size) {
    uint64_t c = get<uint64_t>();
    if (elem_size && c > (n - off) / elem_size) throw Error(FORMAT, "checkpoint truncated (array length)");
    return c;
  }
};

void write_header(Writer& w, Kind k) {
  w.raw(MAGIC, 8);
  w.put<uint32_t>(FORMAT_VERSION);
  w.put<uint32_t>(k);
}
void read_header(Reader& r, Kind k) {
  char m[8];
  r.raw(m, 8);
  if (memcmp(m, MAGIC, 8) != 0) throw Error(FORMAT, "not a umap_b200 checkpoint (bad magic)");
  uint32_t v = r.get<uint32_t>();
  if (v != FORMAT_VERSION) throw Error(FORMAT, "unsupported checkpoint version " + std::to_string(v));
  uint32_t kk = r.get<uint32_t>();
  if (kk != k) throw Error(FORMAT, "checkpoint holds a different object kind");
}

template <class T>
void put_device_array(Writer& w, const T* dev, uint64_t n, cudaStream_t s) {
  w.put<uint64_t>(n);
  size_t at = w.b.size();
  w.b.resize(at + n * sizeof(T));
  d2h((T*)(w.b.data() + at), dev, n, s);
  UB_CUDA(cudaStreamSynchronize(s));
}
template <class T>
void get_device_array(Reader& r, DevBuf<T>& buf, uint64_t expect, cudaStream_t s) {
  uint64_t n = r.count(sizeof(T));
  if (expect != UINT64_MAX && n != expect) throw Error(FORMAT, "checkpoint array length mismatch");
  buf.alloc(n, s);
  if (n) {
    h2d(buf.p, (const T*)(r.p + r.off), n, s);
    UB_CUDA(cudaStreamSynchronize(s));
  }
  r.off += n * sizeof(T);
}

// LearnedManifold fields (manifold.rs:14-38): graph, sigmas, rhos, n_vertices, a, b.
void write_manifold(Writer& w, const umap_manifold& m) {
  cudaStream_t s = m.s();
  w.put<uint64_t>(m.n_vertices);  // graph shape (n, n)
  w.put<uint64_t>(m.n_vertices);
  put_device_array(w, m.indptr.p, m.n_vertices + 1, s);
  put_device_array(w, m.indices.p, m.nnz, s);
  put_device_array(w, m.data.p, m.nnz, s);
  put_device_array(w, m.sigmas.p, m.n_vertices, s);
  put_device_array(w, m.rhos.p, m.n_vertices, s);
  w.put<uint64_t>(m.n_vertices);
  w.put<float>(m.a);
  w.put<float>(m.b);
  w.put<uint64_t>(m.edges_removed);
  w.put<uint64_t>(m.vertices_disconnected);
}

std::unique_ptr<umap_manifold> read_manifold(Reader& r) {
  auto m = std::make_unique<umap_manifold>();
  m->stream = std::make_unique<Stream>();
  cudaStream_t s = m->s();
  uint64_t rows = r.get<uint64_t>(), cols = r.get<uint64_t>();
  if (rows != cols) throw Error(FORMAT, "graph must be square");
  get_device_array(r, m->indptr, rows + 1, s);
  get_device_array(r, m->indices, UINT64_MAX, s);
  m->nnz = m->indices.n;
  get_device_array(r, m->data, m->nnz, s);
  get_device_array(r, m->sigmas, rows, s);
  get_device_array(r, m->rhos, rows, s);
  m->n_vertices = r.get<uint64_t>();
  if (m->n_vertices != rows) throw Error(FORMAT, "n_vertices does not match the graph shape");
  m->a = r.get<float>();
  m->b = r.get<float>();
  m->edges_removed = r.get<uint64_t>();
  m->vertices_disconnected = r.get<uint64_t>();
  uint64_t last = 0;
  d2h(&last, m->indptr.p + rows, 1, s);
  UB_CUDA(cudaStreamSynchronize(s));
  if (last != m->nnz) throw Error(FORMAT, "graph indptr does not match nnz");
  return m;
}

void write_config(Writer& w, const umap_config& c) {
  w.put(c.n_components);
  w.put(c.min_dist); w.put(c.spread); w.put(c.has_a); w.put(c.a); w.put(c.has_b); w.put(c.b);
  w.put(c.n_neighbors); w.put(c.local_connectivity); w.put(c.set_op_mix_ratio);
  w.put(c.has_disconnection_distance); w.put(c.disconnection_distance); w.put(c.symmetrize);
  w.put(c.has_n_epochs); w.put(c.n_epochs); w.put(c.learning_rate); w.put(c.negative_sample_rate);
  w.put(c.repulsion_strength);
}
umap_config read_config(Reader& r) {
  umap_config c{};
  c.n_components = r.get<uint64_t>();
  c.min_dist = r.get<float>(); c.spread = r.get<float>(); c.has_a = r.get<int32_t>(); c.a = r.get<float>();
  c.has_b = r.get<int32_t>(); c.b = r.get<float>();
  c.n_neighbors = r.get<uint64_t>(); c.local_connectivity = r.get<float>(); c.set_op_mix_ratio = r.get<float>();
  c.has_disconnection_distance = r.get<int32_t>(); c.disconnection_distance = r.get<float>();
  c.symmetrize = r.get<int32_t>();
  c.has_n_epochs = r.get<int32_t>(); c.n_epochs = r.get<uint64_t>(); c.learning_rate = r.get<float>();
  c.negative_sample_rate = r.get<uint64_t>(); c.repulsion_strength = r.get<float>();
  return c;
}

// Common end of loading an optimizer: validate the edge list (row-major by head, heads and
// tails < n) on the host and rebuild the SGD layout from head / tail / epochs_per_sample (the
// schedule state follows from epochs_per_sample and current_epoch).
void finish_loaded_optimizer(umap_optimizer& o, const DevBuf<uint32_t>& head, const DevBuf<uint32_t>& tail,
                             const DevBuf<double>& eps) {
  cudaStream_t s = o.s();
  const uint64_t n = o.manifold->n_vertices, E = head.n;
  if (o.current_epoch > o.total_epochs) throw Error(FORMAT, "current_epoch exceeds total_epochs");
  if (o.total_epochs > MAX_EPOCHS)
    throw Error(UNSUPPORTED, "total_epochs must be at most " + std::to_string(MAX_EPOCHS) + " on this build");
  if (o.metric_type != UMAP_METRIC_EUCLIDEAN && o.metric_type != UMAP_METRIC_GENERIC)
    throw Error(FORMAT, "invalid MetricType");
  std::vector<uint32_t> hh(E), tt(E);
  d2h(hh.data(), head.p, E, s);
  d2h(tt.data(), tail.p, E, s);
  UB_CUDA(cudaStreamSynchronize(s));
  for (uint64_t i = 0; i < E; ++i) {
    if (hh[i] >= n || tt[i] >= n) throw Error(FORMAT, "edge index out of range");
    if (i && hh[i] < hh[i - 1]) throw Error(FORMAT, "edges are not ordered by head");
  }
  DevBuf<uint64_t> ptr(n + 1, s);
  segment_starts(head.p, E, n, ptr.p, s);
  const bool generic = o.metric_type == UMAP_METRIC_GENERIC;
  build_sgd_layout(ptr.p, tail.p, eps.p, n, generic ? pick_chunk_generic(E) : 0, o.layout, s, nullptr, !generic);
  set_l2_window(o, true);
  UB_CUDA(cudaStreamSynchronize(s));
}

// ---- the reference's own checkpoint bytes: serde derive + bincode 1.3 `serialize`
// bincode 1.3 (legacy options): little-endian fixed-width integers and floats, usize as u64,
// bool as u8, Option as a u8 tag then the value, a unit enum variant as its u32 index, a
// sequence as a u64 length then its elements, [T; N] as N elements, struct fields in
// declaration order with no names.  ndarray 0.17 serialises an array as the struct
// {v: u8 = 1, dim: [usize; D], data: sequence in logical (row-major) order}; sprs 0.11 a
// CsMatI as {storage: CompressedStorage (CSR = 0), nrows, ncols, indptr: {storage: Vec<usize>},
// indices: Vec<u32>, data: Vec<f32>}.  Those two crates are not in the reference tree, so this
// layout is restated from their published serde implementations.
constexpr uint8_t NDARRAY_FORMAT_VERSION = 1;

template <class T>
void bc_array1(Writer& w, const T* dev, uint64_t n, cudaStream_t s) {
  w.put<uint8_t>(NDARRAY_FORMAT_VERSION);
  w.put<uint64_t>(n);
  put_device_array(w, dev, n, s);
}
template <class T>
void bc_array2(Writer& w, const T* dev, uint64_t rows, uint64_t cols, cudaStream_t s) {
  w.put<uint8_t>(NDARRAY_FORMAT_VERSION);
  w.put<uint64_t>(rows);
  w.put<uint64_t>(cols);
  put_device_array(w, dev, rows * cols, s);
}
uint64_t bc_array_header(Reader& r, int ndim, uint64_t* dims) {
  if (r.get<uint8_t>() != NDARRAY_FORMAT_VERSION) throw Error(FORMAT, "unknown ndarray serialization version");
  uint64_t total = 1;
  for (int i = 0; i < ndim; ++i) {
    dims[i] = r.get<uint64_t>();
    if (dims[i] && total > UINT64_MAX / dims[i]) throw Error(FORMAT, "array shape overflows");
    total *= dims[i];
  }
  return total;
}
template <class T>
void bc_get_array1(Reader& r, DevBuf<T>& buf, uint64_t expect, cudaStream_t s) {
  uint64_t d;
  const uint64_t total = bc_array_header(r, 1, &d);
  if (expect != UINT64_MAX && total != expect) throw Error(FORMAT, "array length mismatch");
  get_device_array(r, buf, total, s);
}

// LearnedManifold (manifold.rs:14-38): graph, sigmas, rhos, n_vertices, a, b.
void bc_manifold(Writer& w, const umap_manifold& m) {
  cudaStream_t s = m.s();
  w.put<uint32_t>(0);  // CompressedStorage::CSR
  w.put<uint64_t>(m.n_vertices);
  w.put<uint64_t>(m.n_vertices);
  put_device_array(w, m.indptr.p, m.n_vertices + 1, s);
  put_device_array(w, m.indices.p, m.nnz, s);
  put_device_array(w, m.data.p, m.nnz, s);
  bc_array1(w, m.sigmas.p, m.n_vertices, s);
  bc_array1(w, m.rhos.p, m.n_vertices, s);
  w.put<uint64_t>(m.n_vertices);
  w.put<float>(m.a);
  w.put<float>(m.b);
}

std::unique_ptr<umap_manifold> bc_read_manifold(Reader& r) {
  if (r.get<uint32_t>() != 0) throw Error(FORMAT, "graph is not stored as CSR");
  const uint64_t rows = r.get<uint64_t>(), cols = r.get<uint64_t>();
  if (rows != cols) throw Error(FORMAT, "graph must be square");
  auto m = std::make_unique<umap_manifold>();
  m->stream = std::make_unique<Stream>();
  cudaStream_t s = m->s();
  get_device_array(r, m->indptr, rows + 1, s);
  get_device_array(r, m->indices, UINT64_MAX, s);
  m->nnz = m->indices.n;
  get_device_array(r, m->data, m->nnz, s);
  bc_get_array1(r, m->sigmas, rows, s);
  bc_get_array1(r, m->rhos, rows, s);
  m->n_vertices = r.get<uint64_t>();
  if (m->n_vertices != rows) throw Error(FORMAT, "n_vertices does not match the graph shape");
  m->a = r.get<float>();
  m->b = r.get<float>();
  std::vector<uint64_t> ip(rows + 1);
  std::vector<uint32_t> ix(m->nnz);
  d2h(ip.data(), m->indptr.p, rows + 1, s);
  d2h(ix.data(), m->indices.p, m->nnz, s);
  UB_CUDA(cudaStreamSynchronize(s));
  if (ip[0] != 0 || ip[rows] != m->nnz) throw Error(FORMAT, "graph indptr does not match nnz");
  for (uint64_t i = 0; i < rows; ++i)
    if (ip[i + 1] < ip[i]) throw Error(FORMAT, "graph indptr is not monotone");
  for (uint64_t q = 0; q < m->nnz; ++q)
    if (ix[q] >= cols) throw Error(FORMAT, "graph column index out of range");
  // not part of the reference's struct: the disconnection counts are recomputed
  DevBuf<unsigned long long> de(1, s);
  count_empty_rows(m->indptr.p, m->data.p, rows, de.p, s);
  unsigned long long v = 0;
  UB_CUDA(cudaMemcpyAsync(&v, de.p, 8, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  m->vertices_disconnected = v;
  m->edges_removed = 0;
  return m;
}

// UmapConfig (config.rs:8-235): n_components, manifold {min_dist, spread, a, b},
// graph {n_neighbors, local_connectivity, set_op_mix_ratio, disconnection_distance,
// symmetrize}, optimization {n_epochs, learning_rate, negative_sample_rate, repulsion_strength}.
void bc_config(Writer& w, const umap_config& c) {
  w.put<uint64_t>(c.n_components);
  w.put<float>(c.min_dist);
  w.put<float>(c.spread);
  w.put<uint8_t>(c.has_a ? 1 : 0);
  if (c.has_a) w.put<float>(c.a);
  w.put<uint8_t>(c.has_b ? 1 : 0);
  if (c.has_b) w.put<float>(c.b);
  w.put<uint64_t>(c.n_neighbors);
  w.put<float>(c.local_connectivity);
  w.put<float>(c.set_op_mix_ratio);
  w.put<uint8_t>(c.has_disconnection_distance ? 1 : 0);
  if (c.has_disconnection_distance) w.put<float>(c.disconnection_distance);
  w.put<uint8_t>(c.symmetrize ? 1 : 0);
  w.put<uint8_t>(c.has_n_epochs ? 1 : 0);
  if (c.has_n_epochs) w.put<uint64_t>(c.n_epochs);
  w.put<float>(c.learning_rate);
  w.put<uint64_t>(c.negative_sample_rate);
  w.put<float>(c.repulsion_strength);
}

umap_config bc_read_config(Reader& r) {
  auto tag = [&]() {
    const uint8_t t = r.get<uint8_t>();
    if (t > 1) throw Error(FORMAT, "invalid Option tag");
    return (int32_t)t;
  };
  umap_config c{};
  c.n_components = r.get<uint64_t>();
  c.min_dist = r.get<float>();
  c.spread = r.get<float>();
  if ((c.has_a = tag())) c.a = r.get<float>();
  if ((c.has_b = tag())) c.b = r.get<float>();
  c.n_neighbors = r.get<uint64_t>();
  c.local_connectivity = r.get<float>();
  c.set_op_mix_ratio = r.get<float>();
  if ((c.has_disconnection_distance = tag())) c.disconnection_distance = r.get<float>();
  const uint8_t sym = r.get<uint8_t>();
  if (sym > 1) throw Error(FORMAT, "invalid bool");
  c.symmetrize = sym;
  if ((c.has_n_epochs = tag())) c.n_epochs = r.get<uint64_t>();
  c.learning_rate = r.get<float>();
  c.negative_sample_rate = r.get<uint64_t>();
  c.repulsion_strength = r.get<float>();
  return c;
}

int copy_out(const Writer& w, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  if (needed) *needed = w.b.size();
  if (buf && cap) memcpy(buf, w.b.data(), std::min<uint64_t>(cap, w.b.size()));
  return (buf && cap < w.b.size()) ? UMAP_ERR_INVALID_ARGUMENT : UMAP_OK;
}

// ------------------------------------------------------------------ learned warm start
// Uniform floats in [0, 1) from a SplitMix64 stream (Steele, Lea, Flood, OOPSLA 2014): the
// network's initial parameters and the default subsample init.
struct HostUniform {
  uint64_t x;
  explicit HostUniform(uint64_t seed) : x(seed) {}
  float next() {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)(z >> 40) * (1.0f / 16777216.0f);
  }
};

// Flat parameters W1, b1, W2, b2, W3, b3 drawn like a default linear layer:
// U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases.
std::vector<float> mlp_initial_params(int in_dim, int out_dim, uint64_t seed) {
  std::vector<float> p;
  p.reserve((size_t)Mlp::param_count(in_dim, out_dim));
  HostUniform u(seed ^ 0x6D6C705F696E6974ull);
  const int fan[3][2] = {{in_dim, 256}, {256, 256}, {256, out_dim}};
  for (const auto& f : fan) {
    const float bound = 1.0f / sqrtf((float)f[0]);
    for (int i = 0; i < f[1] * f[0] + f[1]; ++i) p.push_back(bound * (2.0f * u.next() - 1.0f));
  }
  return p;
}

// The warm start's checks that need no device (run before the call touches the GPU).
void warm_start_check_args(const umap_config& c, const umap_warm_start_params& wp, uint64_t n, uint64_t d,
                           uint64_t k, uint64_t n_sub) {
  const uint64_t dim = c.n_components;
  if (d < 1 || d > 4096) throw Error(INVALID_ARGUMENT, "data_dim must be 1..4096, got " + std::to_string(d));
  if (dim < 1 || dim > 4) throw Error(INVALID_ARGUMENT, "the warm start's network predicts 1..4 components");
  if (n_sub < 128 || n_sub > n) throw Error(INVALID_ARGUMENT, "the subsample must have 128..n_samples rows");
  if (wp.sub_epochs < 1 || wp.epochs < 1 || wp.mlp_epochs < 1)
    throw Error(INVALID_ARGUMENT, "sub_epochs, epochs and mlp_epochs must be positive");
  std::string err = validate_parameters(c, n, n, k);
  if (!err.empty()) throw Error(INVALID_ARGUMENT, err);
}

std::unique_ptr<umap_fitted> warm_start_impl(const umap_config& c, const umap_warm_start_params& wp,
                                             const float* data, uint64_t n, uint64_t d, const uint32_t* idx,
                                             const float* dist, uint64_t k, const uint32_t* sub_rows,
                                             uint64_t n_sub, const uint32_t* sub_idx, const float* sub_dist,
                                             const float* sub_init, float* phase_ms, float* losses) {
  using clk = std::chrono::steady_clock;
  const auto ms_since = [](clk::time_point t) {
    return std::chrono::duration<float, std::milli>(clk::now() - t).count();
  };
  const uint64_t dim = c.n_components;
  warm_start_check_args(c, wp, n, d, k, n_sub);
  {  // the subsample's rows index the caller's data: every one must be a row of it
    std::vector<uint32_t> rows(n_sub);
    UB_CUDA(cudaMemcpy(rows.data(), sub_rows, n_sub * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < n_sub; ++i)
      if (rows[i] >= n)
        throw Error(INVALID_ARGUMENT, "sub_rows[" + std::to_string(i) + "] = " + std::to_string(rows[i]) +
                                          " is not a row of data (" + std::to_string(n) + " rows)");
  }
  int dev = 0;
  UB_CUDA(cudaGetDevice(&dev));
  float ph[UMAP_WARM_START_PHASES] = {};
  const auto t_start = clk::now();
  auto t0 = t_start;
  umap_config cfg_full = c;
  cfg_full.has_n_epochs = 1;
  cfg_full.n_epochs = wp.epochs;
  if (wp.has_learning_rate) cfg_full.learning_rate = wp.learning_rate;
  umap_config cfg_sub = c;
  cfg_sub.has_n_epochs = 1;
  cfg_sub.n_epochs = wp.sub_epochs;

  // The full graph and the final fit's optimizer set-up (prune, schedule, task layout) do not
  // depend on the initial embedding: built on their own stream and host thread while the
  // subsample is fitted and the network trained.
  std::unique_ptr<umap_optimizer> full;
  std::exception_ptr full_err;
  float full_ms = 0.0f;
  std::thread worker([&] {
    try {
      UB_CUDA(cudaSetDevice(dev));
      const auto tg = clk::now();
      full = optimizer_prepare_impl(learn_manifold_impl(cfg_full, n, idx, dist, n, k), n, dim, wp.epochs, cfg_full,
                                    UMAP_METRIC_EUCLIDEAN);
      UB_CUDA(cudaStreamSynchronize(full->s()));
      full_ms = ms_since(tg);
    } catch (...) {
      full_err = std::current_exception();
    }
  });
  struct Join {
    std::thread& t;
    ~Join() { if (t.joinable()) t.join(); }
  } join{worker};

  Stream st;
  cudaStream_t s = st.s;
  const uint64_t dp = (d + 63) / 64 * 64;
  DevBuf<float> sub(n_sub * dp, s);
  pad_gather_rows(data, d, dp, sub_rows, n_sub, sub.p, s);
  DevBuf<float> sinit;
  if (!sub_init) {
    std::vector<float> h(n_sub * dim);
    HostUniform u(wp.seed);
    for (float& v : h) v = -10.0f + 20.0f * u.next();
    sinit.alloc(n_sub * dim, s);
    h2d(sinit.p, h.data(), h.size(), s);
    sub_init = sinit.p;
  }
  UB_CUDA(cudaStreamSynchronize(s));
  ph[0] = ms_since(t0);
  t0 = clk::now();

  auto fsub = fit_impl(cfg_sub, n_sub, sub_idx, sub_dist, n_sub, k, sub_init, n_sub, dim, false);
  const float* y = fsub->embedding.p;
  // rows whose graph row is empty come back NaN: train on the others
  DevBuf<uint32_t> keep(n_sub, s);
  DevBuf<uint64_t> pos(n_sub + 1, s);
  finite_rows(y, n_sub, (uint32_t)dim, keep.p, s);
  scan_u32_to_u64(keep.p, pos.p, n_sub, s);
  uint64_t n_keep = 0;
  d2h(&n_keep, pos.p + n_sub, 1, s);
  UB_CUDA(cudaStreamSynchronize(s));
  DevBuf<float> xk, yk;
  const float* xt = sub.p;
  if (n_keep < n_sub) {
    xk.alloc(n_keep * dp, s);
    yk.alloc(n_keep * dim, s);
    compact_rows(sub.p, n_sub, dp, keep.p, pos.p, xk.p, s);
    compact_rows(y, n_sub, dim, keep.p, pos.p, yk.p, s);
    xt = xk.p;
    y = yk.p;
  }
  if (n_keep < 128) throw Error(INVALID_ARGUMENT, "fewer than 128 subsample rows have a non-empty graph row");
  UB_CUDA(cudaStreamSynchronize(s));
  ph[1] = ms_since(t0);
  t0 = clk::now();

  const std::vector<float> params = mlp_initial_params((int)dp, (int)dim, wp.seed);
  Mlp net((int)dp, (int)dim, params.data(), s);
  net.fit_input_norm(xt, (int64_t)n_keep);
  const uint64_t batch = std::min<uint64_t>(wp.batch, n_keep) / 128 * 128;
  std::vector<float> loss(wp.mlp_epochs);
  net.train(xt, y, (int64_t)n_keep, (int)wp.mlp_epochs, (int64_t)batch, wp.mlp_learning_rate, wp.seed, loss.data());
  if (losses) memcpy(losses, loss.data(), loss.size() * sizeof(float));
  UB_CUDA(cudaStreamSynchronize(s));
  ph[2] = ms_since(t0);
  t0 = clk::now();
  fsub.reset();
  xk.reset();
  yk.reset();
  sub.reset();

  DevBuf<float> xpad;
  const float* x = data;
  if (dp != d) {
    xpad.alloc(n * dp, s);
    pad_gather_rows(data, d, dp, nullptr, n, xpad.p, s);
    x = xpad.p;
  }
  DevBuf<float> init(n * dim, s);
  net.predict(x, (int64_t)n, init.p);
  UB_CUDA(cudaStreamSynchronize(s));
  xpad.reset();
  ph[3] = ms_since(t0);
  t0 = clk::now();

  worker.join();
  if (full_err) std::rethrow_exception(full_err);
  ph[4] = ms_since(t0);
  t0 = clk::now();
  // the rest of Umap::fit (embedding.rs:311-337) on the prepared optimizer
  optimizer_set_init_impl(*full, init.p, false);
  step_epochs_impl(*full, wp.epochs);
  auto fitted = into_fitted_impl(std::move(full), cfg_full);
  nan_empty_rows(fitted->manifold->indptr.p, fitted->n, (uint32_t)fitted->dim, fitted->embedding.p, fitted->s());
  UB_CUDA(cudaStreamSynchronize(fitted->s()));
  ph[5] = ms_since(t0);
  ph[6] = full_ms;
  ph[7] = ms_since(t_start);
  if (phase_ms) memcpy(phase_ms, ph, sizeof ph);
  return fitted;
}

}  // namespace
}  // namespace ub

using namespace ub;

// =================================================================== C ABI
extern "C" {

const char* umap_last_error(void) { return ub::g_last_error.c_str(); }
int umap_abi_version(void) { return UMAP_B200_ABI_VERSION; }

int umap_config_default(umap_config* out) {
  API_BEGIN
  need(out, "out");
  memset(out, 0, sizeof *out);
  out->n_components = 2;
  out->min_dist = 0.1f;
  out->spread = 1.0f;
  out->n_neighbors = 15;
  out->local_connectivity = 1.0f;
  out->set_op_mix_ratio = 1.0f;
  out->symmetrize = 1;
  out->learning_rate = 1.0f;
  out->negative_sample_rate = 5;
  out->repulsion_strength = 1.0f;
  API_END
}

int umap_find_ab_params(float spread, float min_dist, float* a_out, float* b_out) {
  API_BEGIN
  need(a_out, "a_out");
  need(b_out, "b_out");
  find_ab_params(spread, min_dist, a_out, b_out);
  API_END
}

int umap_learn_manifold(const umap_config* cfg, uint64_t n_samples, const uint32_t* idx, const float* dist,
                        uint64_t rows, uint64_t cols, umap_manifold** out) {
  API_BEGIN
  need(cfg, "cfg"); need(idx, "knn_indices"); need(dist, "knn_dists"); need(out, "out");
  *out = nullptr;
  std::string err = validate_parameters(*cfg, n_samples, rows, cols);
  if (!err.empty()) throw Error(INVALID_ARGUMENT, err);
  cudaStream_t s0;
  UB_CUDA(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s0};
  DevBuf<uint32_t> di(rows * cols, s0);
  DevBuf<float> dd(rows * cols, s0);
  h2d(di.p, idx, rows * cols, s0);
  h2d(dd.p, dist, rows * cols, s0);
  UB_CUDA(cudaStreamSynchronize(s0));
  auto m = learn_manifold_impl(*cfg, n_samples, di.p, dd.p, rows, cols);
  UB_CUDA(cudaStreamSynchronize(m->s()));
  *out = m.release();
  API_END
}

int umap_learn_manifold_device(const umap_config* cfg, uint64_t n_samples, const uint32_t* idx,
                               const float* dist, uint64_t rows, uint64_t cols, umap_manifold** out) {
  API_BEGIN
  need(cfg, "cfg"); need(idx, "knn_indices"); need(dist, "knn_dists"); need(out, "out");
  *out = nullptr;
  wait_for_inputs();
  auto m = learn_manifold_impl(*cfg, n_samples, idx, dist, rows, cols);
  *out = m.release();
  API_END
}

int umap_manifold_n_vertices(const umap_manifold* m, uint64_t* out) {
  API_BEGIN
  need(m, "manifold"); need(out, "out");
  *out = m->n_vertices;
  API_END
}

int umap_manifold_curve_params(const umap_manifold* m, float* a, float* b) {
  API_BEGIN
  need(m, "manifold"); need(a, "a"); need(b, "b");
  *a = m->a;
  *b = m->b;
  API_END
}

int umap_manifold_graph_nnz(const umap_manifold* m, uint64_t* nnz) {
  API_BEGIN
  need(m, "manifold"); need(nnz, "nnz");
  *nnz = m->nnz;
  API_END
}

int umap_manifold_graph_copy(const umap_manifold* m, uint64_t* indptr, uint32_t* indices, float* data) {
  API_BEGIN
  need(m, "manifold");
  m->stream->activate();
  if (indptr) d2h(indptr, m->indptr.p, m->n_vertices + 1, m->s());
  if (indices) d2h(indices, m->indices.p, m->nnz, m->s());
  if (data) d2h(data, m->data.p, m->nnz, m->s());
  m->stream->sync();
  API_END
}

int umap_manifold_sigmas_rhos(const umap_manifold* m, float* sigmas, float* rhos) {
  API_BEGIN
  need(m, "manifold");
  m->stream->activate();
  if (sigmas) d2h(sigmas, m->sigmas.p, m->n_vertices, m->s());
  if (rhos) d2h(rhos, m->rhos.p, m->n_vertices, m->s());
  m->stream->sync();
  API_END
}

int umap_manifold_disconnection_counts(const umap_manifold* m, uint64_t* edges_removed,
                                       uint64_t* vertices_disconnected) {
  API_BEGIN
  need(m, "manifold");
  if (edges_removed) *edges_removed = m->edges_removed;
  if (vertices_disconnected) *vertices_disconnected = m->vertices_disconnected;
  API_END
}

int umap_manifold_clone(const umap_manifold* m, umap_manifold** out) {
  API_BEGIN
  need(m, "manifold"); need(out, "out");
  *out = nullptr;
  m->stream->activate();
  *out = clone_manifold(*m).release();
  API_END
}

int umap_manifold_free(umap_manifold* m) {
  API_BEGIN
  if (m) {
    m->stream->activate();
    delete m;
  }
  API_END
}

int umap_optimizer_new(umap_manifold* manifold, const float* init, uint64_t rows, uint64_t dims,
                       uint64_t total_epochs, const umap_config* cfg, int metric_type, umap_optimizer** out) {
  std::unique_ptr<umap_manifold> owned(manifold);
  API_BEGIN
  need(manifold, "manifold"); need(init, "init"); need(cfg, "cfg"); need(out, "out");
  *out = nullptr;
  owned->stream->activate();
  *out = optimizer_new_impl(std::move(owned), init, true, rows, dims, total_epochs, *cfg, metric_type).release();
  API_END
}

int umap_optimizer_new_device(umap_manifold* manifold, const float* init, uint64_t rows, uint64_t dims,
                              uint64_t total_epochs, const umap_config* cfg, int metric_type,
                              umap_optimizer** out) {
  std::unique_ptr<umap_manifold> owned(manifold);
  API_BEGIN
  need(manifold, "manifold"); need(init, "init"); need(cfg, "cfg"); need(out, "out");
  *out = nullptr;
  owned->stream->activate();
  wait_for_inputs();
  *out = optimizer_new_impl(std::move(owned), init, false, rows, dims, total_epochs, *cfg, metric_type).release();
  API_END
}

int umap_optimizer_step_epochs(umap_optimizer* opt, uint64_t n) {
  API_BEGIN
  need(opt, "optimizer");
  opt->manifold->stream->activate();
  step_epochs_impl(*opt, n);
  API_END
}

int umap_optimizer_step_epochs_metric(umap_optimizer* opt, uint64_t n, int output_metric) {
  API_BEGIN
  need(opt, "optimizer");
  opt->manifold->stream->activate();
  step_epochs_impl(*opt, n, output_metric);
  API_END
}

int umap_optimizer_current_epoch(const umap_optimizer* opt, uint64_t* out) {
  API_BEGIN
  need(opt, "optimizer"); need(out, "out");
  *out = opt->current_epoch;
  API_END
}

int umap_optimizer_total_epochs(const umap_optimizer* opt, uint64_t* out) {
  API_BEGIN
  need(opt, "optimizer"); need(out, "out");
  *out = opt->total_epochs;
  API_END
}

int umap_optimizer_remaining_epochs(const umap_optimizer* opt, uint64_t* out) {
  API_BEGIN
  need(opt, "optimizer"); need(out, "out");
  *out = opt->total_epochs - opt->current_epoch;
  API_END
}

int umap_optimizer_embedding(const umap_optimizer* opt, float* out) {
  API_BEGIN
  need(opt, "optimizer"); need(out, "out");
  opt->manifold->stream->activate();
  d2h(out, opt->emb2.p, opt->n * opt->dim, opt->s());
  opt->manifold->stream->sync();
  API_END
}

int umap_optimizer_embedding_device(umap_optimizer* opt, float** dev_ptr) {
  API_BEGIN
  need(opt, "optimizer"); need(dev_ptr, "dev_ptr");
  *dev_ptr = opt->emb2.p;
  API_END
}

int umap_optimizer_dims(const umap_optimizer* opt, uint64_t* n_vertices, uint64_t* dims) {
  API_BEGIN
  need(opt, "optimizer");
  if (n_vertices) *n_vertices = opt->n;
  if (dims) *dims = opt->dim;
  API_END
}

int umap_optimizer_manifold(const umap_optimizer* opt, const umap_manifold** out) {
  API_BEGIN
  need(opt, "optimizer"); need(out, "out");
  *out = opt->manifold.get();
  API_END
}

int umap_optimizer_into_fitted(umap_optimizer* opt, const umap_config* cfg, umap_fitted** out) {
  std::unique_ptr<umap_optimizer> owned(opt);
  API_BEGIN
  need(opt, "optimizer"); need(cfg, "cfg"); need(out, "out");
  *out = nullptr;
  owned->manifold->stream->activate();
  *out = into_fitted_impl(std::move(owned), *cfg).release();
  API_END
}

int umap_optimizer_free(umap_optimizer* opt) {
  API_BEGIN
  if (opt) {
    opt->manifold->stream->activate();
    delete opt;
  }
  API_END
}

int umap_optimizer_set_seed(umap_optimizer* opt, uint64_t seed) {
  API_BEGIN
  need(opt, "optimizer");
  opt->seed = seed;
  API_END
}

int umap_optimizer_n_edges(const umap_optimizer* opt, uint64_t* out) {
  API_BEGIN
  need(opt, "optimizer"); need(out, "out");
  *out = opt->layout.n_edges;
  API_END
}

int umap_optimizer_export_edges(const umap_optimizer* opt, uint32_t* head, uint32_t* tail, double* eps,
                                double* eons, double* eonns, double* epns) {
  API_BEGIN
  need(opt, "optimizer");
  opt->manifold->stream->activate();
  cudaStream_t s = opt->s();
  KeptEdges K;
  compute_kept_edges(*opt, K, true, true);
  const uint64_t E = K.E;
  if (head) {
    DevBuf<uint32_t> h(E, s);
    head_from_ptr(K.ptr.p, opt->manifold->n_vertices, h.p, s);
    d2h(head, h.p, E, s);
    UB_CUDA(cudaStreamSynchronize(s));
  }
  if (tail) d2h(tail, K.tail.p, E, s);
  if (eps) d2h(eps, K.eps.p, E, s);
  if (eons || eonns || epns) {
    DevBuf<double> a(E, s), b(E, s), c(E, s);
    export_state(K.eps.p, E, opt->negative_sample_rate, opt->current_epoch, a.p, b.p, c.p, s);
    if (eons) d2h(eons, a.p, E, s);
    if (eonns) d2h(eonns, b.p, E, s);
    if (epns) d2h(epns, c.p, E, s);
    UB_CUDA(cudaStreamSynchronize(s));
  }
  UB_CUDA(cudaStreamSynchronize(s));
  API_END
}

int umap_optimizer_schedule_totals(const umap_optimizer* opt, uint64_t start, uint64_t end, uint64_t* fired,
                                   uint64_t* negatives) {
  API_BEGIN
  need(opt, "optimizer");
  opt->manifold->stream->activate();
  cudaStream_t s = opt->s();
  DevBuf<unsigned long long> d(2, s);
  schedule_totals(opt->layout, (uint32_t)opt->negative_sample_rate, (uint32_t)start, (uint32_t)end, d.p,
                  d.p + 1, s);
  unsigned long long h[2];
  d2h(h, d.p, 2, s);
  UB_CUDA(cudaStreamSynchronize(s));
  if (fired) *fired = h[0];
  if (negatives) *negatives = h[1];
  API_END
}

int umap_optimizer_last_step_ms(const umap_optimizer* opt, float* ms) {
  API_BEGIN
  need(opt, "optimizer"); need(ms, "ms");
  *ms = opt->last_step_ms;
  API_END
}

int umap_release_cached_memory(uint64_t* released_bytes) {
  API_BEGIN
  uint64_t b = release_cached_memory();
  if (released_bytes) *released_bytes = b;
  API_END
}

int umap_kernel_launches(uint64_t* out) {
  API_BEGIN
  need(out, "out");
  *out = ub::g_launches.load(std::memory_order_relaxed);
  API_END
}

int umap_fitted_embedding(const umap_fitted* f, float* out) {
  API_BEGIN
  need(f, "fitted"); need(out, "out");
  f->manifold->stream->activate();
  d2h(out, f->embedding.p, f->n * f->dim, f->s());
  f->manifold->stream->sync();
  API_END
}

int umap_fitted_dims(const umap_fitted* f, uint64_t* n_vertices, uint64_t* dims) {
  API_BEGIN
  need(f, "fitted");
  if (n_vertices) *n_vertices = f->n;
  if (dims) *dims = f->dim;
  API_END
}

int umap_fitted_manifold(const umap_fitted* f, const umap_manifold** out) {
  API_BEGIN
  need(f, "fitted"); need(out, "out");
  *out = f->manifold.get();
  API_END
}

int umap_fitted_config(const umap_fitted* f, umap_config* out) {
  API_BEGIN
  need(f, "fitted"); need(out, "out");
  *out = f->config;
  API_END
}

int umap_fitted_free(umap_fitted* f) {
  API_BEGIN
  if (f) {
    f->manifold->stream->activate();
    delete f;
  }
  API_END
}

int umap_fit(const umap_config* cfg, uint64_t n_samples, const uint32_t* idx, const float* dist, uint64_t rows,
             uint64_t cols, const float* init, uint64_t irows, uint64_t icols, umap_fitted** out) {
  API_BEGIN
  need(cfg, "cfg"); need(idx, "knn_indices"); need(dist, "knn_dists"); need(init, "init"); need(out, "out");
  *out = nullptr;
  *out = fit_impl(*cfg, n_samples, idx, dist, rows, cols, init, irows, icols, true).release();
  API_END
}

int umap_fit_device(const umap_config* cfg, uint64_t n_samples, const uint32_t* idx, const float* dist,
                    uint64_t rows, uint64_t cols, const float* init, uint64_t irows, uint64_t icols,
                    umap_fitted** out) {
  API_BEGIN
  need(cfg, "cfg"); need(idx, "knn_indices"); need(dist, "knn_dists"); need(init, "init"); need(out, "out");
  *out = nullptr;
  wait_for_inputs();
  *out = fit_impl(*cfg, n_samples, idx, dist, rows, cols, init, irows, icols, false).release();
  API_END
}

int umap_fit_manifold(umap_manifold* manifold, const umap_config* cfg, const float* init, uint64_t irows,
                      uint64_t icols, umap_fitted** out) {
  std::unique_ptr<umap_manifold> owned(manifold);
  API_BEGIN
  need(manifold, "manifold"); need(cfg, "cfg"); need(init, "init"); need(out, "out");
  *out = nullptr;
  owned->stream->activate();
  *out = fit_manifold_impl(*cfg, std::move(owned), init, irows, icols, true).release();
  API_END
}

int umap_fit_manifold_device(umap_manifold* manifold, const umap_config* cfg, const float* init, uint64_t irows,
                             uint64_t icols, umap_fitted** out) {
  std::unique_ptr<umap_manifold> owned(manifold);
  API_BEGIN
  need(manifold, "manifold"); need(cfg, "cfg"); need(init, "init"); need(out, "out");
  *out = nullptr;
  owned->stream->activate();
  wait_for_inputs();
  *out = fit_manifold_impl(*cfg, std::move(owned), init, irows, icols, false).release();
  API_END
}

int umap_fit_manifold_metric(umap_manifold* manifold, const umap_config* cfg, const float* init, uint64_t irows,
                             uint64_t icols, int metric_type, int output_metric, umap_fitted** out) {
  std::unique_ptr<umap_manifold> owned(manifold);
  API_BEGIN
  need(manifold, "manifold"); need(cfg, "cfg"); need(init, "init"); need(out, "out");
  *out = nullptr;
  if (metric_type != UMAP_METRIC_EUCLIDEAN && metric_type != UMAP_METRIC_GENERIC)
    throw Error(INVALID_ARGUMENT, "unknown metric_type");
  owned->stream->activate();
  *out = fit_manifold_impl(*cfg, std::move(owned), init, irows, icols, true, metric_type, output_metric).release();
  API_END
}

int umap_fit_manifold_metric_device(umap_manifold* manifold, const umap_config* cfg, const float* init,
                                    uint64_t irows, uint64_t icols, int metric_type, int output_metric,
                                    umap_fitted** out) {
  std::unique_ptr<umap_manifold> owned(manifold);
  API_BEGIN
  need(manifold, "manifold"); need(cfg, "cfg"); need(init, "init"); need(out, "out");
  *out = nullptr;
  if (metric_type != UMAP_METRIC_EUCLIDEAN && metric_type != UMAP_METRIC_GENERIC)
    throw Error(INVALID_ARGUMENT, "unknown metric_type");
  owned->stream->activate();
  wait_for_inputs();
  *out = fit_manifold_impl(*cfg, std::move(owned), init, irows, icols, false, metric_type, output_metric).release();
  API_END
}

// ---- checkpoints
int umap_manifold_serialize(const umap_manifold* m, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  API_BEGIN
  need(m, "manifold");
  m->stream->activate();
  Writer w;
  write_header(w, KIND_MANIFOLD);
  write_manifold(w, *m);
  int rc = copy_out(w, buf, cap, needed);
  if (rc) throw Error(rc, "buffer too small for the serialized manifold");
  API_END
}

int umap_manifold_deserialize(const uint8_t* buf, uint64_t len, umap_manifold** out) {
  API_BEGIN
  need(buf, "buf"); need(out, "out");
  *out = nullptr;
  Reader r{buf, len};
  read_header(r, KIND_MANIFOLD);
  auto m = read_manifold(r);
  if (r.off != len) throw Error(FORMAT, "trailing bytes after the manifold");
  *out = m.release();
  API_END
}

// Optimizer fields in the reference's declaration order (optimizer.rs:27-56), then this
// library's extensions (seed, max_val, threshold).
int umap_optimizer_serialize(const umap_optimizer* o, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  API_BEGIN
  need(o, "optimizer");
  if (o->n_seg) throw Error(UNSUPPORTED, "checkpoints of batched optimizers are not supported");
  o->manifold->stream->activate();
  cudaStream_t s = o->s();
  Writer w;
  write_header(w, KIND_OPTIMIZER);
  write_manifold(w, *o->manifold);
  KeptEdges K;
  compute_kept_edges(*o, K, true, true);
  const uint64_t E = K.E;
  {
    DevBuf<uint32_t> h(E, s);
    head_from_ptr(K.ptr.p, o->manifold->n_vertices, h.p, s);
    put_device_array(w, h.p, E, s);
  }
  put_device_array(w, K.tail.p, E, s);
  put_device_array(w, K.eps.p, E, s);
  w.put<uint64_t>(o->n);
  w.put<uint64_t>(o->dim);
  put_device_array(w, o->emb2.p, o->n * o->dim, s);
  {
    DevBuf<double> a(E, s), b(E, s), c(E, s);
    export_state(K.eps.p, E, o->negative_sample_rate, o->current_epoch, a.p, b.p, c.p, s);
    put_device_array(w, a.p, E, s);  // epoch_of_next_sample
    put_device_array(w, b.p, E, s);  // epoch_of_next_negative_sample
    put_device_array(w, c.p, E, s);  // epochs_per_negative_sample
  }
  w.put<uint64_t>(o->current_epoch);
  w.put<uint64_t>(o->total_epochs);
  w.put<float>(o->gamma);
  w.put<float>(o->initial_alpha);
  w.put<double>((double)o->negative_sample_rate);
  w.put<uint32_t>((uint32_t)o->metric_type);
  w.put<uint64_t>(o->seed);
  w.put<float>(o->max_val);
  w.put<float>(o->threshold);
  w.put<float>(o->max_w);
  int rc = copy_out(w, buf, cap, needed);
  if (rc) throw Error(rc, "buffer too small for the serialized optimizer");
  API_END
}

int umap_optimizer_deserialize(const uint8_t* buf, uint64_t len, umap_optimizer** out) {
  API_BEGIN
  need(buf, "buf"); need(out, "out");
  *out = nullptr;
  Reader r{buf, len};
  read_header(r, KIND_OPTIMIZER);
  auto o = std::make_unique<umap_optimizer>();
  o->manifold = read_manifold(r);
  cudaStream_t s = o->s();
  const uint64_t n = o->manifold->n_vertices;
  DevBuf<uint32_t> head, tail;
  DevBuf<double> eps;
  get_device_array(r, head, UINT64_MAX, s);
  const uint64_t E = head.n;
  get_device_array(r, tail, E, s);
  get_device_array(r, eps, E, s);
  o->n = r.get<uint64_t>();
  o->dim = r.get<uint64_t>();
  if (o->n != n || o->dim < 1 || o->dim > (1u << 20)) throw Error(FORMAT, "embedding shape mismatch");
  {
    DevBuf<float> e;
    get_device_array(r, e, n * o->dim, s);
    o->emb2.alloc(2 * n * o->dim, s);
    d2d(o->emb2.p, e.p, n * o->dim, s);
  }
  for (int t = 0; t < 3; ++t) {  // schedule state: recomputed from epochs_per_sample
    uint64_t c = r.count(8);
    if (c != E) throw Error(FORMAT, "schedule array length mismatch");
    r.off += c * 8;
  }
  o->current_epoch = r.get<uint64_t>();
  o->total_epochs = r.get<uint64_t>();
  o->gamma = r.get<float>();
  o->initial_alpha = r.get<float>();
  o->negative_sample_rate = (uint64_t)r.get<double>();
  o->metric_type = (int)r.get<uint32_t>();
  o->seed = r.get<uint64_t>();
  o->max_val = r.get<float>();
  o->threshold = r.get<float>();
  o->max_w = r.get<float>();
  if (r.off != len) throw Error(FORMAT, "trailing bytes after the optimizer");
  finish_loaded_optimizer(*o, head, tail, eps);
  *out = o.release();
  API_END
}

// FittedUmap fields (embedding.rs:438-443): embedding, manifold, config.
int umap_fitted_serialize(const umap_fitted* f, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  API_BEGIN
  need(f, "fitted");
  f->manifold->stream->activate();
  Writer w;
  write_header(w, KIND_FITTED);
  w.put<uint64_t>(f->n);
  w.put<uint64_t>(f->dim);
  put_device_array(w, f->embedding.p, f->n * f->dim, f->s());
  write_manifold(w, *f->manifold);
  write_config(w, f->config);
  int rc = copy_out(w, buf, cap, needed);
  if (rc) throw Error(rc, "buffer too small for the serialized fitted model");
  API_END
}

int umap_fitted_deserialize(const uint8_t* buf, uint64_t len, umap_fitted** out) {
  API_BEGIN
  need(buf, "buf"); need(out, "out");
  *out = nullptr;
  Reader r{buf, len};
  read_header(r, KIND_FITTED);
  auto f = std::make_unique<umap_fitted>();
  f->n = r.get<uint64_t>();
  f->dim = r.get<uint64_t>();
  if (f->dim > (1u << 20)) throw Error(FORMAT, "embedding shape mismatch");
  // The embedding precedes the manifold (which owns the stream): stage it on the host.
  uint64_t cnt = r.count(4);
  if (cnt != f->n * f->dim) throw Error(FORMAT, "embedding length mismatch");
  const float* host_emb = (const float*)(r.p + r.off);
  r.off += cnt * 4;
  f->manifold = read_manifold(r);
  f->config = read_config(r);
  if (r.off != len) throw Error(FORMAT, "trailing bytes after the fitted model");
  if (f->manifold->n_vertices != f->n) throw Error(FORMAT, "embedding rows do not match the manifold");
  f->embedding.alloc(cnt, f->s());
  std::vector<float> tmp(host_emb, host_emb + cnt);
  h2d(f->embedding.p, tmp.data(), cnt, f->s());
  UB_CUDA(cudaStreamSynchronize(f->s()));
  *out = f.release();
  API_END
}

// ---- checkpoints in the reference's own encoding (serde derive + bincode 1.3)
int umap_manifold_serialize_bincode(const umap_manifold* m, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  API_BEGIN
  need(m, "manifold");
  m->stream->activate();
  Writer w;
  bc_manifold(w, *m);
  int rc = copy_out(w, buf, cap, needed);
  if (rc) throw Error(rc, "buffer too small for the serialized manifold");
  API_END
}

int umap_manifold_deserialize_bincode(const uint8_t* buf, uint64_t len, umap_manifold** out) {
  API_BEGIN
  need(buf, "buf"); need(out, "out");
  *out = nullptr;
  Reader r{buf, len};
  auto m = bc_read_manifold(r);
  if (r.off != len) throw Error(FORMAT, "trailing bytes after the manifold");
  *out = m.release();
  API_END
}

// Optimizer (optimizer.rs:27-56): manifold, head, tail, epochs_per_sample, embedding,
// epoch_of_next_sample, epoch_of_next_negative_sample, epochs_per_negative_sample,
// current_epoch, total_epochs, gamma, initial_alpha, negative_sample_rate, metric_type.
int umap_optimizer_serialize_bincode(const umap_optimizer* o, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  API_BEGIN
  need(o, "optimizer");
  if (o->n_seg) throw Error(UNSUPPORTED, "checkpoints of batched optimizers are not supported");
  o->manifold->stream->activate();
  cudaStream_t s = o->s();
  Writer w;
  bc_manifold(w, *o->manifold);
  KeptEdges K;
  compute_kept_edges(*o, K, true, true);
  const uint64_t E = K.E;
  {
    DevBuf<uint32_t> h(E, s);
    head_from_ptr(K.ptr.p, o->manifold->n_vertices, h.p, s);
    bc_array1(w, h.p, E, s);
  }
  bc_array1(w, K.tail.p, E, s);
  bc_array1(w, K.eps.p, E, s);
  bc_array2(w, o->emb2.p, o->n, o->dim, s);
  {
    DevBuf<double> a(E, s), b(E, s), c(E, s);
    export_state(K.eps.p, E, o->negative_sample_rate, o->current_epoch, a.p, b.p, c.p, s);
    bc_array1(w, a.p, E, s);
    bc_array1(w, b.p, E, s);
    bc_array1(w, c.p, E, s);
  }
  w.put<uint64_t>(o->current_epoch);
  w.put<uint64_t>(o->total_epochs);
  w.put<float>(o->gamma);
  w.put<float>(o->initial_alpha);
  w.put<double>((double)o->negative_sample_rate);
  w.put<uint32_t>((uint32_t)o->metric_type);
  int rc = copy_out(w, buf, cap, needed);
  if (rc) throw Error(rc, "buffer too small for the serialized optimizer");
  API_END
}

int umap_optimizer_deserialize_bincode(const uint8_t* buf, uint64_t len, umap_optimizer** out) {
  API_BEGIN
  need(buf, "buf"); need(out, "out");
  *out = nullptr;
  Reader r{buf, len};
  auto o = std::make_unique<umap_optimizer>();
  o->manifold = bc_read_manifold(r);
  cudaStream_t s = o->s();
  const uint64_t n = o->manifold->n_vertices;
  DevBuf<uint32_t> head, tail;
  DevBuf<double> eps;
  bc_get_array1(r, head, UINT64_MAX, s);
  const uint64_t E = head.n;
  bc_get_array1(r, tail, E, s);
  bc_get_array1(r, eps, E, s);
  {
    uint64_t dims[2];
    const uint64_t total = bc_array_header(r, 2, dims);
    if (dims[0] != n || dims[1] < 1 || dims[1] > (1u << 20)) throw Error(FORMAT, "embedding shape mismatch");
    o->n = dims[0];
    o->dim = dims[1];
    DevBuf<float> e;
    get_device_array(r, e, total, s);
    o->emb2.alloc(2 * n * o->dim, s);
    d2d(o->emb2.p, e.p, n * o->dim, s);
  }
  for (int t = 0; t < 3; ++t) {  // schedule state: recomputed from epochs_per_sample
    uint64_t d;
    const uint64_t total = bc_array_header(r, 1, &d);
    if (total != E || r.count(8) != E) throw Error(FORMAT, "schedule array length mismatch");
    r.off += E * 8;
  }
  o->current_epoch = r.get<uint64_t>();
  o->total_epochs = r.get<uint64_t>();
  o->gamma = r.get<float>();
  o->initial_alpha = r.get<float>();
  const double nsr = r.get<double>();
  if (!(nsr >= 0.0 && nsr < 4294967296.0) || nsr != (double)(uint64_t)nsr)
    throw Error(FORMAT, "negative_sample_rate is not a whole number");
  o->negative_sample_rate = (uint64_t)nsr;
  const uint32_t mt = r.get<uint32_t>();
  if (mt > 1) throw Error(FORMAT, "invalid MetricType");
  o->metric_type = (int)mt;
  if (r.off != len) throw Error(FORMAT, "trailing bytes after the optimizer");
  compute_thresholds(*o);
  finish_loaded_optimizer(*o, head, tail, eps);
  *out = o.release();
  API_END
}

// FittedUmap (embedding.rs:438-443): embedding, manifold, config.
int umap_fitted_serialize_bincode(const umap_fitted* f, uint8_t* buf, uint64_t cap, uint64_t* needed) {
  API_BEGIN
  need(f, "fitted");
  f->manifold->stream->activate();
  Writer w;
  bc_array2(w, f->embedding.p, f->n, f->dim, f->s());
  bc_manifold(w, *f->manifold);
  bc_config(w, f->config);
  int rc = copy_out(w, buf, cap, needed);
  if (rc) throw Error(rc, "buffer too small for the serialized fitted model");
  API_END
}

int umap_fitted_deserialize_bincode(const uint8_t* buf, uint64_t len, umap_fitted** out) {
  API_BEGIN
  need(buf, "buf"); need(out, "out");
  *out = nullptr;
  Reader r{buf, len};
  auto f = std::make_unique<umap_fitted>();
  uint64_t dims[2];
  const uint64_t total = bc_array_header(r, 2, dims);
  if (dims[1] > (1u << 20)) throw Error(FORMAT, "embedding shape mismatch");
  f->n = dims[0];
  f->dim = dims[1];
  // The embedding precedes the manifold (which owns the stream): stage it on the host.
  const uint64_t cnt = r.count(4);
  if (cnt != total) throw Error(FORMAT, "embedding length mismatch");
  const float* host_emb = (const float*)(r.p + r.off);
  r.off += cnt * 4;
  f->manifold = bc_read_manifold(r);
  f->config = bc_read_config(r);
  if (r.off != len) throw Error(FORMAT, "trailing bytes after the fitted model");
  if (f->manifold->n_vertices != f->n) throw Error(FORMAT, "embedding rows do not match the manifold");
  f->embedding.alloc(cnt, f->s());
  std::vector<float> tmp(host_emb, host_emb + cnt);
  h2d(f->embedding.p, tmp.data(), cnt, f->s());
  UB_CUDA(cudaStreamSynchronize(f->s()));
  *out = f.release();
  API_END
}

// ---- batched instances
int umap_batch_optimizer_new(const umap_config* cfg, uint64_t n_instances, const uint64_t* offsets,
                             const uint32_t* idx, const float* dist, uint64_t knn_cols, const float* init,
                             uint64_t init_cols, uint64_t total_epochs, umap_optimizer** out) {
  API_BEGIN
  need(cfg, "cfg"); need(offsets, "offsets"); need(idx, "knn_indices"); need(dist, "knn_dists");
  need(init, "init"); need(out, "out");
  *out = nullptr;
  *out = batch_new_impl(*cfg, n_instances, offsets, idx, dist, knn_cols, init, init_cols, total_epochs, true)
             .release();
  API_END
}

int umap_batch_optimizer_new_device(const umap_config* cfg, uint64_t n_instances, const uint64_t* offsets,
                                    const uint32_t* idx, const float* dist, uint64_t knn_cols, const float* init,
                                    uint64_t init_cols, uint64_t total_epochs, umap_optimizer** out) {
  API_BEGIN
  need(cfg, "cfg"); need(offsets, "offsets"); need(idx, "knn_indices"); need(dist, "knn_dists");
  need(init, "init"); need(out, "out");
  *out = nullptr;
  wait_for_inputs();
  *out = batch_new_impl(*cfg, n_instances, offsets, idx, dist, knn_cols, init, init_cols, total_epochs, false)
             .release();
  API_END
}

int umap_batch_fit(const umap_config* cfg, uint64_t n_instances, const uint64_t* offsets, const uint32_t* idx,
                   const float* dist, uint64_t knn_cols, const float* init, uint64_t init_cols, float* out) {
  API_BEGIN
  need(cfg, "cfg"); need(offsets, "offsets"); need(idx, "knn_indices"); need(dist, "knn_dists");
  need(init, "init"); need(out, "out");
  batch_fit_impl(*cfg, n_instances, offsets, idx, dist, knn_cols, init, init_cols, out, true);
  API_END
}

int umap_batch_fit_device(const umap_config* cfg, uint64_t n_instances, const uint64_t* offsets,
                          const uint32_t* idx, const float* dist, uint64_t knn_cols, const float* init,
                          uint64_t init_cols, float* out) {
  API_BEGIN
  need(cfg, "cfg"); need(offsets, "offsets"); need(idx, "knn_indices"); need(dist, "knn_dists");
  need(init, "init"); need(out, "out");
  wait_for_inputs();
  batch_fit_impl(*cfg, n_instances, offsets, idx, dist, knn_cols, init, init_cols, out, false);
  API_END
}

int umap_optimizer_tuning(const umap_optimizer* opt, uint32_t* chunk, uint32_t* block_threads) {
  API_BEGIN
  need(opt, "optimizer");
  if (chunk) *chunk = opt->layout.chunk;
  if (block_threads) *block_threads = opt->layout.block_threads;
  API_END
}

int umap_optimizer_layout_flags(const umap_optimizer* opt, uint32_t* flags) {
  API_BEGIN
  need(opt, "optimizer"); need(flags, "flags");
  *flags = (opt->layout.lane_major ? UMAP_LAYOUT_LANE_MAJOR : 0u) |
           (opt->layout.short_epoch && !opt->layout.dram_epoch ? UMAP_LAYOUT_EIGHT_NEGATIVES : 0u) |
           (opt->layout.dram_epoch ? UMAP_LAYOUT_TWELVE_NEGATIVES : 0u) |
           (opt->layout.order.p ? UMAP_LAYOUT_RENAMED : 0u) |
           (opt->metric_type == UMAP_METRIC_GENERIC ? UMAP_LAYOUT_GENERIC_RULE : 0u) |
           (opt->layout.task_order == TaskOrder::LengthRate ? UMAP_LAYOUT_RATE_ORDER : 0u) |
           (opt->layout.task_order == TaskOrder::RowBlock ? UMAP_LAYOUT_BLOCK_ORDER : 0u) |
           (opt->layout.task_order == TaskOrder::Row ? UMAP_LAYOUT_ROW_ORDER : 0u);
  API_END
}

// ---- kernel-level entry points
int umap_smooth_knn_dist_device(const float* dists, uint64_t n, uint64_t k, uint64_t n_iter,
                                float local_connectivity, float bandwidth, float* sigmas, float* rhos) {
  API_BEGIN
  need(dists, "dists"); need(sigmas, "sigmas"); need(rhos, "rhos");
  if (k < 1) throw Error(INVALID_ARGUMENT, "k must be >= 1");
  cudaStream_t s;
  UB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s};
  wait_for_inputs();
  GraphParams gp{};
  gp.local_connectivity = local_connectivity;
  const float lcf = floorf(local_connectivity);
  gp.interpolation = local_connectivity - lcf;
  gp.lc_usize = rust_f32_as_usize(local_connectivity);
  gp.lc_index = rust_f32_as_usize(lcf);
  gp.target = log2f((float)k) * bandwidth;
  gp.n_iter = (int)std::min<uint64_t>(n_iter, 1u << 30);
  smooth_knn(dists, n, k, gp, sigmas, rhos, s);
  UB_CUDA(cudaStreamSynchronize(s));
  API_END
}

// Exact brute-force kNN (examples/src/bin/mnist_demo.rs:203-229) on the tensor cores.
thread_local KnnStats g_knn_last;
static void knn_entry(const float* X, uint64_t n, uint64_t dim, uint64_t k, uint32_t* idx, float* dist,
                      uint64_t* rows_recomputed, bool host) {
  cudaStream_t s;
  UB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s};
  if (!host) wait_for_inputs();
  if (n && dim && n > UINT64_MAX / dim) throw Error(INVALID_ARGUMENT, "n * dim overflows");
  KnnStats st;
  if (host) {
    DevBuf<float> dx(n * dim, s);
    DevBuf<uint32_t> di(n * k, s);
    DevBuf<float> dd(n * k, s);
    h2d(dx.p, X, n * dim, s);
    st = knn_bruteforce(dx.p, n, dim, k, di.p, dd.p, s);
    d2h(idx, di.p, n * k, s);
    d2h(dist, dd.p, n * k, s);
    UB_CUDA(cudaStreamSynchronize(s));
  } else {
    st = knn_bruteforce(X, n, dim, k, idx, dist, s);
  }
  if (rows_recomputed) *rows_recomputed = st.fallback_rows;
  g_knn_last = st;
}

int umap_knn_last_profile(float* candidate_pass_ms, uint64_t* rows_recomputed, uint32_t* reordered) {
  API_BEGIN
  if (candidate_pass_ms) *candidate_pass_ms = g_knn_last.candidate_ms;
  if (rows_recomputed) *rows_recomputed = g_knn_last.fallback_rows;
  if (reordered) *reordered = g_knn_last.reordered;
  API_END
}

int umap_knn_bruteforce(const float* data, uint64_t n, uint64_t dim, uint64_t k, uint32_t* knn_indices,
                        float* knn_dists, uint64_t* rows_recomputed) {
  API_BEGIN
  need(data, "data"); need(knn_indices, "knn_indices"); need(knn_dists, "knn_dists");
  knn_entry(data, n, dim, k, knn_indices, knn_dists, rows_recomputed, true);
  API_END
}

int umap_knn_bruteforce_device(const float* data, uint64_t n, uint64_t dim, uint64_t k, uint32_t* knn_indices,
                               float* knn_dists, uint64_t* rows_recomputed) {
  API_BEGIN
  need(data, "data"); need(knn_indices, "knn_indices"); need(knn_dists, "knn_dists");
  knn_entry(data, n, dim, k, knn_indices, knn_dists, rows_recomputed, false);
  API_END
}

// The sort's passes read one buffer while they scatter into another, so no output may share
// memory with an input or with the other output.
void sort_buffers_disjoint(const uint32_t* keys_in, const uint32_t* vals_in, const uint32_t* keys_out,
                           const uint32_t* vals_out, uint64_t n) {
  const auto overlap = [n](const uint32_t* a, const uint32_t* b) {
    if (!a || !b || n == 0) return false;
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b), len = n * 4;
    return x < y + len && y < x + len;
  };
  if (overlap(keys_out, keys_in) || overlap(keys_out, vals_in) || overlap(vals_out, keys_in) ||
      overlap(vals_out, vals_in) || overlap(keys_out, vals_out))
    throw Error(INVALID_ARGUMENT, "radix sort: output buffers must not overlap the inputs or each other");
}

int umap_radix_sort_pairs_device(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                 uint32_t* vals_out, uint64_t n, int end_bit) {
  API_BEGIN
  need(keys_in, "keys_in"); need(keys_out, "keys_out"); need(vals_out, "values_out");
  sort_buffers_disjoint(keys_in, vals_in, keys_out, vals_out, n);
  cudaStream_t s;
  UB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s};
  wait_for_inputs();
  radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, n, end_bit, s);
  UB_CUDA(cudaStreamSynchronize(s));
  API_END
}

int umap_sgd_negative_draws_device(uint64_t seed, uint64_t first_entry, uint64_t n_entries, uint32_t epoch,
                                   uint32_t per_entry, uint32_t lo, uint32_t range, uint32_t* dev_out) {
  API_BEGIN
  need(dev_out, "out");
  if (range == 0) throw Error(INVALID_ARGUMENT, "range must be at least 1");
  if (per_entry > 64) throw Error(INVALID_ARGUMENT, "per_entry must be at most 64");
  cudaStream_t s;
  UB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s};
  wait_for_inputs();
  negative_draws(seed, first_entry, n_entries, epoch, per_entry, lo, range, dev_out, s);
  UB_CUDA(cudaStreamSynchronize(s));
  API_END
}

int umap_sgd_negatives_per_firing_device(const uint32_t* dev_q, const uint32_t* dev_epoch, uint64_t count,
                                         uint32_t negative_sample_rate, uint32_t* dev_out) {
  API_BEGIN
  need(dev_q, "q"); need(dev_epoch, "epoch"); need(dev_out, "out");
  cudaStream_t s;
  UB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SGuard { cudaStream_t s; ~SGuard() { (void)cudaStreamSynchronize(s); (void)cudaStreamDestroy(s); } } g{s};
  wait_for_inputs();
  negatives_per_firing(dev_q, dev_epoch, count, negative_sample_rate, dev_out, s);
  UB_CUDA(cudaStreamSynchronize(s));
  API_END
}

int umap_random_rows_probe_device(float* dev_table, uint64_t n_rows, uint64_t accesses, int mode, float* dev_out,
                                  float* ms, uint64_t* accesses_done) {
  API_BEGIN
  need(dev_table, "table"); need(ms, "ms"); need(accesses_done, "accesses_done");
  if (mode != 0 && mode != 1) throw Error(INVALID_ARGUMENT, "mode must be 0 (reads) or 1 (red.add)");
  if (mode == 0) need(dev_out, "out");
  Stream st;
  wait_for_inputs();
  *ms = random_rows_probe(dev_table, n_rows, accesses, mode, dev_out, accesses_done, st.s);
  API_END
}

int umap_radix_sort_pairs_device_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                         uint32_t* vals_out, uint64_t n, int end_bit, void* stream) {
  API_BEGIN
  // n = 0 is the per-device warm-up call: it only loads the scratch array and looks up its
  // address, so its buffers may be NULL.
  if (n > radix_sort_noalloc_max_pairs())
    throw Error(INVALID_ARGUMENT, "allocation-free radix sort takes at most " +
                                      std::to_string(radix_sort_noalloc_max_pairs()) + " pairs, got " +
                                      std::to_string(n));
  if (n > 0) {
    need(keys_in, "keys_in"); need(keys_out, "keys_out"); need(vals_out, "values_out");
  }
  sort_buffers_disjoint(keys_in, vals_in, keys_out, vals_out, n);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  radix_sort_pairs_noalloc(keys_in, vals_in, keys_out, vals_out, n, end_bit, s);
  UB_CUDA(cudaStreamSynchronize(s));
  API_END
}

int umap_radix_sort_noalloc_max_pairs(uint64_t* out) {
  API_BEGIN
  need(out, "out");
  *out = radix_sort_noalloc_max_pairs();
  API_END
}

// ---------------------------------------------------------------- learned warm start
int umap_mlp_param_count(uint64_t in_dim, uint64_t out_dim, uint64_t* out) {
  API_BEGIN
  need(out, "out");
  if (in_dim > 4096 || out_dim > 4) throw Error(INVALID_ARGUMENT, "in_dim must be <= 4096 and out_dim <= 4");
  *out = (uint64_t)Mlp::param_count((int)in_dim, (int)out_dim);
  API_END
}

int umap_mlp_new(uint64_t in_dim, uint64_t out_dim, const float* params, umap_mlp** out) {
  API_BEGIN
  need(params, "params"); need(out, "out");
  *out = nullptr;
  if (in_dim > 4096 || out_dim > 4)
    throw Error(INVALID_ARGUMENT, "MLP input width must be a positive multiple of 64 (at most 4096) and output width 1..4");
  auto m = std::make_unique<umap_mlp>();
  m->stream = std::make_unique<Stream>();
  m->net = std::make_unique<Mlp>((int)in_dim, (int)out_dim, params, m->stream->s);
  *out = m.release();
  API_END
}

int umap_mlp_dims(const umap_mlp* m, uint64_t* in_dim, uint64_t* out_dim) {
  API_BEGIN
  need(m, "mlp"); need(in_dim, "in_dim"); need(out_dim, "out_dim");
  *in_dim = (uint64_t)m->net->in_dim();
  *out_dim = (uint64_t)m->net->out_dim();
  API_END
}

int umap_mlp_get_params(const umap_mlp* m, float* params) {
  API_BEGIN
  need(m, "mlp"); need(params, "params");
  m->stream->activate();
  m->net->get_params(params);
  API_END
}

int umap_mlp_set_params(umap_mlp* m, const float* params) {
  API_BEGIN
  need(m, "mlp"); need(params, "params");
  m->stream->activate();
  m->net->set_params(params);
  API_END
}

int umap_mlp_fit_input_norm_device(umap_mlp* m, const float* x, uint64_t rows) {
  API_BEGIN
  need(m, "mlp"); need(x, "x");
  m->stream->activate();
  wait_for_inputs();
  m->net->fit_input_norm(x, (int64_t)rows);
  API_END
}

int umap_mlp_input_norm(const umap_mlp* m, float* shift, float* scale) {
  API_BEGIN
  need(m, "mlp"); need(shift, "shift"); need(scale, "scale");
  m->stream->activate();
  m->net->get_input_norm(shift, scale);
  API_END
}

int umap_mlp_set_input_norm(umap_mlp* m, const float* shift, const float* scale) {
  API_BEGIN
  need(m, "mlp"); need(shift, "shift"); need(scale, "scale");
  m->stream->activate();
  m->net->set_input_norm(shift, scale);
  API_END
}

int umap_mlp_gradients_device(umap_mlp* m, const float* x, const float* y, uint64_t rows, float* grads,
                              float* loss) {
  API_BEGIN
  need(m, "mlp"); need(x, "x"); need(y, "y"); need(grads, "grads"); need(loss, "loss");
  m->stream->activate();
  wait_for_inputs();
  m->net->gradients(x, y, (int64_t)rows, grads, loss);
  API_END
}

int umap_mlp_train_device(umap_mlp* m, const float* x, const float* y, uint64_t rows, uint64_t epochs,
                          uint64_t batch, float learning_rate, uint64_t seed, float* losses) {
  API_BEGIN
  need(m, "mlp"); need(x, "x"); need(y, "y");
  if (epochs > (1u << 20)) throw Error(INVALID_ARGUMENT, "epochs must be <= 1048576");
  if (!(learning_rate > 0.0f)) throw Error(INVALID_ARGUMENT, "learning_rate must be positive, got " + rust_f32(learning_rate));
  m->stream->activate();
  wait_for_inputs();
  m->net->train(x, y, (int64_t)std::min<uint64_t>(rows, 1ull << 40), (int)epochs,
                (int64_t)std::min<uint64_t>(batch, 1ull << 40), learning_rate, seed, losses);
  API_END
}

int umap_mlp_predict_device(umap_mlp* m, const float* x, uint64_t rows, float* y) {
  API_BEGIN
  need(m, "mlp"); need(x, "x"); need(y, "y");
  m->stream->activate();
  wait_for_inputs();
  m->net->predict(x, (int64_t)std::min<uint64_t>(rows, 1ull << 40), y);
  API_END
}

int umap_mlp_free(umap_mlp* m) {
  API_BEGIN
  if (m) {
    m->stream->activate();
    delete m;
  }
  API_END
}

int umap_warm_start_params_default(umap_warm_start_params* out) {
  API_BEGIN
  need(out, "out");
  *out = umap_warm_start_params{};
  out->sub_epochs = 500;
  out->epochs = 100;
  out->mlp_epochs = 20;
  out->batch = 4096;
  out->mlp_learning_rate = 1e-3f;
  out->has_learning_rate = 0;
  out->learning_rate = 1.0f;
  out->seed = 0;
  API_END
}

int umap_warm_start_fit_device(const umap_config* cfg, const umap_warm_start_params* params, const float* data,
                               uint64_t n_samples, uint64_t data_dim, const uint32_t* knn_indices,
                               const float* knn_dists, uint64_t knn_cols, const uint32_t* sub_rows, uint64_t n_sub,
                               const uint32_t* sub_knn_indices, const float* sub_knn_dists, const float* sub_init,
                               umap_fitted** out, float* phase_ms, float* mlp_losses) {
  API_BEGIN
  need(cfg, "config"); need(params, "params"); need(data, "data"); need(knn_indices, "knn_indices");
  need(knn_dists, "knn_dists"); need(sub_rows, "sub_rows"); need(sub_knn_indices, "sub_knn_indices");
  need(sub_knn_dists, "sub_knn_dists"); need(out, "out");
  *out = nullptr;
  warm_start_check_args(*cfg, *params, n_samples, data_dim, knn_cols, n_sub);
  wait_for_inputs();
  *out = warm_start_impl(*cfg, *params, data, n_samples, data_dim, knn_indices, knn_dists, knn_cols, sub_rows, n_sub,
                         sub_knn_indices, sub_knn_dists, sub_init, phase_ms, mlp_losses)
             .release();
  API_END
}

int umap_gemm_bf16_device(const void* a, const void* b, float* c, uint64_t m, uint64_t n, uint64_t k,
                          uint64_t k_splits) {
  API_BEGIN
  need(a, "a"); need(b, "b"); need(c, "c");
  if (m > (1ull << 40) || n > (1ull << 30) || k > (1ull << 30) || k_splits < 1 || k_splits > 65535)
    throw Error(INVALID_ARGUMENT, "GEMM dimensions out of range");
  Stream st;
  wait_for_inputs();
  umma_gemm_f32(a, b, c, (int64_t)m, (int64_t)n, (int64_t)k, (int)k_splits, st.s);
  API_END
}

}  // extern "C"
