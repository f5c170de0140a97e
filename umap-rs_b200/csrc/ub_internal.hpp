// Internal declarations shared by the CUDA kernels (*.cu) and the C++ host (*.cpp).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

namespace ub {

// C-ABI status codes (mirrors include/umap_b200.h).
enum Status : int {
  OK = 0,
  INVALID_ARGUMENT = 1,
  OVERSTEP = 2,
  CUDA = 3,
  OUT_OF_MEMORY = 4,
  FORMAT = 5,
  IO = 6,
  NULLPTR = 7,
  UNSUPPORTED = 8,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);
inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) throw_cuda(e, what, file, line);
}
#define UB_CUDA(x) ::ub::cuda_check((x), #x, __FILE__, __LINE__)
// Every kernel launch site calls this right after its launch: it counts the launch (for
// throughput accounting) and surfaces launch errors.
void count_launch();
#define UB_LAUNCH_CHECK() \
  (::ub::count_launch(), ::ub::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))

// Allocation diagnostics (UMAP_B200_LOG): reports device allocations whose host call took
// longer than 1 ms.
bool alloc_log_enabled();
void log_slow_alloc(uint64_t bytes, double ms);

// Device memory from the library's cache (alloc.cpp): stream-ordered, blocks reused across
// calls.  dev_free orders the block's reuse after the work queued so far on `s`.
void* dev_alloc(uint64_t bytes, cudaStream_t s);
void dev_free(void* p, uint64_t bytes, cudaStream_t s) noexcept;
uint64_t release_cached_memory();

// Stream-ordered device buffer from the cache above, owned by one stream.
template <class T>
struct DevBuf {
  T* p = nullptr;
  uint64_t n = 0;
  cudaStream_t s = nullptr;

  DevBuf() = default;
  DevBuf(uint64_t count, cudaStream_t st) { alloc(count, st); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p; n = o.n; s = o.s;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }

  void alloc(uint64_t count, cudaStream_t st) {
    reset();
    s = st;
    if (count == 0) return;
    p = static_cast<T*>(dev_alloc(count * sizeof(T), st));
    n = count;
  }
  void reset() noexcept {
    if (p) dev_free(p, n * sizeof(T), s);
    p = nullptr;
    n = 0;
  }
  // Moves ownership to another stream's ordering (caller guarantees ordering).
  void set_stream(cudaStream_t st) { s = st; }
  uint64_t bytes() const { return n * sizeof(T); }
  T* get() const { return p; }
};

// ---------------------------------------------------------------- primitives (prim.cu)
// out[0..n] = exclusive prefix sum of in[0..n-1]; out[n] = total.
void scan_u32_to_u64(const uint32_t* in, uint64_t* out, uint64_t n, cudaStream_t s);
void scan_u64_to_u64(const uint64_t* in, uint64_t* out, uint64_t n, cudaStream_t s);
// Stable LSD radix sort by key bits [0, end_bit).  vals_in == nullptr means 0..n-1.
// keys_out/vals_out may not alias the inputs.  n must be < 2^32.
void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                      uint32_t* vals_out, uint64_t n, int end_bit, cudaStream_t s);
// Same sort with its scratch in a static device array instead of allocations; n must be
// at most radix_sort_noalloc_max_pairs().  Calls whose GPU work overlaps race on the array.
void radix_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                              uint32_t* vals_out, uint64_t n, int end_bit, cudaStream_t s);
uint64_t radix_sort_noalloc_max_pairs();
// Reductions into a device scalar (*out).
void reduce_max_f32(const float* x, uint64_t n, float init, float* out, cudaStream_t s);
void reduce_max_u32(const uint32_t* x, uint64_t n, uint32_t* out, cudaStream_t s);
void reduce_sum_u64(const uint64_t* x, uint64_t n, uint64_t* out, cudaStream_t s);
int bits_for(uint64_t max_value);

// ---------------------------------------------------------------- graph build (graph.cu)
struct GraphParams {
  float local_connectivity;
  float interpolation;  // local_connectivity - floor(local_connectivity)
  uint64_t lc_usize;    // `local_connectivity as usize` (saturating)
  uint64_t lc_index;    // `local_connectivity.floor() as usize`
  float target;         // log2f(k) * bandwidth, computed on the host with glibc log2f
  float disc_thr;       // disconnection distance (+inf by default)
  float mix;            // set_op_mix_ratio
  float prod_coeff;     // 1 - 2*mix (f32, host-rounded)
  int n_iter;           // 64
};

// Batched instances: rows [seg_off[s], seg_off[s+1]) belong to instance s (device arrays).
struct Segments {
  uint32_t n_seg = 0;
  const uint64_t* seg_off = nullptr;  // [n_seg + 1] row offsets
  const uint32_t* row_seg = nullptr;  // [n_rows] instance of each row
};

// K1: per-row rho and sigma (smooth_knn_dist.rs:60-198).  Rows whose rho is not positive
// fall back on the mean of all distances of their instance (seg == nullptr: one instance).
void smooth_knn(const float* dist, uint64_t n, uint64_t k, const GraphParams& gp,
                float* sigmas, float* rhos, cudaStream_t s, const Segments* seg = nullptr);
// Batched instances: local kNN ids -> global ids (out-of-instance ids -> 0xFFFFFFFF).
void localize_knn(const uint32_t* idx, uint64_t n, uint64_t k, const Segments& seg, uint32_t* out,
                  cudaStream_t s);
void fill_row_segments(const uint64_t* seg_off, uint32_t n_seg, uint32_t* row_seg, cudaStream_t s);
// K2: directed membership entries per row, kept ones sorted by column (stable) into the
// padded [n][k] arrays pcol/pw; cnt[r] = kept count.  edges_removed (device u64) counts
// dist >= disc_thr entries; dup_row (device u64, zeroed by the caller) receives ~r of the
// smallest row r that keeps one neighbour twice (0 = none).
void membership(const uint32_t* idx, const float* dist, uint64_t n, uint64_t k,
                const GraphParams& gp, const float* sigmas, const float* rhos, uint32_t* pcol,
                float* pw, uint32_t* cnt, unsigned long long* edges_removed, unsigned long long* dup_row,
                cudaStream_t s);
// Compacts padded rows into CSR order: keys[q] = column, vals[q] = padded position r*k+e.
void compact_directed(const uint32_t* pcol, const uint32_t* cnt, const uint64_t* dptr,
                      uint64_t n, uint64_t k, uint32_t* keys, uint32_t* vals, cudaStream_t s);
// data[q] = pw[vals[q]].
void gather_weights(const float* pw, const uint32_t* vals, uint64_t nnz, float* data,
                    cudaStream_t s);
// tptr[c] = first index i with sorted_keys[i] >= c, for c in [0, n]; tptr[n] = nnz.
void segment_starts(const uint32_t* sorted_keys, uint64_t nnz, uint64_t n, uint64_t* tptr,
                    cudaStream_t s);
// K4 fuzzy union, count pass (fill=false) and fill pass.
void union_rows(const uint32_t* pcol, const float* pw, const uint32_t* cnt, uint64_t k,
                const uint64_t* tptr, const uint32_t* tvals, uint64_t n, const GraphParams& gp,
                uint32_t* out_cnt, const uint64_t* out_ptr, uint32_t* out_idx, float* out_w,
                bool fill, cudaStream_t s);
// Rows whose weights sum to zero (embedding.rs:216-223); returns count into *out.
void count_empty_rows(const uint64_t* indptr, const float* data, uint64_t n,
                      unsigned long long* out, cudaStream_t s);

// ---------------------------------------------------------------- SGD layout (sgd.cu)
// Schedule value per kept edge: Q = ceil(2^32 / epochs_per_sample), stored as Q - 1 in a
// u32 (Q in [1, 2^32]).  Fires by epoch n: (n * Q) >> 32.  Q - 1 == 0 never fires in
// any realistic run (padding).
//
// Tasks: each head row's kept edges are cut into chunks of at most `chunk` edges; a task is
// one chunk.  Tasks are sorted by length (descending, stable) and packed 32 to a slice; a
// warp owns a slice, a lane owns a task.  Entry (e, lane) of slice s lives at
// slice_base[s] + e*32 + lane as uint2 {tail, Q - 1}.  Bit `lane` of split_mask[s] is set
// when the lane's task is a partial row (its head update is merged with an atomic add).
// Largest total epoch count of an optimizer: keeps the epoch kernel's per-firing schedule
// arithmetic exact in 32 bits (see negatives_at in sgd.cu).
constexpr uint64_t MAX_EPOCHS = 1ull << 21;

// Order in which build_sgd_layout deals tasks to warps (sgd.cu, pick_task_order).
enum class TaskOrder { Length, LengthRate, RowBlock, Row };

struct SgdLayout {
  uint64_t n_vertices = 0, n_edges = 0, n_entries = 0, n_slices = 0, n_tasks = 0;
  uint32_t max_degree = 0, chunk = 0;
  uint32_t block_threads = 256;  // threads per block of the epoch kernel (multiple of 32)
  bool short_epoch = false;      // epoch kernel budget for graphs of at most ~2 waves of warps
  bool dram_epoch = false;       // 12-negatives budget of renamed DRAM-bound layouts
  bool lane_major = true;        // entry order: lane major (true) or interleaved by lane
  TaskOrder task_order = TaskOrder::Length;
  uint64_t split_tasks = 0;
  DevBuf<uint64_t> slice_base;   // [n_slices + 1]
  DevBuf<uint32_t> slice_width;  // [n_slices]
  DevBuf<uint32_t> split_mask;   // [n_slices]
  DevBuf<uint32_t> rowid;        // [n_slices * 32]; 0xFFFFFFFF = padding lane
  DevBuf<uint2> entry;           // [n_entries] {tail, Q - 1}
  // Renamed vertices (DRAM-bound plain fits, see order.cu; empty otherwise): rowid and entry
  // tails are new ids, vertex order[u] of the caller is vertex u of the layout, and the epoch
  // loop runs on a working copy of the embedding permuted into that order.
  DevBuf<uint32_t> order;        // [n_vertices] or empty
};

struct SgdParams {
  float a, b, gamma;
  float neg_attr;   // (-2 a) b
  float pos_rep;    // (2 gamma) b
  uint32_t neg_rate;  // negative_sample_rate
  uint32_t n_vertices;
  // Batched instances (null for a plain fit): negatives of a row of instance s are drawn
  // from [seg_off[s], seg_off[s+1]).
  const uint32_t* row_seg;
  const uint64_t* seg_off;
  uint32_t dim;
  uint64_t seed;
  // MetricType::Generic (optimizer.rs:340-358): the generic-metric update rule with the
  // built-in Euclidean output metric instead of the Euclidean specialisation.
  uint32_t generic_metric;
  float two_b;      // 2 b
};

// Batched instances: per-instance prune threshold and max kept weight (device arrays).
struct SegmentPrune {
  const float* seg_thr = nullptr;
  const float* seg_maxw = nullptr;
  const uint32_t* row_seg = nullptr;
};

// Prune (optimizer.rs:85-167): keep w >= thr.  kept_ptr[n+1] = row pointers of the kept
// edges in the reference's row-major order; *n_edges = kept count (host, synchronises).
void prune_edges(const uint64_t* indptr, const float* data, uint64_t n, float thr,
                 uint64_t* kept_ptr, uint64_t* n_edges, cudaStream_t s,
                 const SegmentPrune* sp = nullptr);
// Batched instances: max weight per instance.
void segment_max(const uint64_t* indptr, const float* data, const uint64_t* seg_off, uint32_t n_seg,
                 float* out, cudaStream_t s);
// Kept edges in the reference order: head/tail u32 and epochs_per_sample f64
// (make_epochs_per_sample.rs:21-52 with max weight max_w).  Any output may be null.
void export_edges(const uint64_t* indptr, const uint32_t* indices, const float* data,
                  uint64_t n, float thr, float max_w, uint64_t total_epochs,
                  const uint64_t* kept_ptr, uint32_t* head, uint32_t* tail, double* eps,
                  cudaStream_t s, const SegmentPrune* sp = nullptr);
void head_from_ptr(const uint64_t* kept_ptr, uint64_t n, uint32_t* head, cudaStream_t s);
// Schedule state at cur_epoch in the reference's representation (optimizer.rs:41-43).
void export_state(const double* eps, uint64_t E, uint64_t neg_rate, uint64_t cur_epoch,
                  double* eons, double* eonns, double* epns, cudaStream_t s);
// Slice layout from kept edges (kept_ptr, tail, eps).  chunk = 0 picks the task length
// from the edge count.
// Task length for a layout of n_edges kept edges (sgd.cu; UMAP_B200_CHUNK overrides it), and
// the one for the generic-metric rule, whose rows must stay whole tasks (see sgd.cu).
uint32_t pick_chunk(uint64_t n_edges);
uint32_t pick_chunk_generic(uint64_t n_edges);
// `rename`: a plain fit's layout may rename its vertices into a locality order (DRAM-bound
// sizes); the generic-metric rule passes false.
void build_sgd_layout(const uint64_t* kept_ptr, const uint32_t* tail, const double* eps,
                      uint64_t n, uint32_t chunk, SgdLayout& L, cudaStream_t s,
                      const Segments* seg = nullptr, bool rename = true);
void kept_degree(const uint64_t* indptr, const float* data, uint64_t n, float thr,
                 uint32_t* deg, cudaStream_t s, const SegmentPrune* sp = nullptr);
// K6 normalise init into [0, 10] per dimension (optimizer.rs:181-230), in place.
void normalize_init(float* emb, uint64_t n, uint32_t dim, cudaStream_t s,
                    const Segments* seg = nullptr);
// K7 one Hogwild epoch.
void sgd_epoch(const SgdLayout& L, float* live, float* snap, const SgdParams& p,
               uint32_t epoch, float alpha, cudaStream_t s);
// Exact totals of fired edges / negatives over epochs [start, end).
// Warm-start row helpers (warm.cu): rows (or rows[i]) of x [*, d] zero-padded to dp columns;
// keep[r] = 1 for rows of y [n, dim] without NaN/inf; rows with keep set moved to pos[r].
void pad_gather_rows(const float* x, uint64_t d, uint64_t dp, const uint32_t* rows, uint64_t count, float* out,
                     cudaStream_t s);
void finite_rows(const float* y, uint64_t n, uint32_t dim, uint32_t* keep, cudaStream_t s);
void compact_rows(const float* src, uint64_t n, uint64_t width, const uint32_t* keep, const uint64_t* pos,
                  float* dst, cudaStream_t s);
// Timed rate probe of random 8-byte row reads (mode 0) or red.adds (mode 1) on table [n_rows][2]
// (probe.cu): returns the CUDA-event milliseconds of one launch; *done = accesses made; out
// receives 148 * 8 * 256 per-thread sums in mode 0.
constexpr uint64_t PROBE_THREADS = 148ull * 8 * 256;
float random_rows_probe(float* table, uint64_t n_rows, uint64_t accesses, int mode, float* out, uint64_t* done,
                        cudaStream_t s);
// Locality order of a graph's vertices (order.cu): order[u] = old id of new vertex u,
// rank = its inverse.
void locality_order(const uint64_t* kptr, const uint32_t* ktail, uint64_t n, uint32_t* order, uint32_t* rank,
                    cudaStream_t s);
// Rows of an n x dim array into the new order (to_new: dst[u] = src[order[u]]) or back.
void permute_rows(const float* src, const uint32_t* order, uint64_t n, uint32_t dim, bool to_new, float* dst,
                  cudaStream_t s);
// Negative samples of the SGD epoch's generator (see negative_draws_kernel in sgd.cu).
void negative_draws(uint64_t seed, uint64_t first, uint64_t count, uint32_t epoch, uint32_t per, uint32_t lo,
                    uint32_t range, uint32_t* out, cudaStream_t s);
// Per-firing negative counts of the epoch kernel's schedule (negatives_per_firing_kernel).
void negatives_per_firing(const uint32_t* qs, const uint32_t* ns, uint64_t count, uint32_t neg, uint32_t* out,
                          cudaStream_t s);
void schedule_totals(const SgdLayout& L, uint32_t neg_rate, uint32_t start, uint32_t end,
                     unsigned long long* d_fired, unsigned long long* d_negs, cudaStream_t s);
// Rows with an empty graph row -> NaN (embedding.rs:327-334).
void nan_empty_rows(const uint64_t* indptr, uint64_t n, uint32_t dim, float* emb,
                    cudaStream_t s);

// ---------------------------------------------------------------- warm-start MLP (mlp.cu)
// in -> 256 -> 256 -> out network with GELU, bf16 weights/activations, fp32 accumulation.
// Flat fp32 parameters in the order W1 [256, in], b1 [256], W2 [256, 256], b2 [256],
// W3 [out, 256], b3 [out] (weights row-major, one row per output unit).  All X / Y pointers
// are device memory; X rows are `in` floats, Y rows `out` floats.
class Mlp {
 public:
  struct Impl;
  Mlp(int in_dim, int out_dim, const float* host_params, cudaStream_t s);
  ~Mlp();
  Mlp(const Mlp&) = delete;
  Mlp& operator=(const Mlp&) = delete;
  static int64_t param_count(int in_dim, int out_dim);
  int in_dim() const;
  int out_dim() const;
  int64_t n_params() const;
  void set_params(const float* host);
  void get_params(float* host) const;
  // Input standardisation x' = (x - shift) * scale applied before the first layer.
  void fit_input_norm(const float* X, int64_t n);
  void set_input_norm(const float* shift, const float* scale);
  void get_input_norm(float* shift, float* scale) const;
  // Forward + backward of one batch (rows % 128 == 0) without an update: gradients of the
  // mean squared error (flat layout, host) and the loss.
  void gradients(const float* X, const float* Y, int64_t rows, float* host_grads, float* loss);
  // Adam training over shuffled batches; per-epoch mean loss into losses[epochs] (host).
  void train(const float* X, const float* Y, int64_t n, int epochs, int64_t batch, float lr,
             uint64_t seed, float* losses);
  void predict(const float* X, int64_t n, float* Y);
  void check_error();

 private:
  Impl* p;
};
// C[M,N] (f32, device) = A[M,K] B[N,K]^T, bf16 operands both K-major, on the tensor cores.
// M % 128, N % 32, K % (64 * ksplit); ksplit > 1 adds into C with atomics.
void umma_gemm_f32(const void* A, const void* B, float* C, int64_t M, int64_t N, int64_t K, int ksplit,
                   cudaStream_t s);

// Exact brute-force kNN (knn.cu): for each of the n rows of X [n, d] (f32, device), the k
// nearest other rows by the reference example's f32 Euclidean distance, ordered by (distance,
// index); out_idx / out_dist [n, k] on the device.  Synchronises `s`.
constexpr int KNN_MAX_K = 32;         // through the tensor-core candidate pass
constexpr int KNN_MAX_K_EXACT = 128;  // every row on the exact CUDA-core path
struct KnnStats {
  uint32_t splits = 0;         // database splits of the candidate pass
  uint32_t fallback_rows = 0;  // rows whose certificate failed and were recomputed exactly
  float scale = 1.0f;          // power of two applied to the centred rows before FP16 rounding
  uint32_t reordered = 0;      // 1 when the scan ran in pivot (locality) order
  float candidate_ms = 0.0f;   // CUDA-event time of the tensor-core candidate pass
  uint32_t all_exact = 0;      // 1 when k > KNN_MAX_K sent every row to the exact path
};
KnnStats knn_bruteforce(const float* X, uint64_t n, uint64_t d, uint64_t k, uint32_t* out_idx, float* out_dist,
                        cudaStream_t s);

}  // namespace ub
