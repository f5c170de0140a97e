/*
 * umap_b200.h -- C ABI of the B200 (sm_100a) UMAP fit path.
 *
 * Each entry point stands in for one item of the Rust API of wilsonzlin/umap-rs 0.4.5
 * (paths below are relative to that project).  A Rust crate keeps its public API and
 * implements the bodies by calling these functions.
 *
 * Conventions
 *  - Every function returns an int status: UMAP_OK (0) or a UMAP_ERR_* code.  Where the
 *    reference panics, the same condition returns a code and umap_last_error() holds the
 *    reference's panic message text (e.g. "Cannot step 5 epochs: would exceed
 *    total_epochs 20 (current: 18)", umap-rs/src/optimizer.rs:298-304).
 *  - Arrays are row-major and contiguous.  Pointers named host_* are host memory; the
 *    *_device variants take device pointers on the current CUDA device.
 *  - Handles are opaque.  A function documented as "consumes" takes ownership (the
 *    reference moves the value); the caller must not use or free that handle afterwards,
 *    even when the call fails.
 *  - One CUDA stream per handle; a handle is not thread-safe (the reference takes
 *    &mut self).  Distinct handles may be used from distinct threads.
 *  - No CPU fallback: without a usable CUDA device, compute calls return UMAP_ERR_CUDA.
 */
#ifndef UMAP_B200_H
#define UMAP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UMAP_B200_ABI_VERSION 1

enum umap_status {
  UMAP_OK = 0,
  UMAP_ERR_INVALID_ARGUMENT = 1, /* reference: validate_parameters / shape panics   */
  UMAP_ERR_OVERSTEP = 2,         /* reference: Optimizer::step_epochs assert         */
  UMAP_ERR_CUDA = 3,             /* CUDA runtime error or no device                  */
  UMAP_ERR_OUT_OF_MEMORY = 4,
  UMAP_ERR_FORMAT = 5,           /* checkpoint bytes truncated / corrupt / wrong kind */
  UMAP_ERR_IO = 6,
  UMAP_ERR_NULL = 7,             /* NULL handle or pointer                           */
  UMAP_ERR_UNSUPPORTED = 8       /* e.g. an output metric with no device implementation */
};

/* MetricType (umap-rs/src/metric.rs:6-12) selects the SGD update rule: the Euclidean
 * specialisation (layout/optimize_layout_euclidean.rs) or the generic-metric rule
 * (layout/optimize_layout_generic.rs), which calls the output metric's distance and gradient. */
enum umap_metric_type {
  UMAP_METRIC_EUCLIDEAN = 0,
  UMAP_METRIC_GENERIC = 1
};

/* Output metrics with a device implementation, for the generic rule (the reference's
 * `output_metric: &dyn Metric`).  The reference ships one Metric, EuclideanMetric
 * (distances.rs:10-50): distance sqrt(sum (x-y)^2), gradient (x-y) / (distance + 1e-6). */
enum umap_output_metric {
  UMAP_OUTPUT_METRIC_EUCLIDEAN = 0
};

/* UmapConfig (umap-rs/src/config.rs:205-235).  Option<T> fields are a has_* flag plus a
 * value.  Defaults (umap_config_default) are the reference's Default impls:
 * config.rs:43-52, :117-127, :171-180, :226-235. */
typedef struct umap_config {
  uint64_t n_components;            /* 2 */
  /* ManifoldParams */
  float min_dist;                   /* 0.1 */
  float spread;                     /* 1.0 */
  int32_t has_a; float a;           /* None */
  int32_t has_b; float b;           /* None */
  /* GraphParams */
  uint64_t n_neighbors;             /* 15 */
  float local_connectivity;         /* 1.0 */
  float set_op_mix_ratio;           /* 1.0 */
  int32_t has_disconnection_distance; float disconnection_distance; /* None */
  int32_t symmetrize;               /* true */
  /* OptimizationParams */
  int32_t has_n_epochs; uint64_t n_epochs; /* None */
  float learning_rate;              /* 1.0 */
  uint64_t negative_sample_rate;    /* 5 */
  float repulsion_strength;         /* 1.0 */
} umap_config;

typedef struct umap_manifold umap_manifold;   /* LearnedManifold, manifold.rs:14-38  */
typedef struct umap_optimizer umap_optimizer; /* Optimizer, optimizer.rs:27-56       */
typedef struct umap_fitted umap_fitted;       /* FittedUmap, embedding.rs:438-443    */

/* ---- library ---------------------------------------------------------------------- */
/* Device pointers (the *_device calls, dev_* arguments): a call first waits for the work
 * queued so far on the legacy default stream (stream 0, where PyTorch queues by default),
 * then works on its handle's own stream and returns when its results are complete.  Inputs
 * produced on any other stream must be complete before the call.  Calls on different
 * handles may run concurrently from different host threads. */
/* Message of the last failed call on this thread ("" if none). */
const char* umap_last_error(void);
int umap_abi_version(void);
/* Replaces `impl Default for UmapConfig` (config.rs:226-235). */
int umap_config_default(umap_config* out);
/* Replaces umap/find_ab_params.rs:9-82 (host code; no GPU needed). */
int umap_find_ab_params(float spread, float min_dist, float* a_out, float* b_out);

/* ---- Umap::learn_manifold (embedding.rs:149-240) ----------------------------------- */
/* n_samples = data.shape()[0] (the reference reads nothing else from `data`).
 * knn_indices u32[knn_rows, knn_cols], knn_dists f32[knn_rows, knn_cols]. */
int umap_learn_manifold(const umap_config* cfg, uint64_t n_samples,
                        const uint32_t* host_knn_indices, const float* host_knn_dists,
                        uint64_t knn_rows, uint64_t knn_cols, umap_manifold** out);
int umap_learn_manifold_device(const umap_config* cfg, uint64_t n_samples,
                               const uint32_t* dev_knn_indices, const float* dev_knn_dists,
                               uint64_t knn_rows, uint64_t knn_cols, umap_manifold** out);

/* ---- LearnedManifold accessors (manifold.rs:40-55) --------------------------------- */
int umap_manifold_n_vertices(const umap_manifold* m, uint64_t* out);
int umap_manifold_curve_params(const umap_manifold* m, float* a, float* b);
/* graph(): CsMatI<f32,u32,usize>; nnz then copy of indptr[n+1], indices[nnz], data[nnz]. */
int umap_manifold_graph_nnz(const umap_manifold* m, uint64_t* nnz);
int umap_manifold_graph_copy(const umap_manifold* m, uint64_t* host_indptr,
                             uint32_t* host_indices, float* host_data);
/* sigmas / rhos fields (manifold.rs:20-26). */
int umap_manifold_sigmas_rhos(const umap_manifold* m, float* host_sigmas, float* host_rhos);
/* Counts behind raise_disconnected_warning (embedding.rs:187-230). */
int umap_manifold_disconnection_counts(const umap_manifold* m, uint64_t* edges_removed,
                                       uint64_t* vertices_disconnected);
/* #[derive(Clone)] on LearnedManifold (manifold.rs:14). */
int umap_manifold_clone(const umap_manifold* m, umap_manifold** out);
int umap_manifold_free(umap_manifold* m);

/* ---- Optimizer (optimizer.rs:74-403) ----------------------------------------------- */
/* Optimizer::new (optimizer.rs:74-290).  Consumes `manifold`.  init f32[rows, dims]. */
int umap_optimizer_new(umap_manifold* manifold, const float* host_init, uint64_t rows,
                       uint64_t dims, uint64_t total_epochs, const umap_config* cfg,
                       int metric_type, umap_optimizer** out);
int umap_optimizer_new_device(umap_manifold* manifold, const float* dev_init, uint64_t rows,
                              uint64_t dims, uint64_t total_epochs, const umap_config* cfg,
                              int metric_type, umap_optimizer** out);
/* Optimizer::step_epochs (optimizer.rs:297-366).  UMAP_ERR_OVERSTEP with the reference's
 * message when current_epoch + n > total_epochs.  A MetricType::Generic optimizer steps with
 * the Euclidean output metric; _metric names the output metric (umap_output_metric) and
 * returns UMAP_ERR_UNSUPPORTED for one without a device implementation.  A Euclidean
 * optimizer ignores it, as the reference does. */
int umap_optimizer_step_epochs(umap_optimizer* opt, uint64_t n);
int umap_optimizer_step_epochs_metric(umap_optimizer* opt, uint64_t n, int output_metric);
int umap_optimizer_current_epoch(const umap_optimizer* opt, uint64_t* out);   /* :369 */
int umap_optimizer_total_epochs(const umap_optimizer* opt, uint64_t* out);    /* :374 */
int umap_optimizer_remaining_epochs(const umap_optimizer* opt, uint64_t* out);/* :379 */
/* embedding() (optimizer.rs:384): copies f32[n_vertices, dims] to host. */
int umap_optimizer_embedding(const umap_optimizer* opt, float* host_out);
/* Device pointer to the live embedding (valid until the next call on `opt`). */
int umap_optimizer_embedding_device(umap_optimizer* opt, float** dev_ptr);
int umap_optimizer_dims(const umap_optimizer* opt, uint64_t* n_vertices, uint64_t* dims);
/* manifold() (optimizer.rs:389): borrowed, owned by `opt`. */
int umap_optimizer_manifold(const umap_optimizer* opt, const umap_manifold** out);
/* into_fitted (optimizer.rs:397-403).  Consumes `opt`. */
int umap_optimizer_into_fitted(umap_optimizer* opt, const umap_config* cfg, umap_fitted** out);
int umap_optimizer_free(umap_optimizer* opt);
/* Extension (the reference has no seed API; its RNG is unseeded): the seed of the
 * counter-based generator that draws negative samples.  Default 0. */
int umap_optimizer_set_seed(umap_optimizer* opt, uint64_t seed);
/* Number of kept edges (the reference's head/tail length, optimizer.rs:133-163). */
int umap_optimizer_n_edges(const umap_optimizer* opt, uint64_t* out);
/* The reference's per-edge arrays in its row-major edge order: head/tail u32[E],
 * epochs_per_sample f64[E] (optimizer.rs:33-35) and the schedule state at current_epoch
 * (optimizer.rs:41-43).  Any pointer may be NULL to skip that array. */
int umap_optimizer_export_edges(const umap_optimizer* opt, uint32_t* head, uint32_t* tail,
                                double* epochs_per_sample, double* epoch_of_next_sample,
                                double* epoch_of_next_negative_sample,
                                double* epochs_per_negative_sample);
/* Extension: exact totals of fired edges and negative samples that step_epochs would
 * process over epochs [start, end) (for throughput accounting). */
int umap_optimizer_schedule_totals(const umap_optimizer* opt, uint64_t start, uint64_t end,
                                   uint64_t* fired, uint64_t* negatives);

/* Extension: CUDA-event time (ms) of the epoch loop of the last step_epochs call, measured
 * on the optimizer's stream (the SGD kernels only; no host overhead). */
int umap_optimizer_last_step_ms(const umap_optimizer* opt, float* ms);
/* Extension: device memory freed by the library is cached for reuse by later calls (growing
 * the device pool costs ~100 ms per large block).  This returns the cached blocks to the
 * CUDA pool; *released_bytes (may be NULL) receives their total size. */
int umap_release_cached_memory(uint64_t* released_bytes);
/* Extension: number of this library's kernel launches so far in this process. */
int umap_kernel_launches(uint64_t* out);

/* ---- FittedUmap (embedding.rs:438-524) --------------------------------------------- */
int umap_fitted_embedding(const umap_fitted* f, float* host_out);             /* :462 */
int umap_fitted_dims(const umap_fitted* f, uint64_t* n_vertices, uint64_t* dims);
int umap_fitted_manifold(const umap_fitted* f, const umap_manifold** out);    /* :485 */
int umap_fitted_config(const umap_fitted* f, umap_config* out);               /* :490 */
int umap_fitted_free(umap_fitted* f);

/* ---- Umap::fit (embedding.rs:274-337) ---------------------------------------------- */
/* learn_manifold -> Optimizer::new -> one step_epochs(total) -> into_fitted -> rows whose
 * graph row sums to 0 become NaN.  init f32[init_rows, init_cols]. */
int umap_fit(const umap_config* cfg, uint64_t n_samples, const uint32_t* host_knn_indices,
             const float* host_knn_dists, uint64_t knn_rows, uint64_t knn_cols,
             const float* host_init, uint64_t init_rows, uint64_t init_cols,
             umap_fitted** out);
int umap_fit_device(const umap_config* cfg, uint64_t n_samples, const uint32_t* dev_knn_indices,
                    const float* dev_knn_dists, uint64_t knn_rows, uint64_t knn_cols,
                    const float* dev_init, uint64_t init_rows, uint64_t init_cols,
                    umap_fitted** out);
/* The rest of Umap::fit once the manifold is learned (embedding.rs:299-337): optimise for
 * n_epochs (or the 500 / 200 default), then NaN rows for vertices with an empty graph row.
 * Consumes `manifold`.  Lets a caller build the graph while it prepares `init`. */
int umap_fit_manifold(umap_manifold* manifold, const umap_config* cfg, const float* host_init,
                      uint64_t init_rows, uint64_t init_cols, umap_fitted** out);
int umap_fit_manifold_device(umap_manifold* manifold, const umap_config* cfg, const float* dev_init,
                             uint64_t init_rows, uint64_t init_cols, umap_fitted** out);
/* The same with the Umap's output metric (embedding.rs:311-321): its MetricType picks the
 * update rule and `output_metric` (umap_output_metric) is passed to step_epochs. */
int umap_fit_manifold_metric(umap_manifold* manifold, const umap_config* cfg, const float* host_init,
                             uint64_t init_rows, uint64_t init_cols, int metric_type, int output_metric,
                             umap_fitted** out);
int umap_fit_manifold_metric_device(umap_manifold* manifold, const umap_config* cfg, const float* dev_init,
                                    uint64_t init_rows, uint64_t init_cols, int metric_type,
                                    int output_metric, umap_fitted** out);

/* ---- kNN producer (the step before the fit; the reference takes kNN as input) ---------
 * Exact brute-force k nearest neighbours as the reference's example computes them
 * (examples/src/bin/mnist_demo.rs:203-229): for each row of data [n, dim] (row-major f32) the
 * k other rows with the smallest sqrt(sum_i (x_i - y_i)^2) (f32, summed in coordinate order),
 * ordered by distance then index, the row itself excluded; with fewer than k other rows the
 * remaining slots are 0 / 0.0.  Outputs [n, k] row-major.  1 <= k <= 128.  For k <= 32
 * candidates come from an FP16 tensor-core distance pass; every row is then either certified
 * exact against an error bound or recomputed exactly, so the result equals the f32 brute
 * force.  For 32 < k <= 128 every row is computed exactly on the CUDA cores (slower).
 * `rows_recomputed` (nullable) receives the number of rows that needed the exact recompute.
 * UMAP_ERR_INVALID_ARGUMENT for NaN or infinite inputs (the reference's sort panics). */
int umap_knn_bruteforce(const float* host_data, uint64_t n, uint64_t dim, uint64_t k,
                        uint32_t* host_knn_indices, float* host_knn_dists, uint64_t* rows_recomputed);
int umap_knn_bruteforce_device(const float* dev_data, uint64_t n, uint64_t dim, uint64_t k,
                               uint32_t* dev_knn_indices, float* dev_knn_dists, uint64_t* rows_recomputed);
/* Profile of this thread's last kNN call: CUDA-event time of the tensor-core candidate pass,
 * rows recomputed exactly, and whether the scan ran in pivot (locality) order.  Nullable. */
int umap_knn_last_profile(float* candidate_pass_ms, uint64_t* rows_recomputed, uint32_t* reordered);

/* ---- batched instances (no counterpart in the reference: a fit per dataset) --------
 * n_instances independent fits in one problem.  Instance s owns points
 * [offsets[s], offsets[s+1]) of the concatenated arrays (host offsets, u64[n_instances+1],
 * offsets[0] = 0); its kNN ids are local to it (0..n_s-1).  Each instance is validated like
 * learn_manifold (messages prefixed "instance s: ").  Every epoch is one kernel launch over
 * all instances; the SGD task length and block shape are autotuned on the first batch of a
 * given size.  The result is an ordinary optimizer handle (step_epochs, embedding,
 * export_edges, schedule_totals, into_fitted work on it; checkpoints do not). */
int umap_batch_optimizer_new(const umap_config* cfg, uint64_t n_instances, const uint64_t* host_offsets,
                             const uint32_t* host_knn_indices, const float* host_knn_dists,
                             uint64_t knn_cols, const float* host_init, uint64_t init_cols,
                             uint64_t total_epochs, umap_optimizer** out);
int umap_batch_optimizer_new_device(const umap_config* cfg, uint64_t n_instances,
                                    const uint64_t* host_offsets, const uint32_t* dev_knn_indices,
                                    const float* dev_knn_dists, uint64_t knn_cols, const float* dev_init,
                                    uint64_t init_cols, uint64_t total_epochs, umap_optimizer** out);
/* Umap::fit for every instance at once: n_epochs from cfg (or the shared default), rows
 * with an empty graph row become NaN; writes f32[total points, init_cols]. */
int umap_batch_fit(const umap_config* cfg, uint64_t n_instances, const uint64_t* host_offsets,
                   const uint32_t* host_knn_indices, const float* host_knn_dists, uint64_t knn_cols,
                   const float* host_init, uint64_t init_cols, float* host_embedding_out);
int umap_batch_fit_device(const umap_config* cfg, uint64_t n_instances, const uint64_t* host_offsets,
                          const uint32_t* dev_knn_indices, const float* dev_knn_dists, uint64_t knn_cols,
                          const float* dev_init, uint64_t init_cols, float* dev_embedding_out);
/* Extension: the SGD task length and threads per block in use (autotuned for batches). */
int umap_optimizer_tuning(const umap_optimizer* opt, uint32_t* chunk, uint32_t* block_threads);
/* Extension: how the SGD layout is laid out (bit flags): UMAP_LAYOUT_LANE_MAJOR (a lane's
 * edges contiguous; else interleaved by lane), UMAP_LAYOUT_EIGHT_NEGATIVES (the epoch kernel's
 * 8-row-loads-in-flight register budget), UMAP_LAYOUT_TWELVE_NEGATIVES (the 12-row budget of
 * renamed layouts; neither flag: 4), UMAP_LAYOUT_RENAMED (vertices renamed into a locality
 * order; DRAM-bound plain fits), UMAP_LAYOUT_GENERIC_RULE (the optimizer's MetricType is
 * Generic), and the order in which tasks are dealt to warps: UMAP_LAYOUT_RATE_ORDER (by
 * length, then by mean firing rate; small graphs and batched instances), UMAP_LAYOUT_BLOCK_ORDER (by length inside
 * blocks of 4096 consecutive rows; renamed layouts), UMAP_LAYOUT_ROW_ORDER (row order, forced
 * only); none of the three: by length. */
#define UMAP_LAYOUT_LANE_MAJOR 1u
#define UMAP_LAYOUT_EIGHT_NEGATIVES 2u
#define UMAP_LAYOUT_RENAMED 4u
#define UMAP_LAYOUT_GENERIC_RULE 8u
#define UMAP_LAYOUT_TWELVE_NEGATIVES 16u
#define UMAP_LAYOUT_RATE_ORDER 32u
#define UMAP_LAYOUT_BLOCK_ORDER 64u
#define UMAP_LAYOUT_ROW_ORDER 128u
int umap_optimizer_layout_flags(const umap_optimizer* opt, uint32_t* flags);

/* ---- serde checkpoints (optimizer.rs:27, manifold.rs:14, embedding.rs:438) ---------
 * The byte format is this library's own little-endian layout carrying every field of the
 * reference struct (not bincode).  *_serialize writes at most `cap` bytes and sets
 * *needed to the full size (call with buf=NULL, cap=0 to query). */
int umap_manifold_serialize(const umap_manifold* m, uint8_t* buf, uint64_t cap, uint64_t* needed);
int umap_manifold_deserialize(const uint8_t* buf, uint64_t len, umap_manifold** out);
int umap_optimizer_serialize(const umap_optimizer* o, uint8_t* buf, uint64_t cap, uint64_t* needed);
int umap_optimizer_deserialize(const uint8_t* buf, uint64_t len, umap_optimizer** out);
int umap_fitted_serialize(const umap_fitted* f, uint8_t* buf, uint64_t cap, uint64_t* needed);
int umap_fitted_deserialize(const uint8_t* buf, uint64_t len, umap_fitted** out);
/* The same three objects in the reference's own checkpoint bytes: its serde derives
 * (manifold.rs:14, optimizer.rs:27, embedding.rs:438, config.rs) encoded by bincode 1.3
 * `serialize`, as its tests do (tests.rs:150, :179, :207).  Layout: fixed-width little-endian
 * numbers, usize as u64, sequences as a u64 length then elements, Option as a u8 tag, unit
 * enum variants as a u32 index; ndarray arrays as {v: u8 = 1, dim, data}; the sprs graph as
 * {storage (CSR = 0), nrows, ncols, indptr, indices, data}.  The serde formats of ndarray and
 * sprs are not in the reference tree and are restated from those crates (no Rust-written
 * file has been checked).  Loading an Optimizer recomputes its schedule state from
 * epochs_per_sample and current_epoch (the stored arrays are length-checked, then skipped);
 * the disconnection counts of a loaded manifold are recomputed (edges_removed reads 0). */
int umap_manifold_serialize_bincode(const umap_manifold* m, uint8_t* buf, uint64_t cap, uint64_t* needed);
int umap_manifold_deserialize_bincode(const uint8_t* buf, uint64_t len, umap_manifold** out);
int umap_optimizer_serialize_bincode(const umap_optimizer* opt, uint8_t* buf, uint64_t cap, uint64_t* needed);
int umap_optimizer_deserialize_bincode(const uint8_t* buf, uint64_t len, umap_optimizer** out);
int umap_fitted_serialize_bincode(const umap_fitted* f, uint8_t* buf, uint64_t cap, uint64_t* needed);
int umap_fitted_deserialize_bincode(const uint8_t* buf, uint64_t len, umap_fitted** out);

/* ---- kernel-level entry points (parity hooks, device pointers) ---------------------- */
/* SmoothKnnDist::exec (umap/smooth_knn_dist.rs:60-198) on device arrays. */
int umap_smooth_knn_dist_device(const float* dev_dists, uint64_t n, uint64_t k,
                                uint64_t n_iter, float local_connectivity, float bandwidth,
                                float* dev_sigmas, float* dev_rhos);
/* Stable LSD radix sort of (u32 key, u32 value) pairs by key bits [0, end_bit): the
 * transpose step that replaces build_csc_structure (fuzzy_simplicial_set.rs:310-370).
 * dev_values_in may be NULL (values = 0..n-1).  Neither output may overlap an input or the
 * other output (UMAP_ERR_INVALID_ARGUMENT). */
int umap_radix_sort_pairs_device(const uint32_t* dev_keys_in, const uint32_t* dev_values_in,
                                 uint32_t* dev_keys_out, uint32_t* dev_values_out,
                                 uint64_t n, int end_bit);

/* The negative samples of the SGD epoch kernel (optimize_layout_euclidean.rs:313-314, which
 * draws rng.random_range(0..n_vertices) from an unseeded thread-local generator; here a
 * counter-based generator keyed by (seed, edge entry, epoch)).  For entries first_entry ..
 * first_entry + n_entries - 1 firing at `epoch`, draw q (q < per_entry <= 64) of entry e is
 * written to dev_out[(e - first_entry) * per_entry + q], in [lo, lo + range): exactly the
 * values the epoch kernel uses for an optimizer whose seed is `seed`.  For statistical
 * tests of the generator. */
int umap_sgd_negative_draws_device(uint64_t seed, uint64_t first_entry, uint64_t n_entries,
                                   uint32_t epoch, uint32_t per_entry, uint32_t lo, uint32_t range,
                                   uint32_t* dev_out);

/* The SGD schedule's negative count per firing (optimize_layout_euclidean.rs:308-311, :343:
 * n_neg = floor((n - epoch_of_next_negative_sample) / epochs_per_negative_sample)), as the
 * epoch kernel evaluates it from an edge's stored schedule word dev_q[i] (ceil(2^32 /
 * epochs_per_sample) - 1) at epoch dev_epoch[i] (below 2^21, the largest total_epochs an
 * optimizer accepts); 0 where the edge does not fire then. */
int umap_sgd_negatives_per_firing_device(const uint32_t* dev_q, const uint32_t* dev_epoch, uint64_t count,
                                         uint32_t negative_sample_rate, uint32_t* dev_out);

/* Measurement hook (no counterpart in the reference): the device's rate for the SGD epoch's
 * random access pattern, the denominator of its L2 roofline.  One timed launch (after one
 * untimed one that brings the table into L2) of about `accesses` random 8-byte row reads
 * (mode 0) or red.add row moves (mode 1) on dev_table [n_rows][2] f32; *ms = its CUDA-event
 * time, *accesses_done = the accesses it made.  Mode 0 writes 303,104 floats to dev_out;
 * mode 1 changes the table. */
int umap_random_rows_probe_device(float* dev_table, uint64_t n_rows, uint64_t accesses, int mode, float* dev_out,
                                  float* ms, uint64_t* accesses_done);

/* Allocation-free variant of umap_radix_sort_pairs_device (no counterpart in the
 * reference; the reference has no device code).  For callers that cannot allocate device
 * memory when they sort: a host application whose allocator owns the whole GPU heap, or a
 * latency-critical loop that must not enter the CUDA allocator.  It performs no cudaMalloc
 * / cudaFree and no allocating library call: its scratch is a static device array of about
 * 9 MiB.  The CUDA runtime places that array on a GPU when it loads the library's sort
 * module there (lazily, by default: at the module's first kernel launch or symbol lookup on
 * that device), and the GPU then holds it until the process exits.  That load is itself a
 * device allocation, so a caller that later reserves the whole heap should first call this
 * entry point once per device with n = 0 (buffers may then be NULL): that call loads the
 * module, looks up the array's device address (cudaGetSymbolAddress) with that device
 * current, and queues no GPU work.  Make that first call before any stream capture.
 * At most umap_radix_sort_noalloc_max_pairs() pairs (1,048,576); larger n returns
 * UMAP_ERR_INVALID_ARGUMENT, as do outputs that overlap an input or each other.  Work is
 * queued on `stream` (NULL = the default stream), and every call synchronises that stream
 * (cudaStreamSynchronize) before it returns.  All calls share the array: calls whose GPU
 * work overlaps (on different streams or threads) race on it and must be serialised by the
 * caller. */
int umap_radix_sort_pairs_device_noalloc(const uint32_t* dev_keys_in, const uint32_t* dev_values_in,
                                         uint32_t* dev_keys_out, uint32_t* dev_values_out,
                                         uint64_t n, int end_bit, void* stream);
int umap_radix_sort_noalloc_max_pairs(uint64_t* out);

/* ---- Learned warm start (no counterpart in the reference: its caller supplies `init`) ----
 * An MLP in_dim -> 256 -> 256 -> out_dim with exact-erf GELU, bf16 weights and activations,
 * fp32 accumulation on the tensor cores, trained with Adam (beta 0.9 / 0.999, eps 1e-8) on
 * the mean squared error to target embeddings; its predictions initialise a shortened fit.
 * Parameters are one flat fp32 array of umap_mlp_param_count() values in the order
 * W1 [256][in_dim], b1 [256], W2 [256][256], b2 [256], W3 [out_dim][256], b3 [out_dim]
 * (weights row-major, one row per output unit).  in_dim: a multiple of 64 up to 4096;
 * out_dim: 1..4.  dev_* pointers are device memory (row-major rows of in_dim / out_dim
 * floats); the others are host memory. */
typedef struct umap_mlp umap_mlp;
int umap_mlp_param_count(uint64_t in_dim, uint64_t out_dim, uint64_t* out);
int umap_mlp_new(uint64_t in_dim, uint64_t out_dim, const float* params, umap_mlp** out);
int umap_mlp_dims(const umap_mlp* m, uint64_t* in_dim, uint64_t* out_dim);
int umap_mlp_get_params(const umap_mlp* m, float* params);
int umap_mlp_set_params(umap_mlp* m, const float* params);
/* Input standardisation x' = (x - shift) * scale (per input column) applied before the first
 * layer; fit_input_norm sets shift = column mean and scale = 1 / column std of dev_x. */
int umap_mlp_fit_input_norm_device(umap_mlp* m, const float* dev_x, uint64_t rows);
int umap_mlp_input_norm(const umap_mlp* m, float* shift, float* scale);
int umap_mlp_set_input_norm(umap_mlp* m, const float* shift, const float* scale);
/* One forward + backward over `rows` rows (a multiple of 128) without an update: gradients of
 * the mean squared error in the flat parameter order into `grads`, the loss into *loss. */
int umap_mlp_gradients_device(umap_mlp* m, const float* dev_x, const float* dev_y, uint64_t rows,
                              float* grads, float* loss);
/* Adam over `epochs` shuffled passes of mini-batches of `batch` rows (a multiple of 128; the
 * last partial batch of each pass is dropped).  losses (may be NULL) receives each epoch's
 * mean batch loss. */
int umap_mlp_train_device(umap_mlp* m, const float* dev_x, const float* dev_y, uint64_t rows,
                          uint64_t epochs, uint64_t batch, float learning_rate, uint64_t seed,
                          float* losses);
int umap_mlp_predict_device(umap_mlp* m, const float* dev_x, uint64_t rows, float* dev_y);
int umap_mlp_free(umap_mlp* m);
/* The tensor-core GEMM the MLP is built from: dev_c [m][n] (fp32) = A [m][k] * B [n][k]^T with
 * bf16 A and B (both K contiguous).  m % 128 == 0, n % 32 == 0, k % (64 * k_splits) == 0;
 * k_splits > 1 adds the split partial sums into dev_c with atomics (zero it first). */
int umap_gemm_bf16_device(const void* dev_a, const void* dev_b, float* dev_c, uint64_t m, uint64_t n,
                          uint64_t k, uint64_t k_splits);

/* The whole warm start in one call, standing in for the `init` a caller hands to Umap::fit
 * (embedding.rs:274-280): a plain fit of a subsample for sub_epochs, the network trained for
 * mlp_epochs of Adam on (subsample rows, that embedding), its prediction for every row as
 * init, then Umap::fit of all rows for `epochs` epochs (the prune threshold and the
 * learning-rate decay follow that epoch count, optimizer.rs:96-102, :317).  The full data's
 * graph and that fit's optimizer set-up (prune, schedule, task layout) are built on another
 * stream and host thread while the subsample is fitted and the network trained
 * (full_graph_overlapped below times them). */
typedef struct umap_warm_start_params {
  uint64_t sub_epochs;            /* 500: the subsample's plain fit */
  uint64_t epochs;                /* 100: the fit of all rows from the learned init */
  uint64_t mlp_epochs;            /* 20 */
  uint64_t batch;                 /* 4096; rounded down to a multiple of 128 and at most the subsample */
  float mlp_learning_rate;        /* 1e-3 (Adam) */
  int32_t has_learning_rate;      /* 0: the final fit uses cfg's learning_rate */
  float learning_rate;
  uint64_t seed;                  /* network initialisation, batch shuffles, default subsample init */
} umap_warm_start_params;
int umap_warm_start_params_default(umap_warm_start_params* out);
/* Phases reported in phase_ms (milliseconds of host wall time, in this order). */
#define UMAP_WARM_START_PHASES 8  /* prepare, subsample_fit, mlp_train, mlp_predict,
                                     wait_full_graph, fit, full_graph_overlapped, total */
/* dev_data f32 [n_samples][data_dim] (any data_dim up to 4096: rows are zero-padded to a
 * multiple of 64 for the network); dev_knn_* the full data's kNN [n_samples][knn_cols] as for
 * umap_fit_device; dev_sub_rows u32[n_sub] the subsample's row numbers; dev_sub_knn_* its own
 * kNN [n_sub][knn_cols] with ids local to the subsample; dev_sub_init f32 [n_sub][n_components]
 * or NULL for uniform [-10, 10] from `seed`.  phase_ms (UMAP_WARM_START_PHASES floats) and
 * mlp_losses (mlp_epochs floats, each epoch's mean batch loss) are host arrays and may be
 * NULL.  n_sub must leave at least 128 rows with a non-empty graph row. */
int umap_warm_start_fit_device(const umap_config* cfg, const umap_warm_start_params* params,
                               const float* dev_data, uint64_t n_samples, uint64_t data_dim,
                               const uint32_t* dev_knn_indices, const float* dev_knn_dists,
                               uint64_t knn_cols, const uint32_t* dev_sub_rows, uint64_t n_sub,
                               const uint32_t* dev_sub_knn_indices, const float* dev_sub_knn_dists,
                               const float* dev_sub_init, umap_fitted** out, float* phase_ms,
                               float* mlp_losses);

#ifdef __cplusplus
}
#endif
#endif /* UMAP_B200_H */
