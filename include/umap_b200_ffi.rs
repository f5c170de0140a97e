// Generated from include/umap_b200.h by include/gen_rust_ffi.py; do not edit by hand.
// Every entry point of the B200 UMAP library, for a Rust crate's src/ffi.rs.
#![allow(non_camel_case_types, dead_code)]
use std::os::raw::{c_char, c_int, c_void};

pub const UMAP_B200_ABI_VERSION: c_int = 1;
pub const UMAP_OK: c_int = 0;
pub const UMAP_ERR_INVALID_ARGUMENT: c_int = 1;
pub const UMAP_ERR_OVERSTEP: c_int = 2;
pub const UMAP_ERR_CUDA: c_int = 3;
pub const UMAP_ERR_OUT_OF_MEMORY: c_int = 4;
pub const UMAP_ERR_FORMAT: c_int = 5;
pub const UMAP_ERR_IO: c_int = 6;
pub const UMAP_ERR_NULL: c_int = 7;
pub const UMAP_ERR_UNSUPPORTED: c_int = 8;
pub const UMAP_METRIC_EUCLIDEAN: c_int = 0;
pub const UMAP_METRIC_GENERIC: c_int = 1;
pub const UMAP_OUTPUT_METRIC_EUCLIDEAN: c_int = 0;
pub const UMAP_LAYOUT_LANE_MAJOR: u32 = 1;
pub const UMAP_LAYOUT_EIGHT_NEGATIVES: u32 = 2;
pub const UMAP_LAYOUT_RENAMED: u32 = 4;
pub const UMAP_LAYOUT_GENERIC_RULE: u32 = 8;
pub const UMAP_LAYOUT_TWELVE_NEGATIVES: u32 = 16;
pub const UMAP_LAYOUT_RATE_ORDER: u32 = 32;
pub const UMAP_LAYOUT_BLOCK_ORDER: u32 = 64;
pub const UMAP_LAYOUT_ROW_ORDER: u32 = 128;
pub const UMAP_WARM_START_PHASES: usize = 8;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct umap_config {
    pub n_components: u64,
    pub min_dist: f32,
    pub spread: f32,
    pub has_a: i32,
    pub a: f32,
    pub has_b: i32,
    pub b: f32,
    pub n_neighbors: u64,
    pub local_connectivity: f32,
    pub set_op_mix_ratio: f32,
    pub has_disconnection_distance: i32,
    pub disconnection_distance: f32,
    pub symmetrize: i32,
    pub has_n_epochs: i32,
    pub n_epochs: u64,
    pub learning_rate: f32,
    pub negative_sample_rate: u64,
    pub repulsion_strength: f32,
}

#[repr(C)]
pub struct umap_manifold {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct umap_optimizer {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct umap_fitted {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct umap_mlp {
    _opaque: [u8; 0],
}

extern "C" {
    pub fn umap_last_error() -> *const c_char;
    pub fn umap_abi_version() -> c_int;
    pub fn umap_config_default(out: *mut umap_config) -> c_int;
    pub fn umap_find_ab_params(spread: f32, min_dist: f32, a_out: *mut f32, b_out: *mut f32) -> c_int;
    pub fn umap_learn_manifold(cfg: *const umap_config, n_samples: u64, host_knn_indices: *const u32, host_knn_dists: *const f32, knn_rows: u64, knn_cols: u64, out: *mut *mut umap_manifold) -> c_int;
    pub fn umap_learn_manifold_device(cfg: *const umap_config, n_samples: u64, dev_knn_indices: *const u32, dev_knn_dists: *const f32, knn_rows: u64, knn_cols: u64, out: *mut *mut umap_manifold) -> c_int;
    pub fn umap_manifold_n_vertices(m: *const umap_manifold, out: *mut u64) -> c_int;
    pub fn umap_manifold_curve_params(m: *const umap_manifold, a: *mut f32, b: *mut f32) -> c_int;
    pub fn umap_manifold_graph_nnz(m: *const umap_manifold, nnz: *mut u64) -> c_int;
    pub fn umap_manifold_graph_copy(m: *const umap_manifold, host_indptr: *mut u64, host_indices: *mut u32, host_data: *mut f32) -> c_int;
    pub fn umap_manifold_sigmas_rhos(m: *const umap_manifold, host_sigmas: *mut f32, host_rhos: *mut f32) -> c_int;
    pub fn umap_manifold_disconnection_counts(m: *const umap_manifold, edges_removed: *mut u64, vertices_disconnected: *mut u64) -> c_int;
    pub fn umap_manifold_clone(m: *const umap_manifold, out: *mut *mut umap_manifold) -> c_int;
    pub fn umap_manifold_free(m: *mut umap_manifold) -> c_int;
    pub fn umap_optimizer_new(manifold: *mut umap_manifold, host_init: *const f32, rows: u64, dims: u64, total_epochs: u64, cfg: *const umap_config, metric_type: c_int, out: *mut *mut umap_optimizer) -> c_int;
    pub fn umap_optimizer_new_device(manifold: *mut umap_manifold, dev_init: *const f32, rows: u64, dims: u64, total_epochs: u64, cfg: *const umap_config, metric_type: c_int, out: *mut *mut umap_optimizer) -> c_int;
    pub fn umap_optimizer_step_epochs(opt: *mut umap_optimizer, n: u64) -> c_int;
    pub fn umap_optimizer_step_epochs_metric(opt: *mut umap_optimizer, n: u64, output_metric: c_int) -> c_int;
    pub fn umap_optimizer_current_epoch(opt: *const umap_optimizer, out: *mut u64) -> c_int;
    pub fn umap_optimizer_total_epochs(opt: *const umap_optimizer, out: *mut u64) -> c_int;
    pub fn umap_optimizer_remaining_epochs(opt: *const umap_optimizer, out: *mut u64) -> c_int;
    pub fn umap_optimizer_embedding(opt: *const umap_optimizer, host_out: *mut f32) -> c_int;
    pub fn umap_optimizer_embedding_device(opt: *mut umap_optimizer, dev_ptr: *mut *mut f32) -> c_int;
    pub fn umap_optimizer_dims(opt: *const umap_optimizer, n_vertices: *mut u64, dims: *mut u64) -> c_int;
    pub fn umap_optimizer_manifold(opt: *const umap_optimizer, out: *mut *const umap_manifold) -> c_int;
    pub fn umap_optimizer_into_fitted(opt: *mut umap_optimizer, cfg: *const umap_config, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_optimizer_free(opt: *mut umap_optimizer) -> c_int;
    pub fn umap_optimizer_set_seed(opt: *mut umap_optimizer, seed: u64) -> c_int;
    pub fn umap_optimizer_n_edges(opt: *const umap_optimizer, out: *mut u64) -> c_int;
    pub fn umap_optimizer_export_edges(opt: *const umap_optimizer, head: *mut u32, tail: *mut u32, epochs_per_sample: *mut f64, epoch_of_next_sample: *mut f64, epoch_of_next_negative_sample: *mut f64, epochs_per_negative_sample: *mut f64) -> c_int;
    pub fn umap_optimizer_schedule_totals(opt: *const umap_optimizer, start: u64, end: u64, fired: *mut u64, negatives: *mut u64) -> c_int;
    pub fn umap_optimizer_last_step_ms(opt: *const umap_optimizer, ms: *mut f32) -> c_int;
    pub fn umap_release_cached_memory(released_bytes: *mut u64) -> c_int;
    pub fn umap_kernel_launches(out: *mut u64) -> c_int;
    pub fn umap_fitted_embedding(f: *const umap_fitted, host_out: *mut f32) -> c_int;
    pub fn umap_fitted_dims(f: *const umap_fitted, n_vertices: *mut u64, dims: *mut u64) -> c_int;
    pub fn umap_fitted_manifold(f: *const umap_fitted, out: *mut *const umap_manifold) -> c_int;
    pub fn umap_fitted_config(f: *const umap_fitted, out: *mut umap_config) -> c_int;
    pub fn umap_fitted_free(f: *mut umap_fitted) -> c_int;
    pub fn umap_fit(cfg: *const umap_config, n_samples: u64, host_knn_indices: *const u32, host_knn_dists: *const f32, knn_rows: u64, knn_cols: u64, host_init: *const f32, init_rows: u64, init_cols: u64, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_fit_device(cfg: *const umap_config, n_samples: u64, dev_knn_indices: *const u32, dev_knn_dists: *const f32, knn_rows: u64, knn_cols: u64, dev_init: *const f32, init_rows: u64, init_cols: u64, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_fit_manifold(manifold: *mut umap_manifold, cfg: *const umap_config, host_init: *const f32, init_rows: u64, init_cols: u64, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_fit_manifold_device(manifold: *mut umap_manifold, cfg: *const umap_config, dev_init: *const f32, init_rows: u64, init_cols: u64, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_fit_manifold_metric(manifold: *mut umap_manifold, cfg: *const umap_config, host_init: *const f32, init_rows: u64, init_cols: u64, metric_type: c_int, output_metric: c_int, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_fit_manifold_metric_device(manifold: *mut umap_manifold, cfg: *const umap_config, dev_init: *const f32, init_rows: u64, init_cols: u64, metric_type: c_int, output_metric: c_int, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_knn_bruteforce(host_data: *const f32, n: u64, dim: u64, k: u64, host_knn_indices: *mut u32, host_knn_dists: *mut f32, rows_recomputed: *mut u64) -> c_int;
    pub fn umap_knn_bruteforce_device(dev_data: *const f32, n: u64, dim: u64, k: u64, dev_knn_indices: *mut u32, dev_knn_dists: *mut f32, rows_recomputed: *mut u64) -> c_int;
    pub fn umap_knn_last_profile(candidate_pass_ms: *mut f32, rows_recomputed: *mut u64, reordered: *mut u32) -> c_int;
    pub fn umap_batch_optimizer_new(cfg: *const umap_config, n_instances: u64, host_offsets: *const u64, host_knn_indices: *const u32, host_knn_dists: *const f32, knn_cols: u64, host_init: *const f32, init_cols: u64, total_epochs: u64, out: *mut *mut umap_optimizer) -> c_int;
    pub fn umap_batch_optimizer_new_device(cfg: *const umap_config, n_instances: u64, host_offsets: *const u64, dev_knn_indices: *const u32, dev_knn_dists: *const f32, knn_cols: u64, dev_init: *const f32, init_cols: u64, total_epochs: u64, out: *mut *mut umap_optimizer) -> c_int;
    pub fn umap_batch_fit(cfg: *const umap_config, n_instances: u64, host_offsets: *const u64, host_knn_indices: *const u32, host_knn_dists: *const f32, knn_cols: u64, host_init: *const f32, init_cols: u64, host_embedding_out: *mut f32) -> c_int;
    pub fn umap_batch_fit_device(cfg: *const umap_config, n_instances: u64, host_offsets: *const u64, dev_knn_indices: *const u32, dev_knn_dists: *const f32, knn_cols: u64, dev_init: *const f32, init_cols: u64, dev_embedding_out: *mut f32) -> c_int;
    pub fn umap_optimizer_tuning(opt: *const umap_optimizer, chunk: *mut u32, block_threads: *mut u32) -> c_int;
    pub fn umap_optimizer_layout_flags(opt: *const umap_optimizer, flags: *mut u32) -> c_int;
    pub fn umap_manifold_serialize(m: *const umap_manifold, buf: *mut u8, cap: u64, needed: *mut u64) -> c_int;
    pub fn umap_manifold_deserialize(buf: *const u8, len: u64, out: *mut *mut umap_manifold) -> c_int;
    pub fn umap_optimizer_serialize(o: *const umap_optimizer, buf: *mut u8, cap: u64, needed: *mut u64) -> c_int;
    pub fn umap_optimizer_deserialize(buf: *const u8, len: u64, out: *mut *mut umap_optimizer) -> c_int;
    pub fn umap_fitted_serialize(f: *const umap_fitted, buf: *mut u8, cap: u64, needed: *mut u64) -> c_int;
    pub fn umap_fitted_deserialize(buf: *const u8, len: u64, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_manifold_serialize_bincode(m: *const umap_manifold, buf: *mut u8, cap: u64, needed: *mut u64) -> c_int;
    pub fn umap_manifold_deserialize_bincode(buf: *const u8, len: u64, out: *mut *mut umap_manifold) -> c_int;
    pub fn umap_optimizer_serialize_bincode(opt: *const umap_optimizer, buf: *mut u8, cap: u64, needed: *mut u64) -> c_int;
    pub fn umap_optimizer_deserialize_bincode(buf: *const u8, len: u64, out: *mut *mut umap_optimizer) -> c_int;
    pub fn umap_fitted_serialize_bincode(f: *const umap_fitted, buf: *mut u8, cap: u64, needed: *mut u64) -> c_int;
    pub fn umap_fitted_deserialize_bincode(buf: *const u8, len: u64, out: *mut *mut umap_fitted) -> c_int;
    pub fn umap_smooth_knn_dist_device(dev_dists: *const f32, n: u64, k: u64, n_iter: u64, local_connectivity: f32, bandwidth: f32, dev_sigmas: *mut f32, dev_rhos: *mut f32) -> c_int;
    pub fn umap_radix_sort_pairs_device(dev_keys_in: *const u32, dev_values_in: *const u32, dev_keys_out: *mut u32, dev_values_out: *mut u32, n: u64, end_bit: c_int) -> c_int;
    pub fn umap_sgd_negative_draws_device(seed: u64, first_entry: u64, n_entries: u64, epoch: u32, per_entry: u32, lo: u32, range: u32, dev_out: *mut u32) -> c_int;
    pub fn umap_sgd_negatives_per_firing_device(dev_q: *const u32, dev_epoch: *const u32, count: u64, negative_sample_rate: u32, dev_out: *mut u32) -> c_int;
    pub fn umap_random_rows_probe_device(dev_table: *mut f32, n_rows: u64, accesses: u64, mode: c_int, dev_out: *mut f32, ms: *mut f32, accesses_done: *mut u64) -> c_int;
    pub fn umap_radix_sort_pairs_device_noalloc(dev_keys_in: *const u32, dev_values_in: *const u32, dev_keys_out: *mut u32, dev_values_out: *mut u32, n: u64, end_bit: c_int, stream: *mut c_void) -> c_int;
    pub fn umap_radix_sort_noalloc_max_pairs(out: *mut u64) -> c_int;
    pub fn umap_mlp_param_count(in_dim: u64, out_dim: u64, out: *mut u64) -> c_int;
    pub fn umap_mlp_new(in_dim: u64, out_dim: u64, params: *const f32, out: *mut *mut umap_mlp) -> c_int;
    pub fn umap_mlp_dims(m: *const umap_mlp, in_dim: *mut u64, out_dim: *mut u64) -> c_int;
    pub fn umap_mlp_get_params(m: *const umap_mlp, params: *mut f32) -> c_int;
    pub fn umap_mlp_set_params(m: *mut umap_mlp, params: *const f32) -> c_int;
    pub fn umap_mlp_fit_input_norm_device(m: *mut umap_mlp, dev_x: *const f32, rows: u64) -> c_int;
    pub fn umap_mlp_input_norm(m: *const umap_mlp, shift: *mut f32, scale: *mut f32) -> c_int;
    pub fn umap_mlp_set_input_norm(m: *mut umap_mlp, shift: *const f32, scale: *const f32) -> c_int;
    pub fn umap_mlp_gradients_device(m: *mut umap_mlp, dev_x: *const f32, dev_y: *const f32, rows: u64, grads: *mut f32, loss: *mut f32) -> c_int;
    pub fn umap_mlp_train_device(m: *mut umap_mlp, dev_x: *const f32, dev_y: *const f32, rows: u64, epochs: u64, batch: u64, learning_rate: f32, seed: u64, losses: *mut f32) -> c_int;
    pub fn umap_mlp_predict_device(m: *mut umap_mlp, dev_x: *const f32, rows: u64, dev_y: *mut f32) -> c_int;
    pub fn umap_mlp_free(m: *mut umap_mlp) -> c_int;
    pub fn umap_gemm_bf16_device(dev_a: *const c_void, dev_b: *const c_void, dev_c: *mut f32, m: u64, n: u64, k: u64, k_splits: u64) -> c_int;
    pub fn umap_warm_start_params_default(out: *mut umap_warm_start_params) -> c_int;
    pub fn umap_warm_start_fit_device(cfg: *const umap_config, params: *const umap_warm_start_params, dev_data: *const f32, n_samples: u64, data_dim: u64, dev_knn_indices: *const u32, dev_knn_dists: *const f32, knn_cols: u64, dev_sub_rows: *const u32, n_sub: u64, dev_sub_knn_indices: *const u32, dev_sub_knn_dists: *const f32, dev_sub_init: *const f32, out: *mut *mut umap_fitted, phase_ms: *mut f32, mlp_losses: *mut f32) -> c_int;
}
