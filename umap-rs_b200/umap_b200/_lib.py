"""ctypes loader for libumap_b200.so (the C ABI declared in include/umap_b200.h).

There is no fallback: if the library is missing, importing the package raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libumap_b200.so")

u64, u32, f32, i32 = C.c_uint64, C.c_uint32, C.c_float, C.c_int
P = C.c_void_p
PP = C.POINTER(C.c_void_p)


class UmapConfigC(C.Structure):
    """Mirror of `umap_config` (include/umap_b200.h)."""
    _fields_ = [
        ("n_components", u64),
        ("min_dist", f32), ("spread", f32),
        ("has_a", C.c_int32), ("a", f32),
        ("has_b", C.c_int32), ("b", f32),
        ("n_neighbors", u64), ("local_connectivity", f32), ("set_op_mix_ratio", f32),
        ("has_disconnection_distance", C.c_int32), ("disconnection_distance", f32),
        ("symmetrize", C.c_int32),
        ("has_n_epochs", C.c_int32), ("n_epochs", u64),
        ("learning_rate", f32), ("negative_sample_rate", u64), ("repulsion_strength", f32),
    ]


class WarmStartParamsC(C.Structure):
    """Mirror of `umap_warm_start_params` (include/umap_b200.h)."""
    _fields_ = [
        ("sub_epochs", u64), ("epochs", u64), ("mlp_epochs", u64), ("batch", u64),
        ("mlp_learning_rate", f32), ("has_learning_rate", C.c_int32), ("learning_rate", f32),
        ("seed", u64),
    ]


# umap_optimizer_layout_flags bits (UMAP_LAYOUT_* in include/umap_b200.h)
LAYOUT_FLAGS = {"LANE_MAJOR": 1, "EIGHT_NEGATIVES": 2, "RENAMED": 4, "GENERIC_RULE": 8, "TWELVE_NEGATIVES": 16,
                "RATE_ORDER": 32, "BLOCK_ORDER": 64, "ROW_ORDER": 128}

WARM_START_PHASES = ("prepare", "subsample_fit", "mlp_train", "mlp_predict", "wait_full_graph", "fit",
                     "full_graph_overlapped", "total")

# name -> (argtypes) ; every function returns int status
SIGNATURES = {
    "umap_config_default": [C.POINTER(UmapConfigC)],
    "umap_find_ab_params": [f32, f32, C.POINTER(f32), C.POINTER(f32)],
    "umap_learn_manifold": [C.POINTER(UmapConfigC), u64, P, P, u64, u64, PP],
    "umap_learn_manifold_device": [C.POINTER(UmapConfigC), u64, P, P, u64, u64, PP],
    "umap_manifold_n_vertices": [P, C.POINTER(u64)],
    "umap_manifold_curve_params": [P, C.POINTER(f32), C.POINTER(f32)],
    "umap_manifold_graph_nnz": [P, C.POINTER(u64)],
    "umap_manifold_graph_copy": [P, P, P, P],
    "umap_manifold_sigmas_rhos": [P, P, P],
    "umap_manifold_disconnection_counts": [P, C.POINTER(u64), C.POINTER(u64)],
    "umap_manifold_clone": [P, PP],
    "umap_manifold_free": [P],
    "umap_optimizer_new": [P, P, u64, u64, u64, C.POINTER(UmapConfigC), i32, PP],
    "umap_optimizer_new_device": [P, P, u64, u64, u64, C.POINTER(UmapConfigC), i32, PP],
    "umap_optimizer_step_epochs": [P, u64],
    "umap_optimizer_step_epochs_metric": [P, u64, i32],
    "umap_optimizer_current_epoch": [P, C.POINTER(u64)],
    "umap_optimizer_total_epochs": [P, C.POINTER(u64)],
    "umap_optimizer_remaining_epochs": [P, C.POINTER(u64)],
    "umap_optimizer_embedding": [P, P],
    "umap_optimizer_embedding_device": [P, PP],
    "umap_optimizer_dims": [P, C.POINTER(u64), C.POINTER(u64)],
    "umap_optimizer_manifold": [P, PP],
    "umap_optimizer_into_fitted": [P, C.POINTER(UmapConfigC), PP],
    "umap_optimizer_free": [P],
    "umap_optimizer_set_seed": [P, u64],
    "umap_optimizer_n_edges": [P, C.POINTER(u64)],
    "umap_optimizer_export_edges": [P, P, P, P, P, P, P],
    "umap_optimizer_schedule_totals": [P, u64, u64, C.POINTER(u64), C.POINTER(u64)],
    "umap_optimizer_last_step_ms": [P, C.POINTER(f32)],
    "umap_kernel_launches": [C.POINTER(u64)],
    "umap_release_cached_memory": [C.POINTER(u64)],
    "umap_fitted_embedding": [P, P],
    "umap_fitted_dims": [P, C.POINTER(u64), C.POINTER(u64)],
    "umap_fitted_manifold": [P, PP],
    "umap_fitted_config": [P, C.POINTER(UmapConfigC)],
    "umap_fitted_free": [P],
    "umap_fit": [C.POINTER(UmapConfigC), u64, P, P, u64, u64, P, u64, u64, PP],
    "umap_fit_device": [C.POINTER(UmapConfigC), u64, P, P, u64, u64, P, u64, u64, PP],
    "umap_batch_optimizer_new": [C.POINTER(UmapConfigC), u64, P, P, P, u64, P, u64, u64, PP],
    "umap_batch_optimizer_new_device": [C.POINTER(UmapConfigC), u64, P, P, P, u64, P, u64, u64, PP],
    "umap_batch_fit": [C.POINTER(UmapConfigC), u64, P, P, P, u64, P, u64, P],
    "umap_batch_fit_device": [C.POINTER(UmapConfigC), u64, P, P, P, u64, P, u64, P],
    "umap_optimizer_tuning": [P, C.POINTER(u32), C.POINTER(u32)],
    "umap_manifold_serialize": [P, P, u64, C.POINTER(u64)],
    "umap_manifold_deserialize": [P, u64, PP],
    "umap_optimizer_serialize": [P, P, u64, C.POINTER(u64)],
    "umap_optimizer_deserialize": [P, u64, PP],
    "umap_fitted_serialize": [P, P, u64, C.POINTER(u64)],
    "umap_fitted_deserialize": [P, u64, PP],
    "umap_manifold_serialize_bincode": [P, P, u64, C.POINTER(u64)],
    "umap_manifold_deserialize_bincode": [P, u64, PP],
    "umap_optimizer_serialize_bincode": [P, P, u64, C.POINTER(u64)],
    "umap_optimizer_deserialize_bincode": [P, u64, PP],
    "umap_fitted_serialize_bincode": [P, P, u64, C.POINTER(u64)],
    "umap_fitted_deserialize_bincode": [P, u64, PP],
    "umap_smooth_knn_dist_device": [P, u64, u64, u64, f32, f32, P, P],
    "umap_knn_bruteforce": [P, u64, u64, u64, P, P, C.POINTER(u64)],
    "umap_knn_bruteforce_device": [P, u64, u64, u64, P, P, C.POINTER(u64)],
    "umap_knn_last_profile": [C.POINTER(f32), C.POINTER(u64), C.POINTER(u32)],
    "umap_radix_sort_pairs_device": [P, P, P, P, u64, i32],
    "umap_radix_sort_pairs_device_noalloc": [P, P, P, P, u64, i32, P],
    "umap_sgd_negative_draws_device": [u64, u64, u64, u32, u32, u32, u32, P],
    "umap_optimizer_layout_flags": [P, C.POINTER(u32)],
    "umap_random_rows_probe_device": [P, u64, u64, i32, P, C.POINTER(f32), C.POINTER(u64)],
    "umap_sgd_negatives_per_firing_device": [P, P, u64, u32, P],
    "umap_warm_start_params_default": [C.POINTER(WarmStartParamsC)],
    "umap_warm_start_fit_device": [C.POINTER(UmapConfigC), C.POINTER(WarmStartParamsC), P, u64, u64, P, P, u64,
                                   P, u64, P, P, P, PP, P, P],
    "umap_radix_sort_noalloc_max_pairs": [C.POINTER(u64)],
    "umap_fit_manifold": [P, C.POINTER(UmapConfigC), P, u64, u64, PP],
    "umap_fit_manifold_device": [P, C.POINTER(UmapConfigC), P, u64, u64, PP],
    "umap_fit_manifold_metric": [P, C.POINTER(UmapConfigC), P, u64, u64, i32, i32, PP],
    "umap_fit_manifold_metric_device": [P, C.POINTER(UmapConfigC), P, u64, u64, i32, i32, PP],
    "umap_mlp_param_count": [u64, u64, C.POINTER(u64)],
    "umap_mlp_new": [u64, u64, P, PP],
    "umap_mlp_dims": [P, C.POINTER(u64), C.POINTER(u64)],
    "umap_mlp_get_params": [P, P],
    "umap_mlp_set_params": [P, P],
    "umap_mlp_fit_input_norm_device": [P, P, u64],
    "umap_mlp_input_norm": [P, P, P],
    "umap_mlp_set_input_norm": [P, P, P],
    "umap_mlp_gradients_device": [P, P, P, u64, P, C.POINTER(f32)],
    "umap_mlp_train_device": [P, P, P, u64, u64, u64, f32, u64, P],
    "umap_mlp_predict_device": [P, P, u64, P],
    "umap_mlp_free": [P],
    "umap_gemm_bf16_device": [P, P, P, u64, u64, u64, u64],
}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python umap-rs_b200/build.py` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.umap_last_error.restype = C.c_char_p
        L.umap_last_error.argtypes = []
        L.umap_abi_version.restype = C.c_int
        L.umap_abi_version.argtypes = []
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = L
    return _lib
