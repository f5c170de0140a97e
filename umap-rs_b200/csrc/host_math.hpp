// Host-side arithmetic shared by the C-ABI implementation (see host_math.cpp).
#pragma once

#include <cstdint>
#include <string>

#include "../../include/umap_b200.h"

namespace ub {

// Rust `format!("{}", x)` for f32 (shortest round-trip digits, no exponent).
std::string rust_f32(float x);
// umap/find_ab_params.rs:9-82.
void find_ab_params(float spread, float min_dist, float* a, float* b);
// Rust `x as usize` for f32 (saturating, NaN -> 0).
uint64_t rust_f32_as_usize(float v);
// embedding.rs:339-429; returns the panic text, or "" when the parameters are valid.
std::string validate_parameters(const umap_config& c, uint64_t n_samples, uint64_t knn_rows,
                                uint64_t knn_cols);

}  // namespace ub
