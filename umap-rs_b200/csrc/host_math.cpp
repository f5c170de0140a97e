// Host-side arithmetic of the fit path: the (a, b) curve fit, parameter validation with the
// reference's panic texts, and Rust `{}` formatting of floats for those texts.
// Built with -ffp-contract=off (no FMA contraction) so f32 expressions round as in Rust.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "host_math.hpp"

namespace ub {

std::string rust_f32(float x) {
  if (std::isnan(x)) return "NaN";
  if (std::isinf(x)) return x > 0 ? "inf" : "-inf";
  if (x == 0.0f) return std::signbit(x) ? "-0" : "0";
  // Shortest round-trip digits (what Rust's Display picks), then plain decimal notation.
  char buf[64];
  int prec = 1;
  for (; prec <= 9; ++prec) {
    snprintf(buf, sizeof buf, "%.*e", prec - 1, (double)x);
    if (strtof(buf, nullptr) == x) break;
  }
  std::string s(buf);
  bool neg = s[0] == '-';
  if (neg) s = s.substr(1);
  size_t epos = s.find('e');
  int exp10 = atoi(s.c_str() + epos + 1);
  std::string digits;
  for (size_t i = 0; i < epos; ++i)
    if (s[i] != '.') digits += s[i];
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  std::string out;
  int p = (int)digits.size();
  if (exp10 >= p - 1) {
    out = digits + std::string(exp10 - (p - 1), '0');
  } else if (exp10 >= 0) {
    out = digits.substr(0, exp10 + 1) + "." + digits.substr(exp10 + 1);
  } else {
    out = "0." + std::string(-exp10 - 1, '0') + digits;
  }
  return neg ? "-" + out : out;
}

// umap/find_ab_params.rs:9-82: custom f32 gradient descent (not scipy curve_fit).  The
// 300,000 steps take a few milliseconds of host time and the result depends only on the two
// arguments' bits, so results are memoised per (spread, min_dist) for the process.
static void find_ab_params_uncached(float spread, float min_dist, float* a_out, float* b_out);

void find_ab_params(float spread, float min_dist, float* a_out, float* b_out) {
  static std::mutex mu;
  static std::map<uint64_t, std::pair<float, float>> memo;
  uint32_t sb, mb;
  std::memcpy(&sb, &spread, 4);
  std::memcpy(&mb, &min_dist, 4);
  const uint64_t key = (uint64_t)sb << 32 | mb;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = memo.find(key);
    if (it != memo.end()) {
      *a_out = it->second.first;
      *b_out = it->second.second;
      return;
    }
  }
  float a = 0.0f, b = 0.0f;
  find_ab_params_uncached(spread, min_dist, &a, &b);
  std::lock_guard<std::mutex> lock(mu);
  if (memo.size() >= 256) memo.clear();
  memo[key] = {a, b};
  *a_out = a;
  *b_out = b;
}

static void find_ab_params_uncached(float spread, float min_dist, float* a_out, float* b_out) {
  const int n_points = 300;
  float xv[300], yv[300];
  for (int i = 0; i < n_points; ++i) xv[i] = ((spread * 3.0f) * (float)i) / ((float)n_points - 1.0f);
  for (int i = 0; i < n_points; ++i) {
    float x = xv[i];
    yv[i] = x < min_dist ? 1.0f : expf((-(x - min_dist)) / spread);
  }
  float a = 1.5f, b = 0.9f;
  const float learning_rate = 0.01f;
  for (int it = 0; it < 1000; ++it) {
    float grad_a = 0.0f, grad_b = 0.0f, total_error = 0.0f;
    for (int i = 0; i < n_points; ++i) {
      float x = xv[i];
      float x_2b = powf(x, 2.0f * b);
      float denom = 1.0f + a * x_2b;
      float y_pred = 1.0f / denom;
      float error = y_pred - yv[i];
      total_error = total_error + error * error;
      grad_a = grad_a + (2.0f * error) * ((-x_2b) / (denom * denom));
      if (x > 0.0f) {
        float ln_x = logf(x);
        grad_b = grad_b + (2.0f * error) * ((((-2.0f * a) * x_2b) * ln_x) / (denom * denom));
      }
    }
    a = a - (learning_rate * grad_a) / (float)n_points;
    b = b - (learning_rate * grad_b) / (float)n_points;
    if (a < 0.001f) a = 0.001f;
    if (a > 10.0f) a = 10.0f;
    if (b < 0.001f) b = 0.001f;
    if (b > 10.0f) b = 10.0f;
    if (total_error / (float)n_points < 1e-7f) break;
  }
  *a_out = a;
  *b_out = b;
}

uint64_t rust_f32_as_usize(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 18446744073709551615.0f) return UINT64_MAX;
  return (uint64_t)v;
}

// embedding.rs:339-429 (validate_parameters), in the reference's order.
std::string validate_parameters(const umap_config& c, uint64_t n_samples, uint64_t knn_rows,
                                uint64_t knn_cols) {
  if (c.set_op_mix_ratio < 0.0f || c.set_op_mix_ratio > 1.0f)
    return "set_op_mix_ratio must be between 0.0 and 1.0, got " + rust_f32(c.set_op_mix_ratio);
  if (c.n_neighbors < 2) return "n_neighbors must be >= 2, got " + std::to_string(c.n_neighbors);
  if (c.repulsion_strength < 0.0f)
    return "repulsion_strength cannot be negative, got " + rust_f32(c.repulsion_strength);
  if (c.min_dist > c.spread)
    return "min_dist (" + rust_f32(c.min_dist) + ") must be <= spread (" + rust_f32(c.spread) + ")";
  if (c.min_dist < 0.0f) return "min_dist cannot be negative, got " + rust_f32(c.min_dist);
  if (c.learning_rate < 0.0f) return "learning_rate must be positive, got " + rust_f32(c.learning_rate);
  if (c.n_components < 1) return "n_components must be >= 1, got " + std::to_string(c.n_components);
  // knn_dists / knn_indices shapes are equal by construction at this ABI (one shape pair).
  if (knn_cols != c.n_neighbors)
    return "knn_dists has " + std::to_string(knn_cols) + " neighbors but n_neighbors is " +
           std::to_string(c.n_neighbors);
  if (knn_rows != n_samples)
    return "knn_dists has " + std::to_string(knn_rows) + " samples but data has " +
           std::to_string(n_samples) + " samples";
  if (n_samples <= c.n_neighbors)
    return "Number of samples (" + std::to_string(n_samples) + ") must be > n_neighbors (" +
           std::to_string(c.n_neighbors) + ")";
  // fuzzy_simplicial_set.rs:111-114
  if (n_samples >= 0xFFFFFFFFull) return "n_samples must be < 2^32 for u32 indices";
  return "";
}

}  // namespace ub
