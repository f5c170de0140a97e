// Edge pruning + task/slice layout (K5), init normalisation (K6) and the Hogwild SGD epoch
// (K7).
//
// Layout.  The kept edges of the symmetric graph are grouped by head row and cut into tasks
// of at most `chunk` edges (see SgdLayout).  A warp owns a slice of 32 tasks and a lane owns
// one task, keeping the head row's live embedding in registers.  A slice's entries are lane
// major when the embedding the epoch touches stays in L2: task l's entries are contiguous at
// base + l * width (width = the slice's longest task rounded up to 4 entries, padding never
// fires), so a lane's 4-entry window is one aligned 32-byte sector whatever the other lanes'
// progress.  Otherwise (DRAM-bound sizes) entry e of task l sits at base + 32 e + l, so a
// warp's loads cover whole 256-byte rows (see pick_lane_major).  The reference writes a
// head row only from edges whose head it is (optimize_layout_euclidean.rs:281-306, :338),
// so a task that is a whole row reproduces the reference's sequential per-row order with
// no lost head updates; the rare long rows (kNN hubs) are split so that one row cannot
// serialise an epoch, and each partial task merges its head delta with an atomic add.
// Tail moves (fire-and-forget atomic adds, see sub_row) and negative samples (racy loads)
// touch the per-call snapshot buffer, where the reference reads and writes it racily.
//
// Schedule.  The reference keeps four f64 arrays per edge (optimizer.rs:33-43).  Here one
// u32 per edge holds Q = ceil(2^32 / epochs_per_sample) and the state is recomputed in
// exact integer arithmetic: the edge has fired m(n) = (n*Q) >> 32 times by epoch n, so it
// fires at n iff m(n) > m(n-1) (at most once per epoch, never at epoch 0; :277, :308), and
// a firing with index m draws y(n) - y(p) negatives, y(x) = (x*neg*Q) >> 32 and p the epoch
// of firing m-1 (y(n) - 1 for the first firing): the closed form of :310-311 / :343.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ub_internal.hpp"

namespace ub {
namespace {

constexpr uint32_t PAD_ROW = 0xFFFFFFFFu;

// The epoch kernel comes in two register budgets.  Large graphs (many waves of warps) are
// bound by instruction issue and L2 sector throughput: 4 negative rows fetched together and
// 5 resident 256-thread blocks per SM (48 registers).  Graphs that fill about two waves or
// fewer are bound by the chain of dependent loads of their busiest lanes: 8 negative rows
// fetched together (one round trip for a firing's usual 4-6 negatives) and 4 blocks per SM.
// On the 2M-point workload (500 epochs, SGD ms) the wide budget's occupancy beats the extra
// round trip of a firing's fifth negative: 4 / 5: 314.0, 8 / 4: 317.6, 6 / 4: 330.9, 4 / 4:
// 343.5, 5 / 4: 349.9 (5 and 6 rows at 5 blocks per SM spill more than 4 / 5's 16 bytes).
constexpr int NB_WIDE = 4, MINB_WIDE = 5;
constexpr int NB_SHORT = 8, MINB_SHORT = 4;
// Renamed DRAM-bound layouts: 12 negative rows fetched together, 3 blocks per SM.  Their random
// row loads go to DRAM and their warps are limited by registers either way, so more loads in
// flight per lane beat more warps (30 epochs of a 20M-point roll: 8 / 4: 310.8 ms, 10 / 3:
// 295.1, 12 / 3: 295.2, 12 / 2: 313.4, 16 / 2: 316.0, 24 / 2: 317.7; 40M points, 24 epochs:
// 8 / 4: 590.4, 12 / 3: 562.6, 16 / 2: 564.9).  Small latency-bound graphs keep 8 / 4: with
// 12 / 3 the warm start's 100k-point subsample fit took 38.4-38.9 ms against 30.5-31.6 ms.
constexpr int NB_DRAM = 12, MINB_DRAM = 3;

// ------------------------------------------------------------------------------ negatives' RNG
// Counter-based: the firing of entry `idx` at `epoch` draws its negatives in pairs; pair t is
// the SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) of a counter derived from (seed, idx, epoch, t), and each 32-bit
// half maps to [0, n) by a multiply-high.  The reference draws from an unseeded thread-local
// generator (optimize_layout_euclidean.rs:314), so parity with it is statistical.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
struct NegRng {
  uint64_t base;
  __device__ __forceinline__ NegRng(uint64_t seed, uint64_t idx, uint32_t epoch)
      : base(seed ^ (idx * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)epoch * 0xC2B2AE3D27D4EB4Full)) {}
  __device__ __forceinline__ uint64_t pair(uint32_t t) const { return mix64(base + (uint64_t)t * 0xD1B54A32D192ED03ull); }
};

// ------------------------------------------------------------------------------ schedule
__host__ __device__ __forceinline__ uint32_t q_minus_1(double eps) {
  if (!(eps > 0.0)) return 0u;
  const double x = ceil(4294967296.0 / eps);
  if (x >= 4294967296.0) return 0xFFFFFFFFu;
  if (x < 1.0) return 0u;
  return (uint32_t)x - 1u;
}
// All schedule helpers take q = Q - 1 (the stored u32).  n*Q = n*q + n fits in 64 bits for
// any u32 n, and the product is a single 32x32->64 multiply.
__device__ __forceinline__ uint64_t fires_by(uint32_t n, uint32_t q) {
  return ((uint64_t)n * q + n) >> 32;
}
// Smallest epoch x with fires_by(x) >= m.
__device__ __forceinline__ uint32_t fire_epoch(uint64_t m, uint32_t q) {
  const float est = (float)m * __fdividef(4294967296.0f, (float)q + 1.0f);
  uint32_t x = est > 0.0f ? (est < 4294967040.0f ? (uint32_t)ceilf(est) : 0xFFFFFF00u) : 0u;
  for (int t = 0; t < 8 && x > 0 && fires_by(x - 1, q) >= m; ++t) --x;
  for (int t = 0; t < 8 && fires_by(x, q) < m; ++t) ++x;
  return x;
}

// Negatives drawn in total after m firings.
__device__ __forceinline__ uint64_t negatives_after(uint64_t m, uint32_t q, uint32_t neg) {
  if (m == 0) return 0;
  const int64_t t = (int64_t)fires_by(fire_epoch(m, q) * neg, q) - 1;
  return t > 0 ? (uint64_t)t : 0ull;
}
// Fires at epoch n iff fires_by(n) > fires_by(n - 1), i.e. iff the low 32 bits of (n - 1) * Q
// are at least 2^32 - Q (Q <= 2^32, so the count grows by at most one): one 32-bit multiply.
__device__ __forceinline__ bool fires_at(uint32_t n, uint32_t q) {
  const uint32_t nm1 = n - 1u;
  return n > 0 && nm1 * q + nm1 >= ~q;
}
// Negatives drawn by the firing at epoch n (n * neg < 2^32 is checked on the host):
// y(n) - y(p) with y(x) = fires_by(x * neg) and p the epoch of the previous firing, or
// y(n) - 1 for the first.  Firings are floor(2^32 / Q) or one more epochs apart, so p is found
// among a few candidates below n - floor(2^32 / Q) + 1 with the cheap test above (the float
// estimate of the gap is within one epoch: a second firing needs n >= 2 * 2^32 / Q and epochs
// stay below MAX_EPOCHS = 2^21, checked on the host; fire_epoch is the exact fallback).
// A two-candidate form with an exact integer gap (one fewer fires_at test, no fallback)
// measured 1.7% slower on the 2M workload (317.6 against 312.3 ms per 500 epochs).
__device__ __forceinline__ uint32_t negatives_at(uint32_t n, uint32_t q, uint32_t neg) {
  const int64_t y = (int64_t)fires_by(n * neg, q);
  const uint64_t m = fires_by(n, q);
  int64_t prev = 1;
  if (m > 1) {
    const int64_t g0 = (int64_t)__fdividef(4294967296.0f, (float)q + 1.0f);
    uint32_t pe = 0;
#pragma unroll
    for (int t = 1; t >= -2; --t) {
      const int64_t x = (int64_t)n - g0 + t;
      if (pe == 0 && x >= 1 && x < (int64_t)n && fires_at((uint32_t)x, q)) pe = (uint32_t)x;
    }
    if (pe == 0) pe = fire_epoch(m - 1, q);
    prev = (int64_t)fires_by(pe * neg, q);
  }
  const int64_t d = y - prev;
  return d > 0 ? (uint32_t)d : 0u;
}

// Rust f32::clamp(-4, 4) (utils/clip.rs:13-15): NaN passes through.
__device__ __forceinline__ float clip4(float v) {
  float x = v;
  if (x < -4.0f) x = -4.0f;
  if (x > 4.0f) x = 4.0f;
  return x;
}

// Two-lane FP32 arithmetic on a 2-D row (each lane the same IEEE operation as the scalar one).
__device__ __forceinline__ uint64_t pk2(float x, float y) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(__float_as_uint(x)), "r"(__float_as_uint(y)));
  return r;
}
__device__ __forceinline__ void up2(uint64_t v, float& x, float& y) {
  uint32_t a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=r"(a), "=r"(b) : "l"(v));
  x = __uint_as_float(a);
  y = __uint_as_float(b);
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// ------------------------------------------------------------------------------ K7

template <int DIM>
__device__ __forceinline__ void load_row(float (&v)[DIM], const float* p) {
  if constexpr (DIM == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x;
    v[1] = t.y;
  } else if constexpr (DIM == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = p[d];
  }
}
template <int DIM>
__device__ __forceinline__ void store_row(float* p, const float (&v)[DIM]) {
  if constexpr (DIM == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else if constexpr (DIM == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) p[d] = v[d];
  }
}

// Tail move (optimize_layout_euclidean.rs:303-305) as a fire-and-forget atomic add.  The
// reference's racy read-modify-write rarely collides on a CPU (a vertex's few tail moves per
// epoch come from rows processed at different times); with every row of an epoch in flight
// at once, plain stores would drop most of them, so the add is atomic to keep the
// reference's statistics.
template <int DIM>
__device__ __forceinline__ void sub_row(float* p, const float (&g)[DIM]) {
  if constexpr (DIM == 2) {
    atomicAdd(reinterpret_cast<float2*>(p), make_float2(-g[0], -g[1]));
  } else if constexpr (DIM == 4) {
    atomicAdd(reinterpret_cast<float4*>(p), make_float4(-g[0], -g[1], -g[2], -g[3]));
  } else {
#pragma unroll
    for (int d = 0; d < DIM; ++d) atomicAdd(p + d, -g[d]);
  }
}

// Force law of the generic-metric path (layout/optimize_layout_generic.rs:65-119) with the
// built-in output metric EuclideanMetric (distances.rs:22-37): distance d = sqrt(sum diff^2),
// gradient diff / (d + 1e-6), w = 1 / (1 + a d^(2b)).  Returns the coefficient c that
// multiplies the gradient: 2b (w - 1) / (d + 1e-6) for an attraction, 2 gamma b w / (d + 1e-6)
// for a repulsion (`scale` = 2b or 2 gamma b, `bias` = -1 or 0); *den receives d + 1e-6.
__device__ __forceinline__ float metric_coeff(float ds, float a, float two_b, float scale, float bias,
                                              float* den) {
  const float dist = sqrtf(ds);
  *den = dist + 1e-6f;
  const float w = dist > 0.0f ? 1.0f / (1.0f + a * __powf(dist, two_b)) : 1.0f;
  return __fdividef(scale * (w + bias), *den);
}

// One fired edge (optimize_layout_euclidean.rs:278-343, or with GEN the generic-metric rule
// of optimize_layout_generic.rs:57-121): attractive step on (head, tail), then `nneg`
// negative samples, all reading the snapshot buffer.  The tail row and a batch of negative
// rows are fetched together before the (sequential) updates of `cur`.
template <int DIM, bool GEN, int NEG_BATCH>
__device__ __forceinline__ void fired_edge(float (&cur)[DIM], uint32_t r, uint32_t k, uint32_t nneg,
                                           float* snap, const SgdParams& p, float alpha, uint64_t idx,
                                           uint32_t epoch, uint64_t seed, uint32_t seg_lo, uint32_t seg_n) {
  const float a = p.a, b = p.b;
  float* oth = snap + (uint64_t)k * DIM;
  float o[DIM];
  load_row<DIM>(o, oth);
  // Negative q uses half (q & 1) of pair (q >> 1) for this (entry, epoch).
  uint32_t kk[NEG_BATCH];
  float ob[NEG_BATCH][DIM];
  const NegRng rng(seed, idx, epoch);
  uint64_t rnd = 0;
  uint32_t rpair = 0xFFFFFFFFu;
  auto fetch = [&](uint32_t q0) {
#pragma unroll
    for (int q = 0; q < NEG_BATCH; ++q) {
      const uint32_t qq = q0 + q;
      if (qq < nneg) {
        if ((qq >> 1) != rpair) {
          rpair = qq >> 1;
          rnd = rng.pair(rpair);
        }
        const uint32_t rv = (qq & 1) ? (uint32_t)(rnd >> 32) : (uint32_t)rnd;
        kk[q] = seg_lo + __umulhi(rv, seg_n);
        if constexpr (DIM == 2) {
          // uniform rows, rarely reused by this SM: cached in L2 only, so they do not evict
          // the tail and head lines L1 serves (2M workload, 500 epochs: 311.1-311.2 against
          // 311.8-311.9 ms; renamed 20M roll, 30 epochs: 219.7-220.1 against 221.3-223.6 ms)
          const float2 t = __ldcg(reinterpret_cast<const float2*>(snap + (uint64_t)kk[q] * DIM));
          ob[q][0] = t.x;
          ob[q][1] = t.y;
        } else {
          load_row<DIM>(ob[q], snap + (uint64_t)kk[q] * DIM);
        }
      }
    }
  };
  fetch(0);
  // attractive step (:284-306)
  float ds = 0.0f;
#pragma unroll
  for (int d = 0; d < DIM; ++d) { const float df = cur[d] - o[d]; ds += df * df; }
  float g[DIM];
  if constexpr (GEN) {
    // head += clip(c * grad) alpha; tail += clip(c * rev_grad) alpha with rev_grad = -grad
    float den;
    const float gc = metric_coeff(ds, a, p.two_b, p.two_b, -1.0f, &den);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      g[d] = clip4(gc * __fdividef(cur[d] - o[d], den)) * alpha;
      cur[d] += g[d];
    }
  } else {
    float gc = 0.0f;
    if (ds > 0.0f) {
      const float pb = __powf(ds, b);
      gc = __fdividef(p.neg_attr * pb, ds * (a * pb * ds + 1.0f));
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      g[d] = clip4(gc * (cur[d] - o[d])) * alpha;
      cur[d] += g[d];
    }
  }
  sub_row<DIM>(oth, g);
  // negative samples (:313-341)
  for (uint32_t q0 = 0; q0 < nneg; q0 += NEG_BATCH) {
    if (q0 > 0) fetch(q0);  // more than NEG_BATCH negatives in this firing
#pragma unroll
    for (int q = 0; q < NEG_BATCH; ++q) {
      if (q0 + q >= nneg) break;
      if (kk[q] == r) continue;
      if constexpr (DIM == 2 && !GEN) {
        // the same operations as the generic-DIM code below, two columns per instruction
        const uint64_t c2 = pk2(cur[0], cur[1]);
        const uint64_t df2 = sub2(c2, pk2(ob[q][0], ob[q][1]));
        float df0, df1;
        up2(df2, df0, df1);
        const float dsn = df0 * df0 + df1 * df1;
        float gr = 0.0f;
        if (dsn > 0.0f) {
          const float pb = __powf(dsn, b);
          gr = __fdividef(p.pos_rep, (0.001f + dsn) * (a * pb * dsn + 1.0f));
        }
        if (gr > 0.0f) {
          float t0, t1;
          up2(mul2(pk2(gr, gr), df2), t0, t1);
          up2(fma2(pk2(clip4(t0), clip4(t1)), pk2(alpha, alpha), c2), cur[0], cur[1]);
        }
        continue;
      }
      float dsn = 0.0f;
#pragma unroll
      for (int d = 0; d < DIM; ++d) { const float df = cur[d] - ob[q][d]; dsn += df * df; }
      if constexpr (GEN) {
        float den;
        const float gr = metric_coeff(dsn, a, p.two_b, p.pos_rep, 0.0f, &den);
#pragma unroll
        for (int d = 0; d < DIM; ++d) cur[d] += clip4(gr * __fdividef(cur[d] - ob[q][d], den)) * alpha;
      } else {
        float gr = 0.0f;
        if (dsn > 0.0f) {
          const float pb = __powf(dsn, b);
          gr = __fdividef(p.pos_rep, (0.001f + dsn) * (a * pb * dsn + 1.0f));
        }
        if (gr > 0.0f) {
#pragma unroll
          for (int d = 0; d < DIM; ++d) cur[d] += clip4(gr * (cur[d] - ob[q][d])) * alpha;
        }
      }
    }
  }
}

// Variant with independent lane progress: each lane walks its own task through a small
// register window of entries (refilled on demand, W loads in flight), so a warp runs as long
// as its busiest task rather than its busiest lane of every batch.
#ifndef UB_SGD2_W
#define UB_SGD2_W 4
#endif
template <int DIM, bool GEN, int NEG_BATCH, int MINB, bool LM>
__global__ void __launch_bounds__(256, MINB) sgd_epoch_kernel2(
    const uint64_t* __restrict__ slice_base, const uint32_t* __restrict__ slice_width,
    const uint32_t* __restrict__ split_mask, const uint32_t* __restrict__ rowid,
    const uint2* __restrict__ entry, uint64_t n_slices, float* __restrict__ live, float* snap,
    SgdParams p, uint32_t epoch, float alpha) {
  constexpr int W = UB_SGD2_W;
  const uint64_t slice = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (slice >= n_slices) return;
  const uint32_t r = rowid[slice * 32 + lane];
  const bool active = r != PAD_ROW;
  const uint32_t width = active ? slice_width[slice] : 0u;
  const uint64_t base = slice_base[slice];
  const bool split = (split_mask[slice] >> lane) & 1u;
  uint32_t seg_lo = 0, seg_n = p.n_vertices;
  if (p.row_seg && active) {
    const uint32_t sg = p.row_seg[r];
    seg_lo = (uint32_t)p.seg_off[sg];
    seg_n = (uint32_t)(p.seg_off[sg + 1] - p.seg_off[sg]);
  }
  float cur[DIM], start[DIM];
  float* hrow = live + (uint64_t)(active ? r : 0) * DIM;
  if (active) load_row<DIM>(cur, hrow);
  else
#pragma unroll
    for (int d = 0; d < DIM; ++d) cur[d] = 0.0f;
#pragma unroll
  for (int d = 0; d < DIM; ++d) start[d] = cur[d];
  const uint32_t n = epoch;
  const uint64_t seed = p.seed;
  static_assert(W % 4 == 0, "windows are whole 4-entry sectors");
  // this lane's entries: contiguous (lane major) or every 32nd (interleaved)
  const uint2* lent = LM ? entry + base + (uint64_t)lane * width : entry + base + lane;
  uint2 win[W];
  uint32_t mask = 0, ew = 0, ebase = 0;
  for (;;) {
    while (mask == 0 && ew < width) {
      ebase = ew;
      if (LM) {
        // width is a multiple of W (slice_meta_kernel): the window lies inside the lane's entries
#pragma unroll
        for (int j = 0; j < W; j += 2) {
          const uint4 v = __ldg(reinterpret_cast<const uint4*>(lent + ew + j));
          win[j] = make_uint2(v.x, v.y);
          win[j + 1] = make_uint2(v.z, v.w);
        }
      } else {
#pragma unroll
        for (int j = 0; j < W; ++j) {
          const uint32_t e = ew + j;
          win[j] = e < width ? __ldg(lent + (uint64_t)e * 32) : make_uint2(0u, 0u);
        }
      }
#pragma unroll
      for (int j = 0; j < W; ++j)
        if (fires_at(n, win[j].y)) mask |= 1u << j;
      ew += W;
    }
    if (!__any_sync(0xFFFFFFFFu, mask != 0)) break;
    if (mask) {
      const int j = __ffs(mask) - 1;
      mask &= mask - 1;
      uint2 en = win[0];
#pragma unroll
      for (int t = 1; t < W; ++t)
        if (t == j) en = win[t];
      const uint32_t nneg = negatives_at(n, en.y, p.neg_rate);
      const uint64_t idx = LM ? base + (uint64_t)lane * width + ebase + j : base + (uint64_t)(ebase + j) * 32 + lane;
      fired_edge<DIM, GEN, NEG_BATCH>(cur, r, en.x, nneg, snap, p, alpha, idx, epoch, seed, seg_lo, seg_n);
    }
  }
  if (active) {
    if (split) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) atomicAdd(hrow + d, cur[d] - start[d]);
    } else {
      store_row<DIM>(hrow, cur);
    }
  }
}

// Any dimension (n_components > 4): same algorithm, head row in global memory (owned by this
// lane for whole-row tasks; split tasks accumulate their delta in place with atomics).  GEN
// selects the generic-metric rule as in fired_edge.
template <bool GEN>
__global__ void __launch_bounds__(256) sgd_epoch_anydim(
    const uint64_t* __restrict__ slice_base, const uint32_t* __restrict__ slice_width,
    const uint32_t* __restrict__ split_mask, const uint32_t* __restrict__ rowid,
    const uint2* __restrict__ entry, uint64_t n_slices, float* __restrict__ live, float* snap,
    SgdParams p, uint32_t epoch, float alpha, bool lane_major) {
  const uint64_t slice = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (slice >= n_slices) return;
  const uint32_t r = rowid[slice * 32 + lane];
  if (r == PAD_ROW) return;
  const uint32_t width = slice_width[slice];
  const uint64_t base = slice_base[slice];
  const bool split = (split_mask[slice] >> lane) & 1u;
  uint32_t seg_lo = 0, seg_n = p.n_vertices;
  if (p.row_seg) {
    const uint32_t sg = p.row_seg[r];
    seg_lo = (uint32_t)p.seg_off[sg];
    seg_n = (uint32_t)(p.seg_off[sg + 1] - p.seg_off[sg]);
  }
  const uint32_t dim = p.dim;
  float* cur = live + (uint64_t)r * dim;
  const uint32_t n = epoch;
  const uint64_t seed = p.seed;
  const float a = p.a, b = p.b;
  auto add = [&](uint32_t d, float v) {
    if (split) atomicAdd(cur + d, v);
    else cur[d] += v;
  };
  for (uint32_t e = 0; e < width; ++e) {
    const uint64_t idx = lane_major ? base + (uint64_t)lane * width + e : base + (uint64_t)e * 32 + lane;
    const uint2 en = __ldcs(entry + idx);
    if (!fires_at(n, en.y)) continue;
    float* oth = snap + (uint64_t)en.x * dim;
    float ds = 0.0f;
    for (uint32_t d = 0; d < dim; ++d) { const float df = cur[d] - oth[d]; ds += df * df; }
    float gc = 0.0f, den = 1.0f;
    if constexpr (GEN) {
      gc = metric_coeff(ds, a, p.two_b, p.two_b, -1.0f, &den);
    } else if (ds > 0.0f) {
      const float pb = __powf(ds, b);
      gc = __fdividef(p.neg_attr * pb, ds * (a * pb * ds + 1.0f));
    }
    for (uint32_t d = 0; d < dim; ++d) {
      const float cd = cur[d], od = oth[d];
      const float g = clip4(gc * (GEN ? __fdividef(cd - od, den) : cd - od)) * alpha;
      add(d, g);
      atomicAdd(oth + d, -g);
    }
    const uint32_t nneg = negatives_at(n, en.y, p.neg_rate);
    const NegRng rng(seed, idx, epoch);
    uint64_t rnd = 0;
    for (uint32_t q = 0; q < nneg; ++q) {
      if ((q & 1) == 0) rnd = rng.pair(q >> 1);
      const uint32_t rv = (q & 1) ? (uint32_t)(rnd >> 32) : (uint32_t)rnd;
      const uint32_t kk = seg_lo + __umulhi(rv, seg_n);
      if (kk == r) continue;
      const float* ob = snap + (uint64_t)kk * dim;
      float dsn = 0.0f;
      for (uint32_t d = 0; d < dim; ++d) { const float df = cur[d] - ob[d]; dsn += df * df; }
      if constexpr (GEN) {
        float dn;
        const float gr = metric_coeff(dsn, a, p.two_b, p.pos_rep, 0.0f, &dn);
        for (uint32_t d = 0; d < dim; ++d) add(d, clip4(gr * __fdividef(cur[d] - ob[d], dn)) * alpha);
      } else {
        float gr = 0.0f;
        if (dsn > 0.0f) {
          const float pb = __powf(dsn, b);
          gr = __fdividef(p.pos_rep, (0.001f + dsn) * (a * pb * dsn + 1.0f));
        }
        if (gr > 0.0f)
          for (uint32_t d = 0; d < dim; ++d) add(d, clip4(gr * (cur[d] - ob[d])) * alpha);
      }
    }
  }
}

// ------------------------------------------------------------------------------ K5 pieces
__global__ void kept_degree_kernel(const uint64_t* __restrict__ indptr, const float* __restrict__ data,
                                   uint64_t n, float thr, const float* __restrict__ seg_thr,
                                   const uint32_t* __restrict__ row_seg, uint32_t* __restrict__ deg) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float t = seg_thr ? seg_thr[row_seg[r]] : thr;
  uint32_t c = 0;
  for (uint64_t q = indptr[r]; q < indptr[r + 1]; ++q) c += data[q] >= t ? 1u : 0u;
  deg[r] = c;
}

// Batched instances: max graph weight of each instance (optimizer.rs:90-94 per instance).
__global__ void segment_max_kernel(const uint64_t* __restrict__ indptr, const float* __restrict__ data,
                                   const uint64_t* __restrict__ seg_off, float* __restrict__ out) {
  const uint32_t sgm = blockIdx.x;
  const uint64_t q0 = indptr[seg_off[sgm]], q1 = indptr[seg_off[sgm + 1]];
  float m = 0.0f;
  for (uint64_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) m = fmaxf(m, data[q]);
  __shared__ float s_m[32];
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t w = 1; w < blockDim.x / 32; ++w) m = fmaxf(m, s_m[w]);
    out[sgm] = m;
  }
}

// Row u of the layout is row order[u] of the kept-edge CSR (order null: the same row).
__global__ void ptr_degree_kernel(const uint64_t* __restrict__ kptr, uint64_t n, uint32_t chunk,
                                  const uint32_t* __restrict__ order, uint32_t* __restrict__ deg,
                                  uint32_t* __restrict__ ntask) {
  const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const uint64_t r = order ? order[u] : u;
  const uint32_t d = (uint32_t)(kptr[r + 1] - kptr[r]);
  deg[u] = d;
  ntask[u] = (d + chunk - 1) / chunk;
}

// One task per chunk of a row: row id, first kept-edge index, length, split flag, sort key.
// The key orders tasks by descending length and, with rate_bits = RATE_BITS, then by
// descending mean firing rate (sum over the task's edges of min(1, 1 / epochs_per_sample),
// over its length, in RATE_BITS bits), so that a warp's lanes draw similar numbers of firings
// per epoch; batched instances sort instance-major first.
constexpr int RATE_BITS = 8;
__global__ void task_fill_kernel(const uint64_t* __restrict__ kptr, const uint32_t* __restrict__ deg,
                                 const uint64_t* __restrict__ tptr, uint64_t n, uint32_t chunk,
                                 const uint32_t* __restrict__ row_seg, int len_bits, int rate_bits,
                                 int block_shift, const double* __restrict__ keps, const uint32_t* __restrict__ order,
                                 uint32_t* __restrict__ trow, uint64_t* __restrict__ tstart,
                                 uint32_t* __restrict__ tkey) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const uint64_t src = order ? order[r] : r;  // the kept-edge CSR row of layout row r
  const uint32_t d = deg[r];
  const uint64_t t0 = tptr[r], nt = tptr[r + 1] - t0;
  for (uint64_t c = 0; c < nt; ++c) {
    const uint32_t len = (uint32_t)min((uint64_t)chunk, (uint64_t)d - c * chunk);
    const uint64_t st = kptr[src] + c * chunk;
    trow[t0 + c] = (uint32_t)r | (nt > 1 ? 0x80000000u : 0u);   // high bit: partial row
    tstart[t0 + c] = st;
    uint32_t rate = 0;
    if (rate_bits) {
      float sp = 0.0f;
      for (uint32_t e = 0; e < len; ++e) {
        const double x = keps[st + e];
        sp += x > 1.0 ? (float)(1.0 / x) : (x > 0.0 ? 1.0f : 0.0f);
      }
      const uint32_t top = (1u << rate_bits) - 1u;
      rate = top - min(top, (uint32_t)(sp / (float)max(len, 1u) * (float)(top + 1u)));
    }
    const uint32_t hi = block_shift >= 0 ? (uint32_t)(r >> block_shift) : (row_seg ? row_seg[r] : 0u);
    tkey[t0 + c] = (((hi << len_bits) | (chunk - len)) << rate_bits) | rate;
  }
}

__global__ void iota_u32_kernel(uint32_t* __restrict__ p, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = (uint32_t)i;
}

__global__ void slice_meta_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ trow,
                                  const uint32_t* __restrict__ skey, uint64_t T, uint64_t n_slices,
                                  uint32_t chunk, int rate_bits, uint32_t len_mask, bool lane_major,
                                  uint32_t* __restrict__ width,
                                  uint32_t* __restrict__ rowid, uint32_t* __restrict__ split_mask) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_slices * 32) return;
  const uint32_t tr = q < T ? trow[perm[q]] : PAD_ROW;
  rowid[q] = tr == PAD_ROW ? PAD_ROW : (tr & 0x7FFFFFFFu);
  const unsigned bits = __ballot_sync(0xFFFFFFFFu, tr != PAD_ROW && (tr & 0x80000000u));
  // slice width = longest task of the slice (instance-major order: the max over lanes)
  uint32_t len = q < T ? chunk - ((skey[q] >> rate_bits) & len_mask) : 0u;
  for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xFFFFFFFFu, len, o));
  // whole register windows per lane (UB_SGD2_W entries, a multiple of one 4-entry sector): the
  // lane-major epoch loads a full window without a bounds check
  if (lane_major) len = (len + (UB_SGD2_W - 1u)) / UB_SGD2_W * UB_SGD2_W;
  if ((q & 31) == 0) {
    width[q >> 5] = len;
    split_mask[q >> 5] = bits;
  }
}

__global__ void slice_fill_kernel(const uint32_t* __restrict__ ktail, const double* __restrict__ keps,
                                  const uint32_t* __restrict__ perm, const uint64_t* __restrict__ tstart,
                                  const uint32_t* __restrict__ skey, uint64_t T, uint32_t chunk,
                                  int rate_bits, uint32_t len_mask, const uint64_t* __restrict__ wscan,
                                  const uint32_t* __restrict__ width, uint64_t n_slices, bool lane_major,
                                  const uint32_t* __restrict__ rank, uint2* __restrict__ entry) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_slices * 32) return;
  const uint64_t s = q >> 5;
  const uint32_t lane = (uint32_t)(q & 31);
  const uint64_t base = wscan[s] * 32;
  const uint32_t wd = width[s];
  uint32_t e = 0;
  if (q < T) {
    const uint64_t st = tstart[perm[q]];
    const uint32_t len = chunk - ((skey[q] >> rate_bits) & len_mask);
    for (; e < len; ++e)
      entry[lane_major ? base + (uint64_t)lane * wd + e : base + (uint64_t)e * 32 + lane] =
          make_uint2(rank ? rank[ktail[st + e]] : ktail[st + e], q_minus_1(keps[st + e]));
  }
  for (; e < wd; ++e)
    entry[lane_major ? base + (uint64_t)lane * wd + e : base + (uint64_t)e * 32 + lane] = make_uint2(0u, 0u);
}

__global__ void head_from_ptr_kernel(const uint64_t* __restrict__ kptr, uint64_t n, uint32_t* __restrict__ head) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (uint64_t j = kptr[r]; j < kptr[r + 1]; ++j) head[j] = (uint32_t)r;
}

// Schedule state of the reference at `cur` (optimizer.rs:41-43) from the closed form:
// m = firings so far, T = negatives drawn so far;  eons = (m+1)*eps, epns = eps/neg,
// eonns = epns*(1+T).
__global__ void export_state_kernel(const double* __restrict__ eps, uint64_t E, uint64_t neg,
                                    uint64_t cur, double* __restrict__ eons, double* __restrict__ eonns,
                                    double* __restrict__ epns) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  const double e = eps[i];
  const uint32_t q = q_minus_1(e);
  const uint64_t m = cur > 0 ? fires_by((uint32_t)(cur - 1), q) : 0ull;
  const uint64_t t = negatives_after(m, q, (uint32_t)neg);
  const double pn = e / (double)neg;
  if (eons) eons[i] = e * ((double)m + 1.0);
  if (epns) epns[i] = pn;
  if (eonns) eonns[i] = pn * (1.0 + (double)t);
}

// make_epochs_per_sample.rs:30-49 in f64.
__device__ __forceinline__ double epochs_per_sample(float w, double max_w, double n_ep) {
  const double n_samples = n_ep * ((double)w / max_w);
  return n_samples > 0.0 ? n_ep / n_samples : -1.0;
}

__global__ void export_edges_kernel(const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                                    const float* __restrict__ data, uint64_t n, float thr, double max_w,
                                    double n_ep, const float* __restrict__ seg_thr,
                                    const float* __restrict__ seg_maxw, const uint32_t* __restrict__ row_seg,
                                    const uint64_t* __restrict__ kept_ptr, uint32_t* __restrict__ head,
                                    uint32_t* __restrict__ tail, double* __restrict__ eps) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float t = thr;
  double mw = max_w;
  if (seg_thr) {
    const uint32_t sg = row_seg[r];
    t = seg_thr[sg];
    mw = (double)seg_maxw[sg];
  }
  uint64_t o = kept_ptr[r];
  for (uint64_t j = indptr[r]; j < indptr[r + 1]; ++j) {
    const float w = data[j];
    if (w >= t) {
      if (head) head[o] = (uint32_t)r;
      if (tail) tail[o] = indices[j];
      if (eps) eps[o] = epochs_per_sample(w, mw, n_ep);
      ++o;
    }
  }
}

// ------------------------------------------------------------------------------ K6
// optimizer.rs:189-230.  f32::min / f32::max ignore NaN like fminf / fmaxf.
__global__ void minmax_dim_kernel(const float* __restrict__ emb, uint64_t n, uint32_t dim,
                                  const uint64_t* __restrict__ seg_off, float* __restrict__ mins,
                                  float* __restrict__ scales) {
  // one block per (dimension, instance)
  const uint32_t d = blockIdx.x, sg = blockIdx.y;
  const uint64_t r0 = seg_off ? seg_off[sg] : 0, r1 = seg_off ? seg_off[sg + 1] : n;
  float mn = INFINITY, mx = -INFINITY;
  for (uint64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const float v = emb[i * dim + d];
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
  __shared__ float s_mn[32], s_mx[32];
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) { s_mn[threadIdx.x >> 5] = mn; s_mx[threadIdx.x >> 5] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t w = 1; w < blockDim.x / 32; ++w) { mn = fminf(mn, s_mn[w]); mx = fmaxf(mx, s_mx[w]); }
    const float range = __fsub_rn(mx, mn);
    mins[sg * dim + d] = mn;
    scales[sg * dim + d] = range > 0.0f ? __fdiv_rn(10.0f, range) : 0.0f;
  }
}

// A plain fit's column min / max in two stages: block b of dimension d reduces rows
// b, b + G, ... into part[d][b]; then minmax_finish_kernel folds the G partials.  Min and max
// ignore NaN and are exact in any order, so the result equals one block's.
__global__ void minmax_part_kernel(const float* __restrict__ emb, uint64_t n, uint32_t dim,
                                   float* __restrict__ pmin, float* __restrict__ pmax) {
  const uint32_t d = blockIdx.y, G = gridDim.x;
  float mn = INFINITY, mx = -INFINITY;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)G * blockDim.x) {
    const float v = emb[i * dim + d];
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
  __shared__ float s_mn[32], s_mx[32];
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) { s_mn[threadIdx.x >> 5] = mn; s_mx[threadIdx.x >> 5] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t w = 1; w < blockDim.x / 32; ++w) { mn = fminf(mn, s_mn[w]); mx = fmaxf(mx, s_mx[w]); }
    pmin[d * G + blockIdx.x] = mn;
    pmax[d * G + blockIdx.x] = mx;
  }
}

__global__ void minmax_finish_kernel(const float* __restrict__ pmin, const float* __restrict__ pmax, uint32_t G,
                                     float* __restrict__ mins, float* __restrict__ scales) {
  const uint32_t d = blockIdx.x;
  float mn = INFINITY, mx = -INFINITY;
  for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
    mn = fminf(mn, pmin[d * G + g]);
    mx = fmaxf(mx, pmax[d * G + g]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
  }
  if (threadIdx.x == 0) {
    const float range = __fsub_rn(mx, mn);
    mins[d] = mn;
    scales[d] = range > 0.0f ? __fdiv_rn(10.0f, range) : 0.0f;
  }
}

__global__ void normalize_kernel(float* __restrict__ emb, uint64_t total, uint32_t dim,
                                 const float* __restrict__ mins, const float* __restrict__ scales,
                                 const uint32_t* __restrict__ row_seg) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const uint64_t r = i / dim;
  const uint32_t d = (uint32_t)(i - r * dim);
  const uint64_t c = (uint64_t)(row_seg ? row_seg[r] : 0) * dim + d;
  const float sc = scales[c];
  if (sc > 0.0f) emb[i] = __fmul_rn(__fsub_rn(emb[i], mins[c]), sc);
}

// ------------------------------------------------------------------------------ accounting
__global__ void schedule_totals_kernel(const uint2* __restrict__ entry, uint64_t n_entries, uint64_t neg,
                                       uint64_t start, uint64_t end, unsigned long long* __restrict__ fired,
                                       unsigned long long* __restrict__ negs) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long f = 0, g = 0;
  if (i < n_entries) {
    const uint32_t q = entry[i].y;
    // firings in [start, end) = m(end-1) - m(start-1); negatives telescope the same way.
    const uint64_t fe = end > 0 ? fires_by((uint32_t)(end - 1), q) : 0ull;
    const uint64_t fs = start > 0 ? fires_by((uint32_t)(start - 1), q) : 0ull;
    f = fe - fs;
    g = negatives_after(fe, q, (uint32_t)neg) - negatives_after(fs, q, (uint32_t)neg);
  }
  for (int o = 16; o > 0; o >>= 1) {
    f += __shfl_xor_sync(0xFFFFFFFFu, f, o);
    g += __shfl_xor_sync(0xFFFFFFFFu, g, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (f) atomicAdd(fired, f);
    if (g) atomicAdd(negs, g);
  }
}

// The negative samples the epoch kernel would draw for the firings of entries
// [first, first + count) at `epoch`: draw q of entry e is out[(e - first) * per + q], made by
// the same generator and mapping as fired_edge (half q & 1 of pair q >> 1, multiply-high into
// [lo, lo + range)).  Statistical tests of the generator read these.
__global__ void negative_draws_kernel(uint64_t seed, uint64_t first, uint64_t count, uint32_t epoch,
                                      uint32_t per, uint32_t lo, uint32_t range, uint32_t* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const NegRng rng(seed, first + i, epoch);
  uint64_t rnd = 0;
  for (uint32_t q = 0; q < per; ++q) {
    if ((q & 1) == 0) rnd = rng.pair(q >> 1);
    const uint32_t rv = (q & 1) ? (uint32_t)(rnd >> 32) : (uint32_t)rnd;
    out[i * per + q] = lo + __umulhi(rv, range);
  }
}

// Negatives the epoch kernel draws for a firing of an entry with schedule word q at epoch n
// (0 where the entry does not fire at n): the schedule's per-firing count, for exact tests.
__global__ void negatives_per_firing_kernel(const uint32_t* __restrict__ qs, const uint32_t* __restrict__ ns,
                                            uint64_t count, uint32_t neg, uint32_t* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t q = qs[i], n = ns[i];
  out[i] = fires_at(n, q) ? negatives_at(n, q, neg) : 0u;
}

__global__ void nan_rows_kernel(const uint64_t* __restrict__ indptr, uint64_t n, uint32_t dim,
                                float* __restrict__ emb) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || indptr[r + 1] != indptr[r]) return;
  for (uint32_t d = 0; d < dim; ++d) emb[r * dim + d] = __int_as_float(0x7FC00000);
}

__global__ void scale32_kernel(uint64_t* __restrict__ x, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= 32;
}

inline unsigned grid_for(uint64_t n, unsigned bt) { return (unsigned)((n + bt - 1) / bt); }

}  // namespace

void kept_degree(const uint64_t* indptr, const float* data, uint64_t n, float thr, uint32_t* deg,
                 cudaStream_t s, const SegmentPrune* sp) {
  if (n == 0) return;
  kept_degree_kernel<<<grid_for(n, 256), 256, 0, s>>>(indptr, data, n, thr, sp ? sp->seg_thr : nullptr,
                                                      sp ? sp->row_seg : nullptr, deg);
  UB_LAUNCH_CHECK();
}

void segment_max(const uint64_t* indptr, const float* data, const uint64_t* seg_off, uint32_t n_seg,
                 float* out, cudaStream_t s) {
  if (n_seg == 0) return;
  segment_max_kernel<<<n_seg, 256, 0, s>>>(indptr, data, seg_off, out);
  UB_LAUNCH_CHECK();
}

void prune_edges(const uint64_t* indptr, const float* data, uint64_t n, float thr, uint64_t* kept_ptr,
                 uint64_t* n_edges, cudaStream_t s, const SegmentPrune* sp) {
  DevBuf<uint32_t> deg(n, s);
  kept_degree(indptr, data, n, thr, deg.p, s, sp);
  scan_u32_to_u64(deg.p, kept_ptr, n, s);
  UB_CUDA(cudaMemcpyAsync(n_edges, kept_ptr + n, 8, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
}

void head_from_ptr(const uint64_t* kept_ptr, uint64_t n, uint32_t* head, cudaStream_t s) {
  if (n == 0) return;
  head_from_ptr_kernel<<<grid_for(n, 256), 256, 0, s>>>(kept_ptr, n, head);
  UB_LAUNCH_CHECK();
}

void export_state(const double* eps, uint64_t E, uint64_t neg_rate, uint64_t cur_epoch, double* eons,
                  double* eonns, double* epns, cudaStream_t s) {
  if (E == 0) return;
  export_state_kernel<<<grid_for(E, 256), 256, 0, s>>>(eps, E, neg_rate, cur_epoch, eons, eonns, epns);
  UB_LAUNCH_CHECK();
}

// Longest task (edges) so that no single lane's chain of updates outlasts roughly half an
// epoch: an epoch streams E edges across the whole GPU, while one lane works through its
// task sequentially, so the bound grows linearly with E (~E/135k for this kernel).
uint32_t pick_chunk(uint64_t n_edges) {
  if (const char* e = getenv("UMAP_B200_CHUNK")) {
    long v = atol(e);
    if (v >= 1 && v <= (1 << 30)) return (uint32_t)v;
  }
  uint64_t c = (n_edges / 135000 + 4) / 8 * 8;
  return (uint32_t)std::min<uint64_t>(512, std::max<uint64_t>(16, c));
}

// The generic-metric rule (optimize_layout_generic.rs) attracts much harder than the
// Euclidean one, and a row cut into tasks that all start from the same head position
// overshoots where the reference applies the row's moves one after another: on the 10k-point
// Gaussian workload (4 seeds each) 16-edge tasks gave 15-NN recall 0.0348 and fuzzy
// cross-entropy 268,541 against the oracle's 0.0380 and 270,403; 32: 0.0356 / 268,666;
// 64: 0.0369 / 269,976; 128 and whole rows: no further change.  The Euclidean rule showed no
// such dependence at any task length.  So the generic rule keeps typical rows whole (tasks
// of at least 64 edges, about three times a kNN graph's mean degree) and splits only hubs.
uint32_t pick_chunk_generic(uint64_t n_edges) {
  if (getenv("UMAP_B200_CHUNK")) return pick_chunk(n_edges);
  return std::max<uint32_t>(64, pick_chunk(n_edges));
}

// Whether the epoch kernel takes the 8-negatives budget (the Euclidean rule in 2-D and 1-D):
// where the layout's warps (one per slice) fill at most two waves of the wide budget's
// resident warps (SMs x 5 blocks x 8 warps), and for renamed DRAM-bound layouts, where more
// row loads in flight per lane hide DRAM latency (20M-point swiss roll, 30 epochs: 337.7 ->
// 308.4 ms).  UMAP_B200_SGD_SHORT=0 / 1 forces it.
bool pick_short_epoch(uint64_t n_slices, bool renamed) {
  if (const char* e = getenv("UMAP_B200_SGD_SHORT")) {
    if (e[0] == '0') return false;
    if (e[0] == '1') return true;
  }
  if (renamed) return true;  // the layout takes the DRAM budget (pick_dram_epoch) unless forced
  int dev = 0, sms = 0;
  UB_CUDA(cudaGetDevice(&dev));
  UB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return n_slices <= 2ull * (uint64_t)std::max(sms, 1) * MINB_WIDE * 8;
}

// Renamed (DRAM-bound) layouts take the 12-negatives budget unless UMAP_B200_SGD_SHORT forces one
// of the other two.
bool pick_dram_epoch(bool renamed) {
  return renamed && getenv("UMAP_B200_SGD_SHORT") == nullptr;
}

// Entry order of the layout.  Lane major (a lane's window is one 32-byte sector) wins while
// the rows the negatives and tails reach stay in L2: a plain fit whose 2-D embedding (live +
// snapshot, 16 B per vertex) is at most 64 MB, and batched instances, whose instance-major
// task order keeps the instances in flight in L2.  Beyond that every access goes to DRAM,
// where the interleaved order's whole 256-byte rows per warp use DRAM bursts better than
// 32-byte windows.  UMAP_B200_SGD_LANE_MAJOR=0 / 1 forces either.
bool pick_lane_major(uint64_t n, bool segmented) {
  if (const char* e = getenv("UMAP_B200_SGD_LANE_MAJOR")) {
    if (e[0] == '0') return false;
    if (e[0] == '1') return true;
  }
  return segmented || n <= 4000000ull;
}

// Whether a plain fit's layout renames its vertices into a locality order (order.cu): where
// every random access is a DRAM access, i.e. the sizes that take interleaved entries.
// UMAP_B200_RELABEL=0 / 1 forces either.  The generic-metric rule never renames (its caller
// passes rename = false): it is sensitive to which rows update at the same time (its split
// rows showed that), and its parity with the reference was established in the caller's order;
// on a 6,000-point roll one renamed run sat 2.6% from a plain one, inside that small case's
// run-to-run spread, so renaming is not shown to move it, only not shown to be harmless.
bool pick_relabel(uint64_t n, bool segmented) {
  if (segmented) return false;
  if (const char* e = getenv("UMAP_B200_RELABEL")) {
    if (e[0] == '0') return false;
    if (e[0] == '1') return true;
  }
  return n > 4000000ull;
}

// Order in which the tasks are dealt to warps (32 consecutive tasks per warp):
//  * Length: descending length (a warp's lanes scan equally long tasks; least padding).
//  * LengthRate: length, then descending mean firing rate, so that a warp's lanes draw similar
//    numbers of firings per epoch.  Small graphs, whose epochs are short and bound by their
//    warps' busiest lanes (100k-point fit: 25.4-25.6 against 26.0-26.1 ms).
//  * RowBlock: blocks of 2^TASK_BLOCK_SHIFT consecutive layout rows, length order inside each.
//    Renamed layouts: their warps in flight then cover a narrow range of new ids, whose tails
//    stay in L2 (30 epochs of the 20M-point roll: 292.6 ms in length order, 245.7 in row
//    order, blocks of 2^6 / 2^8 / 2^10 / 2^12 / 2^14 / 2^16 rows: 241.4 / 237.7 / 235.6 /
//    235.3-239.1 / 239.7 / 242.9 ms; 40M points, 24 epochs: 564.7 -> 475.9 ms).
//  * Row: layout row order (measurement only; the 2M-point fit takes 5x as long in it, its
//    whole-row tasks of very different lengths padded to the longest of each warp).
// Plain fits without renaming keep Length at any size that is not short (2M points: 320.6 in
// LengthRate against 321.0 ms, within noise; a block order: 1106 ms).  Batched instances take
// LengthRate inside each instance (4,096 instances, 200 epochs: 2,822-2,825 against
// 2,842-2,843 ms per batch).  UMAP_B200_TASK_ORDER=len / rate / block / row forces one.
constexpr int TASK_BLOCK_SHIFT = 12;
TaskOrder pick_task_order(bool renamed, bool short_graph, bool segmented) {
  if (const char* e = getenv("UMAP_B200_TASK_ORDER")) {
    if (!strcmp(e, "len")) return TaskOrder::Length;
    if (!strcmp(e, "rate")) return TaskOrder::LengthRate;
    if (!strcmp(e, "block") && !segmented) return TaskOrder::RowBlock;
    if (!strcmp(e, "row")) return TaskOrder::Row;
  }
  if (segmented) return TaskOrder::LengthRate;
  if (renamed) return TaskOrder::RowBlock;
  return short_graph ? TaskOrder::LengthRate : TaskOrder::Length;
}

void build_sgd_layout(const uint64_t* kept_ptr, const uint32_t* ktail, const double* keps, uint64_t n,
                      uint32_t chunk, SgdLayout& L, cudaStream_t s, const Segments* seg, bool rename) {
  L.n_vertices = n;
  L.lane_major = pick_lane_major(n, seg != nullptr);
  DevBuf<uint32_t> rank;
  L.order.reset();
  if (n && rename && pick_relabel(n, seg != nullptr)) {
    L.order.alloc(n, s);
    rank.alloc(n, s);
    locality_order(kept_ptr, ktail, n, L.order.p, rank.p, s);
  }
  uint64_t n_edges = 0;
  UB_CUDA(cudaMemcpyAsync(&n_edges, kept_ptr + n, 8, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  L.n_edges = n_edges;
  L.chunk = chunk ? chunk : pick_chunk(n_edges);
  DevBuf<uint32_t> deg(n, s), ntask(n, s);
  if (n) {
    ptr_degree_kernel<<<grid_for(n, 256), 256, 0, s>>>(kept_ptr, n, L.chunk, L.order.p, deg.p, ntask.p);
    UB_LAUNCH_CHECK();
  }
  DevBuf<uint32_t> dmax(1, s);
  reduce_max_u32(deg.p, n, dmax.p, s);
  DevBuf<uint64_t> tptr(n + 1, s);
  scan_u32_to_u64(ntask.p, tptr.p, n, s);
  uint64_t T = 0;
  UB_CUDA(cudaMemcpyAsync(&T, tptr.p + n, 8, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaMemcpyAsync(&L.max_degree, dmax.p, 4, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  if (T >= 0xFFFFFFFFull) throw Error(UNSUPPORTED, "too many SGD tasks (>= 2^32)");
  L.n_tasks = T;
  DevBuf<uint32_t> trow(T, s), tkey(T, s), skey(T, s), perm(T, s);
  DevBuf<uint64_t> tstart(T, s);
  const int len_bits = bits_for(L.chunk);
  const uint32_t len_mask = (1u << len_bits) - 1u;
  const uint32_t n_seg = seg ? seg->n_seg : 0u;
  if ((uint64_t)n_seg << len_bits >= (1ull << 32)) throw Error(UNSUPPORTED, "too many instances for the task sort key");
  const int seg_bits = n_seg ? bits_for(n_seg) : 0;
  const bool renamed = L.order.p != nullptr;
  TaskOrder torder = pick_task_order(renamed, pick_short_epoch((T + 31) / 32, renamed), seg != nullptr);
  if (torder == TaskOrder::LengthRate && len_bits + seg_bits + RATE_BITS > 32) torder = TaskOrder::Length;
  L.task_order = torder;
  const int rate_bits = torder == TaskOrder::LengthRate ? RATE_BITS : 0;
  int block_shift = -1, block_bits = 0;
  if (torder == TaskOrder::RowBlock) {
    block_shift = TASK_BLOCK_SHIFT;
    if (const char* e = getenv("UMAP_B200_TASK_BLOCK")) block_shift = std::min(31, std::max(0, atoi(e)));
    while (bits_for(n >> block_shift) + len_bits > 32) ++block_shift;  // the key fits 32 bits
    block_bits = bits_for(n >> block_shift);
  }
  if (n) {
    task_fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(kept_ptr, deg.p, tptr.p, n, L.chunk,
                                                      seg ? seg->row_seg : nullptr, len_bits, rate_bits, block_shift,
                                                      keps, L.order.p, trow.p, tstart.p, tkey.p);
    UB_LAUNCH_CHECK();
  }
  if (T && torder == TaskOrder::Row) {
    iota_u32_kernel<<<grid_for(T, 256), 256, 0, s>>>(perm.p, T);
    UB_LAUNCH_CHECK();
    UB_CUDA(cudaMemcpyAsync(skey.p, tkey.p, T * 4, cudaMemcpyDeviceToDevice, s));
  } else if (T) {
    radix_sort_pairs(tkey.p, nullptr, skey.p, perm.p, T, len_bits + (block_shift >= 0 ? block_bits : seg_bits) + rate_bits, s);
  }
  L.n_slices = (T + 31) / 32;
  L.slice_width.alloc(L.n_slices, s);
  L.split_mask.alloc(L.n_slices, s);
  L.rowid.alloc(L.n_slices * 32, s);
  L.slice_base.alloc(L.n_slices + 1, s);
  if (L.n_slices) {
    slice_meta_kernel<<<grid_for(L.n_slices * 32, 256), 256, 0, s>>>(perm.p, trow.p, skey.p, T, L.n_slices,
                                                                        L.chunk, rate_bits, len_mask, L.lane_major,
                                                                        L.slice_width.p, L.rowid.p,
                                                                        L.split_mask.p);
    UB_LAUNCH_CHECK();
  }
  DevBuf<uint64_t> wscan(L.n_slices + 1, s);
  scan_u32_to_u64(L.slice_width.p, wscan.p, L.n_slices, s);
  uint64_t wtot = 0;
  UB_CUDA(cudaMemcpyAsync(&wtot, wscan.p + L.n_slices, 8, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  L.n_entries = wtot * 32;
  L.entry.alloc(L.n_entries, s);
  if (L.n_slices) {
    slice_fill_kernel<<<grid_for(L.n_slices * 32, 256), 256, 0, s>>>(ktail, keps, perm.p, tstart.p, skey.p, T,
                                                                        L.chunk, rate_bits, len_mask, wscan.p,
                                                                        L.slice_width.p, L.n_slices,
                                                                        L.lane_major, rank.p, L.entry.p);
    UB_LAUNCH_CHECK();
  }
  // slice_base = 32 * wscan (entries, not widths)
  scale32_kernel<<<grid_for(L.n_slices + 1, 256), 256, 0, s>>>(wscan.p, L.n_slices + 1);
  UB_LAUNCH_CHECK();
  UB_CUDA(cudaMemcpyAsync(L.slice_base.p, wscan.p, (L.n_slices + 1) * 8, cudaMemcpyDeviceToDevice, s));
  // count partial-row tasks (diagnostics)
  std::vector<uint32_t> h(L.n_slices);
  if (L.n_slices) UB_CUDA(cudaMemcpyAsync(h.data(), L.split_mask.p, L.n_slices * 4, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  L.split_tasks = 0;
  for (uint32_t v : h) L.split_tasks += __builtin_popcount(v);
  L.short_epoch = pick_short_epoch(L.n_slices, L.order.p != nullptr);
  L.dram_epoch = pick_dram_epoch(L.order.p != nullptr);
}

void export_edges(const uint64_t* indptr, const uint32_t* indices, const float* data, uint64_t n,
                  float thr, float max_w, uint64_t total_epochs, const uint64_t* kept_ptr,
                  uint32_t* head, uint32_t* tail, double* eps, cudaStream_t s, const SegmentPrune* sp) {
  if (n == 0) return;
  export_edges_kernel<<<grid_for(n, 256), 256, 0, s>>>(
      indptr, indices, data, n, thr, (double)max_w, (double)total_epochs, sp ? sp->seg_thr : nullptr,
      sp ? sp->seg_maxw : nullptr, sp ? sp->row_seg : nullptr, kept_ptr, head, tail, eps);
  UB_LAUNCH_CHECK();
}

void normalize_init(float* emb, uint64_t n, uint32_t dim, cudaStream_t s, const Segments* seg) {
  if (n == 0 || dim == 0) return;
  const uint32_t n_seg = seg ? seg->n_seg : 1u;
  DevBuf<float> mins((uint64_t)dim * n_seg, s), scales((uint64_t)dim * n_seg, s);
  if (seg || dim > 65535) {  // batched instances: one block per (dimension, instance)
    minmax_dim_kernel<<<dim3(dim, n_seg), 1024, 0, s>>>(emb, n, dim, seg ? seg->seg_off : nullptr, mins.p, scales.p);
    UB_LAUNCH_CHECK();
  } else {
    const uint32_t G = (uint32_t)std::min<uint64_t>(256, (n + 4095) / 4096);
    DevBuf<float> pmin((uint64_t)dim * G, s), pmax((uint64_t)dim * G, s);
    minmax_part_kernel<<<dim3(G, dim), 256, 0, s>>>(emb, n, dim, pmin.p, pmax.p);
    UB_LAUNCH_CHECK();
    minmax_finish_kernel<<<dim, 32, 0, s>>>(pmin.p, pmax.p, G, mins.p, scales.p);
    UB_LAUNCH_CHECK();
  }
  normalize_kernel<<<grid_for(n * dim, 256), 256, 0, s>>>(emb, n * dim, dim, mins.p, scales.p,
                                                          seg ? seg->row_seg : nullptr);
  UB_LAUNCH_CHECK();
}

void sgd_epoch(const SgdLayout& L, float* live, float* snap, const SgdParams& p, uint32_t epoch, float alpha,
               cudaStream_t s) {
  if (L.n_slices == 0) return;
  const unsigned bt = L.block_threads ? L.block_threads : 256;
  const unsigned grid = grid_for(L.n_slices * 32, bt);
#define UB_SGD_ARGS L.slice_base.p, L.slice_width.p, L.split_mask.p, L.rowid.p, L.entry.p, L.n_slices, live, snap, \
                    p, epoch, alpha
#define UB_SGD_WIDE(D, GEN)                                                                   \
  if (L.lane_major) sgd_epoch_kernel2<D, GEN, NB_WIDE, MINB_WIDE, true><<<grid, bt, 0, s>>>(UB_SGD_ARGS); \
  else sgd_epoch_kernel2<D, GEN, NB_WIDE, MINB_WIDE, false><<<grid, bt, 0, s>>>(UB_SGD_ARGS)
// short graphs are small, so lane major by default (pick_lane_major); both orders are built
#define UB_SGD_SHORT(D, GEN)                                                                    \
  if (L.lane_major) sgd_epoch_kernel2<D, GEN, NB_SHORT, MINB_SHORT, true><<<grid, bt, 0, s>>>(UB_SGD_ARGS); \
  else sgd_epoch_kernel2<D, GEN, NB_SHORT, MINB_SHORT, false><<<grid, bt, 0, s>>>(UB_SGD_ARGS)
#define UB_SGD_DISPATCH(GEN, SHORT)                                                   \
  switch (p.dim) {                                                                    \
    case 1: if (SHORT) UB_SGD_SHORT(1, GEN); else UB_SGD_WIDE(1, GEN); break;         \
    case 2: if (SHORT) UB_SGD_SHORT(2, GEN); else UB_SGD_WIDE(2, GEN); break;         \
    case 3: UB_SGD_WIDE(3, GEN); break;                                               \
    case 4: UB_SGD_WIDE(4, GEN); break;                                               \
    default: sgd_epoch_anydim<GEN><<<grid, bt, 0, s>>>(UB_SGD_ARGS, L.lane_major); break; \
  }
  // The generic-metric rule keeps the large-graph budget at every size (its statistical
  // parity with the reference's sequential loop was established with it).
  if (p.generic_metric) {
    UB_SGD_DISPATCH(true, false)
  } else if (L.dram_epoch && (p.dim == 1 || p.dim == 2)) {
#define UB_SGD_DRAM(D)                                                                                       \
  if (L.lane_major) sgd_epoch_kernel2<D, false, NB_DRAM, MINB_DRAM, true><<<grid, bt, 0, s>>>(UB_SGD_ARGS); \
  else sgd_epoch_kernel2<D, false, NB_DRAM, MINB_DRAM, false><<<grid, bt, 0, s>>>(UB_SGD_ARGS)
    if (p.dim == 1) { UB_SGD_DRAM(1); } else { UB_SGD_DRAM(2); }
#undef UB_SGD_DRAM
  } else {
    UB_SGD_DISPATCH(false, L.short_epoch)
  }
#undef UB_SGD_DISPATCH
#undef UB_SGD_SHORT
#undef UB_SGD_WIDE
#undef UB_SGD_ARGS
  UB_LAUNCH_CHECK();
}

void schedule_totals(const SgdLayout& L, uint32_t neg_rate, uint32_t start, uint32_t end,
                     unsigned long long* d_fired, unsigned long long* d_negs, cudaStream_t s) {
  UB_CUDA(cudaMemsetAsync(d_fired, 0, 8, s));
  UB_CUDA(cudaMemsetAsync(d_negs, 0, 8, s));
  if (L.n_entries == 0 || end <= start) return;
  schedule_totals_kernel<<<grid_for(L.n_entries, 256), 256, 0, s>>>(L.entry.p, L.n_entries, neg_rate, start, end,
                                                                   d_fired, d_negs);
  UB_LAUNCH_CHECK();
}

void negative_draws(uint64_t seed, uint64_t first, uint64_t count, uint32_t epoch, uint32_t per, uint32_t lo,
                    uint32_t range, uint32_t* out, cudaStream_t s) {
  if (count == 0 || per == 0) return;
  negative_draws_kernel<<<grid_for(count, 256), 256, 0, s>>>(seed, first, count, epoch, per, lo, range, out);
  UB_LAUNCH_CHECK();
}

void negatives_per_firing(const uint32_t* qs, const uint32_t* ns, uint64_t count, uint32_t neg, uint32_t* out,
                          cudaStream_t s) {
  if (count == 0) return;
  negatives_per_firing_kernel<<<grid_for(count, 256), 256, 0, s>>>(qs, ns, count, neg, out);
  UB_LAUNCH_CHECK();
}

void nan_empty_rows(const uint64_t* indptr, uint64_t n, uint32_t dim, float* emb, cudaStream_t s) {
  if (n == 0) return;
  nan_rows_kernel<<<grid_for(n, 256), 256, 0, s>>>(indptr, n, dim, emb);
  UB_LAUNCH_CHECK();
}

}  // namespace ub
