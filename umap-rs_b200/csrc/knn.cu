// Exact k-nearest neighbours by brute force, the step before the fit path.  The reference
// takes kNN as input (umap-rs/src/lib.rs:41) and its example computes it by brute force
// (examples/src/bin/mnist_demo.rs:203-229): for every point the k others with the smallest
// Euclidean distance sqrt(sum_i (x_i - y_i)^2) (f32, summed in coordinate order), ordered by
// distance with ties in index order (a stable sort of the candidates 0..n), the point itself
// excluded; with fewer than k other points the missing slots stay zero.  This file returns
// exactly those arrays.
//
// Pipeline (one stream):
//  K-a  column means (f64 sums) and the largest centred magnitude, then per row: centred
//       values scaled by a power of two into the FP16 range and rounded to FP16 [n_pad, Dp]
//       (Dp = D rounded up to 64, zero padded), the squared norm of the rounded row, and the
//       f32 norm of the centred row (for the error bound).
//       From 16,384 points the rows are first put in locality order: each is assigned to the
//       nearest of 256 pivot rows (BF16 tensor-core GEMM) and the rows are sorted by pivot, so
//       a query block meets its neighbours in the first tiles it scans.
//  K-b  tensor-core candidate pass.  A CTA owns 128 query rows and streams database tiles of
//       256 rows: warp 0 issues TMA loads (128-byte swizzle, 3 stages of a 128 x 64 query chunk
//       and a 256 x 64 database chunk), warp 1 issues tcgen05.mma (M=128, N=256, K=16, FP16,
//       FP32 accumulation) into one of two 256-column tensor-memory accumulators, and warps
//       2-9 read the other accumulator with tcgen05.ld (thread = query row; warps 2-5 take
//       the first 128 columns of a tile, warps 6-9 the rest).  For a dot product
//       s with database row y the approximate squared distance is |q|^2 + |y|^2 - 2s; the
//       epilogue tests v = 2s - |y|^2 against the row's threshold |q|^2 - tau in registers and
//       only on a hit inserts into its half's list of the 32 smallest (a max-heap in shared
//       memory whose root is tau), so the common path costs two instructions per candidate;
//       the two halves' lists together are the row's C = 64 candidates.
//       The scan takes 16 tiles around the query block's own tile first, then the rest in the
//       order all CTAs share; the producer warp also bulk-copies each tile's row norms into a
//       ring of shared-memory slots.
//  K-c  exact rerank, a warp per row: the reference's f32 distance for each candidate (the
//       candidates' rows staged through shared memory 32 coordinates at a time, each lane
//       summing its candidate's coordinates in order), the k smallest (distance, index)
//       pairs, and a certificate: any point that never entered the list has an approximate
//       squared distance >= tau, hence a true distance >= a lower bound that accounts for the
//       FP16 rounding of both rows, the accumulation error and the rounding of the
//       reference's own formula; if the k-th distance found is below that bound no outside
//       point can enter the top k.
//  K-d  rows whose certificate fails are recomputed exactly against all points: CTAs over
//       (row, column range) keep the k smallest keys of their range, then a warp per row
//       merges the ranges.  For k > 32 (more than the candidate pass keeps) every row takes
//       this path.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "ub_internal.hpp"
#include "umma.cuh"

namespace ub {
namespace {

using namespace umma;

constexpr int QM = 128;      // query rows per CTA (UMMA M, tensor-memory lanes)
constexpr int DBN = 256;     // database rows per tile (UMMA N)
constexpr int KC = 64;       // K per staged chunk (128 bytes of bf16)
constexpr int TS = 3;        // pipeline stages
constexpr int NCAND = 64;    // candidates kept per row and database split
constexpr int HC = NCAND / 2;  // per epilogue warpgroup (each takes half of a tile's columns)
constexpr int KNN_THREADS = 320;
constexpr uint32_t Q_BYTES = QM * 128, D_BYTES = DBN * 128, STAGE = Q_BYTES + D_BYTES;
constexpr int NBS = 4;      // slots of the ring of per-tile row norms
constexpr size_t KNN_SMEM = (size_t)TS * STAGE + (size_t)NCAND * QM * 8 + (size_t)2 * 8 * QM * 4 + NBS * DBN * 4 + 1024;
static_assert(STAGE % 1024 == 0, "stages stay 1024-byte aligned");
constexpr float PAD_NORM = 3.0e38f;  // |y|^2 of padding rows: never a candidate
constexpr uint64_t KNN_REORDER_MIN = 16384;  // scan in locality order from this many points

__device__ __forceinline__ uint64_t dist_key(float dist, uint32_t idx) {
  // non-negative floats order like their bit patterns: (distance, index) order in one u64
  return ((uint64_t)__float_as_uint(dist) << 32) | idx;
}

// ---------------------------------------------------------------------------- K-a
__global__ void col_sums_kernel(const float* __restrict__ X, int64_t n, int d, double* __restrict__ sums,
                                unsigned* __restrict__ cmin, unsigned* __restrict__ cmax,
                                unsigned* __restrict__ bad) {
  __shared__ double part[8][33];
  __shared__ float lo[8][33], hi[8][33];
  const int col = blockIdx.x * 32 + threadIdx.x;
  double acc = 0.0;
  float mn = INFINITY, mx = -INFINITY;
  bool finite = true;
  if (col < d)
    for (int64_t r = (int64_t)blockIdx.y * 8 + threadIdx.y; r < n; r += (int64_t)gridDim.y * 8) {
      const float v = X[r * d + col];
      finite &= isfinite(v);
      acc += (double)v;
      mn = fminf(mn, v);
      mx = fmaxf(mx, v);
    }
  if (!finite) atomicOr(bad, 1u);
  part[threadIdx.y][threadIdx.x] = acc;
  lo[threadIdx.y][threadIdx.x] = mn;
  hi[threadIdx.y][threadIdx.x] = mx;
  __syncthreads();
  if (threadIdx.y == 0 && col < d) {
    for (int i = 1; i < 8; ++i) {
      acc += part[i][threadIdx.x];
      mn = fminf(mn, lo[i][threadIdx.x]);
      mx = fmaxf(mx, hi[i][threadIdx.x]);
    }
    atomicAdd(sums + col, acc);
    // order-preserving integer images of the floats for atomicMin / atomicMax
    const unsigned umn = __float_as_uint(mn), umx = __float_as_uint(mx);
    atomicMin(cmin + col, (umn & 0x80000000u) ? ~umn : (umn | 0x80000000u));
    atomicMax(cmax + col, (umx & 0x80000000u) ? ~umx : (umx | 0x80000000u));
  }
}

__device__ __forceinline__ float from_ordered(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Column means and the largest centred magnitude max_c max(max_c - mean_c, mean_c - min_c)
// (bit pattern of a non-negative float, atomicMax).
__global__ void col_means_kernel(const double* __restrict__ sums, const unsigned* __restrict__ cmin,
                                 const unsigned* __restrict__ cmax, int64_t n, int d, float* __restrict__ mean,
                                 unsigned* __restrict__ maxabs) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d) return;
  const float m = (float)(sums[c] / (double)n);
  mean[c] = m;
  const float a = fmaxf(fabsf(from_ordered(cmax[c]) - m), fabsf(m - from_ordered(cmin[c])));
  atomicMax(maxabs, __float_as_uint(a * (1.0f + 1e-6f)));
}

// One warp per output row r (source row src = perm ? perm[r] : r, rows >= n are padding):
// the centred row times `scale` rounded to FP16 (xh) and its squared norm (nb, scaled units),
// the same values rounded to BF16 (xb, for the pivot assignment), and the f32 norm of the
// centred row (rn, true units, rounded up slightly).  Null outputs are skipped.
__global__ void knn_prep_kernel(const float* __restrict__ X, int64_t n, int d, int dp, int64_t n_pad,
                                const float* __restrict__ mean, float scale, const uint32_t* __restrict__ perm,
                                __half* __restrict__ xh, float* __restrict__ nb, __nv_bfloat16* __restrict__ xb,
                                float* __restrict__ rn, unsigned* __restrict__ rmax_bits) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = w0; r < n_pad; r += nw) {
    const int64_t src = (r < n && perm) ? (int64_t)perm[r] : r;
    float s2 = 0.0f, sb = 0.0f;
    for (int c = lane; c < dp; c += 32) {
      float xc = 0.0f;
      if (r < n && c < d) xc = X[src * d + c] - mean[c];
      const __half h = __float2half_rn(xc * scale);
      const float hf = __half2float(h);
      if (xh) xh[r * dp + c] = h;
      if (xb) xb[r * dp + c] = __float2bfloat16_rn(xc * scale);
      s2 += xc * xc;
      sb += hf * hf;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o);
      sb += __shfl_xor_sync(0xFFFFFFFFu, sb, o);
    }
    if (lane == 0) {
      if (nb) nb[r] = r < n ? sb : PAD_NORM;
      if (rn) {
        const float norm = r < n ? sqrtf(s2) * (1.0f + 1e-5f) : 0.0f;
        rn[r] = norm;
        atomicMax(rmax_bits, __float_as_uint(norm));
      }
    }
  }
}

// Locality order for the scan.  Pivot p is row p * n / P; its BF16 row and squared norm.
constexpr int NPIV = 256;
__global__ void gather_pivots_kernel(const __nv_bfloat16* __restrict__ xb, int64_t n, int dp,
                                     __nv_bfloat16* __restrict__ piv, float* __restrict__ pn) {
  const int p = blockIdx.x;
  const int64_t src = (int64_t)p * n / NPIV;
  float s = 0.0f;
  for (int c = threadIdx.x; c < dp; c += blockDim.x) {
    const __nv_bfloat16 v = xb[src * dp + c];
    piv[(int64_t)p * dp + c] = v;
    const float f = __bfloat162float(v);
    s += f * f;
  }
  __shared__ float red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    pn[p] = s;
  }
}

// A warp per row of a chunk of x . p^T [rows, NPIV]: key = the nearest pivot (|p|^2 - 2 x.p).
__global__ void nearest_pivot_kernel(const float* __restrict__ dots, int64_t rows, int64_t row0, int64_t n,
                                     const float* __restrict__ pn, uint32_t* __restrict__ key) {
  const int lane = threadIdx.x & 31;
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (r >= rows || row0 + r >= n) return;
  float best = INFINITY;
  uint32_t arg = 0;
  for (int p = lane; p < NPIV; p += 32) {
    const float v = pn[p] - 2.0f * dots[r * NPIV + p];
    if (v < best) {
      best = v;
      arg = (uint32_t)p;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
    const uint32_t oa = __shfl_xor_sync(0xFFFFFFFFu, arg, o);
    if (ob < best || (ob == best && oa < arg)) {
      best = ob;
      arg = oa;
    }
  }
  if (lane == 0) key[row0 + r] = arg;
}

// tcgen05.ld of 32 consecutive accumulator columns of this warp's 32 lanes (thread = lane).
__device__ __forceinline__ void tmem_ld32(uint32_t (&r)[32], uint32_t taddr) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
// Waits for the outstanding tensor-memory loads; the registers are in-out operands so that no
// use of them is scheduled before the wait.
__device__ __forceinline__ void tmem_wait32(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// ---------------------------------------------------------------------------- K-b
__global__ void __launch_bounds__(KNN_THREADS, 1) knn_candidates_kernel(
    const __grid_constant__ CUtensorMap tq, const __grid_constant__ CUtensorMap tdb, const float* __restrict__ nb,
    int64_t n, int n_kchunks, int64_t tiles_total, const uint32_t* __restrict__ perm, uint32_t* __restrict__ cand_idx,
    float* __restrict__ tau_out, unsigned* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full[TS], empty[TS], tfull[2], tempty[2], nfull[NBS], nempty[NBS];
  __shared__ uint32_t tmem_base;
  __shared__ volatile int s_fail;
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  float* cd = reinterpret_cast<float*>(smem + TS * STAGE);  // [2][HC][QM] heaps of the two halves
  uint32_t* ci = reinterpret_cast<uint32_t*>(cd + NCAND * QM);
  float* vst = reinterpret_cast<float*>(ci + NCAND * QM);  // [2][8][QM]
  float* nbuf = vst + 2 * 8 * QM;                          // [NBS][DBN] norms of the tile's rows
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * QM;
  const int split = blockIdx.y, n_splits = gridDim.y;
  const int64_t t_begin = tiles_total * split / n_splits, t_end = tiles_total * (split + 1) / n_splits;
  const int T = (int)(t_end - t_begin);
  // Scan order: first a window of WIN tiles around the query block's own tile (rows in
  // locality order: its nearest neighbours come first and the candidate threshold tightens
  // early), then the rest of the range in increasing order, which all CTAs share, so the
  // CTAs resident together read the same tiles and the database streams through L2 once
  // per wave.
  constexpr int64_t WIN = 16;
  int64_t own = m0 / DBN - WIN / 2;
  own = own < t_begin ? t_begin : own;
  own = own > t_end - WIN ? t_end - WIN : own;
  const int64_t w0 = T > WIN ? own : t_begin;
  const int64_t wn = T > WIN ? WIN : 0;
  auto tile_of = [&](int t) -> int64_t {
    if (t < wn) return w0 + t;
    const int64_t u = t_begin + (t - wn);
    return u < w0 ? u : u + wn;
  };
  const int G = T * n_kchunks;

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base)), "r"(2 * DBN) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < TS; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&full[i])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&empty[i])), "r"(1) : "memory");
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&tfull[i])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&tempty[i])), "r"(2 * QM) : "memory");
    }
    for (int i = 0; i < NBS; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&nfull[i])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&nempty[i])), "r"(2 * QM) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = tmem_base;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int g = 0, n_issued = 0;
      for (; g < G; ++g) {
        const int st = g % TS;
        if (g >= TS && !mbar_wait(smem_u32(&empty[st]), (uint32_t)(((g / TS) - 1) & 1))) {
          s_fail = 1;
          break;
        }
        if (s_fail) break;
        const int t = g / n_kchunks, c = g % n_kchunks;
        if (c == 0) {
          // the tile's row norms go to slot t % NBS once the epilogue is done with tile t - NBS
          const int slot = t % NBS;
          if (t >= NBS && !mbar_wait(smem_u32(&nempty[slot]), (uint32_t)(((t / NBS) - 1) & 1))) {
            s_fail = 1;
            break;
          }
          const uint32_t nfb = smem_u32(&nfull[slot]);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(nfb), "r"(DBN * 4) : "memory");
          asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                       :: "r"(smem_u32(nbuf + slot * DBN)), "l"(nb + tile_of(t) * DBN), "r"(DBN * 4), "r"(nfb)
                       : "memory");
          n_issued = t + 1;
        }
        const uint32_t q_dst = smem_u32(smem + st * STAGE), d_dst = q_dst + Q_BYTES;
        const uint32_t fb = smem_u32(&full[st]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(fb), "r"(STAGE) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
            :: "r"(q_dst), "l"(reinterpret_cast<uint64_t>(&tq)), "r"(c * KC), "r"((int)m0), "r"(fb) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
            :: "r"(d_dst), "l"(reinterpret_cast<uint64_t>(&tdb)), "r"(c * KC), "r"((int)(tile_of(t) * DBN)),
               "r"(fb) : "memory");
      }
      // the copies of the last stages and norm buffers must have landed before the CTA may exit
      for (int h = g > TS ? g - TS : 0; h < g; ++h) (void)mbar_wait(smem_u32(&full[h % TS]), (uint32_t)((h / TS) & 1));
      for (int t = n_issued > NBS ? n_issued - NBS : 0; t < n_issued; ++t)
        (void)mbar_wait(smem_u32(&nfull[t % NBS]), (uint32_t)((t / NBS) & 1));
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = instr_desc_f16(QM, DBN);
      int g = 0;
      bool ok = true;
      for (int t = 0; t < T && ok; ++t) {
        const int buf = t & 1;
        if (t >= 2 && !mbar_wait(smem_u32(&tempty[buf]), (uint32_t)(((t >> 1) - 1) & 1))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t dacc = tbase + (uint32_t)(buf * DBN);
        for (int c = 0; c < n_kchunks; ++c) {
          const int st = g % TS;
          if (s_fail || !mbar_wait(smem_u32(&full[st]), (uint32_t)((g / TS) & 1))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(smem + st * STAGE), b0 = a0 + Q_BYTES;
#pragma unroll
          for (int k = 0; k < KC / 16; ++k) {
            const uint64_t ad = smem_desc_sw128(a0 + k * 32), bd = smem_desc_sw128(b0 + k * 32);
            const uint32_t acc = (c > 0 || k > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                :: "r"(dacc), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                : "memory");
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                       :: "r"(smem_u32(&empty[st])) : "memory");
          ++g;
        }
        if (!ok) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_u32(&tfull[buf])) : "memory");
      }
      if (!ok) s_fail = 1;
      // the last MMAs must have completed before tensor memory is freed
      if (g > 0) (void)mbar_wait(smem_u32(&empty[(g - 1) % TS]), (uint32_t)(((g - 1) / TS) & 1));
    }
  } else {
    // epilogue: warps 2..9; warp w owns tensor-memory lane quarter w % 4 (query rows) and half
    // (w - 2) / 4 of each tile's columns, with its own heap of HC candidates per row
    const int q = warp & 3, half = (warp - 2) >> 2;
    const int trow = q * 32 + lane;
    const int64_t row = m0 + trow;
    const bool live = row < n;
    const float nq = live ? nb[row] : 0.0f;
    float* hd = cd + half * HC * QM;
    uint32_t* hi = ci + half * HC * QM;
    float* vs = vst + half * 8 * QM;
    for (int s = 0; s < HC; ++s) {
      hd[s * QM + trow] = INFINITY;
      hi[s * QM + trow] = 0xFFFFFFFFu;
    }
    float tau = INFINITY, thr_h = live ? -INFINITY : INFINITY;  // (|q|^2 - tau) / 2
    // 32 columns of the accumulator: v = 2 s - |y|^2; a column enters the heap when
    // |q|^2 - v < tau, i.e. v > thr.  The common case costs the FMAs and a running max.
    auto process = [&](const uint32_t (&r)[32], const float* nrm, int64_t c0) {
      // u = s - |y|^2 / 2 = v / 2 exactly (halving commutes with rounding), two columns per
      // packed FMA; u > thr / 2 is the same test as v > thr
      float v[32];
      float vmax = -INFINITY;
      const uint64_t mhalf = 0xBF000000BF000000ull;  // (-0.5f, -0.5f)
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float4 w = reinterpret_cast<const float4*>(nrm)[i];
        uint64_t s0, s1, n0, n1, d0, d1;
        asm("mov.b64 %0, {%1, %2};" : "=l"(s0) : "r"(r[4 * i + 0]), "r"(r[4 * i + 1]));
        asm("mov.b64 %0, {%1, %2};" : "=l"(s1) : "r"(r[4 * i + 2]), "r"(r[4 * i + 3]));
        asm("mov.b64 %0, {%1, %2};" : "=l"(n0) : "r"(__float_as_uint(w.x)), "r"(__float_as_uint(w.y)));
        asm("mov.b64 %0, {%1, %2};" : "=l"(n1) : "r"(__float_as_uint(w.z)), "r"(__float_as_uint(w.w)));
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d0) : "l"(n0), "l"(mhalf), "l"(s0));
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d1) : "l"(n1), "l"(mhalf), "l"(s1));
        uint32_t a0, a1, a2, a3;
        asm("mov.b64 {%0, %1}, %2;" : "=r"(a0), "=r"(a1) : "l"(d0));
        asm("mov.b64 {%0, %1}, %2;" : "=r"(a2), "=r"(a3) : "l"(d1));
        v[4 * i + 0] = __uint_as_float(a0);
        v[4 * i + 1] = __uint_as_float(a1);
        v[4 * i + 2] = __uint_as_float(a2);
        v[4 * i + 3] = __uint_as_float(a3);
        vmax = fmaxf(vmax, fmaxf(fmaxf(v[4 * i], v[4 * i + 1]), fmaxf(v[4 * i + 2], v[4 * i + 3])));
      }
      if (!(vmax > thr_h)) return;
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        // stage 8 values (dynamic index below) and mark those above the threshold
        uint32_t hits = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          vs[i * QM + trow] = v[8 * h + i];
          hits |= (v[8 * h + i] > thr_h ? 1u : 0u) << i;
        }
        while (hits) {
          const int i = __ffs(hits) - 1;
          hits &= hits - 1;
          const int64_t col = c0 + 8 * h + i;
          const float a = nq - 2.0f * vs[i * QM + trow];
          if (!(a < tau) || col >= n || col == row) continue;
          // max-heap on the approximate distance: replace the root, sift down
          int pos = 0;
          for (;;) {
            const int l = 2 * pos + 1;
            if (l >= HC) break;
            const float dl = hd[l * QM + trow];
            const float dr = l + 1 < HC ? hd[(l + 1) * QM + trow] : -INFINITY;
            const int c = dr > dl ? l + 1 : l;
            const float dc = dr > dl ? dr : dl;
            if (!(dc > a)) break;
            hd[pos * QM + trow] = dc;
            hi[pos * QM + trow] = hi[c * QM + trow];
            pos = c;
          }
          hd[pos * QM + trow] = a;
          hi[pos * QM + trow] = (uint32_t)col;
          tau = hd[trow];
          thr_h = 0.5f * (nq - tau);
        }
      }
    };
    constexpr int CH = DBN / 64;  // 32-column chunks per half tile
    for (int t = 0; t < T; ++t) {
      const int buf = t & 1;
      const int slot = t % NBS;
      if (!mbar_wait(smem_u32(&tfull[buf]), (uint32_t)((t >> 1) & 1)) ||
          !mbar_wait(smem_u32(&nfull[slot]), (uint32_t)((t / NBS) & 1))) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int64_t cb0 = tile_of(t) * DBN + half * (DBN / 2);
      const float* nrm = nbuf + slot * DBN + half * (DBN / 2);
      const uint32_t ta = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * DBN + half * (DBN / 2));
      // tensor-memory loads run one 32-column chunk ahead of the arithmetic
      uint32_t ra[32], rb[32];
      tmem_ld32(ra, ta);
      tmem_wait32(ra);
#pragma unroll 1
      for (int jj = 0; jj < CH; jj += 2) {
        tmem_ld32(rb, ta + (uint32_t)(jj + 1) * 32);
        process(ra, nrm + jj * 32, cb0 + jj * 32);
        __syncwarp();
        tmem_wait32(rb);
        if (jj + 2 < CH) tmem_ld32(ra, ta + (uint32_t)(jj + 2) * 32);
        process(rb, nrm + (jj + 1) * 32, cb0 + (jj + 1) * 32);
        __syncwarp();
        if (jj + 2 < CH) tmem_wait32(ra);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(&tempty[buf])) : "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(&nempty[slot])) : "memory");
      if (s_fail) break;
    }
    if (live && !s_fail) {  // outputs by original row index, candidates as original indices
      const int64_t orow = perm ? (int64_t)perm[row] : row;
      const int64_t base = (orow * n_splits + split) * NCAND + half * HC;
      for (int s = 0; s < HC; ++s) {
        const uint32_t c = hi[s * QM + trow];
        cand_idx[base + s] = (perm && c < (uint64_t)n) ? perm[c] : c;
      }
      tau_out[(orow * n_splits + split) * 2 + half] = tau;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && s_fail) atomicOr(err, 1u);
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tbase), "r"(2 * DBN) : "memory");
}

// ---------------------------------------------------------------------------- K-c
// Lower bound on the reference's distance from row x to any point y whose approximate squared
// distance (scaled units) is >= tau.  With x~, y~ the centred rows (|y~| <= R), x^, y^ their
// FP16 roundings after scaling by `scale` (a power of two):
//   |approx - |x^ - y^|^2| <= gamma (|x^| + |y^|)^2        (FP32 accumulation of the products
//                                                          and of the norms; generous)
//   | |x^ - y^| / scale - |x - y| | <= 2^-11 (1 + 2^-10) (|x~| + |y~|) + 2 sqrt(Dp) 2^-25 / scale
//                                                          (rounding to FP16 incl. subnormals,
//                                                          and the centring)
//   ref(x, y) >= |x - y| (1 - (D + 8) 2^-23)               (the reference's own f32 formula)
__device__ __forceinline__ float distance_lower_bound(float tau, float xr, float R, float gamma, float scale,
                                                      int d, int dp) {
  const float inv = 1.0f / scale;
  const float s = 1.001f * (xr + R);
  const float e1 = gamma * s * s;
  const float lb = sqrtf(fmaxf(0.0f, tau * inv * inv - e1)) - 0.00048876f * (xr + R) -
                   2.0f * sqrtf((float)dp) * 2.9802322e-8f * inv;
  return lb * (1.0f - (float)(d + 8) * 1.1920929e-7f) * (1.0f - 1e-6f);
}

// The reference's distances from row x to 32 rows (one per lane): the warp stages the 32 rows
// 32 coordinates at a time in shared memory (coalesced 128-byte reads) and each lane sums its
// row's squared differences in coordinate order.  Rows >= n give +inf.
__device__ __forceinline__ float ref_distance_warp(const float* __restrict__ X, int64_t n, int d, int64_t row,
                                                   uint32_t mine, float (*tile)[33], int lane) {
  float acc = 0.0f;
  for (int i0 = 0; i0 < d; i0 += 32) {
    const int i = i0 + lane;
    for (int j = 0; j < 32; ++j) {
      const uint32_t c = __shfl_sync(0xFFFFFFFFu, mine, j);
      tile[j][lane] = (c < (uint64_t)n && i < d) ? __ldg(X + (int64_t)c * d + i) : 0.0f;
    }
    tile[32][lane] = i < d ? __ldg(X + row * d + i) : 0.0f;
    __syncwarp();
    const int m = min(32, d - i0);
    for (int t = 0; t < m; ++t) {
      const float df = __fsub_rn(tile[32][t], tile[lane][t]);
      acc = __fadd_rn(acc, __fmul_rn(df, df));
    }
    __syncwarp();
  }
  return mine < (uint64_t)n ? __fsqrt_rn(acc) : INFINITY;
}

template <int E>  // candidates per lane = splits * NCAND / 32
__global__ void __launch_bounds__(256) knn_rerank_kernel(
    const float* __restrict__ X, int64_t n, int d, int dp, int k, const uint32_t* __restrict__ cand_idx,
    const float* __restrict__ tau_in, const float* __restrict__ rn, const unsigned* __restrict__ rmax_bits,
    float gamma, float scale, const uint32_t* __restrict__ order, uint32_t* __restrict__ out_idx,
    float* __restrict__ out_d, uint32_t* __restrict__ fail_rows, unsigned* __restrict__ fail_count) {
  constexpr int S = E * 32 / NCAND;
  __shared__ float tiles[8][33][33];
  const int lane = threadIdx.x & 31;
  float (*tile)[33] = tiles[threadIdx.x >> 5];
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w = w0; w < n; w += nw) {
    // rows in locality order when there is one: neighbouring warps share candidate rows in L2
    const int64_t row = order ? (int64_t)order[w] : w;
    uint64_t keys[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const uint32_t c = cand_idx[row * (S * NCAND) + e * 32 + lane];
      const float dist = ref_distance_warp(X, n, d, row, c, tile, lane);
      keys[e] = c >= (uint64_t)n ? ~0ull : dist_key(dist, c);
    }
    uint64_t last = ~0ull;
    for (int p = 0; p < k; ++p) {
      uint64_t mn = ~0ull;
#pragma unroll
      for (int e = 0; e < E; ++e) mn = keys[e] < mn ? keys[e] : mn;
      uint64_t wm = mn;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, wm, o);
        wm = other < wm ? other : wm;
      }
      if (wm != ~0ull && mn == wm) {  // keys are distinct (distinct indices): one lane owns it
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (keys[e] == wm) keys[e] = ~0ull;
      }
      if (lane == 0) {
        out_idx[row * k + p] = wm == ~0ull ? 0u : (uint32_t)wm;
        out_d[row * k + p] = wm == ~0ull ? 0.0f : __uint_as_float((uint32_t)(wm >> 32));
      }
      last = wm;
    }
    if (lane == 0 && last != ~0ull) {
      float tau = INFINITY;
      for (int s = 0; s < 2 * S; ++s) tau = fminf(tau, tau_in[row * 2 * S + s]);  // (split, half)
      if (tau < INFINITY) {
        const float lb = distance_lower_bound(tau, rn[row], __uint_as_float(*rmax_bits), gamma, scale, d, dp);
        if (!(__uint_as_float((uint32_t)(last >> 32)) < lb)) fail_rows[atomicAdd(fail_count, 1u)] = (uint32_t)row;
      }
    }
  }
}

// ---------------------------------------------------------------------------- K-d
// Exact brute force for the listed rows.  CTA (b, s) takes row rows[b] against the columns of
// range s: tiles of 256 columns are staged 32 coordinates at a time in shared memory
// (coalesced), each thread sums its column's squared differences in coordinate order and
// keeps its k smallest (distance, index) keys; k rounds of a block-wide minimum leave the
// range's k smallest keys in part[b][s][0..k).
// TH threads per CTA: 256 for k <= 32, 128 for the longer lists of k <= 128.
template <int TH>
__global__ void __launch_bounds__(TH) knn_exact_part_kernel(const float* __restrict__ X, int64_t n, int d, int k,
                                                            const uint32_t* __restrict__ rows, unsigned n_rows,
                                                            int n_ranges, uint64_t* __restrict__ part) {
  constexpr int EX_THREADS = TH, NW = TH / 32;
  extern __shared__ uint64_t lst[];  // [k][EX_THREADS]
  __shared__ float xt[32][EX_THREADS + 1];
  __shared__ float xs[32];
  __shared__ uint64_t red[EX_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int s = blockIdx.y;
  const int64_t j_begin = n * s / n_ranges, j_end = n * (s + 1) / n_ranges;
  for (unsigned b = blockIdx.x; b < n_rows; b += gridDim.x) {
    const int64_t row = rows[b];
    for (int t = 0; t < k; ++t) lst[t * EX_THREADS + tid] = ~0ull;
    uint64_t mx = ~0ull;
    int ms = 0;
    for (int64_t j0 = j_begin; j0 < j_end; j0 += EX_THREADS) {
      const int64_t j = j0 + tid;
      float acc = 0.0f;
      for (int i0 = 0; i0 < d; i0 += 32) {
        __syncthreads();
        // 256 columns x 32 coordinates: warp w loads rows j0 + 32 w' .. as 128-byte pieces
        float ld[32];  // this warp's 32 rows: all loads in flight before the stores
#pragma unroll
        for (int u = 0; u < 32; ++u) {
          const int64_t jj = j0 + warp + NW * u;
          ld[u] = (jj < j_end && i0 + lane < d) ? __ldg(X + jj * d + i0 + lane) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 32; ++u) xt[lane][warp + NW * u] = ld[u];
        if (tid < 32) xs[tid] = i0 + tid < d ? __ldg(X + row * d + i0 + tid) : 0.0f;
        __syncthreads();
        const int m = min(32, d - i0);
        for (int t = 0; t < m; ++t) {
          const float df = __fsub_rn(xs[t], xt[t][tid]);
          acc = __fadd_rn(acc, __fmul_rn(df, df));
        }
      }
      if (j < j_end && j != row) {
        const uint64_t key = dist_key(__fsqrt_rn(acc), (uint32_t)j);
        if (key < mx) {
          lst[ms * EX_THREADS + tid] = key;
          mx = lst[tid];
          ms = 0;
          for (int t = 1; t < k; ++t) {
            const uint64_t e = lst[t * EX_THREADS + tid];
            if (e > mx) {
              mx = e;
              ms = t;
            }
          }
        }
      }
    }
    __syncthreads();
    for (int p = 0; p < k; ++p) {
      uint64_t mn = ~0ull;
      int sm = 0;
      for (int t = 0; t < k; ++t) {
        const uint64_t e = lst[t * EX_THREADS + tid];
        if (e < mn) {
          mn = e;
          sm = t;
        }
      }
      uint64_t wm = mn;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, wm, o);
        wm = other < wm ? other : wm;
      }
      if (lane == 0) red[warp] = wm;
      __syncthreads();
      uint64_t bm = red[0];
      for (int w = 1; w < EX_THREADS / 32; ++w) bm = red[w] < bm ? red[w] : bm;
      if (bm != ~0ull && mn == bm) lst[sm * EX_THREADS + tid] = ~0ull;
      if (tid == 0) part[((int64_t)b * n_ranges + s) * k + p] = bm;
      __syncthreads();
    }
  }
}

// A warp per listed row: the k smallest of its ranges' keys -> the output row.
__global__ void knn_exact_merge_kernel(const uint64_t* __restrict__ part, const uint32_t* __restrict__ rows,
                                       unsigned n_rows, int n_ranges, int k, uint32_t* __restrict__ out_idx,
                                       float* __restrict__ out_d) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_rows) return;
  const uint64_t* p = part + w * (int64_t)n_ranges * k;
  const int m = n_ranges * k;
  const int64_t row = rows[w];
  uint64_t prev = 0;
  bool first = true;
  for (int q = 0; q < k; ++q) {
    // smallest key above the previous one (keys are distinct)
    uint64_t mn = ~0ull;
    for (int t = lane; t < m; t += 32) {
      const uint64_t e = p[t];
      if ((first || e > prev) && e < mn) mn = e;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, mn, o);
      mn = other < mn ? other : mn;
    }
    if (lane == 0) {
      out_idx[row * k + q] = mn == ~0ull ? 0u : (uint32_t)mn;
      out_d[row * k + q] = mn == ~0ull ? 0.0f : __uint_as_float((uint32_t)(mn >> 32));
    }
    prev = mn;
    first = false;
    if (mn == ~0ull) {
      for (int r = q + 1 + lane; r < k; r += 32) {
        out_idx[row * k + r] = 0u;
        out_d[row * k + r] = 0.0f;
      }
      break;
    }
  }
}

inline unsigned blocks_for(int64_t n, unsigned bt) { return (unsigned)std::min<int64_t>((n + bt - 1) / bt, 1 << 20); }

__global__ void iota_kernel(uint32_t* __restrict__ v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

// K-d for the listed rows: enough CTAs to fill the GPU (each row's columns split into ranges
// of >= 1024), then the merge.  Synchronises `s`.
void exact_rows(const float* X, int64_t n, int d, int k, const uint32_t* rows, unsigned n_rows, uint32_t* out_idx,
                float* out_dist, cudaStream_t s) {
  const int64_t want = std::max<int64_t>(1, (4 * 148 + (int64_t)n_rows - 1) / (int64_t)n_rows);
  const int ranges = (int)std::max<int64_t>(1, std::min<int64_t>({want, n / 1024 + 1, 256}));
  const unsigned gx = std::min<unsigned>(n_rows, 65535u);
  DevBuf<uint64_t> part((uint64_t)n_rows * ranges * k, s);
  if (k <= KNN_MAX_K)
    knn_exact_part_kernel<256><<<dim3(gx, (unsigned)ranges), 256, (size_t)k * 256 * 8, s>>>(X, n, d, k, rows, n_rows,
                                                                                            ranges, part.p);
  else
    knn_exact_part_kernel<128><<<dim3(gx, (unsigned)ranges), 128, (size_t)k * 128 * 8, s>>>(X, n, d, k, rows, n_rows,
                                                                                            ranges, part.p);
  UB_LAUNCH_CHECK();
  knn_exact_merge_kernel<<<blocks_for((int64_t)n_rows * 32, 256), 256, 0, s>>>(part.p, rows, n_rows, ranges, k,
                                                                               out_idx, out_dist);
  UB_LAUNCH_CHECK();
  UB_CUDA(cudaStreamSynchronize(s));
}

template <int E>
void launch_rerank(const float* X, int64_t n, int d, int dp, int k, const uint32_t* ci, const float* tau,
                   const float* rn, const unsigned* rmax, float gamma, float scale, const uint32_t* order,
                   uint32_t* oi, float* od, uint32_t* fr, unsigned* fc, cudaStream_t s) {
  knn_rerank_kernel<E><<<blocks_for(n * 32, 256), 256, 0, s>>>(X, n, d, dp, k, ci, tau, rn, rmax, gamma, scale,
                                                               order, oi, od, fr, fc);
  UB_LAUNCH_CHECK();
}

}  // namespace

KnnStats knn_bruteforce(const float* X, uint64_t n, uint64_t d, uint64_t k, uint32_t* out_idx, float* out_dist,
                        cudaStream_t s) {
  KnnStats st{};
  if (k < 1 || k > (uint64_t)KNN_MAX_K_EXACT)
    throw Error(INVALID_ARGUMENT, "k must be in 1.." + std::to_string(KNN_MAX_K_EXACT) + ", got " + std::to_string(k));
  if (d < 1 || d > 65536) throw Error(INVALID_ARGUMENT, "dimension must be in 1..65536");
  if (n >= 0x7FFFFF00ull) throw Error(UNSUPPORTED, "n must be < 2^31 - 256");
  if (n == 0) return st;
  if (n == 1) {
    UB_CUDA(cudaMemsetAsync(out_idx, 0, k * 4, s));
    UB_CUDA(cudaMemsetAsync(out_dist, 0, k * 4, s));
    UB_CUDA(cudaStreamSynchronize(s));
    return st;
  }
  {
    // kernel attributes belong to the device's context: set them once per device
    static std::mutex mu;
    static uint64_t done = 0;  // bit per device id < 64
    int dev = 0;
    UB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 64 || !((done >> dev) & 1u)) {
      UB_CUDA(cudaFuncSetAttribute(knn_candidates_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KNN_SMEM));
      UB_CUDA(cudaFuncSetAttribute(knn_exact_part_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(KNN_MAX_K * 256 * 8)));
      UB_CUDA(cudaFuncSetAttribute(knn_exact_part_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(KNN_MAX_K_EXACT * 128 * 8)));
      if (dev < 64) done |= 1ull << dev;
    }
  }
  const int di = (int)d;
  const int64_t dp = (int64_t)((d + KC - 1) / KC) * KC;
  const int64_t n_pad = (int64_t)((n + DBN - 1) / DBN) * DBN;
  const int64_t q_blocks = n_pad / QM, tiles = n_pad / DBN;
  int S = 1;
  while (S < 8 && q_blocks * S < 148 && tiles / (2 * S) >= 2) S *= 2;
  st.splits = (uint32_t)S;

  DevBuf<double> sums(d, s);
  DevBuf<float> mean(d, s);
  DevBuf<unsigned> flags(5, s);  // 0 non-finite input, 1 max norm, 2 kernel error, 3 failed rows, 4 max |x~|
  UB_CUDA(cudaMemsetAsync(sums.p, 0, d * 8, s));
  UB_CUDA(cudaMemsetAsync(flags.p, 0, 20, s));
  {
    const unsigned gy = (unsigned)std::min<int64_t>(1024, std::max<int64_t>(1, (int64_t)n / 256));
    DevBuf<unsigned> cmm(2 * d, s);
    UB_CUDA(cudaMemsetAsync(cmm.p, 0xFF, d * 4, s));  // min of ordered images starts at the top
    UB_CUDA(cudaMemsetAsync(cmm.p + d, 0, d * 4, s));
    col_sums_kernel<<<dim3((unsigned)((d + 31) / 32), gy), dim3(32, 8), 0, s>>>(X, (int64_t)n, di, sums.p, cmm.p,
                                                                               cmm.p + d, flags.p);
    UB_LAUNCH_CHECK();
    col_means_kernel<<<(unsigned)((d + 255) / 256), 256, 0, s>>>(sums.p, cmm.p, cmm.p + d, (int64_t)n, di, mean.p,
                                                                 flags.p + 4);
    UB_LAUNCH_CHECK();
  }
  unsigned pre[5] = {0, 0, 0, 0, 0};
  UB_CUDA(cudaMemcpyAsync(pre, flags.p, 20, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  if (pre[0]) throw Error(INVALID_ARGUMENT, "kNN input contains NaN or infinite values");
  if (k > (uint64_t)KNN_MAX_K) {
    // lists longer than the candidate pass keeps: every row on the exact CUDA-core path
    DevBuf<uint32_t> all(n, s);
    iota_kernel<<<blocks_for((int64_t)n, 256), 256, 0, s>>>(all.p, (int64_t)n);
    UB_LAUNCH_CHECK();
    exact_rows(X, (int64_t)n, (int)d, (int)k, all.p, (unsigned)n, out_idx, out_dist, s);
    st.fallback_rows = (uint32_t)n;
    st.all_exact = 1;
    return st;
  }
  // scale = 2^e with max |x~| * scale <= 2^14, so every scaled value is finite in FP16
  float maxabs;
  std::memcpy(&maxabs, &pre[4], 4);
  float scale = 1.0f;
  if (maxabs > 0.0f) {
    int e = 0;
    std::frexp(16384.0f / maxabs, &e);
    scale = std::ldexp(1.0f, std::max(-120, std::min(120, e - 1)));
  }
  st.scale = scale;

  DevBuf<__half> xh((uint64_t)(n_pad * dp), s);
  DevBuf<float> nb(n_pad, s), rn(n_pad, s);
  DevBuf<uint32_t> perm;
  const unsigned prep_grid = blocks_for(n_pad * 32, 256);
  if (n >= KNN_REORDER_MIN) {
    // locality order: nearest of NPIV pivot rows (tensor-core GEMM in row chunks), rows
    // sorted by pivot (stable) -> perm[r] = the original row at position r
    DevBuf<__nv_bfloat16> xb((uint64_t)(n_pad * dp), s), piv((uint64_t)NPIV * dp, s);
    DevBuf<float> pn(NPIV, s);
    knn_prep_kernel<<<prep_grid, 256, 0, s>>>(X, (int64_t)n, di, (int)dp, n_pad, mean.p, scale, nullptr, nullptr,
                                              nullptr, xb.p, rn.p, flags.p + 1);
    UB_LAUNCH_CHECK();
    gather_pivots_kernel<<<NPIV, 128, 0, s>>>(xb.p, (int64_t)n, (int)dp, piv.p, pn.p);
    UB_LAUNCH_CHECK();
    constexpr int64_t CH = 65536;
    DevBuf<float> dots((uint64_t)CH * NPIV, s);
    DevBuf<uint32_t> key(n, s), key_sorted(n, s);
    for (int64_t r0 = 0; r0 < (int64_t)n; r0 += CH) {
      const int64_t rows = std::min<int64_t>(CH, n_pad - r0);
      umma_gemm_f32(xb.p + r0 * dp, piv.p, dots.p, rows, NPIV, dp, 1, s);
      nearest_pivot_kernel<<<blocks_for(rows * 32, 256), 256, 0, s>>>(dots.p, rows, r0, (int64_t)n, pn.p, key.p);
      UB_LAUNCH_CHECK();
    }
    perm.alloc(n, s);
    radix_sort_pairs(key.p, nullptr, key_sorted.p, perm.p, n, 8, s);
    knn_prep_kernel<<<prep_grid, 256, 0, s>>>(X, (int64_t)n, di, (int)dp, n_pad, mean.p, scale, perm.p, xh.p, nb.p,
                                              nullptr, nullptr, nullptr);
    UB_LAUNCH_CHECK();
    st.reordered = 1;
  } else {
    knn_prep_kernel<<<prep_grid, 256, 0, s>>>(X, (int64_t)n, di, (int)dp, n_pad, mean.p, scale, nullptr, xh.p, nb.p,
                                              nullptr, rn.p, flags.p + 1);
    UB_LAUNCH_CHECK();
  }

  DevBuf<uint32_t> cidx(n * S * NCAND, s);
  DevBuf<float> tau(n * S * 2, s);
  const CUtensorMap tq = bf16_tile_map(xh.p, n_pad, dp, dp, QM, true);
  const CUtensorMap tdb = bf16_tile_map(xh.p, n_pad, dp, dp, DBN, true);
  cudaEvent_t ev[2];
  UB_CUDA(cudaEventCreate(&ev[0]));
  UB_CUDA(cudaEventCreate(&ev[1]));
  UB_CUDA(cudaEventRecord(ev[0], s));
  knn_candidates_kernel<<<dim3((unsigned)q_blocks, (unsigned)S), KNN_THREADS, KNN_SMEM, s>>>(
      tq, tdb, nb.p, (int64_t)n, (int)(dp / KC), tiles, perm.p, cidx.p, tau.p, flags.p + 2);
  UB_LAUNCH_CHECK();
  UB_CUDA(cudaEventRecord(ev[1], s));
  unsigned kerr = 0;
  UB_CUDA(cudaMemcpyAsync(&kerr, flags.p + 2, 4, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  (void)cudaEventElapsedTime(&st.candidate_ms, ev[0], ev[1]);
  (void)cudaEventDestroy(ev[0]);
  (void)cudaEventDestroy(ev[1]);
  if (kerr) throw Error(CUDA, "kNN candidate pass: a pipeline wait timed out");

  DevBuf<uint32_t> fail_rows(n, s);
  const float gamma = (float)(dp + 8) * 9.5367432e-7f;  // (Dp + 8) 2^-20
  const int ki = (int)k, dpi = (int)dp;
  switch (S) {
    case 1: launch_rerank<2>(X, n, di, dpi, ki, cidx.p, tau.p, rn.p, flags.p + 1, gamma, scale, perm.p, out_idx, out_dist, fail_rows.p, flags.p + 3, s); break;
    case 2: launch_rerank<4>(X, n, di, dpi, ki, cidx.p, tau.p, rn.p, flags.p + 1, gamma, scale, perm.p, out_idx, out_dist, fail_rows.p, flags.p + 3, s); break;
    case 4: launch_rerank<8>(X, n, di, dpi, ki, cidx.p, tau.p, rn.p, flags.p + 1, gamma, scale, perm.p, out_idx, out_dist, fail_rows.p, flags.p + 3, s); break;
    default: launch_rerank<16>(X, n, di, dpi, ki, cidx.p, tau.p, rn.p, flags.p + 1, gamma, scale, perm.p, out_idx, out_dist, fail_rows.p, flags.p + 3, s); break;
  }
  unsigned n_fail = 0;
  UB_CUDA(cudaMemcpyAsync(&n_fail, flags.p + 3, 4, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  st.fallback_rows = n_fail;
  if (n_fail) exact_rows(X, (int64_t)n, di, ki, fail_rows.p, n_fail, out_idx, out_dist, s);
  return st;
}

}  // namespace ub
