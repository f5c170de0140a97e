// Learned warm start: a small MLP (in -> 256 -> 256 -> out, exact-erf GELU) with BF16 weights
// and activations and FP32 accumulation, trained with Adam on the mean squared error to 2-D
// targets.  The reference has no counterpart (its caller supplies the initial embedding);
// this produces that initial embedding from the input features.
//
// Tensor-core GEMM.  C[M,N] = A[M,K] * B[N,K]^T with A and B BF16, both K-major (row-major,
// K contiguous), FP32 accumulation in tensor memory.  One CTA (4 warps) owns a 128 x BN
// output tile and a K range (blockIdx.z splits K).  Warp 0 allocates BN tensor-memory
// columns.  K is staged 64 at a time into shared memory in the canonical no-swizzle K-major
// layout: 8-row x 16-byte core matrices, element (r, k) of a 64-wide chunk at byte
// (r/8)*1024 + (k/8)*128 + (r%8)*16 + (k%8)*2, so the descriptor of MMA step s
// (k = 16s..16s+15) starts at +256*s with leading byte offset 128 (the next 8 k) and stride
// byte offset 1024 (the next 8 rows).  Two stages: while the four tcgen05.mma (M=128, N=BN,
// K=16) of chunk c run, the threads stage chunk c+1; one thread issues the MMAs and commits
// them to the stage's mbarrier, and a stage is refilled only after its MMAs completed (every
// wait bounded by a timer).  The epilogue reads the accumulator with tcgen05.ld (warp w owns
// rows 32w..32w+31, thread = row) and fuses bias, GELU, the GELU derivative, column sums and
// transposed copies.  The first layer's A operand is gathered by the staging threads: in
// training from a bf16 copy of the input rows standardised once per training run, otherwise
// straight from the fp32 rows (standardised and rounded to bf16 on the way).
//
// One training step (batch B): L1 GEMM (gather) -> L2 GEMM -> output layer + loss + its
// backward (CUDA cores) -> { dH1 GEMM (GELU derivative, db1) -> dW1 GEMM } || dW2 GEMM on a
// second stream -> Adam.  The dW GEMMs contract over the batch in K splits whose partial sums
// are stored to separate slices and summed by the Adam kernel.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <utility>
#include <vector>

#include "ub_internal.hpp"
#include "umma.cuh"

namespace ub {
namespace {

using namespace umma;

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static std::mutex mu;
  static EncodeTiledFn fn = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    UB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !f) throw Error(CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}


using bf16 = __nv_bfloat16;

constexpr int GM = 128;   // tile rows (UMMA M)
constexpr int KC = 64;    // K staged per chunk
constexpr int GT = 256;   // threads per GEMM CTA: warps w and w + 4 share TMEM lanes, split columns
constexpr int HID = 256;  // hidden width

enum Epi : int {
  EPI_F32 = 0,         // out_f32 (slice blockIdx.z) = acc (+ bias)
  EPI_F32_ATOMIC = 1,  // out_f32 += acc (split-K partial sums)
  EPI_BIAS_GELU = 2,   // z = acc + bias -> out_f32 (if set); h = gelu(z) -> out_bf16 (+ out_t)
  EPI_GELU_GRAD = 3,   // d = acc * gelu'(z_in) -> out_bf16 / out_t (if set); colsum += sum_rows d
};

struct EpiArgs {
  const float* bias;
  float* out_f32;
  int64_t split_stride;  // EPI_F32: elements between the slices of K splits
  const float* z_in;
  bf16* out_bf16;
  bf16* out_t;  // transposed copy [N, ldt]
  float* colsum;
  int ldo, ldt;
};

// First-layer A operand gathered from fp32 rows: A[r] = bf16((X[src(r)] - shift) * scale) with
// src(r) = rows[r] (training) or min(r, n_valid - 1) (inference, padded tail).  CTAs with
// blockIdx.y == 0 also write the transposed copy xt [K, ldt] (for dW1).
struct GatherA {
  const float* X;
  const __nv_bfloat16* Xb;  // if set: rows already standardised and rounded (training), read instead of X
  int ldx;
  const uint32_t* rows;
  int64_t n_valid;
  const float* shift;
  const float* scale;
  bf16* xt;
  int64_t ldt;
};


__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}


__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Epilogue: thread (warp w, lane l) owns output row m0 + 32w + l; reads the accumulator from
// tensor memory 32 columns at a time and applies the layer's elementwise work.  `scratch`
// (>= 4 x 32 x 33 floats of shared memory no longer read by the MMAs) serves the column sums.
template <int BN, int EPI>
__device__ __forceinline__ void epilogue(uint32_t taddr, int64_t m0, int64_t n0, const EpiArgs& ep,
                                         uint8_t* scratch, int warp, int lane) {
  uint8_t* smem = scratch;
  // warp w reads TMEM lanes 32 * (w % 4) .. + 31 (its rows) and the columns of half w / 4
  const int quarter = warp & 3, half = warp >> 2;
  constexpr int HALF = BN >= 64 ? BN / 2 : BN;
  if (BN < 64 && half) return;
  const int64_t row = m0 + quarter * 32 + lane;
#pragma unroll 1
  for (int c0 = half * HALF; c0 < (half + 1) * HALF; c0 += 32) {
    uint32_t r[32];
    const uint32_t ta = taddr + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(ta));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int64_t cb = n0 + c0;  // first column of this group
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
    if (EPI == EPI_F32 || EPI == EPI_F32_ATOMIC) {
      if (EPI == EPI_F32 && ep.bias) {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += __ldg(ep.bias + cb + j);
      }
      float* base = ep.out_f32 + (EPI == EPI_F32 ? (int64_t)blockIdx.z * ep.split_stride : 0);
      float4* o = reinterpret_cast<float4*>(base + row * ep.ldo + cb);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 x = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        if (EPI == EPI_F32_ATOMIC) atomicAdd(o + q, x);
        else o[q] = x;
      }
    } else {
      if (EPI == EPI_BIAS_GELU) {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += __ldg(ep.bias + cb + j);
        if (ep.out_f32) {
          float4* o = reinterpret_cast<float4*>(ep.out_f32 + row * ep.ldo + cb);
#pragma unroll
          for (int q = 0; q < 8; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
      } else {  // EPI_GELU_GRAD
        const float4* zi = reinterpret_cast<const float4*>(ep.z_in + row * ep.ldo + cb);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 z = zi[q];
          v[4 * q] *= gelu_grad(z.x);
          v[4 * q + 1] *= gelu_grad(z.y);
          v[4 * q + 2] *= gelu_grad(z.z);
          v[4 * q + 3] *= gelu_grad(z.w);
        }
        if (ep.colsum) {
          // column sums over the warp's 32 rows through shared memory (the K stages are
          // free once the MMAs completed), one atomic per column per warp
          float* red = reinterpret_cast<float*>(smem) + warp * (32 * 33);
#pragma unroll
          for (int j = 0; j < 32; ++j) red[lane * 33 + j] = v[j];
          __syncwarp();
          float sum = 0.0f;
#pragma unroll 8
          for (int rr = 0; rr < 32; ++rr) sum += red[rr * 33 + lane];
          atomicAdd(ep.colsum + cb + lane, sum);
          __syncwarp();
        }
      }
      uint32_t pk[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) pk[j] = pack_bf16(v[2 * j], v[2 * j + 1]);
      if (ep.out_bf16) {
        uint4* o = reinterpret_cast<uint4*>(ep.out_bf16 + row * ep.ldo + cb);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
      }
      if (ep.out_t) {
        uint16_t* t = reinterpret_cast<uint16_t*>(ep.out_t);
#pragma unroll
        for (int j = 0; j < 32; ++j)
          t[(cb + j) * ep.ldt + row] = (uint16_t)((j & 1) ? (pk[j >> 1] >> 16) : (pk[j >> 1] & 0xFFFFu));
      }
    }
  }
}

template <int BN, int EPI, bool GATHER>
__global__ void __launch_bounds__(GT) umma_gemm_kernel(const bf16* __restrict__ A, int lda,
                                                       const bf16* __restrict__ B, int ldb, int k_per_cta,
                                                       EpiArgs ep, GatherA ga, unsigned* __restrict__ err) {
  // UMMA with M=128 takes N % 16 == 0 up to 256; the epilogue reads 32 columns at a time.
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "tile width");
  constexpr uint32_t TCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  constexpr int STAGE = (GM + BN) * KC * 2;  // bytes of one K chunk of A and B
  static_assert(2 * STAGE >= 8 * 32 * 33 * 4, "epilogue reduction scratch reuses the stages");
  extern __shared__ __align__(1024) uint8_t smem[];  // two stages: [A | B] [A | B]
  __shared__ __align__(8) uint64_t mbar[2];          // MMA completion, one per stage
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * GM, n0 = (int64_t)blockIdx.y * BN;
  const int64_t k_begin = (int64_t)blockIdx.z * k_per_cta;
  const int n_chunks = k_per_cta / KC;

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[0])), "r"(1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[1])), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // Everything above overlaps the previous kernel; its results are read below.  Tensor memory
  // is taken only after it has finished, so a waiting CTA never holds any.
  grid_wait();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base)), "r"(TCOLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  grid_release();
  const uint32_t taddr = tmem_base;

  // A[m0:m0+128, k:k+64] and B[n0:n0+BN, k:k+64] of chunk c into stage `st`, 16-byte vectors.
  auto stage_chunk = [&](int c, int st) {
    const int64_t kg = k_begin + (int64_t)c * KC;
    uint8_t* sA = smem + st * STAGE;
    uint8_t* sB = sA + GM * KC * 2;
    if (GATHER) {
      // consecutive threads take consecutive rows: the transposed copy is written coalesced;
      // a thread's four items are loaded together
#pragma unroll 4
      for (int v = tid; v < GM * (KC / 8); v += GT) {
        const int r = v & (GM - 1), c8 = v / GM;
        const int64_t b = m0 + r;
        const int64_t src = ga.rows ? (int64_t)ga.rows[b] : (b < ga.n_valid ? b : ga.n_valid - 1);
        const int64_t k0 = kg + c8 * 8;
        uint32_t pk[4];
        if (ga.Xb) {
          const uint4 u = __ldg(reinterpret_cast<const uint4*>(ga.Xb + src * ga.ldx + k0));
          pk[0] = u.x;
          pk[1] = u.y;
          pk[2] = u.z;
          pk[3] = u.w;
        } else {
          const float4* xp = reinterpret_cast<const float4*>(ga.X + src * ga.ldx + k0);
          const float4 x0 = __ldg(xp), x1 = __ldg(xp + 1);
          float f[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
          if (ga.scale) {
            // shift / scale hold in_dim floats from a 256-byte aligned allocation; k0 % 8 == 0
            const float4* sp = reinterpret_cast<const float4*>(ga.shift + k0);
            const float4* cp = reinterpret_cast<const float4*>(ga.scale + k0);
            const float4 s0 = __ldg(sp), s1 = __ldg(sp + 1), c0 = __ldg(cp), c1 = __ldg(cp + 1);
            const float sh[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
            const float sc[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
            for (int e = 0; e < 8; ++e) f[e] = (f[e] - sh[e]) * sc[e];
          }
#pragma unroll
          for (int e = 0; e < 4; ++e) pk[e] = pack_bf16(f[2 * e], f[2 * e + 1]);
        }
        *reinterpret_cast<uint4*>(sA + (r >> 3) * (KC * 16) + c8 * 128 + (r & 7) * 16) =
            make_uint4(pk[0], pk[1], pk[2], pk[3]);
        if (ga.xt && blockIdx.y == 0) {
          uint16_t* t = reinterpret_cast<uint16_t*>(ga.xt);
#pragma unroll
          for (int e = 0; e < 8; ++e)
            t[(k0 + e) * ga.ldt + b] = (uint16_t)((e & 1) ? (pk[e >> 1] >> 16) : (pk[e >> 1] & 0xFFFFu));
        }
      }
    } else {
#pragma unroll 4
      for (int v = tid; v < GM * (KC / 8); v += GT) {
        const int r = v >> 3, c8 = v & 7;
        const uint4 x = __ldg(reinterpret_cast<const uint4*>(A + (m0 + r) * lda + kg + c8 * 8));
        *reinterpret_cast<uint4*>(sA + (r >> 3) * (KC * 16) + c8 * 128 + (r & 7) * 16) = x;
      }
    }
#pragma unroll 4
    for (int v = tid; v < BN * (KC / 8); v += GT) {
      const int r = v >> 3, c8 = v & 7;
      const uint4 x = __ldg(reinterpret_cast<const uint4*>(B + (n0 + r) * ldb + kg + c8 * 8));
      *reinterpret_cast<uint4*>(sB + (r >> 3) * (KC * 16) + c8 * 128 + (r & 7) * 16) = x;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  };
  // The j-th completion of a stage's barrier (j = chunk / 2) has phase parity j & 1.
  auto wait_chunk = [&](int c) { return mbar_wait(smem_u32(&mbar[c & 1]), (uint32_t)((c >> 1) & 1)); };

  bool ok = true;
  int last_issued = -1;
  if (n_chunks > 0) stage_chunk(0, 0);
  for (int c = 0; c < n_chunks; ++c) {
    __syncthreads();  // stage c & 1 holds chunk c
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(smem + (c & 1) * STAGE);
      const uint32_t b0 = a0 + GM * KC * 2;
      constexpr uint32_t idesc = instr_desc(GM, BN);
#pragma unroll
      for (int s = 0; s < KC / 16; ++s) {
        const uint64_t ad = smem_desc(a0 + s * 256, 128, KC * 16);
        const uint64_t bd = smem_desc(b0 + s * 256, 128, KC * 16);
        const uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            :: "r"(taddr), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&mbar[c & 1])) : "memory");
    }
    last_issued = c;
    if (c + 1 < n_chunks) {
      // the other stage was last read by chunk c - 1: wait for it, then refill it while
      // the MMAs of chunk c run
      bool free_ok = true;
      if (c >= 1) free_ok = wait_chunk(c - 1);
      if (!__syncthreads_and(free_ok)) {
        ok = false;
        break;
      }
      stage_chunk(c + 1, (c + 1) & 1);
    }
  }
  if (ok && last_issued >= 0) ok = __syncthreads_and(wait_chunk(last_issued));
  if (!ok) {
    // MMAs did not complete in time: record it, give the last ones one more bounded wait,
    // release tensor memory and leave the tile unwritten.
    if (tid == 0) atomicOr(err, 1u);
    if (last_issued >= 0) (void)wait_chunk(last_issued);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok) epilogue<BN, EPI>(taddr, m0, n0, ep, smem, warp, lane);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(TCOLS) : "memory");
}



constexpr int TS = 4;  // TMA pipeline stages

// Tensor-core GEMM fed by TMA.  Thread 0 arms each stage's `full` barrier with the stage's
// byte count and issues two 2-D bulk tensor loads (A tile 128 x 64, B tile BN x 64, 128-byte
// swizzle) for up to TS chunks ahead, issues the four MMAs of a chunk once its stage is full,
// commits them to the stage's `empty` barrier and refills the stage after they completed.
// Every wait is bounded; on a timeout the kernel records the error, drains the loads it
// issued (bounded), frees tensor memory and leaves the tile unwritten.
template <int BN, int EPI>
__global__ void __launch_bounds__(GT) umma_tma_gemm_kernel(const __grid_constant__ CUtensorMap ta,
                                                           const __grid_constant__ CUtensorMap tb, int k_per_cta,
                                                           EpiArgs ep, unsigned* __restrict__ err) {
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "tile width");
  constexpr uint32_t TCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  constexpr uint32_t A_BYTES = GM * 128, B_BYTES = BN * 128, STAGE = A_BYTES + B_BYTES;
  static_assert(STAGE % 1024 == 0, "stages stay 1024-byte aligned");
  static_assert(2 * STAGE >= 8 * 32 * 33 * 4, "epilogue reduction scratch reuses the stages");
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full[TS], empty[TS];
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * GM, n0 = (int64_t)blockIdx.y * BN;
  const int64_t k_begin = (int64_t)blockIdx.z * k_per_cta;
  const int n_chunks = k_per_cta / KC;

  if (tid == 0) {
    for (int i = 0; i < TS; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&full[i])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&empty[i])), "r"(1) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    s_fail = 0;
  }
  // As in umma_gemm_kernel: set-up overlaps the previous kernel, tensor memory and global
  // memory are touched only after it has finished.
  grid_wait();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base)), "r"(TCOLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  grid_release();
  const uint32_t taddr = tmem_base;

  if (tid == 0) {
    auto issue = [&](int c) {
      const int st = c % TS;
      const uint32_t a_dst = smem_u32(smem + st * STAGE), b_dst = a_dst + A_BYTES;
      const uint32_t fb = smem_u32(&full[st]);
      const int x = (int)(k_begin + (int64_t)c * KC);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(fb), "r"(STAGE) : "memory");
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
          :: "r"(a_dst), "l"(reinterpret_cast<uint64_t>(&ta)), "r"(x), "r"((int)m0), "r"(fb) : "memory");
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
          :: "r"(b_dst), "l"(reinterpret_cast<uint64_t>(&tb)), "r"(x), "r"((int)n0), "r"(fb) : "memory");
    };
    int issued = 0, consumed = 0;
    bool ok = true;
    for (; issued < n_chunks && issued < TS; ++issued) issue(issued);
    constexpr uint32_t idesc = instr_desc(GM, BN);
    for (int c = 0; c < n_chunks; ++c) {
      const int st = c % TS;
      if (!mbar_wait(smem_u32(&full[st]), (uint32_t)((c / TS) & 1))) {
        ok = false;
        break;
      }
      consumed = c + 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(smem + st * STAGE), b0 = a0 + A_BYTES;
#pragma unroll
      for (int k = 0; k < KC / 16; ++k) {
        const uint64_t ad = smem_desc_sw128(a0 + k * 32), bd = smem_desc_sw128(b0 + k * 32);
        const uint32_t acc = (c > 0 || k > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            :: "r"(taddr), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&empty[st])) : "memory");
      if (issued < n_chunks) {
        // the stage is refilled once the MMAs that read it completed
        if (!mbar_wait(smem_u32(&empty[st]), (uint32_t)((c / TS) & 1))) {
          ok = false;
          break;
        }
        issue(issued++);
      }
    }
    if (!ok) {
      s_fail = 1;
      atomicOr(err, 1u);
      for (int c = consumed; c < issued; ++c) (void)mbar_wait(smem_u32(&full[c % TS]), (uint32_t)((c / TS) & 1));
    }
  }
  __syncthreads();
  bool ok = s_fail == 0;
  if (ok && n_chunks > 0) {
    const int last = n_chunks - 1;
    ok = __syncthreads_and(mbar_wait(smem_u32(&empty[last % TS]), (uint32_t)((last / TS) & 1)));
    if (!ok && tid == 0) atomicOr(err, 1u);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) epilogue<BN, EPI>(taddr, m0, n0, ep, smem, warp, lane);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(TCOLS) : "memory");
}

template <int BN>
constexpr size_t tma_gemm_smem() {
  return (size_t)TS * (GM + BN) * 128 + 1024;
}

template <int BN>
constexpr size_t gemm_smem() {
  return (size_t)2 * (GM + BN) * KC * 2;
}

// Launch of `k` on `s`; with `pdl` it carries the programmatic-stream-serialization attribute,
// so it may be scheduled while the previous kernel on `s` still runs (the kernel orders its
// memory accesses after that kernel's end with grid_wait()).
template <typename... KArgs, typename... Args>
void launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  UB_CUDA(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
  count_launch();
}

template <int BN, int EPI, bool GATHER = false>
void prepare_gemm() {
  UB_CUDA(cudaFuncSetAttribute(umma_gemm_kernel<BN, EPI, GATHER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)gemm_smem<BN>()));
}

// C = A[M,K] B[N,K]^T, the K range split into `ksplit` equal parts: EPI_F32 stores each
// part's sum to its own slice (ep.split_stride apart), EPI_F32_ATOMIC adds them up.
template <int BN, int EPI, bool GATHER = false>
void launch_gemm(const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int64_t M, int64_t N, int64_t K,
                 int ksplit, const EpiArgs& ep, unsigned* err, cudaStream_t s, const GatherA* ga = nullptr,
                 bool pdl = false) {
  if (M <= 0 || M % GM || N % BN || K <= 0 || ksplit < 1 || K % ((int64_t)KC * ksplit) || lda % 8 || ldb % 8 ||
      M / GM > 0x7FFFFFFF || lda > 0x7FFFFFFF || ldb > 0x7FFFFFFF || ksplit > 65535)
    throw Error(INVALID_ARGUMENT, "tensor-core GEMM shape: M % 128, N % tile, K % (64 * splits), rows of 16 bytes");
  if (ksplit > 1 && !(EPI == EPI_F32_ATOMIC || (EPI == EPI_F32 && ep.split_stride > 0)))
    throw Error(INVALID_ARGUMENT, "split K needs per-split output slices or the atomic epilogue");
  if (GATHER && (!ga || ga->ldx % 4)) throw Error(INVALID_ARGUMENT, "gathered rows must be 16-byte aligned");
  GatherA g{};
  if (ga) g = *ga;
  dim3 grid((unsigned)(M / GM), (unsigned)(N / BN), (unsigned)ksplit);
  launch_k(umma_gemm_kernel<BN, EPI, GATHER>, grid, dim3(GT), gemm_smem<BN>(), s, pdl, A, (int)lda, B, (int)ldb,
           (int)(K / ksplit), ep, g, err);
}


template <int BN, int EPI>
void prepare_tma_gemm() {
  UB_CUDA(cudaFuncSetAttribute(umma_tma_gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)tma_gemm_smem<BN>()));
}

// C = A[M,K] B[N,K]^T through the TMA-fed kernel; K split into `ksplit` parts as launch_gemm.
template <int BN, int EPI>
void launch_tma_gemm(const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int64_t M, int64_t N, int64_t K,
                     int ksplit, const EpiArgs& ep, unsigned* err, cudaStream_t s, bool pdl = false) {
  if (M <= 0 || M % GM || N <= 0 || N % BN || K <= 0 || ksplit < 1 || K % ((int64_t)KC * ksplit) ||
      M / GM > 0x7FFFFFFF || ksplit > 65535 || K > 0x7FFFFFFF || M > 0x7FFFFFFF || N > 0x7FFFFFFF)
    throw Error(INVALID_ARGUMENT, "tensor-core GEMM shape: M % 128, N % tile, K % (64 * splits), rows of 16 bytes");
  if (ksplit > 1 && !(EPI == EPI_F32_ATOMIC || (EPI == EPI_F32 && ep.split_stride > 0)))
    throw Error(INVALID_ARGUMENT, "split K needs per-split output slices or the atomic epilogue");
  const CUtensorMap ta = bf16_tile_map(A, M, K, lda, GM);
  const CUtensorMap tb = bf16_tile_map(B, N, K, ldb, BN);
  dim3 grid((unsigned)(M / GM), (unsigned)(N / BN), (unsigned)ksplit);
  launch_k(umma_tma_gemm_kernel<BN, EPI>, grid, dim3(GT), tma_gemm_smem<BN>(), s, pdl, ta, tb, (int)(K / ksplit), ep,
           err);
}

// ------------------------------------------------------------------------------ CUDA-core parts
// Output layer (256 -> OUT) on CUDA cores, one warp per row, 32 rows per block (4 per warp);
// lane l owns hidden columns 8l..8l+7.  y = h2 W3^T + b3.  With targets it also runs the loss
// and this layer's backward: t = Y[rows[b]]; e = y - t; loss += sum e^2 / count;
// dy = 2 e / count; dz2 = (dy W3) * gelu'(z2) -> bf16 row-major and transposed [256, ldt];
// dW3 += dy^T h2; db3 += sum dy; db2 += sum dz2 (fp32, before rounding); and it advances the
// Adam step counter.
template <int OUT>
__global__ void __launch_bounds__(256) out_layer_kernel(
    const bf16* __restrict__ h2, const float* __restrict__ z2, const bf16* __restrict__ w3,
    const float* __restrict__ b3, const float* __restrict__ Y, const uint32_t* __restrict__ rows, int64_t n_valid,
    float inv_count, float* __restrict__ y_out, bf16* __restrict__ dz2, bf16* __restrict__ dz2t, int64_t ldt,
    float* __restrict__ g_w3, float* __restrict__ g_b3, float* __restrict__ g_b2, float* __restrict__ loss,
    unsigned* __restrict__ step) {
  __shared__ uint16_t s_t[HID][34];
  __shared__ float s_gw3[OUT * HID];
  __shared__ float s_gb2[HID];
  __shared__ float s_gb3[OUT];
  __shared__ float s_loss;
  grid_wait();
  grid_release();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool train = Y != nullptr;
  if (train) {
    for (int i = tid; i < OUT * HID; i += 256) s_gw3[i] = 0.0f;
    s_gb2[tid] = 0.0f;
    if (tid < OUT) s_gb3[tid] = 0.0f;
    if (tid == 0) s_loss = 0.0f;
    if (step && blockIdx.x == 0 && tid == 0) *step += 1u;
    __syncthreads();
  }
  float w[OUT][8];
#pragma unroll
  for (int j = 0; j < OUT; ++j) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(w3 + j * HID + 8 * lane));
    const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 f = __bfloat1622float2(p[i]);
      w[j][2 * i] = f.x;
      w[j][2 * i + 1] = f.y;
    }
  }
  float bias[OUT];
#pragma unroll
  for (int j = 0; j < OUT; ++j) bias[j] = b3[j];
  // issue every load of the warp's 4 rows first
  const int64_t row0 = (int64_t)blockIdx.x * 32 + warp * 4;
  uint4 hu[4];
  float4 za[4], zb[4];
  float tg[4][OUT];
#pragma unroll
  for (int rr = 0; rr < 4; ++rr) {
    hu[rr] = *reinterpret_cast<const uint4*>(h2 + (row0 + rr) * HID + 8 * lane);
    if (train) {
      const float4* zr = reinterpret_cast<const float4*>(z2 + (row0 + rr) * HID + 8 * lane);
      za[rr] = zr[0];
      zb[rr] = zr[1];
      const int64_t src = rows ? (int64_t)rows[row0 + rr] : row0 + rr;
#pragma unroll
      for (int j = 0; j < OUT; ++j) tg[rr][j] = Y[src * OUT + j];
    }
  }
  float gw[OUT][8] = {}, gb2[8] = {}, gb3[OUT] = {}, lsum = 0.0f;
#pragma unroll
  for (int rr = 0; rr < 4; ++rr) {
    const int rl = warp * 4 + rr;
    const int64_t row = row0 + rr;
    float h[8];
    {
      const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&hu[rr]);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(p[i]);
        h[2 * i] = f.x;
        h[2 * i + 1] = f.y;
      }
    }
    float y[OUT];
#pragma unroll
    for (int j = 0; j < OUT; ++j) {
      float s = 0.0f;
#pragma unroll
      for (int i = 0; i < 8; ++i) s += h[i] * w[j][i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
      y[j] = s + bias[j];
    }
    if (y_out && lane == 0 && row < n_valid) {
#pragma unroll
      for (int j = 0; j < OUT; ++j) y_out[row * OUT + j] = y[j];
    }
    if (!train) continue;
    float dy[OUT];
#pragma unroll
    for (int j = 0; j < OUT; ++j) {
      const float e = y[j] - tg[rr][j];
      lsum += e * e * inv_count;
      dy[j] = 2.0f * e * inv_count;
      gb3[j] += dy[j];
    }
    const float z[8] = {za[rr].x, za[rr].y, za[rr].z, za[rr].w, zb[rr].x, zb[rr].y, zb[rr].z, zb[rr].w};
    float d[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      float dh = 0.0f;
#pragma unroll
      for (int j = 0; j < OUT; ++j) dh += dy[j] * w[j][i];
      d[i] = dh * gelu_grad(z[i]);
      gb2[i] += d[i];
#pragma unroll
      for (int j = 0; j < OUT; ++j) gw[j][i] += dy[j] * h[i];
    }
    uint32_t pk[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) pk[i] = pack_bf16(d[2 * i], d[2 * i + 1]);
    *reinterpret_cast<uint4*>(dz2 + row * HID + 8 * lane) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      s_t[8 * lane + i][rl] = (uint16_t)((i & 1) ? (pk[i >> 1] >> 16) : (pk[i >> 1] & 0xFFFFu));
  }
  if (!train) return;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    atomicAdd(&s_gb2[8 * lane + i], gb2[i]);
#pragma unroll
    for (int j = 0; j < OUT; ++j) atomicAdd(&s_gw3[j * HID + 8 * lane + i], gw[j][i]);
  }
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < OUT; ++j) atomicAdd(&s_gb3[j], gb3[j]);
    atomicAdd(&s_loss, lsum);
  }
  __syncthreads();
  // transposed dz2: thread = hidden column, 32 consecutive rows as 16 packed pairs
  {
    uint32_t* dst = reinterpret_cast<uint32_t*>(dz2t + (int64_t)tid * ldt + (int64_t)blockIdx.x * 32);
    const uint16_t* src = s_t[tid];
#pragma unroll
    for (int p = 0; p < 16; ++p) dst[p] = (uint32_t)src[2 * p] | ((uint32_t)src[2 * p + 1] << 16);
  }
  for (int i = tid; i < OUT * HID; i += 256) atomicAdd(g_w3 + i, s_gw3[i]);
  atomicAdd(g_b2 + tid, s_gb2[tid]);
  if (tid < OUT) atomicAdd(g_b3 + tid, s_gb3[tid]);
  if (tid == 0) atomicAdd(loss, s_loss);
}

// Adam (Kingma & Ba 2015) over the flat fp32 parameters, bias-corrected with the step count
// held on the device.  Gradients of W1 and W2 are the sums of their K-split slices; the other
// gradients were accumulated atomically and are zeroed here for the next step.  Refreshes the
// bf16 working copies of the weight matrices (and W2^T).
struct AdamArgs {
  float* w;
  float* m;
  float* v;
  float* g;
  int64_t n;
  float lr, b1, b2, eps;
  const unsigned* step;
  int64_t o_w1, o_w2, o_w3, n_w1, n_w3;
  const float* part1;  // [ks1][n_w1]
  const float* part2;  // [ks2][HID * HID]
  int ks1, ks2;
  bf16* w1b;
  bf16* w2b;
  bf16* w2t;
  bf16* w3b;
};

// Sum of the K-split slices, added in slice order; the loads of eight slices are issued
// before their additions (the slice count is a power of two, a multiple of 8 above 8).
__device__ __forceinline__ float slice_sum(const float* part, int ks, int64_t stride, int64_t k) {
  float s = 0.0f;
  int z = 0;
#pragma unroll 4
  for (; z + 8 <= ks; z += 8) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = part[(int64_t)(z + u) * stride + k];
#pragma unroll
    for (int u = 0; u < 8; ++u) s += v[u];
  }
  for (; z < ks; ++z) s += part[(int64_t)z * stride + k];
  return s;
}

__global__ void adam_kernel(AdamArgs a) {
  grid_wait();
  grid_release();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const float t = (float)*a.step;
  const float c1 = 1.0f - powf(a.b1, t), c2 = 1.0f - powf(a.b2, t);
  const bool in_w1 = i >= a.o_w1 && i < a.o_w1 + a.n_w1;
  const bool in_w2 = i >= a.o_w2 && i < a.o_w2 + (int64_t)HID * HID;
  float gi;
  if (in_w1) {
    gi = slice_sum(a.part1, a.ks1, a.n_w1, i - a.o_w1);
  } else if (in_w2) {
    gi = slice_sum(a.part2, a.ks2, (int64_t)HID * HID, i - a.o_w2);
  } else {
    gi = a.g[i];
    a.g[i] = 0.0f;
  }
  const float mi = a.b1 * a.m[i] + (1.0f - a.b1) * gi;
  const float vi = a.b2 * a.v[i] + (1.0f - a.b2) * gi * gi;
  a.m[i] = mi;
  a.v[i] = vi;
  const float wi = a.w[i] - a.lr * (mi / c1) / (sqrtf(vi / c2) + a.eps);
  a.w[i] = wi;
  const bf16 h = __float2bfloat16_rn(wi);
  if (in_w1) {
    a.w1b[i - a.o_w1] = h;
  } else if (in_w2) {
    const int64_t k = i - a.o_w2;
    a.w2b[k] = h;
    a.w2t[(k % HID) * HID + k / HID] = h;
  } else if (i >= a.o_w3 && i < a.o_w3 + a.n_w3) {
    a.w3b[i - a.o_w3] = h;
  }
}

// g[W1] and g[W2] from their K-split slices (the gradient query without an update).
__global__ void reduce_slices_kernel(const float* __restrict__ part, int ks, int64_t n, float* __restrict__ out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = slice_sum(part, ks, n, k);
}

__global__ void to_bf16_kernel(const float* __restrict__ w, int64_t n, bf16* __restrict__ wb, bf16* __restrict__ wt,
                               int cols) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bf16 b = __float2bfloat16_rn(w[i]);
  wb[i] = b;
  if (wt) {
    const int64_t r = i / cols, c = i - r * cols;
    wt[c * (n / cols) + r] = b;
  }
}

// Per-column mean and 1/std (population) of X [n, d]; one block per column, fp64 sums.
__global__ void column_stats_kernel(const float* __restrict__ X, int64_t n, int d, float* __restrict__ mean,
                                    float* __restrict__ inv_std) {
  __shared__ double s1[256], s2[256];
  const int c = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = X[i * d + c];
    a += x;
    b += x * x;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double mu = s1[0] / (double)n;
    const double var = std::max(s2[0] / (double)n - mu * mu, 0.0);
    mean[c] = (float)mu;
    inv_std[c] = var > 1e-24 ? (float)(1.0 / sqrt(var)) : 1.0f;
  }
}

inline unsigned grid_for(int64_t n, unsigned bt) { return (unsigned)((n + bt - 1) / bt); }

// The first layer's input rows standardised and rounded once per training run, with the same
// operations as the layer-1 gather: Xb = bf16((X - shift) * scale) (X itself without a norm).
// Eight features per thread; d % 8 == 0.
__global__ void standardize_bf16_kernel(const float* __restrict__ X, int64_t n, int d,
                                        const float* __restrict__ shift, const float* __restrict__ scale,
                                        bf16* __restrict__ Xb) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per_row = d / 8;
  if (v >= n * per_row) return;
  const int64_t r = v / per_row;
  const int k0 = (int)(v - r * per_row) * 8;
  const float4* xp = reinterpret_cast<const float4*>(X + r * d + k0);
  const float4 x0 = __ldg(xp), x1 = __ldg(xp + 1);
  float f[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
  if (scale) {
#pragma unroll
    for (int e = 0; e < 8; ++e) f[e] = (f[e] - __ldg(shift + k0 + e)) * __ldg(scale + k0 + e);
  }
  uint32_t pk[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) pk[e] = pack_bf16(f[2 * e], f[2 * e + 1]);
  *reinterpret_cast<uint4*>(Xb + r * d + k0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
}

// Sort keys of the shuffles of epochs e0 .. e0 + total / n - 1 (entry q * n + row): the
// splitmix64 finaliser of (seed, epoch, row), top 32 bits; with eb > 0 the epoch's offset q
// in the group takes the key's top eb bits and the hash's top 32 - eb bits follow.
__global__ void shuffle_keys_kernel(uint32_t* __restrict__ keys, int64_t n, uint64_t seed, uint32_t e0,
                                    int64_t total, int eb) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int64_t q = i / n, r = i - q * n;
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + ((uint64_t)(e0 + (uint32_t)q) << 32) + (uint64_t)r + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const uint32_t h = (uint32_t)(z >> 32);
  keys[i] = eb ? ((uint32_t)q << (32 - eb)) | (h >> eb) : h;
}

// Sorted positions q * n + row of a group of epochs back to rows.
__global__ void perm_rows_kernel(uint32_t* __restrict__ p, int64_t total, uint32_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) p[i] %= n;
}

bool graphs_enabled() {
  const char* e = std::getenv("UMAP_B200_GRAPH");
  return !(e && e[0] == '0');
}

// Programmatic dependent launch between the kernels of a network step (UMAP_B200_PDL=0 turns
// it off).
bool pdl_enabled() {
  const char* e = std::getenv("UMAP_B200_PDL");
  return !(e && e[0] == '0');
}

// Split of a batch-row contraction of length K over `tiles` output tiles: the largest power
// of two that keeps about 64 CTAs and whole 64-row chunks per split (the TMA pipeline keeps
// a CTA's chunks in flight, so fewer, longer splits cost less than more slices to sum).
int k_splits(int64_t K, int tiles) {
  int ks = 1;
  while ((int64_t)ks * 2 * tiles <= 64 && K % ((int64_t)KC * ks * 2) == 0) ks *= 2;
  return ks;
}

void prepare_all_gemms() {
  static std::mutex mu;
  static uint64_t prepared = 0;  // kernel attributes belong to a device's context: bit per device id < 64
  int dev = 0;
  UB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 64 && ((prepared >> dev) & 1u)) return;
  prepare_gemm<64, EPI_BIAS_GELU, true>();
  prepare_gemm<256, EPI_BIAS_GELU, true>();
  prepare_tma_gemm<64, EPI_BIAS_GELU>();
  prepare_tma_gemm<256, EPI_BIAS_GELU>();
  prepare_tma_gemm<64, EPI_GELU_GRAD>();
  prepare_tma_gemm<64, EPI_F32>();
  prepare_tma_gemm<256, EPI_F32>();
  prepare_tma_gemm<128, EPI_F32>();
  prepare_tma_gemm<32, EPI_F32>();
  prepare_tma_gemm<256, EPI_F32_ATOMIC>();
  prepare_tma_gemm<64, EPI_F32_ATOMIC>();
  (void)encode_tiled();
  if (dev < 64) prepared |= 1ull << dev;
}

}  // namespace

// ------------------------------------------------------------------------------ model
// ------------------------------------------------------------------------------ TMA tensor maps
// Tensor map of a row-major bf16 matrix [rows, cols] (row stride ld elements) read in boxes of
// box_rows x 64 with 128-byte swizzle.
CUtensorMap bf16_tile_map(const void* base, int64_t rows, int64_t cols, int64_t ld, int box_rows, bool f16) {
  if (reinterpret_cast<uintptr_t>(base) % 16 || (ld * 2) % 16 || cols < 64 || rows < box_rows)
    throw Error(INVALID_ARGUMENT, "TMA operand must be 16-byte aligned with 16-byte rows");
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_tiled()(&m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}


struct Mlp::Impl {
  int in_dim = 0, out_dim = 0;
  cudaStream_t s = nullptr;   // owner's stream
  cudaStream_t s2 = nullptr;  // second stream: dW2 runs beside dH1 / dW1
  cudaEvent_t fork = nullptr, join = nullptr;
  int64_t P = 0, o_w1 = 0, o_b1 = 0, o_w2 = 0, o_b2 = 0, o_w3 = 0, o_b3 = 0;
  DevBuf<float> w, m, v, g;         // flat fp32 parameters, Adam moments, gradients
  DevBuf<bf16> w1b, w2b, w2t, w3b;  // bf16 working copies (w2t = W2^T)
  DevBuf<float> shift, scale;       // input standardisation
  bool has_norm = false;
  bool pdl = pdl_enabled();
  DevBuf<unsigned> err, step;
  DevBuf<float> loss;
  // per-batch activations, capacity `cap` rows
  int64_t cap = 0;
  bool cap_train = false;
  int ks1 = 1, ks2 = 1;  // K splits of dW1 / dW2 for the current batch size
  DevBuf<bf16> xt, h1, h1t, h2, dz2, dz2t, dz1t;
  DevBuf<float> z1, z2, part1, part2;

  ~Impl() {
    if (fork) (void)cudaEventDestroy(fork);
    if (join) (void)cudaEventDestroy(join);
    if (s2) {
      (void)cudaStreamSynchronize(s2);
      (void)cudaStreamDestroy(s2);
    }
  }

  void ensure(int64_t B, bool train) {
    if (B <= cap && (!train || cap_train)) return;
    cap = std::max(cap, B);
    cap_train = cap_train || train;
    h1.alloc(cap * HID, s);
    h2.alloc(cap * HID, s);
    if (cap_train) {
      xt.alloc(cap * in_dim, s);
      h1t.alloc(cap * HID, s);
      dz2.alloc(cap * HID, s);
      dz2t.alloc(cap * HID, s);
      dz1t.alloc(cap * HID, s);
      z1.alloc(cap * HID, s);
      z2.alloc(cap * HID, s);
    }
  }
  // Slices for the K splits of a batch of B rows.
  void ensure_slices(int64_t B) {
    const int k1 = k_splits(B, (HID / GM) * (in_dim / 64)), k2 = k_splits(B, (HID / GM) * (HID / 64));
    if (k1 != ks1 || !part1.p) part1.alloc((uint64_t)k1 * HID * in_dim, s);
    if (k2 != ks2 || !part2.p) part2.alloc((uint64_t)k2 * HID * HID, s);
    ks1 = k1;
    ks2 = k2;
  }
};

int64_t Mlp::param_count(int in_dim, int out_dim) {
  return (int64_t)HID * in_dim + HID + (int64_t)HID * HID + HID + (int64_t)out_dim * HID + out_dim;
}

Mlp::Mlp(int in_dim, int out_dim, const float* host_params, cudaStream_t s) : p(nullptr) {
  if (in_dim < 64 || in_dim % 64 || in_dim > 4096 || out_dim < 1 || out_dim > 4)
    throw Error(INVALID_ARGUMENT, "MLP input width must be a positive multiple of 64 (at most 4096) and output width 1..4");
  prepare_all_gemms();
  p = new Impl;
  Impl& m = *p;
  m.in_dim = in_dim;
  m.out_dim = out_dim;
  m.s = s;
  m.o_w1 = 0;
  m.o_b1 = (int64_t)HID * in_dim;
  m.o_w2 = m.o_b1 + HID;
  m.o_b2 = m.o_w2 + (int64_t)HID * HID;
  m.o_w3 = m.o_b2 + HID;
  m.o_b3 = m.o_w3 + (int64_t)out_dim * HID;
  m.P = m.o_b3 + out_dim;
  try {
    UB_CUDA(cudaStreamCreateWithFlags(&m.s2, cudaStreamNonBlocking));
    UB_CUDA(cudaEventCreateWithFlags(&m.fork, cudaEventDisableTiming));
    UB_CUDA(cudaEventCreateWithFlags(&m.join, cudaEventDisableTiming));
    m.w.alloc(m.P, s);
    m.m.alloc(m.P, s);
    m.v.alloc(m.P, s);
    m.g.alloc(m.P, s);
    UB_CUDA(cudaMemsetAsync(m.m.p, 0, m.P * 4, s));
    UB_CUDA(cudaMemsetAsync(m.v.p, 0, m.P * 4, s));
    UB_CUDA(cudaMemsetAsync(m.g.p, 0, m.P * 4, s));
    m.w1b.alloc((int64_t)HID * in_dim, s);
    m.w2b.alloc((int64_t)HID * HID, s);
    m.w2t.alloc((int64_t)HID * HID, s);
    m.w3b.alloc((int64_t)out_dim * HID, s);
    m.err.alloc(1, s);
    m.step.alloc(1, s);
    m.loss.alloc(1, s);
    UB_CUDA(cudaMemsetAsync(m.err.p, 0, 4, s));
    UB_CUDA(cudaMemsetAsync(m.step.p, 0, 4, s));
    UB_CUDA(cudaMemsetAsync(m.loss.p, 0, 4, s));
    set_params(host_params);
  } catch (...) {
    delete p;
    p = nullptr;
    throw;
  }
}

Mlp::~Mlp() { delete p; }

int Mlp::in_dim() const { return p->in_dim; }
int Mlp::out_dim() const { return p->out_dim; }
int64_t Mlp::n_params() const { return p->P; }

void Mlp::set_params(const float* host) {
  Impl& m = *p;
  cudaStream_t s = m.s;
  UB_CUDA(cudaMemcpyAsync(m.w.p, host, m.P * 4, cudaMemcpyHostToDevice, s));
  to_bf16_kernel<<<grid_for(m.w1b.n, 256), 256, 0, s>>>(m.w.p + m.o_w1, m.w1b.n, m.w1b.p, nullptr, m.in_dim);
  UB_LAUNCH_CHECK();
  to_bf16_kernel<<<grid_for(m.w2b.n, 256), 256, 0, s>>>(m.w.p + m.o_w2, m.w2b.n, m.w2b.p, m.w2t.p, HID);
  UB_LAUNCH_CHECK();
  to_bf16_kernel<<<grid_for(m.w3b.n, 256), 256, 0, s>>>(m.w.p + m.o_w3, m.w3b.n, m.w3b.p, nullptr, HID);
  UB_LAUNCH_CHECK();
  UB_CUDA(cudaStreamSynchronize(s));
}

void Mlp::get_params(float* host) const {
  UB_CUDA(cudaMemcpyAsync(host, p->w.p, p->P * 4, cudaMemcpyDeviceToHost, p->s));
  UB_CUDA(cudaStreamSynchronize(p->s));
}

void Mlp::fit_input_norm(const float* X, int64_t n) {
  Impl& m = *p;
  if (n < 1) throw Error(INVALID_ARGUMENT, "input normalisation needs at least one row");
  m.shift.alloc(m.in_dim, m.s);
  m.scale.alloc(m.in_dim, m.s);
  column_stats_kernel<<<m.in_dim, 256, 0, m.s>>>(X, n, m.in_dim, m.shift.p, m.scale.p);
  UB_LAUNCH_CHECK();
  UB_CUDA(cudaStreamSynchronize(m.s));
  m.has_norm = true;
}

void Mlp::get_input_norm(float* shift, float* scale) const {
  const Impl& m = *p;
  if (!m.has_norm) {
    for (int c = 0; c < m.in_dim; ++c) {
      shift[c] = 0.0f;
      scale[c] = 1.0f;
    }
    return;
  }
  UB_CUDA(cudaMemcpyAsync(shift, m.shift.p, m.in_dim * 4, cudaMemcpyDeviceToHost, m.s));
  UB_CUDA(cudaMemcpyAsync(scale, m.scale.p, m.in_dim * 4, cudaMemcpyDeviceToHost, m.s));
  UB_CUDA(cudaStreamSynchronize(m.s));
}

void Mlp::set_input_norm(const float* shift, const float* scale) {
  Impl& m = *p;
  m.shift.alloc(m.in_dim, m.s);
  m.scale.alloc(m.in_dim, m.s);
  UB_CUDA(cudaMemcpyAsync(m.shift.p, shift, m.in_dim * 4, cudaMemcpyHostToDevice, m.s));
  UB_CUDA(cudaMemcpyAsync(m.scale.p, scale, m.in_dim * 4, cudaMemcpyHostToDevice, m.s));
  UB_CUDA(cudaStreamSynchronize(m.s));
  m.has_norm = true;
}

// Forward of one batch of B rows (B % 128 == 0).  With targets Y (training; `rows` selects
// the batch rows of X and Y) also the backward: dW1 / dW2 into their K-split slices, the other
// gradients added into g, the loss into `loss`; with_adam then applies the Adam update.
// Inference writes y for rows < n_valid.
// One forward pass (and with targets the backward pass and, with `with_adam`, the update) of a
// batch.  Each kernel after the first on `s` is a programmatic dependent launch; the first
// one is too when `after_step` says the previous kernel on `s` was this network's update.
static void run_batch(Mlp::Impl& m, const float* X, const uint32_t* rows, int64_t B, int64_t n_valid,
                      const float* Y, float* y_out, bool with_adam, float lr, bool after_step = false,
                      const bf16* Xb = nullptr) {
  cudaStream_t s = m.s;
  const bool pdl = m.pdl;
  const bool train = Y != nullptr;
  float* g = m.g.p;
  GatherA ga{};
  ga.X = X;
  ga.Xb = Xb;
  ga.ldx = m.in_dim;
  ga.rows = rows;
  ga.n_valid = n_valid;
  ga.shift = m.has_norm ? m.shift.p : nullptr;
  ga.scale = m.has_norm ? m.scale.p : nullptr;
  ga.xt = train ? m.xt.p : nullptr;
  ga.ldt = B;
  EpiArgs e1{};
  e1.bias = m.w.p + m.o_b1;
  e1.out_f32 = train ? m.z1.p : nullptr;
  e1.out_bf16 = m.h1.p;
  e1.out_t = train ? m.h1t.p : nullptr;
  e1.ldo = HID;
  e1.ldt = (int)B;
  // Inference on large batches: one CTA per 128 rows covers all 256 hidden units (the rows are
  // gathered once instead of once per 64-column tile); training keeps 64-column tiles for
  // parallelism at its batch of a few thousand rows.
  const bool wide = !train && B >= 8192;
  const bool pdl1 = pdl && after_step;
  if (wide)
    launch_gemm<256, EPI_BIAS_GELU, true>(nullptr, 8, m.w1b.p, m.in_dim, B, HID, m.in_dim, 1, e1, m.err.p, s, &ga,
                                          pdl1);
  else
    launch_gemm<64, EPI_BIAS_GELU, true>(nullptr, 8, m.w1b.p, m.in_dim, B, HID, m.in_dim, 1, e1, m.err.p, s, &ga,
                                         pdl1);
  EpiArgs e2{};
  e2.bias = m.w.p + m.o_b2;
  e2.out_f32 = train ? m.z2.p : nullptr;
  e2.out_bf16 = m.h2.p;
  e2.ldo = HID;
  if (wide)
    launch_tma_gemm<256, EPI_BIAS_GELU>(m.h1.p, HID, m.w2b.p, HID, B, HID, HID, 1, e2, m.err.p, s, pdl);
  else
    launch_tma_gemm<64, EPI_BIAS_GELU>(m.h1.p, HID, m.w2b.p, HID, B, HID, HID, 1, e2, m.err.p, s, pdl);
  const float inv = 1.0f / (float)(B * m.out_dim);
#define UB_OUT_ARGS                                                                                                   \
  m.h2.p, m.z2.p, m.w3b.p, m.w.p + m.o_b3, train ? Y : nullptr, rows, n_valid, inv, y_out, m.dz2.p, m.dz2t.p, B, \
      g + m.o_w3, g + m.o_b3, g + m.o_b2, m.loss.p, with_adam ? m.step.p : nullptr
  const unsigned og = (unsigned)(B / 32);
  switch (m.out_dim) {
    case 1: launch_k(out_layer_kernel<1>, dim3(og), dim3(256), 0, s, pdl, UB_OUT_ARGS); break;
    case 2: launch_k(out_layer_kernel<2>, dim3(og), dim3(256), 0, s, pdl, UB_OUT_ARGS); break;
    case 3: launch_k(out_layer_kernel<3>, dim3(og), dim3(256), 0, s, pdl, UB_OUT_ARGS); break;
    default: launch_k(out_layer_kernel<4>, dim3(og), dim3(256), 0, s, pdl, UB_OUT_ARGS); break;
  }
#undef UB_OUT_ARGS
  if (!train) return;
  // dW2 = dZ2^T H1 on the second stream, beside dH1 and dW1.
  UB_CUDA(cudaEventRecord(m.fork, s));
  UB_CUDA(cudaStreamWaitEvent(m.s2, m.fork, 0));
  EpiArgs e4{};
  e4.out_f32 = m.part2.p;
  e4.split_stride = (int64_t)HID * HID;
  e4.ldo = HID;
  launch_tma_gemm<64, EPI_F32>(m.dz2t.p, B, m.h1t.p, B, HID, HID, B, m.ks2, e4, m.err.p, m.s2);
  UB_CUDA(cudaEventRecord(m.join, m.s2));
  // dH1 = dZ2 W2 (B operand W2^T: row i = column i of W2); dZ1 = dH1 * gelu'(Z1), kept
  // transposed for dW1; db1 = its column sums.
  EpiArgs e3{};
  e3.z_in = m.z1.p;
  e3.out_t = m.dz1t.p;
  e3.colsum = g + m.o_b1;
  e3.ldo = HID;
  e3.ldt = (int)B;
  launch_tma_gemm<64, EPI_GELU_GRAD>(m.dz2.p, HID, m.w2t.p, HID, B, HID, HID, 1, e3, m.err.p, s, pdl);
  // dW1 = dZ1^T X
  EpiArgs e5{};
  e5.out_f32 = m.part1.p;
  e5.split_stride = (int64_t)HID * m.in_dim;
  e5.ldo = m.in_dim;
  launch_tma_gemm<64, EPI_F32>(m.dz1t.p, B, m.xt.p, B, HID, m.in_dim, B, m.ks1, e5, m.err.p, s, pdl);
  UB_CUDA(cudaStreamWaitEvent(s, m.join, 0));
  if (!with_adam) return;
  AdamArgs a{};
  a.w = m.w.p;
  a.m = m.m.p;
  a.v = m.v.p;
  a.g = m.g.p;
  a.n = m.P;
  a.lr = lr;
  a.b1 = 0.9f;
  a.b2 = 0.999f;
  a.eps = 1e-8f;
  a.step = m.step.p;
  a.o_w1 = m.o_w1;
  a.o_w2 = m.o_w2;
  a.o_w3 = m.o_w3;
  a.n_w1 = (int64_t)HID * m.in_dim;
  a.n_w3 = (int64_t)m.out_dim * HID;
  a.part1 = m.part1.p;
  a.part2 = m.part2.p;
  a.ks1 = m.ks1;
  a.ks2 = m.ks2;
  a.w1b = m.w1b.p;
  a.w2b = m.w2b.p;
  a.w2t = m.w2t.p;
  a.w3b = m.w3b.p;
  adam_kernel<<<grid_for(m.P, 256), 256, 0, s>>>(a);
  UB_LAUNCH_CHECK();
}

void Mlp::gradients(const float* X, const float* Y, int64_t B, float* host_grads, float* loss_out) {
  Impl& m = *p;
  if (B < 128 || B % 128) throw Error(INVALID_ARGUMENT, "batch rows must be a positive multiple of 128");
  if (B > (1 << 24)) throw Error(INVALID_ARGUMENT, "at most 16777216 rows per gradient batch");
  m.ensure(B, true);
  m.ensure_slices(B);
  UB_CUDA(cudaMemsetAsync(m.g.p, 0, m.P * 4, m.s));
  UB_CUDA(cudaMemsetAsync(m.loss.p, 0, 4, m.s));
  run_batch(m, X, nullptr, B, B, Y, nullptr, false, 0.0f);
  const int64_t n1 = (int64_t)HID * m.in_dim, n2 = (int64_t)HID * HID;
  reduce_slices_kernel<<<grid_for(n1, 256), 256, 0, m.s>>>(m.part1.p, m.ks1, n1, m.g.p + m.o_w1);
  UB_LAUNCH_CHECK();
  reduce_slices_kernel<<<grid_for(n2, 256), 256, 0, m.s>>>(m.part2.p, m.ks2, n2, m.g.p + m.o_w2);
  UB_LAUNCH_CHECK();
  UB_CUDA(cudaMemcpyAsync(host_grads, m.g.p, m.P * 4, cudaMemcpyDeviceToHost, m.s));
  UB_CUDA(cudaMemcpyAsync(loss_out, m.loss.p, 4, cudaMemcpyDeviceToHost, m.s));
  check_error();
  UB_CUDA(cudaMemsetAsync(m.g.p, 0, m.P * 4, m.s));
}

void Mlp::train(const float* X, const float* Y, int64_t n, int epochs, int64_t batch, float lr, uint64_t seed,
                float* losses) {
  Impl& m = *p;
  cudaStream_t s = m.s;
  if (batch < 128 || batch % 128 || batch > (1 << 24))
    throw Error(INVALID_ARGUMENT, "batch must be a positive multiple of 128 (at most 16777216)");
  if (epochs < 0) throw Error(INVALID_ARGUMENT, "epochs must be >= 0");
  if (n > 0xFFFFFFFFll) throw Error(INVALID_ARGUMENT, "at most 2^32 - 1 training rows");
  const int64_t steps = n / batch;  // the last partial batch of each shuffled epoch is dropped
  if (steps < 1) throw Error(INVALID_ARGUMENT, "fewer training rows than one batch");
  if (epochs == 0) return;
  m.ensure(batch, true);
  m.ensure_slices(batch);
  // Shuffles on the device: epoch e orders the rows by a hash of (seed, e, row) (stable radix
  // sort, so equal hashes keep row order); the first steps * batch rows of each epoch's
  // order are its batches.  Groups of 2^eb epochs share one sort: the key of (epoch
  // e0 + q, row) is q in the top eb bits over the hash's top 32 - eb bits.
  const int64_t per_epoch = steps * batch;
  int eb = 0;
  while (eb < 5 && (1 << eb) < epochs && ((int64_t)2 << eb) * n <= (1ll << 26)) ++eb;
  const int group = 1 << eb;
  const int64_t gmax = (int64_t)std::min(group, epochs) * n;
  DevBuf<uint32_t> hkeys((uint64_t)gmax, s), hsorted((uint64_t)gmax, s), dperm((uint64_t)epochs * n, s);
  DevBuf<uint32_t> cur(per_epoch, s);
  for (int e0 = 0; e0 < epochs; e0 += group) {
    const int64_t total = (int64_t)std::min(group, epochs - e0) * n;
    shuffle_keys_kernel<<<grid_for(total, 256), 256, 0, s>>>(hkeys.p, n, seed, (uint32_t)e0, total, eb);
    UB_LAUNCH_CHECK();
    uint32_t* dst = dperm.p + (int64_t)e0 * n;
    radix_sort_pairs(hkeys.p, nullptr, hsorted.p, dst, (uint64_t)total, 32, s);
    perm_rows_kernel<<<grid_for(total, 256), 256, 0, s>>>(dst, total, (uint32_t)n);
    UB_LAUNCH_CHECK();
  }
  DevBuf<float> dloss(epochs, s);
  UB_CUDA(cudaMemsetAsync(m.g.p, 0, m.P * 4, s));
  // the epochs' batches gather rows of this standardised bf16 copy
  DevBuf<bf16> xb((uint64_t)n * m.in_dim, s);
  const int64_t vec = n * (m.in_dim / 8);
  standardize_bf16_kernel<<<grid_for(vec, 256), 256, 0, s>>>(X, n, m.in_dim, m.has_norm ? m.shift.p : nullptr,
                                                            m.has_norm ? m.scale.p : nullptr, xb.p);
  UB_LAUNCH_CHECK();
  auto one_epoch = [&]() {
    for (int64_t t = 0; t < steps; ++t)
      run_batch(m, X, cur.p + t * batch, batch, batch, Y, nullptr, true, lr, t > 0, xb.p);
  };
  cudaGraphExec_t exec = nullptr;
  if (graphs_enabled()) {
    cudaGraph_t graph = nullptr;
    UB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      one_epoch();
    } catch (...) {
      cudaGraph_t g2 = nullptr;
      (void)cudaStreamEndCapture(s, &g2);
      if (g2) (void)cudaGraphDestroy(g2);
      throw;
    }
    UB_CUDA(cudaStreamEndCapture(s, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    (void)cudaGraphDestroy(graph);
    UB_CUDA(ie);
  }
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() {
      if (e) (void)cudaGraphExecDestroy(e);
    }
  } guard{exec};
  const uint64_t launches_per_epoch = (uint64_t)steps * 7;
  for (int e = 0; e < epochs; ++e) {
    UB_CUDA(cudaMemcpyAsync(cur.p, dperm.p + (int64_t)e * n, per_epoch * 4, cudaMemcpyDeviceToDevice, s));
    UB_CUDA(cudaMemsetAsync(m.loss.p, 0, 4, s));
    if (exec) {
      UB_CUDA(cudaGraphLaunch(exec, s));
      for (uint64_t i = 0; i < launches_per_epoch; ++i) count_launch();
    } else {
      one_epoch();
    }
    UB_CUDA(cudaMemcpyAsync(dloss.p + e, m.loss.p, 4, cudaMemcpyDeviceToDevice, s));
  }
  std::vector<float> hl(epochs);
  UB_CUDA(cudaMemcpyAsync(hl.data(), dloss.p, epochs * 4, cudaMemcpyDeviceToHost, s));
  check_error();
  if (losses)
    for (int e = 0; e < epochs; ++e) losses[e] = hl[e] / (float)steps;
}

void Mlp::predict(const float* X, int64_t n, float* Y) {
  Impl& m = *p;
  if (n < 1) return;
  const int64_t tile = 131072;
  m.ensure(std::min<int64_t>(tile, (n + 127) / 128 * 128), false);
  for (int64_t r0 = 0; r0 < n; r0 += tile) {
    const int64_t rows = std::min(tile, n - r0);
    const int64_t padded = (rows + 127) / 128 * 128;
    run_batch(m, X + r0 * m.in_dim, nullptr, padded, rows, nullptr, Y + r0 * m.out_dim, false, 0.0f);
  }
  check_error();
}

void Mlp::check_error() {
  unsigned e = 0;
  UB_CUDA(cudaMemcpyAsync(&e, p->err.p, 4, cudaMemcpyDeviceToHost, p->s));
  UB_CUDA(cudaStreamSynchronize(p->s));
  if (e) throw Error(CUDA, "tensor-core MMA completion wait timed out");
}

// Standalone tensor-core GEMM: C[M,N] (f32) = A[M,K] B[N,K]^T with bf16 A, B, both K-major.
// ksplit > 1 accumulates split-K partial sums into C with atomics (C must be zeroed).
void umma_gemm_f32(const void* A, const void* B, float* C, int64_t M, int64_t N, int64_t K, int ksplit,
                   cudaStream_t s) {
  prepare_all_gemms();
  if (N > (1 << 30) || K > (1 << 30)) throw Error(INVALID_ARGUMENT, "GEMM dimension too large");
  DevBuf<unsigned> err(1, s);
  UB_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
  EpiArgs ep{};
  ep.out_f32 = C;
  ep.ldo = (int)N;
  const bf16* a = static_cast<const bf16*>(A);
  const bf16* b = static_cast<const bf16*>(B);
  if (ksplit > 1) {
    if (N % 256 == 0) launch_tma_gemm<256, EPI_F32_ATOMIC>(a, K, b, K, M, N, K, ksplit, ep, err.p, s);
    else if (N % 64 == 0) launch_tma_gemm<64, EPI_F32_ATOMIC>(a, K, b, K, M, N, K, ksplit, ep, err.p, s);
    else throw Error(INVALID_ARGUMENT, "split-K GEMM needs N % 64 == 0");
  } else if (N % 256 == 0) {
    launch_tma_gemm<256, EPI_F32>(a, K, b, K, M, N, K, 1, ep, err.p, s);
  } else if (N % 128 == 0) {
    launch_tma_gemm<128, EPI_F32>(a, K, b, K, M, N, K, 1, ep, err.p, s);
  } else if (N % 64 == 0) {
    launch_tma_gemm<64, EPI_F32>(a, K, b, K, M, N, K, 1, ep, err.p, s);
  } else if (N % 32 == 0) {
    launch_tma_gemm<32, EPI_F32>(a, K, b, K, M, N, K, 1, ep, err.p, s);
  } else {
    throw Error(INVALID_ARGUMENT, "GEMM N must be a multiple of 32");
  }
  unsigned e = 0;
  UB_CUDA(cudaMemcpyAsync(&e, err.p, 4, cudaMemcpyDeviceToHost, s));
  UB_CUDA(cudaStreamSynchronize(s));
  if (e) throw Error(CUDA, "tensor-core MMA completion wait timed out");
}

}  // namespace ub
