// Shared pieces of the tensor-core kernels (tcgen05 MMA fed by TMA, accumulators in tensor
// memory): shared-memory and instruction descriptors, bounded mbarrier waits, and the host
// side tensor-map encoder for row-major BF16 matrices.
#pragma once

#include <cuda.h>  // CUtensorMap and its enums; the encoder is fetched from the runtime
#include <cuda_runtime.h>

#include <cstdint>

namespace ub {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// K-major, 128-byte-swizzled shared-memory matrix descriptor (layout type 2): rows of 128 B
// (64 bf16) with 16-byte chunks XOR-swizzled by row % 8, 8-row atoms 1024 B apart (stride
// byte offset), leading byte offset unused (16 B); the tile starts 1024-byte aligned and
// K step s (16 bf16 = 32 B) is addressed by advancing the start address 32 B.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// Instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9 and 10-12
// = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// The same with A and B FP16 (format 0 in bits 7-9 and 10-12).
__host__ __device__ constexpr uint32_t instr_desc_f16(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for an mbarrier phase; gives up after about two seconds.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
    if ((it & 255u) == 255u && global_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}

// Programmatic dependent launch.  `grid_wait` returns once every grid this launch depends on
// has completed and its memory is visible (a no-op for a launch without the attribute); a
// kernel reads and writes no global memory, and allocates no tensor memory, before it.
// `grid_release` lets the dependent launch be scheduled once every CTA of this grid has
// executed it (or exited); the dependent's own `grid_wait` still waits for this grid's end.
__device__ __forceinline__ void grid_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace umma

// Tensor map of a row-major bf16 (or, with f16, fp16) matrix [rows, cols] (row stride ld
// elements) read in boxes of box_rows x 64 with 128-byte swizzle (defined in mlp.cu).
CUtensorMap bf16_tile_map(const void* base, int64_t rows, int64_t cols, int64_t ld, int box_rows, bool f16 = false);

}  // namespace ub
