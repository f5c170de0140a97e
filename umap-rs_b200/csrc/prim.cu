// Device-wide primitives for the graph build: exclusive scan, stable LSD radix sort of
// (u32 key, u32 value) pairs, and reductions.  Hand-written (no CUB/Thrust); every
// kernel is a plain one-pass-per-launch design with no inter-block waiting.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "ub_internal.hpp"

namespace ub {
namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ T warp_incl_scan(T v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(FULL, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// ------------------------------------------------------------------------------ scan
constexpr int SCAN_BT = 256;
constexpr int SCAN_NW = SCAN_BT / 32;
constexpr int SCAN_IPT = 16;
constexpr uint64_t SCAN_TILE = (uint64_t)SCAN_BT * SCAN_IPT;

// Per-tile sums.  Element order inside a tile: warp w owns [w*32*IPT, (w+1)*32*IPT),
// visited as i*32 + lane (coalesced).
template <class TIn, class TOut>
__global__ void __launch_bounds__(SCAN_BT) scan_tile_sums(const TIn* __restrict__ in, uint64_t n,
                                                          TOut* __restrict__ sums) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)w * 32 * SCAN_IPT;
  TOut acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_IPT; ++i) {
    uint64_t idx = base + (uint64_t)i * 32 + lane;
    if (idx < n) acc += (TOut)in[idx];
  }
  acc = warp_sum(acc);
  __shared__ TOut s_w[SCAN_NW];
  if (lane == 0) s_w[w] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    TOut t = 0;
    for (int j = 0; j < SCAN_NW; ++j) t += s_w[j];
    sums[blockIdx.x] = t;
  }
}

template <class TIn, class TOut>
__global__ void __launch_bounds__(SCAN_BT) scan_tile_apply(const TIn* __restrict__ in, uint64_t n,
                                                           const TOut* __restrict__ tile_off,
                                                           TOut* __restrict__ out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)w * 32 * SCAN_IPT;
  TOut v[SCAN_IPT];
  TOut wsum = 0;
#pragma unroll
  for (int i = 0; i < SCAN_IPT; ++i) {
    uint64_t idx = base + (uint64_t)i * 32 + lane;
    v[i] = idx < n ? (TOut)in[idx] : (TOut)0;
    wsum += v[i];
  }
  wsum = warp_sum(wsum);
  __shared__ TOut s_w[SCAN_NW];
  if (lane == 0) s_w[w] = wsum;
  __syncthreads();
  TOut carry = tile_off ? tile_off[blockIdx.x] : (TOut)0;
  for (int j = 0; j < w; ++j) carry += s_w[j];
#pragma unroll
  for (int i = 0; i < SCAN_IPT; ++i) {
    uint64_t idx = base + (uint64_t)i * 32 + lane;
    TOut inc = warp_incl_scan(v[i], lane);
    if (idx < n) out[idx] = carry + inc - v[i];
    carry += __shfl_sync(FULL, inc, 31);
  }
  if (blockIdx.x == gridDim.x - 1 && w == SCAN_NW - 1 && lane == 31) out[n] = carry;
}

template <class TIn, class TOut>
void scan_impl(const TIn* in, TOut* out, uint64_t n, cudaStream_t s) {
  if (n == 0) {
    UB_CUDA(cudaMemsetAsync(out, 0, sizeof(TOut), s));
    return;
  }
  uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (tiles == 1) {
    scan_tile_apply<TIn, TOut><<<1, SCAN_BT, 0, s>>>(in, n, nullptr, out);
    UB_LAUNCH_CHECK();
    return;
  }
  DevBuf<TOut> sums(tiles, s), offs(tiles + 1, s);
  scan_tile_sums<TIn, TOut><<<(unsigned)tiles, SCAN_BT, 0, s>>>(in, n, sums.p);
  UB_LAUNCH_CHECK();
  scan_impl<TOut, TOut>(sums.p, offs.p, tiles, s);
  scan_tile_apply<TIn, TOut><<<(unsigned)tiles, SCAN_BT, 0, s>>>(in, n, offs.p, out);
  UB_LAUNCH_CHECK();
}

// ------------------------------------------------------------------------------ radix sort
constexpr int RS_BT = 256;
constexpr int RS_NW = RS_BT / 32;
constexpr int RS_IPT = 12;
constexpr int RS_TILE = RS_BT * RS_IPT;
constexpr int RS_RADIX = 256;

// Per-tile digit histogram, stored digit-major: hist[d * tiles + tile].
__global__ void __launch_bounds__(RS_BT) radix_upsweep(const uint32_t* __restrict__ kin, uint64_t n,
                                                       int shift, uint32_t* __restrict__ hist,
                                                       uint32_t tiles) {
  __shared__ uint32_t s_h[RS_NW][RS_RADIX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < RS_NW * RS_RADIX; i += RS_BT) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll
  for (int i = 0; i < RS_IPT; ++i) {
    uint64_t idx = base + (uint64_t)i * RS_BT + threadIdx.x;
    if (idx < n) atomicAdd(&s_h[w][(kin[idx] >> shift) & 0xFF], 1u);
  }
  (void)lane;
  __syncthreads();
  for (int d = threadIdx.x; d < RS_RADIX; d += RS_BT) {
    uint32_t t = 0;
#pragma unroll
    for (int j = 0; j < RS_NW; ++j) t += s_h[j][d];
    hist[(uint64_t)d * tiles + blockIdx.x] = t;
  }
}

// Stable scatter.  Tile element order is (round i, thread t) = index i*BT + t, the input
// order; ranks inside a round come from warp match + per-warp counts, so equal digits keep
// their input order.  Output goes through shared memory so global stores are coalesced.
__global__ void __launch_bounds__(RS_BT) radix_downsweep(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, uint64_t n, int shift, const uint32_t* __restrict__ offs,
    uint32_t tiles) {
  __shared__ uint32_t s_cnt[RS_NW][RS_RADIX];
  __shared__ uint32_t s_pre[RS_NW][RS_RADIX];
  __shared__ uint32_t s_run[RS_RADIX];
  __shared__ uint32_t s_start[RS_RADIX];
  __shared__ uint32_t s_gbase[RS_RADIX];
  __shared__ uint32_t s_wtot[RS_NW];
  __shared__ uint32_t s_keys[RS_TILE];
  __shared__ uint32_t s_vals[RS_TILE];

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;

  for (int i = tid; i < RS_NW * RS_RADIX; i += RS_BT) (&s_cnt[0][0])[i] = 0;
  for (int i = tid; i < RS_RADIX; i += RS_BT) s_run[i] = 0;

  uint32_t k[RS_IPT], v[RS_IPT], pos[RS_IPT];
  int d[RS_IPT];
#pragma unroll
  for (int i = 0; i < RS_IPT; ++i) {
    uint64_t idx = base + (uint64_t)i * RS_BT + tid;
    bool valid = idx < n;
    k[i] = valid ? kin[idx] : 0u;
    v[i] = valid ? (vin ? vin[idx] : (uint32_t)idx) : 0u;
    d[i] = valid ? (int)((k[i] >> shift) & 0xFF) : RS_RADIX;
  }
  __syncthreads();

#pragma unroll
  for (int i = 0; i < RS_IPT; ++i) {
    unsigned peers = __match_any_sync(FULL, d[i]);
    int rank = __popc(peers & lt_mask);
    if (d[i] < RS_RADIX && rank == 0) s_cnt[w][d[i]] = __popc(peers);
    __syncthreads();
    for (int dd = tid; dd < RS_RADIX; dd += RS_BT) {
      uint32_t run = s_run[dd];
#pragma unroll
      for (int j = 0; j < RS_NW; ++j) {
        uint32_t c = s_cnt[j][dd];
        s_pre[j][dd] = run;
        s_cnt[j][dd] = 0;
        run += c;
      }
      s_run[dd] = run;
    }
    __syncthreads();
    pos[i] = d[i] < RS_RADIX ? s_pre[w][d[i]] + (uint32_t)rank : 0u;
  }

  // Exclusive prefix of the tile's digit totals (256 digits, 256 threads).
  uint32_t tot = tid < RS_RADIX ? s_run[tid] : 0u;
  uint32_t inc = warp_incl_scan(tot, lane);
  if (lane == 31) s_wtot[w] = inc;
  __syncthreads();
  uint32_t wo = 0;
  for (int j = 0; j < w; ++j) wo += s_wtot[j];
  if (tid < RS_RADIX) {
    s_start[tid] = wo + inc - tot;
    s_gbase[tid] = offs[(uint64_t)tid * tiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < RS_IPT; ++i) {
    if (d[i] < RS_RADIX) {
      uint32_t sp = s_start[d[i]] + pos[i];
      s_keys[sp] = k[i];
      s_vals[sp] = v[i];
    }
  }
  __syncthreads();
  const uint32_t cnt = (uint32_t)min((uint64_t)RS_TILE, n - base);
  for (uint32_t j = tid; j < cnt; j += RS_BT) {
    uint32_t key = s_keys[j];
    uint32_t dd = (key >> shift) & 0xFF;
    uint64_t dst = (uint64_t)s_gbase[dd] + (j - s_start[dd]);
    kout[dst] = key;
    vout[dst] = s_vals[j];
  }
}

// ------------------------------------------------------------------------------ reductions
constexpr int RED_BT = 256;

template <class T, class Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T ident) {
  __shared__ T s[RED_BT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(FULL, v, o));
  if (lane == 0) s[w] = v;
  __syncthreads();
  T r = ident;
  if (threadIdx.x == 0)
    for (int j = 0; j < RED_BT / 32; ++j) r = op(r, s[j]);
  return r;
}

struct MaxF { __device__ float operator()(float a, float b) const { return fmaxf(a, b); } };
struct MaxU { __device__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; } };
struct SumU64 { __device__ uint64_t operator()(uint64_t a, uint64_t b) const { return a + b; } };

template <class T, class Op>
__global__ void __launch_bounds__(RED_BT) reduce_stage(const T* __restrict__ x, uint64_t n, T ident,
                                                       T* __restrict__ out, Op op) {
  T acc = ident;
  for (uint64_t i = (uint64_t)blockIdx.x * RED_BT + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * RED_BT)
    acc = op(acc, x[i]);
  acc = block_reduce(acc, op, ident);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

template <class T, class Op>
void reduce_impl(const T* x, uint64_t n, T ident, T* out, Op op, cudaStream_t s) {
  unsigned blocks = (unsigned)std::min<uint64_t>(148 * 8, std::max<uint64_t>(1, (n + RED_BT - 1) / RED_BT));
  DevBuf<T> part(blocks, s);
  reduce_stage<T, Op><<<blocks, RED_BT, 0, s>>>(x, n, ident, part.p, op);
  UB_LAUNCH_CHECK();
  reduce_stage<T, Op><<<1, RED_BT, 0, s>>>(part.p, blocks, ident, out, op);
  UB_LAUNCH_CHECK();
}

}  // namespace

void scan_u32_to_u64(const uint32_t* in, uint64_t* out, uint64_t n, cudaStream_t s) {
  scan_impl<uint32_t, uint64_t>(in, out, n, s);
}
void scan_u64_to_u64(const uint64_t* in, uint64_t* out, uint64_t n, cudaStream_t s) {
  scan_impl<uint64_t, uint64_t>(in, out, n, s);
}

int bits_for(uint64_t v) {
  int b = 0;
  while (v) { ++b; v >>= 1; }
  return b;
}

void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                      uint32_t* vals_out, uint64_t n, int end_bit, cudaStream_t s) {
  if (n >= 0xFFFFFFFFull) throw Error(UNSUPPORTED, "radix_sort_pairs: n must be < 2^32");
  if (n == 0) return;
  if (end_bit < 1) end_bit = 1;
  if (end_bit > 32) end_bit = 32;
  const int passes = (end_bit + 7) / 8;
  const uint32_t tiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  DevBuf<uint32_t> hist((uint64_t)tiles * RS_RADIX, s), offs((uint64_t)tiles * RS_RADIX + 1, s);
  DevBuf<uint32_t> tk, tv;
  if (passes > 1) {
    tk.alloc(n, s);
    tv.alloc(n, s);
  }
  // Ping-pong so that the last pass lands in keys_out/vals_out.
  const uint32_t* ck = keys_in;
  const uint32_t* cv = vals_in;
  for (int p = 0; p < passes; ++p) {
    bool to_out = ((passes - 1 - p) % 2) == 0;
    uint32_t* nk = to_out ? keys_out : tk.p;
    uint32_t* nv = to_out ? vals_out : tv.p;
    radix_upsweep<<<tiles, RS_BT, 0, s>>>(ck, n, p * 8, hist.p, tiles);
    UB_LAUNCH_CHECK();
    scan_impl<uint32_t, uint32_t>(hist.p, offs.p, (uint64_t)tiles * RS_RADIX, s);
    radix_downsweep<<<tiles, RS_BT, 0, s>>>(ck, cv, nk, nv, n, p * 8, offs.p, tiles);
    UB_LAUNCH_CHECK();
    ck = nk;
    cv = nv;
  }
}

void reduce_max_f32(const float* x, uint64_t n, float init, float* out, cudaStream_t s) {
  if (n == 0) {
    UB_CUDA(cudaMemcpyAsync(out, &init, sizeof(float), cudaMemcpyHostToDevice, s));
    UB_CUDA(cudaStreamSynchronize(s));
    return;
  }
  reduce_impl<float, MaxF>(x, n, init, out, MaxF{}, s);
}
void reduce_max_u32(const uint32_t* x, uint64_t n, uint32_t* out, cudaStream_t s) {
  if (n == 0) {
    UB_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), s));
    return;
  }
  reduce_impl<uint32_t, MaxU>(x, n, 0u, out, MaxU{}, s);
}
void reduce_sum_u64(const uint64_t* x, uint64_t n, uint64_t* out, cudaStream_t s) {
  if (n == 0) {
    UB_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), s));
    return;
  }
  reduce_impl<uint64_t, SumU64>(x, n, (uint64_t)0, out, SumU64{}, s);
}

// ------------------------------------------------------------------------------
// Allocation-free variant of radix_sort_pairs.
//
// Some callers cannot allocate device memory at the moment they need this sort: a host
// application whose allocator owns the whole GPU heap (it reserves the device memory up
// front and a foreign cudaMalloc would fail or fragment it), or a latency-critical loop
// that must not enter the CUDA allocator at all.  For them the scratch space lives in the
// file-scope array below, sized for at most NOALLOC_MAX_PAIRS pairs (about 9 MiB).  The CUDA
// runtime places it on a GPU when it loads this file's module there (lazily: at the first
// kernel launch or symbol lookup on that device), and the GPU holds it until the process
// exits; a call with n = 0 performs that load and the address lookup.  In host code the array's
// name is only a host-side stand-in, so its device address is looked up with
// cudaGetSymbolAddress, once per device, with that device current.  Every call shares the
// array and it keeps the previous call's contents: all of it is fully rewritten before it
// is read (histograms, offsets and ping-pong buffers), so nothing needs clearing, but two
// calls whose GPU work overlaps (e.g. on different streams) race on it.
namespace {

constexpr uint64_t NOALLOC_MAX_PAIRS = 1ull << 20;
constexpr uint64_t NA_TILES = (NOALLOC_MAX_PAIRS + RS_TILE - 1) / RS_TILE;
constexpr uint64_t NA_HIST = NA_TILES * RS_RADIX;
constexpr uint64_t NA_SCAN_TILES = (NA_HIST + SCAN_TILE - 1) / SCAN_TILE;
constexpr uint64_t align256(uint64_t b) { return (b + 255) / 256 * 256; }
constexpr uint64_t NOALLOC_SCRATCH_BYTES =
    2 * align256(NOALLOC_MAX_PAIRS * 4) +          // ping-pong keys / values
    align256(NA_HIST * 4) + align256((NA_HIST + 1) * 4) +  // digit histograms / offsets
    2 * align256((NA_SCAN_TILES + 1) * 4) +        // scan tile sums / offsets
    4096;                                          // slack for the carving's alignment

static __device__ __align__(256) unsigned char g_sort_scratch[NOALLOC_SCRATCH_BYTES];

// Bump allocator over the scratch array (device address).
struct Carve {
  unsigned char* p;
  uint64_t left;
  template <class T>
  T* take(uint64_t count) {
    const uint64_t bytes = align256(count * sizeof(T));
    if (bytes > left) throw Error(INVALID_ARGUMENT, "allocation-free sort: scratch exhausted");
    T* r = reinterpret_cast<T*>(p);
    p += bytes;
    left -= bytes;
    return r;
  }
};

template <class TIn, class TOut>
void scan_carved(const TIn* in, TOut* out, uint64_t n, cudaStream_t s, Carve& c) {
  if (n == 0) {
    UB_CUDA(cudaMemsetAsync(out, 0, sizeof(TOut), s));
    return;
  }
  const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (tiles == 1) {
    scan_tile_apply<TIn, TOut><<<1, SCAN_BT, 0, s>>>(in, n, nullptr, out);
    UB_LAUNCH_CHECK();
    return;
  }
  TOut* sums = c.take<TOut>(tiles);
  TOut* offs = c.take<TOut>(tiles + 1);
  scan_tile_sums<TIn, TOut><<<(unsigned)tiles, SCAN_BT, 0, s>>>(in, n, sums);
  UB_LAUNCH_CHECK();
  scan_carved<TOut, TOut>(sums, offs, tiles, s, c);
  scan_tile_apply<TIn, TOut><<<(unsigned)tiles, SCAN_BT, 0, s>>>(in, n, offs, out);
  UB_LAUNCH_CHECK();
}

// Device address of g_sort_scratch on the current device (looked up once per device).
unsigned char* sort_scratch_address() {
  static std::mutex mu;
  static unsigned char* addr[256] = {};
  int dev = 0;
  UB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) throw Error(UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      throw Error(CUDA, std::string("cudaGetSymbolAddress(sort scratch) failed: ") + cudaGetErrorString(e));
    }
    addr[dev] = static_cast<unsigned char*>(p);
  }
  return addr[dev];
}

}  // namespace

uint64_t radix_sort_noalloc_max_pairs() { return NOALLOC_MAX_PAIRS; }

void radix_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                              uint32_t* vals_out, uint64_t n, int end_bit, cudaStream_t s) {
  if (n > NOALLOC_MAX_PAIRS)
    throw Error(INVALID_ARGUMENT, "allocation-free radix sort takes at most " + std::to_string(NOALLOC_MAX_PAIRS) +
                                      " pairs, got " + std::to_string(n));
  unsigned char* base = sort_scratch_address();
  if (n == 0) return;
  if (end_bit < 1) end_bit = 1;
  if (end_bit > 32) end_bit = 32;
  Carve c{base, NOALLOC_SCRATCH_BYTES};
  const int passes = (end_bit + 7) / 8;
  const uint32_t tiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  uint32_t* tk = c.take<uint32_t>(NOALLOC_MAX_PAIRS);
  uint32_t* tv = c.take<uint32_t>(NOALLOC_MAX_PAIRS);
  uint32_t* hist = c.take<uint32_t>((uint64_t)tiles * RS_RADIX);
  uint32_t* offs = c.take<uint32_t>((uint64_t)tiles * RS_RADIX + 1);
  const uint32_t* ck = keys_in;
  const uint32_t* cv = vals_in;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    uint32_t* nk = to_out ? keys_out : tk;
    uint32_t* nv = to_out ? vals_out : tv;
    radix_upsweep<<<tiles, RS_BT, 0, s>>>(ck, n, p * 8, hist, tiles);
    UB_LAUNCH_CHECK();
    Carve scan_ws = c;  // the scan's temporaries are reused by every pass
    scan_carved<uint32_t, uint32_t>(hist, offs, (uint64_t)tiles * RS_RADIX, s, scan_ws);
    radix_downsweep<<<tiles, RS_BT, 0, s>>>(ck, cv, nk, nv, n, p * 8, offs, tiles);
    UB_LAUNCH_CHECK();
    ck = nk;
    cv = nv;
  }
}

}  // namespace ub
