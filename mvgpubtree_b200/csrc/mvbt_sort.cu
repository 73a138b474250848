// Stable LSD radix sort of 32-bit keys with 32-bit payloads, hand-written for sm_100a: the sort
// stage of the sorted batch front-end (mvbt_sort.h). The payload of each key is its position in
// the caller's array, generated by the first pass.
//
// A pass over one 8-bit digit is three steps:
//   k_sort_hist     per tile of 4096 keys, the count of each digit value (shared-memory counters),
//                   stored digit-major: counts[d * tiles + tile];
//   scan            an exclusive prefix over those counts (reduce / top / down-sweep kernels),
//                   which gives every (digit, tile) run its first output position;
//   k_sort_scatter  per tile, the stable rank of every key among the keys of its digit (rounds of
//                   256 keys in input order; inside a warp __match_any_sync finds the lanes with the
//                   same digit), the tile reordered by digit in shared memory, then written out so
//                   that consecutive threads write consecutive positions of one digit's run.
// All traffic is streaming and coalesced (HBM-bound): per pass the keys are read twice and the
// keys and payloads read and written once. Passes over the low digits can be skipped when only
// locality is needed (a bucketing by the top bits).
#include <cuda_runtime.h>

#include <cstdint>

#include "mvbt_sort.h"

namespace {

constexpr int kThreads = 256;
constexpr int kItems   = 16;
constexpr int kTile    = kThreads * kItems;  // keys per tile
constexpr int kWarps   = kThreads / 32;
constexpr int kScanThreads = 1024;
constexpr int kScanItems   = 4;
constexpr int kScanChunk   = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kThreads) k_sort_hist(const uint32_t* __restrict__ keys, uint32_t n, int shift,
                                                        uint32_t tiles, uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
#pragma unroll 4
  for (int r = 0; r < kItems; ++r) {
    const uint64_t i = base + (uint64_t)r * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of 1024 threads x kScanItems values held per thread; returns the block total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t (&v)[kScanItems], uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint32_t x = v[j];
    v[j]             = sum;
    sum += x;
  }
  uint32_t inc = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = s_warp[lane], wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= d) wi += y;
    }
    s_warp[lane] = wi - w;  // exclusive prefix of warp totals
    if (lane == 31) s_warp[32] = wi;
  }
  __syncthreads();
  const uint32_t off = s_warp[warp] + inc - sum;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) v[j] += off;
  const uint32_t total = s_warp[32];
  __syncthreads();
  return total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ a, uint64_t n,
                                                              uint32_t* __restrict__ sums) {
  __shared__ uint32_t s[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = base + (uint64_t)j * kScanThreads + threadIdx.x;
    if (i < n) x += a[i];
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t y = s[threadIdx.x];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) y += __shfl_down_sync(0xffffffffu, y, d);
    if (threadIdx.x == 0) sums[blockIdx.x] = y;
  }
}

// One block: exclusive scan of the block sums in place (any count, in chunks with a carry).
__global__ void __launch_bounds__(kScanThreads) k_scan_top(uint32_t* __restrict__ sums, uint32_t n) {
  __shared__ uint32_t s_warp[33];
  uint32_t carry = 0;
  for (uint32_t base = 0; base < n; base += kScanChunk) {
    uint32_t v[kScanItems];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
      const uint32_t i = base + threadIdx.x * kScanItems + j;
      v[j]             = i < n ? sums[i] : 0u;
    }
    const uint32_t total = block_exclusive_scan(v, s_warp);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
      const uint32_t i = base + threadIdx.x * kScanItems + j;
      if (i < n) sums[i] = v[j] + carry;
    }
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(uint32_t* __restrict__ a, uint64_t n,
                                                            const uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_warp[33];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) v[j] = base + j < n ? a[base + j] : 0u;
  block_exclusive_scan(v, s_warp);
  const uint32_t off = sums[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) a[base + j] = v[j] + off;
}

// Stable scatter of one tile by the digit at `shift`. vin == nullptr: the payload is the key's
// input position (first pass).
__global__ void __launch_bounds__(kThreads) k_sort_scatter(const uint32_t* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin,
                                                           uint32_t* __restrict__ kout,
                                                           uint32_t* __restrict__ vout, uint32_t n, int shift,
                                                           uint32_t tiles, const uint32_t* __restrict__ offs) {
  __shared__ uint16_t s_cnt[kWarps][256];   // keys of each digit in each warp, this round
  __shared__ uint16_t s_pre[kWarps][256];   // their exclusive prefix (earlier rounds and warps)
  __shared__ uint32_t s_run[256];           // keys of each digit in the rounds so far
  __shared__ uint32_t s_start[256];         // tile-local first position of each digit
  __shared__ uint32_t s_glob[256];          // global first position of each digit's run
  __shared__ uint32_t s_warp[kWarps];
  __shared__ uint32_t s_keys[kTile];
  __shared__ uint32_t s_vals[kTile];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  s_run[tid]  = 0;
  s_glob[tid] = offs[(uint64_t)tid * tiles + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kWarps; ++w) s_cnt[w][tid] = 0;
  __syncthreads();
  uint32_t k[kItems], v[kItems], rank[kItems];
  const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const uint64_t i = base + (uint64_t)r * kThreads + tid;
    const bool ok    = i < n;
    k[r]             = ok ? kin[i] : 0u;
    v[r]             = ok ? (vin ? vin[i] : (uint32_t)i) : 0u;
    const uint32_t d = (k[r] >> shift) & 255u;
    const uint32_t peers = __match_any_sync(0xffffffffu, ok ? d : (0x100u | (uint32_t)lane));
    const uint32_t in_warp = __popc(peers & lt_mask);
    if (ok && (peers & lt_mask) == 0) s_cnt[warp][d] = (uint16_t)__popc(peers);
    __syncthreads();
    {  // thread tid owns digit tid: prefix over the warps of this round, cleared for the next
      uint32_t run = s_run[tid];
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = s_cnt[w][tid];
        s_cnt[w][tid]    = 0;
        s_pre[w][tid]    = (uint16_t)run;
        run += c;
      }
      s_run[tid] = run;
    }
    __syncthreads();
    rank[r] = ok ? (uint32_t)s_pre[warp][d] + in_warp : 0u;
  }
  // tile-local start of each digit: exclusive scan of s_run over the 256 digits
  {
    const uint32_t c = s_run[tid];
    uint32_t inc     = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t off = 0;
    for (int w = 0; w < warp; ++w) off += s_warp[w];
    s_start[tid] = off + inc - c;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const uint64_t i = base + (uint64_t)r * kThreads + tid;
    if (i < n) {
      const uint32_t d  = (k[r] >> shift) & 255u;
      const uint32_t lp = s_start[d] + rank[r];
      s_keys[lp]        = k[r];
      s_vals[lp]        = v[r];
    }
  }
  __syncthreads();
  const uint32_t in_tile = (uint32_t)((n - base) < (uint64_t)kTile ? (n - base) : (uint64_t)kTile);
  for (uint32_t j = tid; j < in_tile; j += kThreads) {
    const uint32_t kk = s_keys[j];
    const uint32_t d  = (kk >> shift) & 255u;
    const uint32_t g  = s_glob[d] + (j - s_start[d]);
    kout[g]           = kk;
    vout[g]           = s_vals[j];
  }
}

int launch_error() {
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

namespace mvbt_sort {

uint64_t scratch_words(uint32_t n) {
  const uint64_t tiles  = ((uint64_t)n + kTile - 1) / kTile;
  const uint64_t counts = tiles * 256;
  const uint64_t sums   = (counts + kScanChunk - 1) / kScanChunk;
  return counts + sums + 64;
}

uint64_t scan_scratch_words(uint64_t n) { return (n + kScanChunk - 1) / kScanChunk + 64; }

int exclusive_scan(uint32_t* a, uint64_t n, uint32_t* sums, cudaStream_t s) {
  if (n == 0) return 0;
  const uint32_t chunks = (uint32_t)((n + kScanChunk - 1) / kScanChunk);
  k_scan_reduce<<<chunks, kScanThreads, 0, s>>>(a, n, sums);
  k_scan_top<<<1, kScanThreads, 0, s>>>(sums, chunks);
  k_scan_down<<<chunks, kScanThreads, 0, s>>>(a, n, sums);
  return launch_error() ? 2 : 0;
}

int sort_pairs(const uint32_t* keys, uint32_t n, int low_bit, uint32_t* k_out, uint32_t* v_out, uint32_t* k_tmp,
               uint32_t* v_tmp, uint32_t* scratch, cudaStream_t s) {
  if (n == 0) return 0;
  if (low_bit < 0 || low_bit > 24 || (low_bit & 7)) return 1;
  const uint32_t tiles  = (uint32_t)(((uint64_t)n + kTile - 1) / kTile);
  const uint64_t counts = (uint64_t)tiles * 256;
  const uint32_t chunks = (uint32_t)((counts + kScanChunk - 1) / kScanChunk);
  uint32_t* cnt         = scratch;
  uint32_t* sums        = scratch + counts;
  const int passes      = (32 - low_bit) / 8;
  const uint32_t* kin   = keys;
  const uint32_t* vin   = nullptr;
  for (int p = 0; p < passes; ++p) {
    // the last pass lands in k_out / v_out; earlier ones alternate so that it does
    const bool to_out = ((passes - 1 - p) & 1) == 0;
    uint32_t* ko      = to_out ? k_out : k_tmp;
    uint32_t* vo      = to_out ? v_out : v_tmp;
    const int shift   = low_bit + 8 * p;
    k_sort_hist<<<tiles, kThreads, 0, s>>>(kin, n, shift, tiles, cnt);
    k_scan_reduce<<<chunks, kScanThreads, 0, s>>>(cnt, counts, sums);
    k_scan_top<<<1, kScanThreads, 0, s>>>(sums, chunks);
    k_scan_down<<<chunks, kScanThreads, 0, s>>>(cnt, counts, sums);
    k_sort_scatter<<<tiles, kThreads, 0, s>>>(kin, vin, ko, vo, n, shift, tiles, cnt);
    if (launch_error()) return 2;
    kin = ko;
    vin = vo;
  }
  return 0;
}

}  // namespace mvbt_sort
