// Compact range output: packs the pairs of a batch run's range queries, first min(count, cap)
// of each query in op order, so a caller copies only the pairs that exist rather than whole
// fixed-size slots. Query i's pairs start at the sum of min(count, cap) over the range queries
// before it, which the caller recomputes from the counts it reads anyway.
//
// Three kernels: per tile of 8192 ops, each op's pair count and its exclusive offset within the
// tile (and the tile total); one block scanning the tile totals into tile offsets (and the grand
// total); one warp per range query copying its pairs (8-byte lanes, coalesced).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "mvbt.h"

extern "C" void mvbt_internal_set_error(const char* msg);
extern "C" void* mvbt_internal_plan_scratch(mvbt_batch_plan* p, uint64_t bytes);
extern "C" uint64_t mvbt_internal_plan_max_ops(mvbt_batch_plan* p);

namespace {

constexpr int kThreads = 1024;
constexpr int kItems   = 8;
constexpr uint64_t kTile = (uint64_t)kThreads * kItems;

int fail(int code, const std::string& msg) {
  mvbt_internal_set_error(msg.c_str());
  return code;
}

__device__ __forceinline__ uint32_t pairs_of(const uint32_t* type, const uint32_t* result, const uint32_t* cap,
                                             uint64_t i, uint64_t n) {
  if (i >= n || type[i] != MVBT_OP_RANGE) return 0u;
  return min(result[i], cap[i]);
}

// Inclusive scan of x over a warp.
__device__ __forceinline__ uint64_t warp_inclusive(uint64_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= d) x += y;
  }
  return x;
}

__global__ void __launch_bounds__(kThreads) k_scan_tiles(const uint32_t* type, const uint32_t* result,
                                                         const uint32_t* cap, uint64_t n, uint64_t* off,
                                                         uint64_t* tile_sum) {
  __shared__ uint64_t warp_sum[32];
  const uint64_t base = blockIdx.x * kTile + (uint64_t)threadIdx.x * kItems;
  uint32_t v[kItems];
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    v[k] = pairs_of(type, result, cap, base + k, n);
    s += v[k];
  }
  const uint64_t incl = warp_inclusive(s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) warp_sum[lane] = warp_inclusive(warp_sum[lane]);
  __syncthreads();
  uint64_t run = incl - s + (warp ? warp_sum[warp - 1] : 0ull);
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    if (base + k < n) off[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == kThreads - 1) tile_sum[blockIdx.x] = run;
}

// One block: tile totals -> exclusive tile offsets, grand total to *total.
__global__ void __launch_bounds__(kThreads) k_scan_tile_sums(uint64_t* tile_sum, uint64_t tiles,
                                                             unsigned long long* total) {
  __shared__ uint64_t warp_sum[32];
  __shared__ uint64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t b = 0; b < tiles; b += kThreads) {
    const uint64_t i = b + threadIdx.x;
    const uint64_t s = i < tiles ? tile_sum[i] : 0ull;
    const uint64_t incl = warp_inclusive(s);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) warp_sum[lane] = warp_inclusive(warp_sum[lane]);
    __syncthreads();
    const uint64_t excl = carry + incl - s + (warp ? warp_sum[warp - 1] : 0ull);
    if (i < tiles) tile_sum[i] = excl;
    __syncthreads();
    if (threadIdx.x == kThreads - 1) carry = excl + s;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(256) k_compact_copy(const uint32_t* type, const uint32_t* result,
                                                      const uint32_t* cap, const uint64_t* out_off,
                                                      const uint2* range_out, uint64_t n, const uint64_t* off,
                                                      const uint64_t* tile_off, uint2* compact) {
  const uint32_t lane  = threadIdx.x & 31u;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    if (type[i] != MVBT_OP_RANGE) continue;
    const uint32_t c = min(result[i], cap[i]);
    const uint64_t d = off[i] + tile_off[i / kTile];
    const uint2* src = range_out + out_off[i];
    for (uint32_t j = lane; j < c; j += 32) compact[d + j] = src[j];
  }
}

}  // namespace

extern "C" int mvbt_batch_compact_ranges(mvbt_batch_plan* plan, uint64_t n, const uint32_t* type,
                                         const uint32_t* result, const uint64_t* out_off,
                                         const uint32_t* range_cap, const mvbt_pair* range_out,
                                         mvbt_pair* compact, uint64_t* total, void* stream) {
  if (!plan || !total) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n && (!type || !result || !out_off || !range_cap || !range_out || !compact))
    return fail(MVBT_ERR_BAD_ARG, "null array");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (n == 0) {
    cudaError_t e = cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
    return e == cudaSuccess ? MVBT_OK : fail(MVBT_ERR_CUDA, cudaGetErrorString(e));
  }
  const uint64_t tiles = (n + kTile - 1) / kTile;
  // Scratch for the most ops the plan holds, so it is allocated once, by the first call: growing
  // it later reallocates after a device-wide synchronisation, which would stall a pipelined
  // caller on every step larger than the ones before.
  const uint64_t cap_n     = std::max<uint64_t>(n, mvbt_internal_plan_max_ops(plan));
  const uint64_t cap_tiles = (cap_n + kTile - 1) / kTile;
  auto* scratch = static_cast<uint64_t*>(mvbt_internal_plan_scratch(plan, (cap_n + cap_tiles) * sizeof(uint64_t)));
  if (!scratch) return fail(MVBT_ERR_OUT_OF_MEMORY, "compact ranges: scratch allocation failed");
  uint64_t* off      = scratch;
  uint64_t* tile_sum = scratch + n;
  k_scan_tiles<<<(unsigned)tiles, kThreads, 0, s>>>(type, result, range_cap, n, off, tile_sum);
  k_scan_tile_sums<<<1, kThreads, 0, s>>>(tile_sum, tiles, reinterpret_cast<unsigned long long*>(total));
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)std::min<uint64_t>((n * 32 + 255) / 256, (uint64_t)sms * 16);
  k_compact_copy<<<grid, 256, 0, s>>>(type, result, range_cap, out_off, reinterpret_cast<const uint2*>(range_out), n,
                                      off, tile_sum, reinterpret_cast<uint2*>(compact));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MVBT_OK : fail(MVBT_ERR_CUDA, std::string("compact ranges: ") + cudaGetErrorString(e));
}
