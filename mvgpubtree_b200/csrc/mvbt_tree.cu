// Bulk kernels and the C ABI of the B200 multiversion B-link tree.
//
// Each bulk call maps one operation to one W-thread tile (W = 8 or 16) and runs a grid-stride
// loop over a grid sized to full occupancy, so every SM keeps as many independent root-to-leaf
// traversals in flight as its registers allow. The reference maps one op to one thread and lets
// each 16-thread tile drain its 16 ops serially (include/btree_kernels.hpp:535-574); here the
// hardware scheduler interleaves the tiles instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mvbt.h"
#include "mvbt_device.cuh"

namespace cg = cooperative_groups;
using mvbt::control_block;
using mvbt::device_tree;

struct mvbt_tree {
  int kind;
  int device;
  int tile_width;
  int block_size;
  uint64_t capacity;  // nodes
  uint32_t* pool;
  control_block* ctl;
  uint32_t* d_words;  // device scratch: [0] snapshot id of the last internal snapshot
  uint32_t* h_word;   // pinned host word
  int num_sms;
  uint32_t spin_limit;
  uint32_t chunk;
  device_tree view() const {
    device_tree t;
    t.pool      = pool;
    t.ctl       = ctl;
    t.versioned = kind == MVBT_KIND_VERSIONED ? 1u : 0u;
    t.capacity  = (uint32_t)capacity;
    return t;
  }
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define MVBT_CUDA_TRY(expr)                                                                     \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ----------------------------------------------------------------------------------------------
// Kernels
// ----------------------------------------------------------------------------------------------
__global__ void k_init(uint32_t* pool, control_block* c, uint32_t capacity, uint32_t chunk,
                       uint32_t spin_limit, uint32_t wait_ns) {
  const int t = threadIdx.x;
  if (t < 32) {
    // root leaf: {0,0} tombstone, empty pairs, high = MAX, no sibling, ts 0, no older, level 0
    uint32_t w;
    if (t == 0 || t == 1) w = 0u;
    else if (t < 28) w = mvbt::kEmptyKey;
    else if (t == 28) w = mvbt::kEmptyKey;  // high key
    else if (t == 29) w = mvbt::kNone;      // link
    else if (t == 30) w = 0u;               // ts
    else w = mvbt::kNone;                   // older | level 0
    pool[t] = w;
  }
  if (t == 0) {
    c->epoch         = 0;
    c->error         = 0;
    c->bump          = 1;
    c->capacity      = capacity;
    c->chunk         = chunk;
    c->spin_limit    = spin_limit;
    c->wait_ns       = wait_ns;
    c->reserved      = 0;
    c->stat_cow      = 0;
    c->stat_split    = 0;
    c->stat_restart  = 0;
    c->stat_reserved = 0;
  }
  for (int i = t; i < mvbt::kMaxSmSlots; i += blockDim.x) c->sm_pool[i] = chunk;  // "used == chunk": refill first
}

__global__ void k_snapshot(control_block* c, uint32_t* out) {
  if (threadIdx.x == 0) {
    __threadfence();
    uint32_t s = atomicAdd(&c->epoch, 1u);
    *out       = s;
  }
}

template <int W>
__device__ __forceinline__ uint64_t first_tile() {
  return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / W;
}
template <int W>
__device__ __forceinline__ uint64_t num_tiles() {
  return ((uint64_t)gridDim.x * blockDim.x) / W;
}

template <int W, bool kStrong>
__global__ void __launch_bounds__(256) k_find(device_tree T, const uint32_t* __restrict__ keys,
                                              uint32_t* __restrict__ out, uint32_t n, uint32_t ts) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); i < n; i += num_tiles<W>()) {
    uint32_t key = keys[i];
    uint32_t v   = T.cooperative_find<W>(key, tile, ts, kStrong);
    if (tile.thread_rank() == 0) out[i] = v;
  }
}

template <int W>
__global__ void __launch_bounds__(256) k_insert(device_tree T, const uint32_t* __restrict__ keys,
                                                const uint32_t* __restrict__ values, uint32_t n) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); i < n; i += num_tiles<W>()) {
    uint32_t key = keys[i], value = values[i];
    uint32_t E   = T.versioned ? T.current_epoch() : 0u;
    T.cooperative_insert<W>(key, value, tile, E);
  }
}

template <int W>
__global__ void __launch_bounds__(256) k_erase(device_tree T, const uint32_t* __restrict__ keys,
                                               uint32_t n) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); i < n; i += num_tiles<W>()) {
    uint32_t key = keys[i];
    uint32_t E   = T.versioned ? T.current_epoch() : 0u;
    T.cooperative_erase<W>(key, tile, E);
  }
}

template <int W, bool kStrong>
__global__ void __launch_bounds__(256) k_range(device_tree T, const uint32_t* __restrict__ lower,
                                               const uint32_t* __restrict__ upper, uint2* result,
                                               uint32_t* counts, uint32_t avg_len, uint32_t n,
                                               uint32_t ts) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); i < n; i += num_tiles<W>()) {
    uint32_t lo = lower[i], hi = upper[i];
    uint2* out  = result ? result + i * (uint64_t)avg_len : nullptr;
    uint32_t c  = T.cooperative_range_query<W>(lo, hi, tile, ts, out, avg_len, kStrong);
    if (counts && tile.thread_rank() == 0) counts[i] = c;
  }
}

// Op i of the mixed kernels: inserts are spread evenly over the op index space
// (Bresenham split), so inserts and queries run side by side in every wave.
__device__ __forceinline__ bool split_op(uint64_t i, uint64_t n_a, uint64_t total, uint64_t& a_idx,
                                         uint64_t& b_idx) {
  uint64_t a = (i * n_a) / total, b = ((i + 1) * n_a) / total;
  a_idx      = a;
  b_idx      = i - a;
  return b > a;
}

template <int W>
__global__ void __launch_bounds__(256)
    k_insert_range(device_tree T, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ values,
                   uint32_t n_ins, const uint32_t* __restrict__ lower, const uint32_t* __restrict__ upper,
                   uint32_t n_rq, uint2* result, uint32_t avg_len, uint32_t* counts,
                   const uint32_t* snap_word) {
  auto tile            = cg::tiled_partition<W>(cg::this_thread_block());
  const bool ver       = T.versioned != 0;
  const uint32_t S     = ver ? mvbt::ld_relaxed_u32(snap_word) : mvbt::kLatest;
  const uint32_t E     = ver ? S + 1 : 0u;
  const uint64_t total = (uint64_t)n_ins + n_rq;
  for (uint64_t i = first_tile<W>(); i < total; i += num_tiles<W>()) {
    uint64_t a, r;
    if (split_op(i, n_ins, total, a, r)) {
      T.cooperative_insert<W>(keys[a], values[a], tile, E);
    } else {
      uint2* out = result ? result + r * (uint64_t)avg_len : nullptr;
      uint32_t c = T.cooperative_range_query<W>(lower[r], upper[r], tile, S, out, avg_len, true);
      if (counts && tile.thread_rank() == 0) counts[r] = c;
    }
  }
}

template <int W>
__global__ void __launch_bounds__(256)
    k_find_erase(device_tree T, const uint32_t* __restrict__ fkeys, uint32_t* __restrict__ fres,
                 uint32_t n_find, const uint32_t* __restrict__ ekeys, uint32_t n_erase,
                 const uint32_t* snap_word) {
  auto tile            = cg::tiled_partition<W>(cg::this_thread_block());
  const bool ver       = T.versioned != 0;
  const uint32_t S     = ver ? mvbt::ld_relaxed_u32(snap_word) : mvbt::kLatest;
  const uint32_t E     = ver ? S + 1 : 0u;
  const uint64_t total = (uint64_t)n_find + n_erase;
  for (uint64_t i = first_tile<W>(); i < total; i += num_tiles<W>()) {
    uint64_t e, f;
    if (split_op(i, n_erase, total, e, f)) {
      T.cooperative_erase<W>(ekeys[e], tile, E);
    } else {
      uint32_t v = T.cooperative_find<W>(fkeys[f], tile, S, true);
      if (tile.thread_rank() == 0) fres[f] = v;
    }
  }
}

// ----------------------------------------------------------------------------------------------
// Launch helpers
// ----------------------------------------------------------------------------------------------
template <class K>
unsigned grid_for(const mvbt_tree* t, K kernel, uint64_t ops) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, t->block_size, 0);
  if (per_sm < 1) per_sm = 1;
  uint64_t tiles_per_block = (uint64_t)t->block_size / t->tile_width;
  uint64_t need            = (ops + tiles_per_block - 1) / tiles_per_block;
  uint64_t cap             = (uint64_t)per_sm * t->num_sms;
  uint64_t g               = std::min<uint64_t>(std::max<uint64_t>(need, 1), cap);
  return (unsigned)g;
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MVBT_OK;
}

int status_from_bits(uint32_t bits) {
  if (bits & mvbt::kErrPoolExhausted) return MVBT_ERR_POOL_EXHAUSTED;
  if (bits & mvbt::kErrSpinLimit) return MVBT_ERR_SPIN_LIMIT;
  if (bits & (mvbt::kErrCorrupt | mvbt::kErrStepLimit)) return MVBT_ERR_CORRUPT;
  return MVBT_OK;
}

// ----------------------------------------------------------------------------------------------
// Host structural walk over a pool image (the counterpart of validate_tree_structure)
// ----------------------------------------------------------------------------------------------
struct host_node {
  const uint32_t* w;
  uint32_t key(int p) const { return w[2 * p]; }
  uint32_t val(int p) const { return w[2 * p + 1]; }
  uint32_t high() const { return w[28]; }
  uint32_t link() const { return w[29]; }
  uint32_t ts() const { return w[30]; }
  uint32_t level() const { return w[31] >> 28; }
  uint32_t older() const { return w[31] & mvbt::kIndexMask; }
  uint32_t sibling() const { return w[29] & mvbt::kIndexMask; }
};

}  // namespace

// ================================================================================================
// C ABI
// ================================================================================================
extern "C" {

void mvbt_config_init(mvbt_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->pool_bytes  = 4ull << 30;
  cfg->device      = -1;
  cfg->tile_width  = 8;
  cfg->block_size  = 256;
  cfg->spin_limit  = 1u << 20;
  cfg->chunk_nodes = 64;
}

const char* mvbt_last_error(void) { return g_last_error.c_str(); }

const char* mvbt_status_string(int s) {
  switch (s) {
    case MVBT_OK: return "ok";
    case MVBT_ERR_BAD_ARG: return "bad argument";
    case MVBT_ERR_CUDA: return "CUDA error";
    case MVBT_ERR_POOL_EXHAUSTED: return "node pool exhausted";
    case MVBT_ERR_SPIN_LIMIT: return "bounded wait gave up";
    case MVBT_ERR_CORRUPT: return "structural invariant failed";
    case MVBT_ERR_NOT_SUPPORTED: return "not supported for this tree kind";
    case MVBT_ERR_OUT_OF_MEMORY: return "out of device memory";
    default: return "unknown status";
  }
}

int mvbt_create(int kind, const mvbt_config* cfg_in, mvbt_tree** out) {
  if (!out) return fail(MVBT_ERR_BAD_ARG, "out is null");
  *out = nullptr;
  if (kind != MVBT_KIND_BLINK && kind != MVBT_KIND_VERSIONED) return fail(MVBT_ERR_BAD_ARG, "bad tree kind");
  mvbt_config cfg;
  mvbt_config_init(&cfg);
  if (cfg_in) {
    cfg = *cfg_in;
    if (cfg.pool_bytes == 0) cfg.pool_bytes = 4ull << 30;
    if (cfg.tile_width == 0) cfg.tile_width = 8;
    if (cfg.block_size == 0) cfg.block_size = 256;
    if (cfg.spin_limit == 0) cfg.spin_limit = 1u << 20;
    if (cfg.chunk_nodes == 0) cfg.chunk_nodes = 64;
  }
  if (cfg.tile_width != 8 && cfg.tile_width != 16) return fail(MVBT_ERR_BAD_ARG, "tile_width must be 8 or 16");
  if (cfg.block_size < 32 || cfg.block_size > 256 || cfg.block_size % 32)
    return fail(MVBT_ERR_BAD_ARG, "block_size must be a multiple of 32 in [32, 256]");
  uint64_t capacity = cfg.pool_bytes / 128;
  if (capacity < 1024) return fail(MVBT_ERR_BAD_ARG, "pool too small");
  if (capacity > mvbt::kNone) capacity = mvbt::kNone;  // 28-bit node indices

  int dev = cfg.device;
  if (dev < 0) MVBT_CUDA_TRY(cudaGetDevice(&dev));
  MVBT_CUDA_TRY(cudaSetDevice(dev));

  auto* t       = new mvbt_tree();
  t->kind       = kind;
  t->device     = dev;
  t->tile_width = cfg.tile_width;
  t->block_size = cfg.block_size;
  t->capacity   = capacity;
  t->spin_limit = cfg.spin_limit;
  t->chunk      = cfg.chunk_nodes;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) {
    delete t;
    return fail(MVBT_ERR_CUDA, cudaGetErrorString(e));
  }
  t->num_sms = prop.multiProcessorCount;
  if (cudaMalloc(&t->pool, capacity * 128) != cudaSuccess) {
    cudaGetLastError();
    delete t;
    return fail(MVBT_ERR_OUT_OF_MEMORY, "cudaMalloc of the node pool failed");
  }
  if (cudaMalloc(&t->ctl, sizeof(control_block)) != cudaSuccess ||
      cudaMalloc(&t->d_words, 64) != cudaSuccess || cudaMallocHost(&t->h_word, 64) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(t->pool);
    delete t;
    return fail(MVBT_ERR_OUT_OF_MEMORY, "cudaMalloc of the control block failed");
  }
  k_init<<<1, 256>>>(t->pool, t->ctl, (uint32_t)capacity, t->chunk, t->spin_limit, 50u * 1000u * 1000u);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    mvbt_destroy(t);
    return fail(MVBT_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
  }
  *out = t;
  return MVBT_OK;
}

int mvbt_destroy(mvbt_tree* t) {
  if (!t) return MVBT_OK;
  cudaSetDevice(t->device);
  cudaDeviceSynchronize();
  if (t->pool) cudaFree(t->pool);
  if (t->ctl) cudaFree(t->ctl);
  if (t->d_words) cudaFree(t->d_words);
  if (t->h_word) cudaFreeHost(t->h_word);
  delete t;
  return MVBT_OK;
}

int mvbt_get_info(mvbt_tree* t, int* kind, int* tile_width, int* device) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  if (kind) *kind = t->kind;
  if (tile_width) *tile_width = t->tile_width;
  if (device) *device = t->device;
  return MVBT_OK;
}

int mvbt_insert(mvbt_tree* t, const uint32_t* keys, const uint32_t* values, uint32_t n, void* stream,
                int in_place) {
  (void)in_place;  // both reference variants keep every snapshot-visible version
  if (!t || (n && (!keys || !values))) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n == 0) return MVBT_OK;
  cudaStream_t s = as_stream(stream);
  if (t->tile_width == 8) {
    k_insert<8><<<grid_for(t, k_insert<8>, n), t->block_size, 0, s>>>(t->view(), keys, values, n);
  } else {
    k_insert<16><<<grid_for(t, k_insert<16>, n), t->block_size, 0, s>>>(t->view(), keys, values, n);
  }
  return check_launch();
}

int mvbt_find(mvbt_tree* t, const uint32_t* keys, uint32_t* values, uint32_t n, uint32_t ts,
              void* stream, int concurrent) {
  if (!t || (n && (!keys || !values))) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n == 0) return MVBT_OK;
  if (t->kind == MVBT_KIND_BLINK) ts = mvbt::kLatest;
  cudaStream_t s = as_stream(stream);
  const int bs   = t->block_size;
  if (t->tile_width == 8) {
    if (concurrent) k_find<8, true><<<grid_for(t, k_find<8, true>, n), bs, 0, s>>>(t->view(), keys, values, n, ts);
    else k_find<8, false><<<grid_for(t, k_find<8, false>, n), bs, 0, s>>>(t->view(), keys, values, n, ts);
  } else {
    if (concurrent) k_find<16, true><<<grid_for(t, k_find<16, true>, n), bs, 0, s>>>(t->view(), keys, values, n, ts);
    else k_find<16, false><<<grid_for(t, k_find<16, false>, n), bs, 0, s>>>(t->view(), keys, values, n, ts);
  }
  return check_launch();
}

int mvbt_erase(mvbt_tree* t, const uint32_t* keys, uint32_t n, void* stream, int concurrent) {
  (void)concurrent;  // writers always use coherent loads
  if (!t || (n && !keys)) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n == 0) return MVBT_OK;
  cudaStream_t s = as_stream(stream);
  if (t->tile_width == 8) {
    k_erase<8><<<grid_for(t, k_erase<8>, n), t->block_size, 0, s>>>(t->view(), keys, n);
  } else {
    k_erase<16><<<grid_for(t, k_erase<16>, n), t->block_size, 0, s>>>(t->view(), keys, n);
  }
  return check_launch();
}

int mvbt_range_query(mvbt_tree* t, const uint32_t* lower, const uint32_t* upper, mvbt_pair* result,
                     uint32_t* counts, uint32_t avg_len, uint32_t n, uint32_t ts, void* stream,
                     int concurrent) {
  if (!t || (n && (!lower || !upper))) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n == 0) return MVBT_OK;
  if (t->kind == MVBT_KIND_BLINK) ts = mvbt::kLatest;
  cudaStream_t s = as_stream(stream);
  uint2* out     = reinterpret_cast<uint2*>(result);
  const int bs   = t->block_size;
  if (t->tile_width == 8) {
    if (concurrent) k_range<8, true><<<grid_for(t, k_range<8, true>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
    else k_range<8, false><<<grid_for(t, k_range<8, false>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
  } else {
    if (concurrent) k_range<16, true><<<grid_for(t, k_range<16, true>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
    else k_range<16, false><<<grid_for(t, k_range<16, false>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
  }
  return check_launch();
}

int mvbt_take_snapshot_async(mvbt_tree* t, void* stream, uint32_t* d_out) {
  if (!t || !d_out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  k_snapshot<<<1, 32, 0, as_stream(stream)>>>(t->ctl, d_out);
  return check_launch();
}

int mvbt_take_snapshot(mvbt_tree* t, void* stream, uint32_t* snapshot_out) {
  if (!t || !snapshot_out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (t->kind != MVBT_KIND_VERSIONED) return fail(MVBT_ERR_NOT_SUPPORTED, "snapshots need a versioned tree");
  cudaStream_t s = as_stream(stream);
  k_snapshot<<<1, 32, 0, s>>>(t->ctl, t->d_words);
  int st = check_launch();
  if (st) return st;
  MVBT_CUDA_TRY(cudaMemcpyAsync(t->h_word, t->d_words, 4, cudaMemcpyDeviceToHost, s));
  MVBT_CUDA_TRY(cudaStreamSynchronize(s));
  *snapshot_out = *t->h_word;
  return MVBT_OK;
}

int mvbt_concurrent_insert_range(mvbt_tree* t, const uint32_t* keys, const uint32_t* values,
                                 uint32_t n_ins, const uint32_t* lower, const uint32_t* upper,
                                 uint32_t n_rq, mvbt_pair* result, uint32_t avg_len, uint32_t* counts,
                                 void* stream) {
  if (!t || (n_ins && (!keys || !values)) || (n_rq && (!lower || !upper)))
    return fail(MVBT_ERR_BAD_ARG, "null argument");
  uint64_t total = (uint64_t)n_ins + n_rq;
  if (total == 0) return MVBT_OK;
  cudaStream_t s = as_stream(stream);
  if (t->kind == MVBT_KIND_VERSIONED) {
    k_snapshot<<<1, 32, 0, s>>>(t->ctl, t->d_words);
    int st = check_launch();
    if (st) return st;
  }
  uint2* out = reinterpret_cast<uint2*>(result);
  if (t->tile_width == 8) {
    k_insert_range<8><<<grid_for(t, k_insert_range<8>, total), t->block_size, 0, s>>>(
        t->view(), keys, values, n_ins, lower, upper, n_rq, out, avg_len, counts, t->d_words);
  } else {
    k_insert_range<16><<<grid_for(t, k_insert_range<16>, total), t->block_size, 0, s>>>(
        t->view(), keys, values, n_ins, lower, upper, n_rq, out, avg_len, counts, t->d_words);
  }
  return check_launch();
}

int mvbt_concurrent_find_erase(mvbt_tree* t, const uint32_t* fkeys, uint32_t* fres, uint32_t n_find,
                               const uint32_t* ekeys, uint32_t n_erase, void* stream) {
  if (!t || (n_find && (!fkeys || !fres)) || (n_erase && !ekeys)) return fail(MVBT_ERR_BAD_ARG, "null argument");
  uint64_t total = (uint64_t)n_find + n_erase;
  if (total == 0) return MVBT_OK;
  cudaStream_t s = as_stream(stream);
  if (t->kind == MVBT_KIND_VERSIONED) {
    k_snapshot<<<1, 32, 0, s>>>(t->ctl, t->d_words);
    int st = check_launch();
    if (st) return st;
  }
  if (t->tile_width == 8) {
    k_find_erase<8><<<grid_for(t, k_find_erase<8>, total), t->block_size, 0, s>>>(
        t->view(), fkeys, fres, n_find, ekeys, n_erase, t->d_words);
  } else {
    k_find_erase<16><<<grid_for(t, k_find_erase<16>, total), t->block_size, 0, s>>>(
        t->view(), fkeys, fres, n_find, ekeys, n_erase, t->d_words);
  }
  return check_launch();
}

int mvbt_check_errors(mvbt_tree* t, void* stream, uint32_t* bits) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  cudaStream_t s = as_stream(stream);
  MVBT_CUDA_TRY(cudaMemcpyAsync(t->h_word, &t->ctl->error, 4, cudaMemcpyDeviceToHost, s));
  MVBT_CUDA_TRY(cudaStreamSynchronize(s));
  uint32_t b = *t->h_word;
  if (bits) *bits = b;
  int st = status_from_bits(b);
  if (st) g_last_error = std::string("device error bits ") + std::to_string(b);
  return st;
}

int mvbt_clear_errors(mvbt_tree* t, void* stream) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  MVBT_CUDA_TRY(cudaMemsetAsync(&t->ctl->error, 0, 4, as_stream(stream)));
  return MVBT_OK;
}

int mvbt_memory_usage(mvbt_tree* t, uint64_t* nodes, uint64_t* bytes, uint64_t* pool_bytes) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  uint32_t bump = 0;
  MVBT_CUDA_TRY(cudaMemcpy(&bump, &t->ctl->bump, 4, cudaMemcpyDeviceToHost));
  uint64_t b = std::min<uint64_t>(bump, t->capacity);
  if (nodes) *nodes = b;
  if (bytes) *bytes = b * 128;
  if (pool_bytes) *pool_bytes = t->capacity * 128;
  return MVBT_OK;
}

int mvbt_get_device_view(mvbt_tree* t, mvbt_device_view* out) {
  if (!t || !out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  out->pool      = t->pool;
  out->control   = t->ctl;
  out->versioned = t->kind == MVBT_KIND_VERSIONED ? 1u : 0u;
  out->capacity  = (uint32_t)t->capacity;
  return MVBT_OK;
}

int mvbt_validate(mvbt_tree* t, uint32_t ts, mvbt_report* rep) {
  if (!t || !rep) return fail(MVBT_ERR_BAD_ARG, "null argument");
  std::memset(rep, 0, sizeof(*rep));
  MVBT_CUDA_TRY(cudaSetDevice(t->device));
  MVBT_CUDA_TRY(cudaDeviceSynchronize());
  uint32_t bump = 0;
  MVBT_CUDA_TRY(cudaMemcpy(&bump, &t->ctl->bump, 4, cudaMemcpyDeviceToHost));
  uint64_t nn = std::min<uint64_t>(bump, t->capacity);
  std::vector<uint32_t> img(nn * 32);
  MVBT_CUDA_TRY(cudaMemcpy(img.data(), t->pool, nn * 128, cudaMemcpyDeviceToHost));
  rep->nodes_allocated = nn;
  const bool snap      = t->kind == MVBT_KIND_VERSIONED && ts != mvbt::kLatest;
  auto node            = [&](uint32_t i) { return host_node{img.data() + (size_t)i * 32}; };
  uint32_t violations  = 0;
  auto resolve         = [&](uint32_t i) -> uint32_t {
    uint32_t hops = 0;
    while (snap && i < nn && node(i).ts() > ts) {
      i = node(i).older();
      if (++hops > 1000000) return mvbt::kNone;
    }
    return i < nn ? i : mvbt::kNone;
  };
  uint32_t root = resolve(mvbt::kRoot);
  if (root == mvbt::kNone) {
    rep->violations = 1;
    return fail(MVBT_ERR_CORRUPT, "root version not found");
  }
  int top        = (int)node(root).level();
  rep->height    = (uint32_t)top + 1;
  uint32_t first = mvbt::kRoot;  // slot index of the leftmost node of the level
  std::vector<uint32_t> child_slots;
  for (int level = top; level >= 0; --level) {
    std::vector<uint32_t> slots;
    std::vector<uint32_t> next_children;
    uint32_t slot = first, low = 0;
    uint64_t guard = 0;
    while (slot != mvbt::kNone) {
      if (++guard > nn + 1) {
        ++violations;
        break;
      }
      uint32_t v = resolve(slot);
      if (v == mvbt::kNone) {
        ++violations;
        break;
      }
      host_node x = node(v);
      slots.push_back(slot);
      if ((int)x.level() != level) ++violations;
      if (x.link() & mvbt::kLockBit) ++rep->locked_nodes;
      uint32_t prev = 0;
      bool have     = false;
      int cnt       = 0;
      for (int p = 0; p < mvbt::kDataPairs; ++p) {
        uint32_t k = x.key(p);
        if (k == mvbt::kEmptyKey) {
          for (int q = p; q < mvbt::kDataPairs; ++q)
            if (x.key(q) != mvbt::kEmptyKey) ++violations;  // valid pairs form a prefix
          break;
        }
        ++cnt;
        if (have && k <= prev) ++violations;
        if (k < low || k >= x.high()) ++violations;
        prev = k;
        have = true;
        if (level == 0) {
          ++rep->keys;
          rep->key_checksum += (uint64_t)k * 0x9E3779B1ull + x.val(p);
        } else {
          next_children.push_back(x.val(p));
        }
      }
      if (level > 0 && cnt == 0) ++violations;
      if (level == 0) ++rep->leaves;
      else ++rep->interior;
      if (x.high() <= low && x.high() != mvbt::kEmptyKey) ++violations;
      low  = x.high();
      slot = x.sibling();
      if (slot == mvbt::kNone && x.high() != mvbt::kEmptyKey) ++violations;
    }
    // every node of this level is referenced by exactly one parent entry
    if (level < top) {
      std::vector<uint32_t> a = slots, b = child_slots;
      std::sort(a.begin(), a.end());
      std::sort(b.begin(), b.end());
      if (a != b) ++violations;
    }
    child_slots = next_children;
    if (level > 0) {
      uint32_t v = resolve(first);
      if (v == mvbt::kNone) break;
      first = node(v).val(0);
    }
  }
  rep->violations = violations;
  if (violations) return fail(MVBT_ERR_CORRUPT, "tree structure check failed: " + std::to_string(violations) + " violations");
  return MVBT_OK;
}

}  // extern "C"
