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
#include <mutex>
#include <string>
#include <vector>

#include "mvbt.h"
#include "mvbt_device.cuh"
#include "mvbt_sort.h"

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
  uint32_t* retire_log;  // reclamation on: uint32_t[capacity]
  uint32_t* free_ring;   // reclamation on: uint32_t[capacity + kMaxSmSlots * chunk]
  int num_sms;
  uint32_t spin_limit;
  uint32_t chunk;
  uint32_t blocks_per_sm;
  uint32_t max_blocks;
  uint32_t wait_ms;
  uint32_t frontend = MVBT_FRONTEND_AUTO;  // batch front-end of the bulk calls (MVBT_FRONTEND_*)
  // Nothing has been written to the tree and no snapshot taken since mvbt_create (only the
  // tombstone {0, 0} in epoch 0): a large sorted insert is then a bottom-up bulk load.
  bool pristine = false;
  // Upper bound on the keys ever written into the tree (host-side, by the calls that write):
  // leaves are never merged, so it bounds the leaf count from above too. Bulk inserts into a tree
  // that is small against the batch are split by it (insert_launches).
  uint64_t grown = 1;
  device_tree view() const {
    device_tree t;
    t.pool      = pool;
    t.ctl       = ctl;
    t.versioned = kind == MVBT_KIND_VERSIONED ? 1u : 0u;
    t.capacity  = (uint32_t)capacity;
    t.reclaim   = retire_log ? 1u : 0u;
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
                       uint32_t spin_limit, uint32_t wait_ns, uint32_t* retire_log, uint32_t* free_ring,
                       uint32_t log_cap, uint32_t ring_cap) {
  for (int i = threadIdx.x; i < 32 * mvbt::kInitialNodes; i += blockDim.x) pool[i] = mvbt::initial_tree_word(i);
  if (threadIdx.x == 0)
    mvbt::init_control(*c, capacity, chunk, spin_limit, wait_ns, (unsigned long long)retire_log,
                       (unsigned long long)free_ring, log_cap, ring_cap);
}

// Reclaim pass over the retire log (mvbt_reclaim): frees every version copy made in an epoch <= M
// (kReclaimAll: the current epoch) and appends it to the free ring (one reservation per warp).
__global__ void __launch_bounds__(256) k_reclaim(device_tree T, uint32_t M) {
  auto warp                       = cg::tiled_partition<32>(cg::this_thread_block());
  control_block* c                = T.ctl;
  const unsigned long long head   = c->retire_head;
  unsigned long long n            = c->retire_tail - head;
  if (n > c->reclaim_cap) n = c->reclaim_cap;
  if (M == mvbt::kReclaimAll) M = c->epoch;
  const uint32_t lane             = threadIdx.x & 31u;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  // b is the same in every lane of a warp, so every lane takes the same number of iterations
  for (unsigned long long b = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < n; b += stride) {
    const unsigned long long i = b + lane;
    uint32_t idx               = mvbt::kNone;
    const int r                = i < n ? T.reclaim_entry(head + i, M, idx) : 0;
    mvbt::ring_push(c, r == 1, idx, warp);
    if (r == 2) atomicMin(&c->rc_first_kept, (uint32_t)i);
  }
}

// End of a reclaim pass: moves the log head (one thread).
__global__ void k_reclaim_finish(device_tree T) {
  if (threadIdx.x == 0) T.reclaim_publish();
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

// Loop condition of every tile loop below: true while any tile of the calling warp has work, so
// that all lanes of the warp meet here once per iteration. Tiles of one warp that diverge (one
// waits on a lock while the other copies a node) otherwise drift apart and issue their
// instructions one tile at a time; met once per op they issue together and overlap their memory
// round trips. A tile without work in an iteration skips its body. Block sizes are multiples of
// 32, and no lane returns from inside such a loop.
__device__ __forceinline__ bool warp_any(bool more) { return __any_sync(0xffffffffu, more); }

template <int W, bool kStrong>
__global__ void __launch_bounds__(256) k_find(device_tree T, const uint32_t* __restrict__ keys,
                                              uint32_t* __restrict__ out, uint32_t n, uint32_t ts) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); warp_any(i < n); i += num_tiles<W>()) {
    if (i >= n) continue;
    uint32_t key = keys[i];
    uint32_t v   = kStrong ? T.cooperative_find<W>(key, tile, ts, true) : T.find_quiescent<W>(key, tile, ts);
    if (tile.thread_rank() == 0) out[i] = v;
  }
}

template <int W>
__global__ void __launch_bounds__(256) k_insert(device_tree T, const uint32_t* __restrict__ keys,
                                                const uint32_t* __restrict__ values, uint32_t n) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); warp_any(i < n); i += num_tiles<W>()) {
    if (i >= n) continue;
    uint32_t key = keys[i], value = values[i];
    uint32_t E   = T.versioned ? T.current_epoch() : 0u;
    T.cooperative_insert<W>(key, value, tile, E);
  }
}

template <int W>
__global__ void __launch_bounds__(256) k_erase(device_tree T, const uint32_t* __restrict__ keys,
                                               uint32_t n) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  for (uint64_t i = first_tile<W>(); warp_any(i < n); i += num_tiles<W>()) {
    if (i >= n) continue;
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
  for (uint64_t i = first_tile<W>(); warp_any(i < n); i += num_tiles<W>()) {
    if (i >= n) continue;
    uint32_t lo = lower[i], hi = upper[i];
    uint2* out  = result ? result + i * (uint64_t)avg_len : nullptr;
    uint32_t c  = kStrong ? T.cooperative_range_query<W>(lo, hi, tile, ts, out, avg_len, true)
                          : T.range_quiescent<W>(lo, hi, tile, ts, out, avg_len);
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
  for (uint64_t i = first_tile<W>(); warp_any(i < total); i += num_tiles<W>()) {
    if (i >= total) continue;
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
  for (uint64_t i = first_tile<W>(); warp_any(i < total); i += num_tiles<W>()) {
    if (i >= total) continue;
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
// Sorted batch front-end: the ops of a call sorted by key (mvbt_sort.cu), each tile running one
// contiguous run of them with its path memory (mvbt::finger), results scattered back to the
// caller's positions (spos = sorted position -> input position).
// ----------------------------------------------------------------------------------------------
// The calling tile's run of sorted positions [begin, end): equal shares of n over the grid.
template <int W>
__device__ __forceinline__ void tile_run(uint64_t n, uint64_t& begin, uint64_t& end) {
  const uint64_t per = (n + num_tiles<W>() - 1) / num_tiles<W>();
  begin              = first_tile<W>() * per;
  end                = begin + per < n ? begin + per : n;
}

template <int W, bool kStrong>
__global__ void __launch_bounds__(256) k_find_sorted(device_tree T, const uint32_t* __restrict__ skeys,
                                                     const uint32_t* __restrict__ spos,
                                                     uint32_t* __restrict__ out, uint32_t n, uint32_t ts) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  uint64_t i, end;
  tile_run<W>(n, i, end);
  mvbt::finger<W> f;
  for (; warp_any(i < end); ++i) {
    if (i >= end) continue;
    const uint32_t key = skeys[i];
    const uint32_t v   = kStrong ? T.cooperative_find<W>(key, tile, ts, true, f.start_for(key, tile), &f)
                                 : T.find_quiescent<W>(key, tile, ts, f.start_for(key, tile), &f);
    if (tile.thread_rank() == 0) out[spos[i]] = v;
  }
}

template <int W, bool kStrong>
__global__ void __launch_bounds__(256) k_range_sorted(device_tree T, const uint32_t* __restrict__ slower,
                                                      const uint32_t* __restrict__ spos,
                                                      const uint32_t* __restrict__ upper, uint2* result,
                                                      uint32_t* counts, uint32_t avg_len, uint32_t n,
                                                      uint32_t ts) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  uint64_t i, end;
  tile_run<W>(n, i, end);
  mvbt::finger<W> f;
  for (; warp_any(i < end); ++i) {
    if (i >= end) continue;
    const uint32_t lo = slower[i], p = spos[i];
    uint2* out        = result ? result + p * (uint64_t)avg_len : nullptr;
    const uint32_t c  = kStrong ? T.cooperative_range_query<W>(lo, upper[p], tile, ts, out, avg_len, true,
                                                               f.start_for(lo, tile), &f)
                                : T.range_quiescent<W>(lo, upper[p], tile, ts, out, avg_len, f.start_for(lo, tile), &f);
    if (counts && tile.thread_rank() == 0) counts[p] = c;
  }
}

// A key repeated in one insert call: only its last occurrence in the caller's array is applied
// (the stable sort keeps equal keys in input order), as applying them in order would leave it.
__device__ __forceinline__ bool superseded(const uint32_t* skeys, uint64_t i, uint64_t n) {
  return i + 1 < n && skeys[i + 1] == skeys[i];
}

template <int W>
__global__ void __launch_bounds__(256, 6) k_insert_sorted(device_tree T, const uint32_t* __restrict__ skeys,
                                                       const uint32_t* __restrict__ spos,
                                                       const uint32_t* __restrict__ values, uint32_t n) {
  auto tile        = cg::tiled_partition<W>(cg::this_thread_block());
  const uint32_t E = T.versioned ? T.current_epoch() : 0u;
  uint64_t i, end;
  tile_run<W>(n, i, end);
  mvbt::finger<W> f;
  while (warp_any(i < end)) {
    if (i >= end) continue;
    if (superseded(skeys, i, n)) {
      ++i;
      continue;
    }
    T.insert_run_group<W>(skeys, spos, values, i, end, n, tile, E, f);
  }
}

// Growth phase of a sorted insert into a tree that has fewer leaves than the grid has tiles: m
// evenly spaced keys of the sorted array, one per tile, so that no two tiles queue on one leaf.
// The final contiguous-run launch applies them again (an upsert of the same value changes
// nothing visible).
template <int W>
__global__ void __launch_bounds__(256) k_insert_spread(device_tree T, const uint32_t* __restrict__ skeys,
                                                       const uint32_t* __restrict__ spos,
                                                       const uint32_t* __restrict__ values, uint32_t n,
                                                       uint32_t m) {
  auto tile        = cg::tiled_partition<W>(cg::this_thread_block());
  const uint32_t E = T.versioned ? T.current_epoch() : 0u;
  for (uint64_t j = first_tile<W>(); warp_any(j < m); j += num_tiles<W>()) {
    if (j >= m) continue;
    const uint64_t i = j * n / m;
    if (superseded(skeys, i, n)) continue;
    T.cooperative_insert<W>(skeys[i], values[spos[i]], tile, E);
  }
}

template <int W>
__global__ void __launch_bounds__(256) k_erase_sorted(device_tree T, const uint32_t* __restrict__ skeys,
                                                      uint32_t n) {
  auto tile        = cg::tiled_partition<W>(cg::this_thread_block());
  const uint32_t E = T.versioned ? T.current_epoch() : 0u;
  uint64_t i, end;
  tile_run<W>(n, i, end);
  mvbt::finger<W> f;
  for (; warp_any(i < end); ++i)
    if (i < end) T.erase_in_run<W>(skeys[i], tile, E, f);
}

// ----------------------------------------------------------------------------------------------
// Launch helpers
// ----------------------------------------------------------------------------------------------
template <class K>
unsigned grid_for(const mvbt_tree* t, K kernel, uint64_t ops) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, t->block_size, 0);
  if (per_sm < 1) per_sm = 1;
  if (t->blocks_per_sm && (int)t->blocks_per_sm < per_sm) per_sm = (int)t->blocks_per_sm;
  uint64_t tiles_per_block = (uint64_t)t->block_size / t->tile_width;
  uint64_t need            = (ops + tiles_per_block - 1) / tiles_per_block;
  uint64_t cap             = (uint64_t)per_sm * t->num_sms;
  uint64_t g               = std::min<uint64_t>(std::max<uint64_t>(need, 1), cap);
  if (t->max_blocks) g = std::min<uint64_t>(g, t->max_blocks);
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

// Bulk insert of n keys. On a tree that is small against the batch, the tiles of a full grid
// would queue on the few leaves there are, and every handoff of a queued lock costs an atomic per
// waiter: at one leaf and ~25 000 tiles an insert into an empty tree ran at 4 M keys/s. So the
// batch is cut into launches of about one tile per leaf of the tree each one starts on (~10 keys
// per leaf), each about doubling the tree, until the full grid has a leaf per tile; the rest runs
// in one launch. The keys of one call are unordered either way.
template <int W>
int insert_launches(mvbt_tree* t, const uint32_t* keys, const uint32_t* values, uint32_t n, cudaStream_t s) {
  const uint64_t full  = grid_for(t, k_insert<W>, n);
  const uint64_t tiles = (uint64_t)t->block_size / W;
  uint64_t done        = 0;
  while (done < n) {
    uint64_t blocks = std::max<uint64_t>(1, (t->grown / 10) / tiles);
    uint64_t chunk  = n - done;
    if (blocks < full) chunk = std::min<uint64_t>(chunk, std::max<uint64_t>(t->grown, blocks * tiles * 16));
    blocks = std::min(blocks, full);
    k_insert<W><<<(unsigned)blocks, t->block_size, 0, s>>>(t->view(), keys + done, values + done, (uint32_t)chunk);
    int st = check_launch();
    if (st) return st;
    done += chunk;
    t->grown += chunk;
  }
  return MVBT_OK;
}

// ---- sorted batch front-end: host side ----
// Whether a bulk call of n ops takes the sorted front-end (MVBT_FRONTEND_AUTO: a large call that
// is dense against the tree, so that neighbouring sorted ops share nodes).
bool use_sorted(const mvbt_tree* t, uint32_t n) {
  if (t->frontend == MVBT_FRONTEND_SORTED) return n > 1;
  if (t->frontend == MVBT_FRONTEND_UNSORTED) return false;
  return n >= (1u << 16) && (uint64_t)n * 128 >= t->grown;
}

// A stream-ordered memory pool per device for the sort's scratch: no device-wide synchronisation,
// and freed blocks stay cached in the pool for the next call (up to kPoolKeepBytes).
constexpr int kMaxDevices           = 64;
constexpr uint64_t kPoolKeepBytes   = 4ull << 30;
cudaMemPool_t g_sort_pool[kMaxDevices] = {};
std::mutex g_sort_pool_mu;

int sort_pool(int dev, cudaMemPool_t* out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(MVBT_ERR_BAD_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_sort_pool_mu);
  if (!g_sort_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType        = cudaMemAllocationTypePinned;
    props.location.type    = cudaMemLocationTypeDevice;
    props.location.id      = dev;
    MVBT_CUDA_TRY(cudaMemPoolCreate(&g_sort_pool[dev], &props));
    uint64_t keep = kPoolKeepBytes;
    MVBT_CUDA_TRY(cudaMemPoolSetAttribute(g_sort_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep));
  }
  *out = g_sort_pool[dev];
  return MVBT_OK;
}

// The keys of a call in ascending order with their input positions, in pool memory released by
// release() (stream-ordered, after the kernels that read it).
struct sorted_ops {
  uint32_t* keys = nullptr;
  uint32_t* pos  = nullptr;
  uint32_t* extra = nullptr;  // extra_words of scratch after the sort's own (64-word aligned)
  void* mem      = nullptr;
  int release(cudaStream_t s) {
    if (mem && cudaFreeAsync(mem, s) != cudaSuccess) return fail(MVBT_ERR_CUDA, "cudaFreeAsync of sort scratch");
    mem = nullptr;
    return MVBT_OK;
  }
};

int sort_ops(mvbt_tree* t, const uint32_t* keys, uint32_t n, int low_bit, cudaStream_t s, sorted_ops* out,
             uint64_t extra_words = 0) {
  cudaMemPool_t pool;
  int st = sort_pool(t->device, &pool);
  if (st) return st;
  const uint64_t sort_words = 4ull * n + ((mvbt_sort::scratch_words(n) + 63) & ~63ull);
  const uint64_t words      = sort_words + extra_words;
  void* mem            = nullptr;
  if (cudaMallocFromPoolAsync(&mem, words * 4, pool, s) != cudaSuccess) {
    cudaGetLastError();
    return fail(MVBT_ERR_OUT_OF_MEMORY, "sort scratch: cudaMallocFromPoolAsync failed");
  }
  uint32_t* w = static_cast<uint32_t*>(mem);
  out->mem    = mem;
  out->keys   = w;
  out->pos    = w + n;
  out->extra  = extra_words ? w + sort_words : nullptr;
  if (mvbt_sort::sort_pairs(keys, n, low_bit, w, w + n, w + 2ull * n, w + 3ull * n, w + 4ull * n, s)) {
    out->release(s);
    return fail(MVBT_ERR_CUDA, std::string("sort launch: ") + cudaGetErrorString(cudaGetLastError()));
  }
  return MVBT_OK;
}

constexpr int kReadSortLowBit = 8;  // reads: order by the top 24 bits (locality is all they need)

template <int W>
int insert_sorted_launches(mvbt_tree* t, const sorted_ops& so, const uint32_t* values, uint32_t n, cudaStream_t s) {
  const uint64_t full  = grid_for(t, k_insert_sorted<W>, n);
  const uint64_t tiles = (uint64_t)t->block_size / W;
  uint64_t spread      = 0;
  while (t->grown / 10 < full * tiles && spread < n) {  // fewer leaves than tiles: spread first
    uint64_t blocks = std::max<uint64_t>(1, (t->grown / 10) / tiles);
    blocks          = std::min(blocks, full);
    uint64_t m      = std::min<uint64_t>(n, std::max<uint64_t>(t->grown, blocks * tiles * 16));
    k_insert_spread<W><<<(unsigned)blocks, t->block_size, 0, s>>>(t->view(), so.keys, so.pos, values, n, (uint32_t)m);
    int st = check_launch();
    if (st) return st;
    t->grown += m;
    spread = m;
  }
  if (spread < n) {
    k_insert_sorted<W><<<(unsigned)full, t->block_size, 0, s>>>(t->view(), so.keys, so.pos, values, n);
    int st = check_launch();
    if (st) return st;
    t->grown += n - spread;
  }
  return MVBT_OK;
}

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
  cfg->wait_ms     = 2000;
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
  t->spin_limit    = cfg.spin_limit;
  t->chunk         = cfg.chunk_nodes;
  t->blocks_per_sm = cfg.blocks_per_sm;
  t->max_blocks    = cfg.max_blocks;
  t->wait_ms       = cfg.wait_ms ? cfg.wait_ms : 2000u;
  if (t->wait_ms > 4000u) t->wait_ms = 4000u;  // wait_ns is a 32-bit ns count
  t->frontend      = cfg.frontend <= MVBT_FRONTEND_SORTED ? cfg.frontend : MVBT_FRONTEND_AUTO;
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
  uint32_t log_cap = 0, ring_cap = 0;
  if (cfg.reclaim) {  // power-of-two rings: positions map to slots with a mask
    auto pow2 = [](uint64_t x) { uint64_t p = 1; while (p < x) p <<= 1; return p; };
    log_cap  = (uint32_t)pow2(capacity);
    ring_cap = (uint32_t)pow2(capacity + (uint64_t)mvbt::kMaxSmSlots * t->chunk);
    if (cudaMalloc(&t->retire_log, (uint64_t)log_cap * 4) != cudaSuccess ||
        cudaMalloc(&t->free_ring, (uint64_t)ring_cap * 4) != cudaSuccess) {
      cudaGetLastError();
      mvbt_destroy(t);
      return fail(MVBT_ERR_OUT_OF_MEMORY, "cudaMalloc of the reclamation rings failed");
    }
    // both start empty: every slot all ones (kRingEmpty; an index >= capacity in the log)
    if (cudaMemset(t->retire_log, 0xFF, (uint64_t)log_cap * 4) != cudaSuccess ||
        cudaMemset(t->free_ring, 0xFF, (uint64_t)ring_cap * 4) != cudaSuccess) {
      cudaGetLastError();
      mvbt_destroy(t);
      return fail(MVBT_ERR_CUDA, "cudaMemset of the reclamation rings failed");
    }
  }
  k_init<<<1, 256>>>(t->pool, t->ctl, (uint32_t)capacity, t->chunk, t->spin_limit, t->wait_ms * 1000000u,
                     t->retire_log, t->free_ring, log_cap, ring_cap);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    mvbt_destroy(t);
    return fail(MVBT_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
  }
  t->pristine = true;
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
  if (t->retire_log) cudaFree(t->retire_log);
  if (t->free_ring) cudaFree(t->free_ring);
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

// ---- bulk build from sorted pairs ----
// Entry e of the built tree: the tombstone {0, 0} first unless the input starts with key 0 (its
// value then replaces the tombstone's), then the input pairs in order.
// Bottom-up build of a tree from sorted unique pairs, shared by mvbt_bulk_build and by inserts into
// a pristine tree. The plan lives in device memory, so a build whose entry count is only known on
// the device (after the sorted front-end dropped repeated keys) needs no host round trip.
struct bulk_levels {
  uint32_t n;                 // levels, leaves = level 0
  uint32_t fill;              // pairs per leaf = children per interior node
  uint64_t base[mvbt::kMaxLevels];   // first node index of each level
  uint64_t count[mvbt::kMaxLevels];  // nodes of each level
  uint64_t span[mvbt::kMaxLevels];   // entries under one node of each level (fill^(level+1), saturated)
};
struct bulk_plan {
  bulk_levels L;
  const uint32_t* keys;    // sorted strictly increasing
  const uint32_t* values;
  uint64_t m;              // entries: the input, plus the tombstone {0, 0} first when off = 1
  uint64_t total;          // nodes below the anchor; 0 = build nothing
  uint32_t off;            // 1: entry 0 is the tombstone; 0: the input holds key 0
  uint32_t status;         // 0 ok, 1 too tall, 2 pool too small
  __device__ uint32_t key(uint64_t e) const { return (off && e == 0) ? 0u : keys[e - off]; }
  __device__ uint32_t value(uint64_t e) const { return (off && e == 0) ? 0u : values[e - off]; }
};

// Level layout of a plan whose m and L.fill are set; leaves total = 0 with a status on failure.
__host__ __device__ inline void plan_levels(bulk_plan& P, uint64_t capacity) {
  const uint32_t fill = P.L.fill;
  P.L.n   = 0;
  P.total = 0;
  uint64_t count = (P.m + fill - 1) / fill, base = 1, span = fill, total = 0;
  for (;;) {
    if (P.L.n >= (uint32_t)mvbt::kMaxLevels - 1) {
      P.status = 1;
      P.L.n    = 0;
      return;
    }
    P.L.base[P.L.n]  = base;
    P.L.count[P.L.n] = count;
    P.L.span[P.L.n]  = span;
    ++P.L.n;
    base += count;
    total += count;
    if (count == 1) break;
    count = (count + fill - 1) / fill;
    span  = span > (~0ull) / fill ? ~0ull : span * fill;
  }
  if (1 + total > capacity) {
    P.status = 2;
    P.L.n    = 0;
    return;
  }
  P.status = 0;
  P.total  = total;
}

// Upper bound of plan.total for m entries (the grid of k_bulk_build).
inline uint64_t bulk_nodes_bound(uint64_t m, uint32_t fill) {
  uint64_t total = 0, count = (m + fill - 1) / fill;
  for (int l = 0; l < mvbt::kMaxLevels; ++l) {
    total += count;
    if (count <= 1) break;
    count = (count + fill - 1) / fill;
  }
  return total;
}

// Sorted strictly increasing, no 0xFFFFFFFF: otherwise sets *bad.
__global__ void k_bulk_check(const uint32_t* keys, uint64_t n, uint32_t* bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if (k == mvbt::kEmptyKey || (i + 1 < n && keys[i + 1] <= k)) atomicOr(bad, 1u);
  }
}

// One warp per node, lane w writes word w: pairs 0..12, then {low, mod}, {high, link}, {ts, level|older}.
__global__ void k_bulk_build(uint32_t* pool, const bulk_plan* __restrict__ plan) {
  __shared__ bulk_plan P;
  if (threadIdx.x == 0) P = *plan;
  __syncthreads();
  const bulk_levels& L = P.L;
  const uint32_t w     = threadIdx.x & 31u;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < P.total; g += warps) {
    uint32_t l = 0;
    while (l + 1 < L.n && g >= L.base[l + 1] - L.base[0]) ++l;
    const uint64_t j     = g - (L.base[l] - L.base[0]);
    const uint64_t first = j * L.span[l];                     // first entry under this node
    const uint64_t child_span = l ? L.span[l - 1] : 1;        // entries under one child (leaf: 1)
    uint64_t items = l ? L.count[l - 1] - j * L.fill : P.m - first;  // children or entries left
    if (items > L.fill) items = L.fill;
    uint32_t v = mvbt::kEmptyKey;
    if (w < 2 * mvbt::kDataPairs) {
      const uint64_t p = w >> 1;
      if (p < items) {
        const uint64_t e = first + p * child_span;
        if (l == 0) v = (w & 1) ? P.value(e) : P.key(e);
        else v = (w & 1) ? (uint32_t)(L.base[l - 1] + j * L.fill + p) : P.key(e);
      }
    } else if (w == 26) {
      v = P.key(first);
    } else if (w == 27) {
      v = 0;  // modification count
    } else if (w == 28) {
      const uint64_t next = first + L.span[l];
      v = (j + 1 < L.count[l] && next < P.m) ? P.key(next) : mvbt::kEmptyKey;
    } else if (w == 29) {
      v = (j + 1 < L.count[l]) ? (uint32_t)(L.base[l] + j + 1) : mvbt::kNone;
    } else if (w == 30) {
      v = 0;  // ts
    } else {
      v = (l << 28) | mvbt::kNone;
    }
    pool[(L.base[l] + j) * 32 + w] = v;
  }
}

// The anchor {0 -> top}, one level above the top; the bump pointer past the built nodes. A plan
// that failed leaves the tree as it was and records the failure in the error bits.
__global__ void k_bulk_anchor(uint32_t* pool, control_block* c, const bulk_plan* __restrict__ plan) {
  const uint32_t w = threadIdx.x;
  if (w >= 32) return;
  if (plan->total == 0) {
    if (w == 0 && plan->status) {
      atomicOr(&c->error, plan->status == 2 ? mvbt::kErrPoolExhausted : mvbt::kErrCorrupt);
      atomicAdd(&c->err_site[17], 1u);
    }
    return;
  }
  const uint32_t top_level = plan->L.n - 1;
  const uint32_t top       = (uint32_t)plan->L.base[top_level];
  uint32_t v = mvbt::kEmptyKey;
  if (w == 0) v = 0;
  else if (w == 1) v = top;
  else if (w == 26 || w == 27 || w == 30) v = 0;
  else if (w == 29) v = mvbt::kNone;
  else if (w == 31) v = ((top_level + 1) << 28) | mvbt::kNone;
  pool[w] = v;
  if (w == 0) c->bump = (uint32_t)(1 + plan->total);
}

// ---- insert into a pristine tree: a bulk load of the sorted call ----
// keep[i] = 1 for the last occurrence of each key (the one an in-order upsert leaves), 0 for an
// earlier occurrence and for the reserved key 0xFFFFFFFF (which insert ignores).
__global__ void k_keep_flags(const uint32_t* __restrict__ skeys, uint64_t n, uint32_t* __restrict__ keep) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    keep[i] = (skeys[i] != mvbt::kEmptyKey && !(i + 1 < n && skeys[i + 1] == skeys[i])) ? 1u : 0u;
}
// After the exclusive scan of keep (at[i] = output position): the kept pairs, compacted.
__global__ void k_keep_compact(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ spos,
                               const uint32_t* __restrict__ values, const uint32_t* __restrict__ at, uint64_t n,
                               uint32_t* __restrict__ ck, uint32_t* __restrict__ cv) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = skeys[i];
    if (k != mvbt::kEmptyKey && !(i + 1 < n && skeys[i + 1] == k)) {
      ck[at[i]] = k;
      cv[at[i]] = values[spos[i]];
    }
  }
}
// One thread: the plan for the compacted pairs (their count is at[n - 1] + keep(n - 1)).
__global__ void k_bulk_plan_kept(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ at, uint64_t n,
                                 const uint32_t* ck, const uint32_t* cv, uint32_t fill, uint64_t capacity,
                                 bulk_plan* plan) {
  const uint32_t last = skeys[n - 1];
  const uint64_t kept = (uint64_t)at[n - 1] + (last != mvbt::kEmptyKey ? 1u : 0u);
  bulk_plan P;
  P.keys   = ck;
  P.values = cv;
  P.off    = (kept && ck[0] == 0u) ? 0u : 1u;  // key 0 in the call replaces the tombstone's value
  P.m      = kept + P.off;
  P.L.fill = fill;
  plan_levels(P, capacity);
  *plan = P;
}

int mvbt_bulk_build(mvbt_tree* t, const uint32_t* keys, const uint32_t* values, uint64_t n, uint32_t fill,
                    void* stream) {
  if (!t || (n && (!keys || !values))) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (fill == 0) fill = 8;
  if (fill < 2 || fill > (uint32_t)mvbt::kDataPairs) return fail(MVBT_ERR_BAD_ARG, "fill must be in [2, 13]");
  MVBT_CUDA_TRY(cudaSetDevice(t->device));
  cudaStream_t s = as_stream(stream);
  MVBT_CUDA_TRY(cudaStreamSynchronize(s));
  control_block c;
  MVBT_CUDA_TRY(cudaMemcpy(&c, t->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  uint32_t leaf[4] = {0, 0, 0, 0};  // the first leaf's first two pairs
  MVBT_CUDA_TRY(cudaMemcpy(leaf, t->pool + 32 * mvbt::kFirstLeaf, sizeof(leaf), cudaMemcpyDeviceToHost));
  if (c.bump != (uint32_t)mvbt::kInitialNodes || c.epoch != 0 || leaf[2] != mvbt::kEmptyKey)
    return fail(MVBT_ERR_BAD_ARG, "bulk build needs a fresh tree (no writes, no snapshots)");
  if (n == 0) return MVBT_OK;
  uint32_t first_key = 0;
  MVBT_CUDA_TRY(cudaMemcpy(&first_key, keys, 4, cudaMemcpyDeviceToHost));
  MVBT_CUDA_TRY(cudaMemsetAsync(t->d_words, 0, 4, s));
  k_bulk_check<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 4096), 256, 0, s>>>(keys, n, t->d_words);
  MVBT_CUDA_TRY(cudaMemcpyAsync(t->h_word, t->d_words, 4, cudaMemcpyDeviceToHost, s));
  MVBT_CUDA_TRY(cudaStreamSynchronize(s));
  if (*t->h_word) return fail(MVBT_ERR_BAD_ARG, "bulk build needs keys sorted strictly increasing, without 0xFFFFFFFF");
  bulk_plan P;
  P.keys   = keys;
  P.values = values;
  P.off    = first_key == 0 ? 0u : 1u;
  P.m      = n + P.off;
  P.L.fill = fill;
  plan_levels(P, t->capacity);
  if (P.status == 1) return fail(MVBT_ERR_BAD_ARG, "bulk build: tree too tall");
  if (P.status == 2) return fail(MVBT_ERR_POOL_EXHAUSTED, "bulk build: the pool is too small");
  cudaMemPool_t pool;
  int st = sort_pool(t->device, &pool);
  if (st) return st;
  bulk_plan* dplan = nullptr;
  MVBT_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dplan), sizeof(bulk_plan), pool, s));
  MVBT_CUDA_TRY(cudaMemcpyAsync(dplan, &P, sizeof(bulk_plan), cudaMemcpyHostToDevice, s));  // staged: P may go
  const uint64_t threads = P.total * 32;
  const unsigned grid    = (unsigned)std::min<uint64_t>((threads + 255) / 256, (uint64_t)t->num_sms * 64);
  k_bulk_build<<<grid, 256, 0, s>>>(t->pool, dplan);
  k_bulk_anchor<<<1, 32, 0, s>>>(t->pool, t->ctl, dplan);
  st = check_launch();
  MVBT_CUDA_TRY(cudaFreeAsync(dplan, s));
  t->pristine = false;
  if (st) return st;
  t->grown += n;
  return MVBT_OK;
}

// ---- copies of a tree: clone on the device, image files for checkpoints ----
static mvbt_config config_of(const mvbt_tree* t) {
  mvbt_config c;
  mvbt_config_init(&c);
  c.pool_bytes    = t->capacity * 128;
  c.device        = t->device;
  c.tile_width    = t->tile_width;
  c.block_size    = t->block_size;
  c.spin_limit    = t->spin_limit;
  c.chunk_nodes   = t->chunk;
  c.blocks_per_sm = t->blocks_per_sm;
  c.max_blocks    = t->max_blocks;
  c.wait_ms       = t->wait_ms;
  c.reclaim       = t->retire_log ? 1u : 0u;
  c.frontend      = t->frontend;
  return c;
}

static uint64_t pow2_at_least(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Retire log and free ring sizes of a tree created with reclamation (as mvbt_create makes them).
static void ring_sizes(const mvbt_tree* t, uint64_t* log_cap, uint64_t* ring_cap) {
  *log_cap  = t->retire_log ? pow2_at_least(t->capacity) : 0;
  *ring_cap = t->retire_log ? pow2_at_least(t->capacity + (uint64_t)mvbt::kMaxSmSlots * t->chunk) : 0;
}

// Writes the control block image `c` into tree t, keeping t's own ring addresses.
static int put_control(mvbt_tree* t, control_block c) {
  c.retire_log = (unsigned long long)t->retire_log;
  c.free_ring  = (unsigned long long)t->free_ring;
  MVBT_CUDA_TRY(cudaMemcpy(t->ctl, &c, sizeof(c), cudaMemcpyHostToDevice));
  return MVBT_OK;
}

int mvbt_clone(mvbt_tree* src, mvbt_tree** out) {
  if (!src || !out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  MVBT_CUDA_TRY(cudaSetDevice(src->device));
  MVBT_CUDA_TRY(cudaDeviceSynchronize());
  const mvbt_config cfg = config_of(src);
  mvbt_tree* t          = nullptr;
  int st                = mvbt_create(src->kind, &cfg, &t);
  if (st) return st;
  control_block c;
  cudaError_t e = cudaMemcpy(&c, src->ctl, sizeof(c), cudaMemcpyDeviceToHost);
  const uint64_t nodes = std::min<uint64_t>(c.bump, src->capacity);
  uint64_t log_cap = 0, ring_cap = 0;
  ring_sizes(src, &log_cap, &ring_cap);
  if (e == cudaSuccess) e = cudaMemcpy(t->pool, src->pool, nodes * 128, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess && log_cap) e = cudaMemcpy(t->retire_log, src->retire_log, log_cap * 4, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess && ring_cap) e = cudaMemcpy(t->free_ring, src->free_ring, ring_cap * 4, cudaMemcpyDeviceToDevice);
  if (e != cudaSuccess) {
    mvbt_destroy(t);
    return fail(MVBT_ERR_CUDA, std::string("clone: ") + cudaGetErrorString(e));
  }
  st = put_control(t, c);
  if (st) {
    mvbt_destroy(t);
    return st;
  }
  t->grown    = src->grown;
  t->pristine = false;
  *out = t;
  return MVBT_OK;
}

namespace {
struct image_header {
  char magic[8];            // "MVBTIMG1"
  uint32_t version;         // 1
  int32_t kind;
  uint64_t capacity;        // nodes
  int32_t tile_width, block_size;
  uint32_t spin_limit, chunk, blocks_per_sm, max_blocks, wait_ms, reclaim;
  uint64_t nodes;           // node image length (the allocated prefix of the pool)
  uint64_t control_bytes;   // sizeof(control_block) of the writer
  uint64_t log_cap, ring_cap;
};
constexpr uint64_t kIoChunk = 64ull << 20;

// Copies `bytes` between a file and device memory through a pinned staging buffer.
int device_file_copy(FILE* f, void* dev, uint64_t bytes, bool to_file, void* stage) {
  for (uint64_t done = 0; done < bytes; done += kIoChunk) {
    const uint64_t n = std::min(kIoChunk, bytes - done);
    if (to_file) {
      MVBT_CUDA_TRY(cudaMemcpy(stage, (char*)dev + done, n, cudaMemcpyDeviceToHost));
      if (std::fwrite(stage, 1, n, f) != n) return fail(MVBT_ERR_BAD_ARG, "tree image: write failed");
    } else {
      if (std::fread(stage, 1, n, f) != n) return fail(MVBT_ERR_BAD_ARG, "tree image: file is truncated");
      MVBT_CUDA_TRY(cudaMemcpy((char*)dev + done, stage, n, cudaMemcpyHostToDevice));
    }
  }
  return MVBT_OK;
}
}  // namespace

int mvbt_save(mvbt_tree* t, const char* path) {
  if (!t || !path) return fail(MVBT_ERR_BAD_ARG, "null argument");
  MVBT_CUDA_TRY(cudaSetDevice(t->device));
  MVBT_CUDA_TRY(cudaDeviceSynchronize());
  control_block c;
  MVBT_CUDA_TRY(cudaMemcpy(&c, t->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  image_header h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, "MVBTIMG1", 8);
  h.version = 1;
  h.kind    = t->kind;
  h.capacity = t->capacity;
  h.tile_width = t->tile_width;
  h.block_size = t->block_size;
  h.spin_limit = t->spin_limit;
  h.chunk = t->chunk;
  h.blocks_per_sm = t->blocks_per_sm;
  h.max_blocks = t->max_blocks;
  h.wait_ms = t->wait_ms;
  h.reclaim = t->retire_log ? 1u : 0u;
  h.nodes = std::min<uint64_t>(c.bump, t->capacity);
  h.control_bytes = sizeof(control_block);
  ring_sizes(t, &h.log_cap, &h.ring_cap);
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(MVBT_ERR_BAD_ARG, std::string("cannot open ") + path);
  void* stage = nullptr;
  int st = MVBT_OK;
  if (cudaMallocHost(&stage, kIoChunk) != cudaSuccess) st = fail(MVBT_ERR_OUT_OF_MEMORY, "pinned staging");
  if (!st && (std::fwrite(&h, sizeof(h), 1, f) != 1 || std::fwrite(&c, sizeof(c), 1, f) != 1))
    st = fail(MVBT_ERR_BAD_ARG, "tree image: write failed");
  if (!st) st = device_file_copy(f, t->pool, h.nodes * 128, true, stage);
  if (!st && h.log_cap) st = device_file_copy(f, t->retire_log, h.log_cap * 4, true, stage);
  if (!st && h.ring_cap) st = device_file_copy(f, t->free_ring, h.ring_cap * 4, true, stage);
  if (stage) cudaFreeHost(stage);
  if (std::fclose(f) != 0 && !st) st = fail(MVBT_ERR_BAD_ARG, "tree image: close failed");
  return st;
}

int mvbt_load(const char* path, int device, mvbt_tree** out) {
  if (!path || !out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  *out    = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(MVBT_ERR_BAD_ARG, std::string("cannot open ") + path);
  image_header h;
  control_block c;
  if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, "MVBTIMG1", 8) != 0 || h.version != 1 ||
      h.control_bytes != sizeof(control_block) || std::fread(&c, sizeof(c), 1, f) != 1) {
    std::fclose(f);
    return fail(MVBT_ERR_BAD_ARG, "not a tree image of this library version");
  }
  mvbt_config cfg;
  mvbt_config_init(&cfg);
  cfg.pool_bytes    = h.capacity * 128;
  cfg.device        = device;
  cfg.tile_width    = h.tile_width;
  cfg.block_size    = h.block_size;
  cfg.spin_limit    = h.spin_limit;
  cfg.chunk_nodes   = h.chunk;
  cfg.blocks_per_sm = h.blocks_per_sm;
  cfg.max_blocks    = h.max_blocks;
  cfg.wait_ms       = h.wait_ms;
  cfg.reclaim       = h.reclaim;
  mvbt_tree* t      = nullptr;
  int st            = mvbt_create(h.kind, &cfg, &t);
  if (st) {
    std::fclose(f);
    return st;
  }
  uint64_t log_cap = 0, ring_cap = 0;
  ring_sizes(t, &log_cap, &ring_cap);
  if (h.nodes > t->capacity || log_cap != h.log_cap || ring_cap != h.ring_cap)
    st = fail(MVBT_ERR_BAD_ARG, "tree image does not match the tree it configures");
  void* stage = nullptr;
  if (!st && cudaMallocHost(&stage, kIoChunk) != cudaSuccess) st = fail(MVBT_ERR_OUT_OF_MEMORY, "pinned staging");
  if (!st) st = device_file_copy(f, t->pool, h.nodes * 128, false, stage);
  if (!st && log_cap) st = device_file_copy(f, t->retire_log, log_cap * 4, false, stage);
  if (!st && ring_cap) st = device_file_copy(f, t->free_ring, ring_cap * 4, false, stage);
  if (stage) cudaFreeHost(stage);
  std::fclose(f);
  if (!st) st = put_control(t, c);
  if (st) {
    mvbt_destroy(t);
    return st;
  }
  t->grown    = std::max<uint64_t>(1, (uint64_t)c.bump * 16);  // at most 16 keys per node
  t->pristine = false;
  *out = t;
  return MVBT_OK;
}

namespace {
// Leaves and interior nodes of a bulk load hold 10 of 13 pairs: later inserts split a leaf after
// three more keys, and a tree built by inserts averages about 9.7.
constexpr uint32_t kLoadFill = 10;
constexpr uint32_t kLoadMin  = 1u << 12;  // smaller inserts into a pristine tree go key by key

// Scratch of a bulk load after the sort's own: keep[n] | scan sums | the plan. Every region starts
// on a 64-word (256-byte) boundary: the plan holds 64-bit fields, and n may be odd.
inline uint64_t round64(uint64_t words) { return (words + 63) & ~63ull; }
uint64_t bulk_load_extra_words(uint32_t n) {
  return round64(n) + round64(mvbt_sort::scan_scratch_words(n)) + round64((sizeof(bulk_plan) + 3) / 4);
}

// Insert of a sorted call into a pristine tree: the last occurrence of every key, compacted, built
// bottom up (k_bulk_build) in place of the tombstone leaf. Stream-ordered, no host round trip: the
// entry count and the level plan are computed on the device.
int bulk_load_sorted(mvbt_tree* t, const sorted_ops& so, const uint32_t* values, uint32_t n, cudaStream_t s) {
  uint32_t* ck   = so.keys + 2ull * n;  // the sort's ping-pong buffers are free again
  uint32_t* cv   = so.keys + 3ull * n;
  uint32_t* keep = so.extra;
  uint32_t* sums = so.extra + round64(n);
  auto* plan     = reinterpret_cast<bulk_plan*>(sums + round64(mvbt_sort::scan_scratch_words(n)));
  const unsigned grid = (unsigned)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)t->num_sms * 16);
  k_keep_flags<<<grid, 256, 0, s>>>(so.keys, n, keep);
  if (mvbt_sort::exclusive_scan(keep, n, sums, s)) return check_launch();
  k_keep_compact<<<grid, 256, 0, s>>>(so.keys, so.pos, values, keep, n, ck, cv);
  k_bulk_plan_kept<<<1, 1, 0, s>>>(so.keys, keep, n, ck, cv, kLoadFill, t->capacity, plan);
  const uint64_t threads = bulk_nodes_bound((uint64_t)n + 1, kLoadFill) * 32;
  k_bulk_build<<<(unsigned)std::min<uint64_t>((threads + 255) / 256, (uint64_t)t->num_sms * 64), 256, 0, s>>>(t->pool, plan);
  k_bulk_anchor<<<1, 32, 0, s>>>(t->pool, t->ctl, plan);
  t->grown += n;
  return check_launch();
}
}  // namespace

int mvbt_insert(mvbt_tree* t, const uint32_t* keys, const uint32_t* values, uint32_t n, void* stream,
                int in_place) {
  (void)in_place;  // both reference variants keep every snapshot-visible version
  if (!t || (n && (!keys || !values))) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n == 0) return MVBT_OK;
  cudaStream_t s = as_stream(stream);
  const bool load = t->pristine && n >= kLoadMin && t->frontend != MVBT_FRONTEND_UNSORTED;
  t->pristine     = false;
  if (load || use_sorted(t, n)) {
    sorted_ops so;
    int st = sort_ops(t, keys, n, 0, s, &so, load ? bulk_load_extra_words(n) : 0);
    if (st) return st;
    if (load)
      st = bulk_load_sorted(t, so, values, n, s);
    else
      st = t->tile_width == 8 ? insert_sorted_launches<8>(t, so, values, n, s)
                              : insert_sorted_launches<16>(t, so, values, n, s);
    const int rs = so.release(s);
    return st ? st : rs;
  }
  return t->tile_width == 8 ? insert_launches<8>(t, keys, values, n, s) : insert_launches<16>(t, keys, values, n, s);
}

int mvbt_find(mvbt_tree* t, const uint32_t* keys, uint32_t* values, uint32_t n, uint32_t ts,
              void* stream, int concurrent) {
  if (!t || (n && (!keys || !values))) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (n == 0) return MVBT_OK;
  if (t->kind == MVBT_KIND_BLINK) ts = mvbt::kLatest;
  cudaStream_t s = as_stream(stream);
  const int bs   = t->block_size;
  if (use_sorted(t, n)) {
    sorted_ops so;
    int st = sort_ops(t, keys, n, kReadSortLowBit, s, &so);
    if (st) return st;
    const device_tree v = t->view();
    if (t->tile_width == 8) {
      if (concurrent) k_find_sorted<8, true><<<grid_for(t, k_find_sorted<8, true>, n), bs, 0, s>>>(v, so.keys, so.pos, values, n, ts);
      else k_find_sorted<8, false><<<grid_for(t, k_find_sorted<8, false>, n), bs, 0, s>>>(v, so.keys, so.pos, values, n, ts);
    } else {
      if (concurrent) k_find_sorted<16, true><<<grid_for(t, k_find_sorted<16, true>, n), bs, 0, s>>>(v, so.keys, so.pos, values, n, ts);
      else k_find_sorted<16, false><<<grid_for(t, k_find_sorted<16, false>, n), bs, 0, s>>>(v, so.keys, so.pos, values, n, ts);
    }
    st = check_launch();
    const int rs = so.release(s);
    return st ? st : rs;
  }
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
  t->pristine = false;
  if (n == 0) return MVBT_OK;
  cudaStream_t s = as_stream(stream);
  if (use_sorted(t, n)) {
    sorted_ops so;
    int st = sort_ops(t, keys, n, 0, s, &so);
    if (st) return st;
    if (t->tile_width == 8)
      k_erase_sorted<8><<<grid_for(t, k_erase_sorted<8>, n), t->block_size, 0, s>>>(t->view(), so.keys, n);
    else
      k_erase_sorted<16><<<grid_for(t, k_erase_sorted<16>, n), t->block_size, 0, s>>>(t->view(), so.keys, n);
    st = check_launch();
    const int rs = so.release(s);
    return st ? st : rs;
  }
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
  if (use_sorted(t, n)) {
    sorted_ops so;
    int st = sort_ops(t, lower, n, kReadSortLowBit, s, &so);
    if (st) return st;
    const device_tree v = t->view();
    if (t->tile_width == 8) {
      if (concurrent) k_range_sorted<8, true><<<grid_for(t, k_range_sorted<8, true>, n), bs, 0, s>>>(v, so.keys, so.pos, upper, out, counts, avg_len, n, ts);
      else k_range_sorted<8, false><<<grid_for(t, k_range_sorted<8, false>, n), bs, 0, s>>>(v, so.keys, so.pos, upper, out, counts, avg_len, n, ts);
    } else {
      if (concurrent) k_range_sorted<16, true><<<grid_for(t, k_range_sorted<16, true>, n), bs, 0, s>>>(v, so.keys, so.pos, upper, out, counts, avg_len, n, ts);
      else k_range_sorted<16, false><<<grid_for(t, k_range_sorted<16, false>, n), bs, 0, s>>>(v, so.keys, so.pos, upper, out, counts, avg_len, n, ts);
    }
    st = check_launch();
    const int rs = so.release(s);
    return st ? st : rs;
  }
  if (t->tile_width == 8) {
    if (concurrent) k_range<8, true><<<grid_for(t, k_range<8, true>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
    else k_range<8, false><<<grid_for(t, k_range<8, false>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
  } else {
    if (concurrent) k_range<16, true><<<grid_for(t, k_range<16, true>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
    else k_range<16, false><<<grid_for(t, k_range<16, false>, n), bs, 0, s>>>(t->view(), lower, upper, out, counts, avg_len, n, ts);
  }
  return check_launch();
}

int mvbt_set_frontend(mvbt_tree* t, uint32_t frontend) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  if (frontend > MVBT_FRONTEND_SORTED) return fail(MVBT_ERR_BAD_ARG, "unknown front-end");
  t->frontend = frontend;
  return MVBT_OK;
}

int mvbt_take_snapshot_async(mvbt_tree* t, void* stream, uint32_t* d_out) {
  if (!t || !d_out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  t->pristine = false;
  k_snapshot<<<1, 32, 0, as_stream(stream)>>>(t->ctl, d_out);
  return check_launch();
}

int mvbt_take_snapshot(mvbt_tree* t, void* stream, uint32_t* snapshot_out) {
  if (!t || !snapshot_out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  t->pristine = false;
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
  t->pristine = false;
  cudaStream_t s = as_stream(stream);
  if (t->kind == MVBT_KIND_VERSIONED) {
    k_snapshot<<<1, 32, 0, s>>>(t->ctl, t->d_words);
    int st = check_launch();
    if (st) return st;
  }
  t->grown += n_ins;
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
  t->pristine = false;
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

int mvbt_reclaim(mvbt_tree* t, uint32_t min_live_snapshot, void* stream) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  if (!t->retire_log)
    return fail(MVBT_ERR_NOT_SUPPORTED, "reclamation is off: create the tree with mvbt_config.reclaim = 1");
  MVBT_CUDA_TRY(cudaSetDevice(t->device));
  cudaStream_t s = as_stream(stream);
  k_reclaim<<<(unsigned)t->num_sms * 4u, 256, 0, s>>>(t->view(), min_live_snapshot);
  int st = check_launch();
  if (st) return st;
  k_reclaim_finish<<<1, 32, 0, s>>>(t->view());
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

int mvbt_copy_pool(mvbt_tree* t, void* dst, uint64_t max_nodes, uint64_t* nodes) {
  if (!t || !dst) return fail(MVBT_ERR_BAD_ARG, "null argument");
  MVBT_CUDA_TRY(cudaSetDevice(t->device));
  MVBT_CUDA_TRY(cudaDeviceSynchronize());
  uint32_t bump = 0;
  MVBT_CUDA_TRY(cudaMemcpy(&bump, &t->ctl->bump, 4, cudaMemcpyDeviceToHost));
  uint64_t nn = std::min<uint64_t>(std::min<uint64_t>(bump, t->capacity), max_nodes);
  MVBT_CUDA_TRY(cudaMemcpy(dst, t->pool, nn * 128, cudaMemcpyDeviceToHost));
  if (nodes) *nodes = nn;
  return MVBT_OK;
}

// Internal accessors for the other translation units of the library.
int mvbt_internal_view(mvbt_tree* t, device_tree* view, int* tile_width, int* block_size,
                       int* num_sms, uint32_t* blocks_per_sm, uint32_t* max_blocks, void** control) {
  if (!t) return fail(MVBT_ERR_BAD_ARG, "null tree");
  cudaError_t e = cudaSetDevice(t->device);
  if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, cudaGetErrorString(e));
  *view          = t->view();
  *tile_width    = t->tile_width;
  *block_size    = t->block_size;
  *num_sms       = t->num_sms;
  *blocks_per_sm = t->blocks_per_sm;
  *max_blocks    = t->max_blocks;
  *control       = t->ctl;
  return MVBT_OK;
}

void mvbt_internal_set_error(const char* msg) { g_last_error = msg ? msg : ""; }

void mvbt_internal_note_growth(mvbt_tree* t, uint64_t keys) {
  if (t) {
    t->grown += keys;
    t->pristine = false;  // batches and serving write and take snapshots
  }
}

int mvbt_stats(mvbt_tree* t, uint64_t* out, uint32_t n) {
  if (!t || !out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  MVBT_CUDA_TRY(cudaSetDevice(t->device));
  MVBT_CUDA_TRY(cudaDeviceSynchronize());
  control_block c;
  MVBT_CUDA_TRY(cudaMemcpy(&c, t->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  const bool rc  = c.reclaim_cap != 0;
  uint64_t v[43] = {rc ? c.retire_tail : mvbt::stat_total(c, 0), mvbt::stat_total(c, 1), c.stat_max_hops,
                    c.stat_max_steps,
                    c.epoch, c.error};
  for (int i = 0; i < 16; ++i) v[6 + i] = c.err_site[i];
  v[22] = c.stat_restarts;
  v[23] = c.stat_reclaimed;
  v[24] = rc ? (uint64_t)std::max<long long>(0, (long long)c.free_avail) : 0;
  v[25] = mvbt::stat_total(c, 2);
  v[26] = c.stat_log_dropped;
  for (int i = 0; i < 16; ++i) v[27 + i] = c.err_site[16 + i];
  for (uint32_t i = 0; i < n && i < 43; ++i) out[i] = v[i];
  return MVBT_OK;
}

int mvbt_get_device_view(mvbt_tree* t, mvbt_device_view* out) {
  if (!t || !out) return fail(MVBT_ERR_BAD_ARG, "null argument");
  out->pool      = t->pool;
  out->control   = t->ctl;
  out->versioned = t->kind == MVBT_KIND_VERSIONED ? 1u : 0u;
  out->capacity  = (uint32_t)t->capacity;
  out->reclaim   = t->retire_log ? 1u : 0u;
  out->reserved  = 0;
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
  int st = mvbt_validate_image(img.data(), nn, t->kind == MVBT_KIND_VERSIONED, ts, rep);
  if (st) g_last_error = "tree structure check failed: " + std::to_string(rep->violations) + " violations";
  return st;
}

}  // extern "C"
