// Mixed operation batches: one persistent launch for many batches (device work queue, optional
// CUDA-graph replay) and the plain mode with one host launch per batch.
//
// A batch plan owns the scratch the persistent path needs: the claim order (writes first in each
// batch), per-batch write counters, the claim cursor and a pinned staging area for the batch
// offsets, so a captured graph can be replayed for any batch list up to the plan's limits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "mvbt.h"
#include "mvbt_device.cuh"

namespace cg = cooperative_groups;
using mvbt::batch_sched;
using mvbt::batch_view;
using mvbt::device_tree;

// Internal helpers shared with mvbt_tree.cu.
extern "C" int mvbt_internal_view(mvbt_tree* t, device_tree* view, int* tile_width, int* block_size,
                                  int* num_sms, uint32_t* blocks_per_sm, uint32_t* max_blocks,
                                  void** control);
extern "C" void mvbt_internal_set_error(const char* msg);
extern "C" void mvbt_internal_note_growth(mvbt_tree* t, uint64_t keys);

struct mvbt_batch_plan {
  mvbt_tree* tree;
  uint64_t max_ops;
  uint32_t max_batches;
  // device scratch
  uint64_t* d_batch_off;  // [max_batches + 1]
  uint32_t* d_params;     // [0] num_batches, [1] snapshot of batch 0
  uint32_t* d_perm;       // [max_ops]
  uint32_t* d_counts;     // n_writes | n_finds | writes_done | fill (3 classes) (each [max_batches]),
                          // then done_batches
  uint64_t* d_pre;        // write-ordinal prefix [max_batches + 1] | read-ordinal prefix [...]
  unsigned long long* d_cursor;  // write cursor, read cursor
  // pinned staging
  uint64_t* h_batch_off;
  uint32_t* h_params;
  // graph cache
  cudaGraphExec_t graph;
  bool have_graph;
  const void* graph_key[8];
  // optional CUDA events around the persistent kernel (PERSISTENT mode), a ring of pairs
  static constexpr int kTimed = 64;
  bool timing;
  uint32_t timed_runs;
  cudaEvent_t ev_begin[kTimed], ev_end[kTimed];
  // launch shape of the persistent path (mvbt_batch_plan_set_launch; autotuning): tile width
  // 0 = the tree's, blocks per SM -1 = the tree's
  int tile_width       = 0;
  int blocks_per_sm    = -1;
  // scratch of mvbt_batch_compact_ranges (grown on demand)
  void* d_scratch        = nullptr;
  uint64_t scratch_bytes = 0;
  // end of the plan's last persistent / graph run: its pinned staging is free once it completes
  cudaEvent_t staging_ev = nullptr;
  bool staging_pending   = false;
  // reclamation inside the persistent runs (mvbt_batch_plan_set_reclaim): reads_done[mb] |
  // full_done, padded to 8-byte words (rc_head_words) | tail_at[mb] | rc_limit | series[4 * mb]
  bool reclaim_on              = false;
  uint32_t reclaim_watermark   = 0xFFFFFFFFu;
  void* d_rc                   = nullptr;
  uint32_t series_batches      = 0;  // batches of the last persistent run with reclamation on
};

namespace {

// uint32 words of the reclamation scratch before its 64-bit part (reads_done[mb], full_done, pad)
inline uint64_t rc_head_words(uint64_t mb) { return (mb + 2) & ~1ull; }

constexpr int kPrepassBlocks = 512;
constexpr int kPrepassThreads = 256;

int fail(int code, const std::string& msg) {
  mvbt_internal_set_error(msg.c_str());
  return code;
}

#define MVBT_TRY(expr)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

__device__ __forceinline__ uint32_t batch_of(const uint64_t* off, uint32_t nb, uint64_t i) {
  uint32_t lo = 0, hi = nb;  // largest b with off[b] <= i
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Op class in the claim order of a batch: writes | finds | ranges.
__device__ __forceinline__ uint32_t op_class(uint32_t type) {
  return mvbt::is_write_op(type) ? 0u : (type == mvbt::kOpFind ? 1u : 2u);
}

// Pass 1: writes and finds per batch (warp-aggregated atomics).
__global__ void k_count_writes(const uint32_t* __restrict__ type, const uint64_t* __restrict__ off,
                               const uint32_t* __restrict__ params, uint32_t* n_writes,
                               uint32_t* n_finds) {
  const uint32_t nb    = params[0];
  const uint64_t total = off[nb];
  const uint32_t lane  = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
  for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x - lane); base < total;
       base += warps * 32) {
    const uint64_t i   = base + lane;
    const uint32_t c   = i < total ? op_class(type[i]) : 2u;
    const bool counted = c < 2u;
    const uint32_t act = __ballot_sync(0xFFFFFFFFu, counted);
    if (counted) {
      const uint32_t b   = batch_of(off, nb, i);
      const uint32_t grp = __match_any_sync(act, (b << 1) | c);
      if (lane == (uint32_t)(__ffs(grp) - 1)) atomicAdd(c == 0 ? &n_writes[b] : &n_finds[b], (uint32_t)__popc(grp));
    }
  }
}

// Pass 2: claim order of every batch: writes, then finds, then ranges.
__global__ void k_place(const uint32_t* __restrict__ type, const uint64_t* __restrict__ off,
                        const uint32_t* __restrict__ params, const uint32_t* __restrict__ n_writes,
                        const uint32_t* __restrict__ n_finds, uint32_t* fill, uint32_t mb,
                        uint32_t* perm) {
  const uint32_t nb    = params[0];
  const uint64_t total = off[nb];
  const uint32_t lane  = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
  for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x - lane); base < total;
       base += warps * 32) {
    const uint64_t i    = base + lane;
    const bool live     = i < total;
    const uint32_t livm = __ballot_sync(0xFFFFFFFFu, live);
    if (!live) continue;
    const uint32_t c    = op_class(type[i]);
    const uint32_t b    = batch_of(off, nb, i);
    const uint32_t grp  = __match_any_sync(livm, (b << 2) | c);
    const uint32_t lead = (uint32_t)(__ffs(grp) - 1);
    const uint32_t rank = __popc(grp & ((1u << lane) - 1u));
    uint32_t slot       = 0;
    if (lane == lead) slot = atomicAdd(&fill[c * mb + b], (uint32_t)__popc(grp));
    slot = __shfl_sync(grp, slot, lead);
    const uint64_t start = c == 0 ? 0u : (c == 1 ? n_writes[b] : n_writes[b] + n_finds[b]);
    perm[off[b] + start + slot + rank] = (uint32_t)i;
  }
}

// First write / read ordinal of every batch (one block; exclusive scans over the batches).
__global__ void __launch_bounds__(1024) k_prefix(const uint64_t* __restrict__ off,
                                                 const uint32_t* __restrict__ params,
                                                 const uint32_t* __restrict__ n_writes, uint64_t* wpre,
                                                 uint64_t* rpre) {
  __shared__ uint64_t sw[1024], sr[1024];
  const uint32_t nb   = params[0];
  const uint32_t per  = (nb + blockDim.x - 1) / blockDim.x;
  const uint32_t b0   = threadIdx.x * per;
  const uint32_t b1   = b0 + per < nb ? b0 + per : nb;
  uint64_t w = 0, r = 0;
  for (uint32_t b = b0; b < b1; ++b) {
    w += n_writes[b];
    r += (off[b + 1] - off[b]) - n_writes[b];
  }
  sw[threadIdx.x] = w;
  sr[threadIdx.x] = r;
  __syncthreads();
  for (uint32_t d = 1; d < blockDim.x; d <<= 1) {
    uint64_t aw = threadIdx.x >= d ? sw[threadIdx.x - d] : 0;
    uint64_t ar = threadIdx.x >= d ? sr[threadIdx.x - d] : 0;
    __syncthreads();
    sw[threadIdx.x] += aw;
    sr[threadIdx.x] += ar;
    __syncthreads();
  }
  uint64_t pw = threadIdx.x ? sw[threadIdx.x - 1] : 0, pr = threadIdx.x ? sr[threadIdx.x - 1] : 0;
  for (uint32_t b = b0; b < b1; ++b) {
    wpre[b] = pw;
    rpre[b] = pr;
    pw += n_writes[b];
    pr += (off[b + 1] - off[b]) - n_writes[b];
  }
  if (threadIdx.x == blockDim.x - 1) {
    wpre[nb] = sw[blockDim.x - 1];
    rpre[nb] = sr[blockDim.x - 1];
  }
}

__global__ void k_batch_begin(mvbt::control_block* ctl, uint32_t* params) {
  if (threadIdx.x == 0) {
    __threadfence();
    params[1] = mvbt::ld_relaxed_u32(&ctl->epoch);
  }
}

// Reclamation on: the copies made before this launch (epochs <= its first snapshot S0) are read
// by no snapshot of the launch, so they are reclaimable from the start unless the caller still
// reads a snapshot below S0 (watermark params[2] < S0).
__global__ void k_batch_begin_reclaim(mvbt::control_block* ctl, const uint32_t* params,
                                      unsigned long long* rc_limit) {
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t S0 = params[1], ext = params[2];
    *rc_limit = (ext == mvbt::kReclaimAll || S0 <= ext) ? ctl->retire_tail : ctl->retire_head;
  }
}

__global__ void k_batch_end(mvbt::control_block* ctl, const uint32_t* params) {
  if (threadIdx.x == 0) {
    __threadfence();
    atomicExch(&ctl->epoch, params[1] + params[0]);
  }
}

struct launch_ctx {
  device_tree view;
  int W, block, sms;
  uint32_t bps, maxb;
  mvbt::control_block* ctl;
};

template <class K>
unsigned occupancy_grid(const launch_ctx& c, K kernel) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, c.block, 0);
  if (per_sm < 1) per_sm = 1;
  if (c.bps && (int)c.bps < per_sm) per_sm = (int)c.bps;
  uint64_t g = (uint64_t)per_sm * c.sms;
  if (c.maxb) g = std::min<uint64_t>(g, c.maxb);
  return (unsigned)g;
}

// MinBlocks > 0 caps registers so that many 256-thread blocks fit on an SM (more traversals in
// flight, some spills); selected with mvbt_config::blocks_per_sm.
template <int W, int MinBlocks>
__global__ void __launch_bounds__(256, MinBlocks) k_batched(device_tree T, batch_view B, batch_sched sc) {
  auto warp = cg::tiled_partition<32>(cg::this_thread_block());
  auto tile = cg::tiled_partition<W>(warp);
  mvbt::batched_worker<W>(T, B, sc, warp, tile);
}

template <int W>
void launch_batched(const launch_ctx& c, const batch_view& B, const batch_sched& sc, cudaStream_t s) {
  if (c.bps >= 8) k_batched<W, 8><<<occupancy_grid(c, k_batched<W, 8>), c.block, 0, s>>>(c.view, B, sc);
  else if (c.bps >= 6) k_batched<W, 6><<<occupancy_grid(c, k_batched<W, 6>), c.block, 0, s>>>(c.view, B, sc);
  else if (c.bps >= 4) k_batched<W, 4><<<occupancy_grid(c, k_batched<W, 4>), c.block, 0, s>>>(c.view, B, sc);
  else k_batched<W, 3><<<occupancy_grid(c, k_batched<W, 3>), c.block, 0, s>>>(c.view, B, sc);
}

// One batch [begin, end) in one launch: reads at the snapshot in snap_word, writes one epoch later.
template <int W>
__global__ void __launch_bounds__(256) k_mixed(device_tree T, batch_view B, uint64_t begin,
                                               uint64_t end, const uint32_t* snap_word) {
  auto tile        = cg::tiled_partition<W>(cg::this_thread_block());
  const uint32_t S = mvbt::ld_relaxed_u32(snap_word);
  const uint64_t tiles = ((uint64_t)gridDim.x * blockDim.x) / W;
  for (uint64_t i = begin + ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / W; i < end; i += tiles)
    mvbt::run_batch_op<W>(T, B, i, S, S + 1, tile);
}

__global__ void k_snapshot_word(mvbt::control_block* ctl, uint32_t* out) {
  if (threadIdx.x == 0) {
    __threadfence();
    *out = atomicAdd(&ctl->epoch, 1u);
  }
}

int enqueue_persistent(mvbt_batch_plan* p, const launch_ctx& c, const batch_view& B, cudaStream_t s) {
  const uint32_t mb = p->max_batches;
  MVBT_TRY(cudaMemcpyAsync(p->d_batch_off, p->h_batch_off, (mb + 1) * sizeof(uint64_t),
                           cudaMemcpyHostToDevice, s));
  MVBT_TRY(cudaMemcpyAsync(p->d_params, p->h_params, 3 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  MVBT_TRY(cudaMemsetAsync(p->d_counts, 0, (6ull * mb + 4) * sizeof(uint32_t), s));
  uint32_t* rc_reads            = nullptr;
  unsigned long long* rc_tail   = nullptr;
  unsigned long long* rc_series = nullptr;
  if (p->reclaim_on) {
    rc_reads  = static_cast<uint32_t*>(p->d_rc);
    rc_tail   = reinterpret_cast<unsigned long long*>(rc_reads + rc_head_words(mb));
    rc_series = rc_tail + mb + 1;
    MVBT_TRY(cudaMemsetAsync(rc_reads, 0, rc_head_words(mb) * sizeof(uint32_t), s));
    MVBT_TRY(cudaMemsetAsync(rc_tail, 0xFF, mb * sizeof(unsigned long long), s));
    MVBT_TRY(cudaMemsetAsync(rc_series, 0, 4ull * mb * sizeof(unsigned long long), s));
  }
  MVBT_TRY(cudaMemsetAsync(p->d_cursor, 0, 2 * sizeof(unsigned long long), s));
  uint32_t* nw    = p->d_counts;
  uint32_t* nf    = p->d_counts + mb;
  uint32_t* wdone = p->d_counts + 2 * mb;
  uint32_t* fill  = p->d_counts + 3 * mb;
  uint32_t* done  = p->d_counts + 6 * mb;
  uint64_t* wpre  = p->d_pre;
  uint64_t* rpre  = p->d_pre + (mb + 1);
  k_count_writes<<<kPrepassBlocks, kPrepassThreads, 0, s>>>(B.type, p->d_batch_off, p->d_params, nw, nf);
  k_place<<<kPrepassBlocks, kPrepassThreads, 0, s>>>(B.type, p->d_batch_off, p->d_params, nw, nf, fill,
                                                     mb, p->d_perm);
  k_prefix<<<1, 1024, 0, s>>>(p->d_batch_off, p->d_params, nw, wpre, rpre);
  k_batch_begin<<<1, 32, 0, s>>>(c.ctl, p->d_params);
  if (p->reclaim_on) k_batch_begin_reclaim<<<1, 32, 0, s>>>(c.ctl, p->d_params, rc_tail + mb);
  batch_sched sc;
  sc.batch_off    = p->d_batch_off;
  sc.perm         = p->d_perm;
  sc.n_writes     = nw;
  sc.wpre         = wpre;
  sc.rpre         = rpre;
  sc.writes_done  = wdone;
  sc.done_batches = done;
  sc.wcursor      = p->d_cursor;
  sc.rcursor      = p->d_cursor + 1;
  sc.params       = p->d_params;
  if (p->reclaim_on) {
    sc.reads_done = rc_reads;
    sc.full_done  = rc_reads + mb;
    sc.tail_at    = rc_tail;
    sc.rc_limit   = rc_tail + mb;
    sc.series     = rc_series;
  }
  const int slot = (int)(p->timed_runs % mvbt_batch_plan::kTimed);
  if (p->timing) cudaEventRecord(p->ev_begin[slot], s);
  if (c.W == 8) launch_batched<8>(c, B, sc, s);
  else launch_batched<16>(c, B, sc, s);
  if (p->timing) {
    cudaEventRecord(p->ev_end[slot], s);
    ++p->timed_runs;
  }
  k_batch_end<<<1, 32, 0, s>>>(c.ctl, p->d_params);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("batched launch: ") + cudaGetErrorString(e));
  return MVBT_OK;
}

}  // namespace

extern "C" {

int mvbt_batch_plan_set_launch(mvbt_batch_plan* p, int tile_width, int blocks_per_sm) {
  if (!p) return fail(MVBT_ERR_BAD_ARG, "null plan");
  if (tile_width != 0 && tile_width != 8 && tile_width != 16) return fail(MVBT_ERR_BAD_ARG, "tile_width must be 0, 8 or 16");
  if (blocks_per_sm < -1 || blocks_per_sm > 32) return fail(MVBT_ERR_BAD_ARG, "blocks_per_sm must be in [-1, 32]");
  if (p->have_graph) {
    cudaGraphExecDestroy(p->graph);
    p->have_graph = false;
  }
  p->tile_width    = tile_width;
  p->blocks_per_sm = blocks_per_sm;
  return MVBT_OK;
}

int mvbt_batch_plan_create(mvbt_tree* tree, uint64_t max_ops, uint32_t max_batches,
                           mvbt_batch_plan** out) {
  if (!tree || !out || max_ops == 0 || max_batches == 0 || max_ops > 0xFFFFFFFFull)
    return fail(MVBT_ERR_BAD_ARG, "bad batch plan arguments");
  device_tree v;
  int W, bs, sms;
  uint32_t bps, maxb;
  void* ctl;
  int st = mvbt_internal_view(tree, &v, &W, &bs, &sms, &bps, &maxb, &ctl);
  if (st) return st;
  if (!v.versioned) return fail(MVBT_ERR_NOT_SUPPORTED, "mixed batches need a versioned tree");
  auto* p        = new mvbt_batch_plan();
  p->tree        = tree;
  p->max_ops     = max_ops;
  p->max_batches = max_batches;
  bool ok = cudaMalloc(&p->d_batch_off, (max_batches + 1) * sizeof(uint64_t)) == cudaSuccess &&
            cudaMalloc(&p->d_params, 64) == cudaSuccess &&
            cudaMalloc(&p->d_perm, max_ops * sizeof(uint32_t)) == cudaSuccess &&
            cudaMalloc(&p->d_counts, (6ull * max_batches + 4) * sizeof(uint32_t)) == cudaSuccess &&
            cudaMalloc(&p->d_pre, 2ull * (max_batches + 1) * sizeof(uint64_t)) == cudaSuccess &&
            cudaMalloc(&p->d_cursor, 2 * sizeof(unsigned long long)) == cudaSuccess &&
            cudaMallocHost(&p->h_batch_off, (max_batches + 1) * sizeof(uint64_t)) == cudaSuccess &&
            cudaMallocHost(&p->h_params, 64) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    mvbt_batch_plan_destroy(p);
    return fail(MVBT_ERR_OUT_OF_MEMORY, "batch plan allocation failed");
  }
  *out = p;
  return MVBT_OK;
}

int mvbt_batch_plan_destroy(mvbt_batch_plan* p) {
  if (!p) return MVBT_OK;
  cudaDeviceSynchronize();
  if (p->have_graph) cudaGraphExecDestroy(p->graph);
  cudaFree(p->d_batch_off);
  cudaFree(p->d_params);
  cudaFree(p->d_perm);
  cudaFree(p->d_counts);
  cudaFree(p->d_pre);
  cudaFree(p->d_cursor);
  cudaFreeHost(p->h_batch_off);
  cudaFreeHost(p->h_params);
  if (p->d_scratch) cudaFree(p->d_scratch);
  if (p->d_rc) cudaFree(p->d_rc);
  if (p->staging_ev) cudaEventDestroy(p->staging_ev);
  mvbt_batch_plan_timing(p, 0);
  delete p;
  return MVBT_OK;
}

// Serving-engine hooks (mvbt_serve.cu). The engine writes a launch's batch offsets straight into
// the plan's pinned staging and enqueues the persistent run without the stream synchronisation
// mvbt_batch_run does: it owns one plan per pipeline slot and reuses a plan only after that
// slot's previous launch has completed.
uint64_t* mvbt_internal_plan_staging(mvbt_batch_plan* p) { return p->h_batch_off; }

// Most ops one run of the plan holds (mvbt_compact.cu sizes its scratch for it on first use).
uint64_t mvbt_internal_plan_max_ops(mvbt_batch_plan* p) { return p ? p->max_ops : 0; }

// Device scratch of at least `bytes` owned by the plan (mvbt_compact.cu); grows by reallocation
// after the device is idle, so callers allocate it once, outside any timed region, by a first call.
void* mvbt_internal_plan_scratch(mvbt_batch_plan* p, uint64_t bytes) {
  if (!p) return nullptr;
  if (p->scratch_bytes >= bytes) return p->d_scratch;
  cudaDeviceSynchronize();
  if (p->d_scratch) cudaFree(p->d_scratch);
  p->d_scratch     = nullptr;
  p->scratch_bytes = 0;
  if (cudaMalloc(&p->d_scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  p->scratch_bytes = bytes;
  return p->d_scratch;
}

int mvbt_internal_batch_enqueue(mvbt_batch_plan* p, uint32_t num_batches, const uint32_t* type,
                                const uint32_t* key, const uint32_t* arg, const uint64_t* out_off,
                                const uint32_t* range_cap, uint32_t* result, mvbt_pair* range_out,
                                void* stream) {
  if (!p || num_batches == 0 || num_batches > p->max_batches) return fail(MVBT_ERR_BAD_ARG, "bad batch count");
  const uint64_t total = p->h_batch_off[num_batches];
  if (total > p->max_ops) return fail(MVBT_ERR_BAD_ARG, "more ops than the plan holds");
  launch_ctx c;
  void* ctl;
  int st = mvbt_internal_view(p->tree, &c.view, &c.W, &c.block, &c.sms, &c.bps, &c.maxb, &ctl);
  if (st) return st;
  mvbt_internal_note_growth(p->tree, total);  // an upper bound on the batches' inserts
  if (p->tile_width) c.W = p->tile_width;
  if (p->blocks_per_sm >= 0) c.bps = (uint32_t)p->blocks_per_sm;
  c.ctl = static_cast<mvbt::control_block*>(ctl);
  for (uint32_t b = num_batches + 1; b <= p->max_batches; ++b) p->h_batch_off[b] = total;
  p->h_params[0] = num_batches;
  p->h_params[1] = 0;
  p->h_params[2] = p->reclaim_watermark;
  if (p->reclaim_on) p->series_batches = num_batches;
  batch_view B;
  B.type      = type;
  B.key       = key;
  B.arg       = arg;
  B.out_off   = out_off;
  B.cap       = range_cap;
  B.result    = result;
  B.range_out = reinterpret_cast<uint2*>(range_out);
  return enqueue_persistent(p, c, B, reinterpret_cast<cudaStream_t>(stream));
}

int mvbt_batch_run(mvbt_batch_plan* p, uint32_t num_batches, const uint64_t* batch_off,
                   const uint32_t* type, const uint32_t* key, const uint32_t* arg,
                   const uint64_t* out_off, const uint32_t* range_cap, uint32_t* result,
                   mvbt_pair* range_out, int mode, void* stream) {
  if (!p || !batch_off || !type || !key || !arg || !result) return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (num_batches == 0) return MVBT_OK;
  if (num_batches > p->max_batches) return fail(MVBT_ERR_BAD_ARG, "more batches than the plan holds");
  const uint64_t total = batch_off[num_batches];
  if (total > p->max_ops) return fail(MVBT_ERR_BAD_ARG, "more ops than the plan holds");
  for (uint32_t b = 0; b < num_batches; ++b)
    if (batch_off[b + 1] < batch_off[b]) return fail(MVBT_ERR_BAD_ARG, "batch offsets must not decrease");
  if (batch_off[0] != 0) return fail(MVBT_ERR_BAD_ARG, "batch_off[0] must be 0");
  launch_ctx c;
  void* ctl;
  int st = mvbt_internal_view(p->tree, &c.view, &c.W, &c.block, &c.sms, &c.bps, &c.maxb, &ctl);
  if (st) return st;
  mvbt_internal_note_growth(p->tree, total);  // an upper bound on the batches' inserts
  if (p->tile_width) c.W = p->tile_width;
  if (p->blocks_per_sm >= 0) c.bps = (uint32_t)p->blocks_per_sm;
  c.ctl = static_cast<mvbt::control_block*>(ctl);
  batch_view B;
  B.type      = type;
  B.key       = key;
  B.arg       = arg;
  B.out_off   = out_off;
  B.cap       = range_cap;
  B.result    = result;
  B.range_out = reinterpret_cast<uint2*>(range_out);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (total == 0) return MVBT_OK;

  if (mode == MVBT_BATCH_PER_LAUNCH) {
    // the plain method: per batch, one snapshot and one mixed launch
    for (uint32_t b = 0; b < num_batches; ++b) {
      const uint64_t lo = batch_off[b], hi = batch_off[b + 1];
      k_snapshot_word<<<1, 32, 0, s>>>(c.ctl, p->d_params + 1);
      if (hi == lo) continue;
      uint64_t tiles = (hi - lo);
      uint64_t need  = (tiles * c.W + c.block - 1) / c.block;
      unsigned grid;
      if (c.W == 8) grid = (unsigned)std::min<uint64_t>(need, occupancy_grid(c, k_mixed<8>));
      else grid = (unsigned)std::min<uint64_t>(need, occupancy_grid(c, k_mixed<16>));
      if (c.W == 8) k_mixed<8><<<grid, c.block, 0, s>>>(c.view, B, lo, hi, p->d_params + 1);
      else k_mixed<16><<<grid, c.block, 0, s>>>(c.view, B, lo, hi, p->d_params + 1);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("per-batch launch: ") + cudaGetErrorString(e));
    return MVBT_OK;
  }

  // stage the batch list in pinned memory (the captured graph copies from here); the plan's
  // previous run may still read it: wait for that run alone, so a caller can queue work on other
  // plans and streams meanwhile
  if (p->staging_pending) MVBT_TRY(cudaEventSynchronize(p->staging_ev));
  std::memcpy(p->h_batch_off, batch_off, (num_batches + 1) * sizeof(uint64_t));
  for (uint32_t b = num_batches + 1; b <= p->max_batches; ++b) p->h_batch_off[b] = total;
  p->h_params[0] = num_batches;
  p->h_params[1] = 0;
  p->h_params[2] = p->reclaim_watermark;
  if (p->reclaim_on) p->series_batches = num_batches;

  if (!p->staging_ev) MVBT_TRY(cudaEventCreateWithFlags(&p->staging_ev, cudaEventDisableTiming));
  if (mode == MVBT_BATCH_PERSISTENT) {
    int rs = enqueue_persistent(p, c, B, s);
    if (rs) return rs;
    MVBT_TRY(cudaEventRecord(p->staging_ev, s));
    p->staging_pending = true;
    return MVBT_OK;
  }
  if (p->timing) return fail(MVBT_ERR_BAD_ARG, "kernel timing is available in MVBT_BATCH_PERSISTENT mode");
  if (mode != MVBT_BATCH_GRAPH) return fail(MVBT_ERR_BAD_ARG, "unknown batch mode");

  const void* key_now[8] = {type, key, arg, out_off, range_cap, result, range_out, stream};
  // (a change of launch shape drops the captured graph: mvbt_batch_plan_set_launch)
  if (!p->have_graph || std::memcmp(key_now, p->graph_key, sizeof(key_now)) != 0) {
    if (p->have_graph) {
      cudaGraphExecDestroy(p->graph);
      p->have_graph = false;
    }
    cudaStream_t cap;
    MVBT_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    MVBT_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rs = enqueue_persistent(p, c, B, cap);
    cudaGraph_t g;
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rs) return rs;
    if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    p->have_graph = true;
    std::memcpy(p->graph_key, key_now, sizeof(key_now));
  }
  MVBT_TRY(cudaGraphLaunch(p->graph, s));
  MVBT_TRY(cudaEventRecord(p->staging_ev, s));
  p->staging_pending = true;
  return MVBT_OK;
}

int mvbt_batch_plan_set_reclaim(mvbt_batch_plan* p, int enable, uint32_t min_live_snapshot) {
  if (!p) return fail(MVBT_ERR_BAD_ARG, "null plan");
  device_tree v;
  int W, bs, sms;
  uint32_t bps, maxb;
  void* ctl;
  int st = mvbt_internal_view(p->tree, &v, &W, &bs, &sms, &bps, &maxb, &ctl);
  if (st) return st;
  if (enable && !v.reclaim)
    return fail(MVBT_ERR_NOT_SUPPORTED, "reclamation is off: create the tree with mvbt_config.reclaim = 1");
  if (enable && !p->d_rc) {
    const uint64_t mb    = p->max_batches;
    const uint64_t bytes = rc_head_words(mb) * 4 + (mb + 1) * 8 + 4 * mb * 8;
    if (cudaMalloc(&p->d_rc, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(MVBT_ERR_OUT_OF_MEMORY, "batch plan: reclamation scratch");
    }
  }
  if (p->have_graph && p->reclaim_on != (enable != 0)) {  // the captured run changes shape
    cudaGraphExecDestroy(p->graph);
    p->have_graph = false;
  }
  p->reclaim_on        = enable != 0;
  p->reclaim_watermark = min_live_snapshot;
  return MVBT_OK;
}

int mvbt_batch_plan_memory_series(mvbt_batch_plan* p, uint64_t* out, uint32_t max_batches, uint32_t* n) {
  if (!p || !out || !n) return fail(MVBT_ERR_BAD_ARG, "null argument");
  *n = 0;
  if (!p->d_rc || p->series_batches == 0) return MVBT_OK;
  if (p->staging_pending) MVBT_TRY(cudaEventSynchronize(p->staging_ev));
  const uint32_t k = std::min(max_batches, p->series_batches);
  const uint64_t mb = p->max_batches;
  auto* series = reinterpret_cast<unsigned long long*>(static_cast<uint32_t*>(p->d_rc) + rc_head_words(mb)) + mb + 1;
  MVBT_TRY(cudaMemcpy(out, series, 4ull * k * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  *n = k;
  return MVBT_OK;
}

int mvbt_batch_plan_timing(mvbt_batch_plan* p, int enable) {
  if (!p) return fail(MVBT_ERR_BAD_ARG, "null plan");
  if (enable && !p->timing) {
    for (int i = 0; i < mvbt_batch_plan::kTimed; ++i) {
      MVBT_TRY(cudaEventCreate(&p->ev_begin[i]));
      MVBT_TRY(cudaEventCreate(&p->ev_end[i]));
    }
    p->timing = true;
  } else if (!enable && p->timing) {
    for (int i = 0; i < mvbt_batch_plan::kTimed; ++i) {
      cudaEventDestroy(p->ev_begin[i]);
      cudaEventDestroy(p->ev_end[i]);
    }
    p->timing = false;
  }
  p->timed_runs = 0;
  return MVBT_OK;
}

int mvbt_batch_plan_kernel_times(mvbt_batch_plan* p, float* ms, uint32_t max, uint32_t* n) {
  if (!p || !ms || !n || !p->timing) return fail(MVBT_ERR_BAD_ARG, "timing is not enabled");
  const uint32_t have = std::min<uint32_t>(p->timed_runs, mvbt_batch_plan::kTimed);
  const uint32_t first = p->timed_runs - have;
  uint32_t k = 0;
  for (uint32_t r = first; r < p->timed_runs && k < max; ++r, ++k) {
    const int slot = (int)(r % mvbt_batch_plan::kTimed);
    MVBT_TRY(cudaEventSynchronize(p->ev_end[slot]));
    MVBT_TRY(cudaEventElapsedTime(&ms[k], p->ev_begin[slot], p->ev_end[slot]));
  }
  *n            = k;
  p->timed_runs = 0;
  return MVBT_OK;
}

}  // extern "C"

// ================================================================================================
// Mixed batches without allocation (mvbt_batch_run_noalloc)
//
// Some callers cannot allocate device memory on their call path: a serving loop with a latency
// budget (cudaMalloc and cudaFree can block the whole device for milliseconds), or a host
// application that hands the library a fixed memory budget up front and owns every later
// allocation itself. For them the persistent batched launch can also run with its scratch (claim
// order, per-batch counters, queue cursors, a checked copy of the batch offsets) in the
// fixed-size device array below instead of a batch plan. Every GPU that loads the library holds
// this array (about 4.3 MB) until the process exits. The caller still passes the op, result and
// output arrays.
// ================================================================================================
namespace {

constexpr uint64_t kNoallocPermBytes  = (uint64_t)MVBT_NOALLOC_MAX_OPS * sizeof(uint32_t);
constexpr uint64_t kNoallocOffBytes   = ((MVBT_NOALLOC_MAX_BATCHES + 1ull) * sizeof(uint64_t) + 255) & ~255ull;
constexpr uint64_t kNoallocCountBytes = ((6ull * MVBT_NOALLOC_MAX_BATCHES + 4) * sizeof(uint32_t) + 255) & ~255ull;
constexpr uint64_t kNoallocPreBytes   = (2ull * (MVBT_NOALLOC_MAX_BATCHES + 1) * sizeof(uint64_t) + 255) & ~255ull;
constexpr uint64_t kNoallocMiscBytes  = 256;  // params (2 words) at 0, the two queue cursors at 64
constexpr uint64_t kNoallocBytes =
    kNoallocOffBytes + kNoallocCountBytes + kNoallocPreBytes + kNoallocMiscBytes + kNoallocPermBytes;

// Shared by every call on a device. In host code this name is only a host-side stand-in: the
// kernels get the device address from noalloc_scratch().
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kNoallocMaxDevices = 64;
void* g_noalloc_ptr[kNoallocMaxDevices] = {};
std::mutex g_noalloc_mu;

// Device address of g_noalloc_scratch on device `dev` (which must be current). The first call on
// a device looks it up with cudaGetSymbolAddress; that first call should come before any stream
// capture.
int noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(MVBT_ERR_BAD_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* ptr     = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(MVBT_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = ptr;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return MVBT_OK;
}

// Checks the caller's device batch offsets (off[0] == 0, non-decreasing, off[nb] == num_ops) and
// copies them into the scratch; on a mismatch it hands the kernels an empty batch list and records
// a device error, so no later kernel indexes past the scratch.
__global__ void k_noalloc_setup(const uint64_t* __restrict__ caller_off, uint32_t nb, uint64_t num_ops,
                                uint64_t* off, uint32_t* params, mvbt::control_block* ctl) {
  __shared__ int ok;
  if (threadIdx.x == 0) ok = (caller_off[0] == 0 && caller_off[nb] == num_ops) ? 1 : 0;
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x)
    if (caller_off[b + 1] < caller_off[b]) ok = 0;
  __syncthreads();
  for (uint32_t b = threadIdx.x; b <= nb; b += blockDim.x) off[b] = ok ? caller_off[b] : 0;
  if (threadIdx.x == 0) {
    params[0] = ok ? nb : 0;
    params[1] = 0;
    if (!ok) {
      atomicOr(&ctl->error, mvbt::kErrCorrupt);
      atomicAdd(&ctl->err_site[16], 1u);  // its own site: the offsets check of this entry point
    }
  }
}

}  // namespace

extern "C" int mvbt_batch_run_noalloc(mvbt_tree* tree, uint32_t num_batches, const uint64_t* batch_off,
                                      uint64_t num_ops, const uint32_t* type, const uint32_t* key,
                                      const uint32_t* arg, const uint64_t* out_off,
                                      const uint32_t* range_cap, uint32_t* result,
                                      mvbt_pair* range_out, void* stream) {
  if (!tree || !batch_off || (num_ops && (!type || !key || !arg || !result)))
    return fail(MVBT_ERR_BAD_ARG, "null argument");
  if (num_batches > MVBT_NOALLOC_MAX_BATCHES)
    return fail(MVBT_ERR_BAD_ARG, "mvbt_batch_run_noalloc: more than MVBT_NOALLOC_MAX_BATCHES batches");
  if (num_ops > MVBT_NOALLOC_MAX_OPS)
    return fail(MVBT_ERR_BAD_ARG, "mvbt_batch_run_noalloc: more than MVBT_NOALLOC_MAX_OPS ops");
  if (num_batches == 0 || num_ops == 0) return MVBT_OK;
  launch_ctx c;
  void* ctl;
  int st = mvbt_internal_view(tree, &c.view, &c.W, &c.block, &c.sms, &c.bps, &c.maxb, &ctl);
  if (st) return st;
  if (!c.view.versioned) return fail(MVBT_ERR_NOT_SUPPORTED, "mixed batches need a versioned tree");
  mvbt_internal_note_growth(tree, num_ops);  // an upper bound on the batches' inserts
  c.ctl = static_cast<mvbt::control_block*>(ctl);
  int dev = 0;
  MVBT_TRY(cudaGetDevice(&dev));
  unsigned char* base = nullptr;
  st = noalloc_scratch(dev, &base);
  if (st) return st;
  constexpr uint32_t mb        = MVBT_NOALLOC_MAX_BATCHES;
  uint64_t* off                = reinterpret_cast<uint64_t*>(base);
  uint32_t* counts             = reinterpret_cast<uint32_t*>(base + kNoallocOffBytes);
  uint64_t* pre                = reinterpret_cast<uint64_t*>(base + kNoallocOffBytes + kNoallocCountBytes);
  unsigned char* misc          = base + kNoallocOffBytes + kNoallocCountBytes + kNoallocPreBytes;
  uint32_t* params             = reinterpret_cast<uint32_t*>(misc);
  unsigned long long* cursor   = reinterpret_cast<unsigned long long*>(misc + 64);
  uint32_t* perm               = reinterpret_cast<uint32_t*>(misc + kNoallocMiscBytes);
  batch_view B;
  B.type      = type;
  B.key       = key;
  B.arg       = arg;
  B.out_off   = out_off;
  B.cap       = range_cap;
  B.result    = result;
  B.range_out = reinterpret_cast<uint2*>(range_out);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: counters and cursors start from zero again
  MVBT_TRY(cudaMemsetAsync(counts, 0, (6ull * mb + 4) * sizeof(uint32_t), s));
  MVBT_TRY(cudaMemsetAsync(cursor, 0, 2 * sizeof(unsigned long long), s));
  k_noalloc_setup<<<1, 256, 0, s>>>(batch_off, num_batches, num_ops, off, params, c.ctl);
  uint32_t* nw    = counts;
  uint32_t* nf    = counts + mb;
  uint32_t* wdone = counts + 2 * mb;
  uint32_t* fill  = counts + 3 * mb;
  uint32_t* done  = counts + 6 * mb;
  uint64_t* wpre  = pre;
  uint64_t* rpre  = pre + (mb + 1);
  k_count_writes<<<kPrepassBlocks, kPrepassThreads, 0, s>>>(type, off, params, nw, nf);
  k_place<<<kPrepassBlocks, kPrepassThreads, 0, s>>>(type, off, params, nw, nf, fill, mb, perm);
  k_prefix<<<1, 1024, 0, s>>>(off, params, nw, wpre, rpre);
  k_batch_begin<<<1, 32, 0, s>>>(c.ctl, params);
  batch_sched sc;
  sc.batch_off    = off;
  sc.perm         = perm;
  sc.n_writes     = nw;
  sc.wpre         = wpre;
  sc.rpre         = rpre;
  sc.writes_done  = wdone;
  sc.done_batches = done;
  sc.wcursor      = cursor;
  sc.rcursor      = cursor + 1;
  sc.params       = params;
  if (c.W == 8) launch_batched<8>(c, B, sc, s);
  else launch_batched<16>(c, B, sc, s);
  k_batch_end<<<1, 32, 0, s>>>(c.ctl, params);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("batched launch (noalloc): ") + cudaGetErrorString(e));
  return MVBT_OK;
}
