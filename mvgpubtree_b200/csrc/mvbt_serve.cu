// Serving engine: a host request loop with continuous batching over the persistent batch path.
//
// mvbt_serve_trace plays a trace of requests against the tree as a server would. The loop runs on
// the calling thread with a session clock (steady_clock, ns from the start):
//   * completions: the oldest launch whose result copies have finished completes its requests
//     (done_ns = the clock when the host sees it);
//   * admission: while a pipeline slot is free, the requests that have arrived are admitted in
//     arrival order into one launch, up to the slot's op, request and range-output budgets and
//     while the free-node estimate covers their writes;
//   * launch: the admitted requests' op arrays are contiguous in the trace, so one async copy per
//     array (input stream) stages them; the compute stream waits for the copy, runs a reclaim pass
//     when one is due, runs the persistent batch kernel (one batch, and so one snapshot, per
//     request) and writes the tree's node usage to mapped host memory; the output stream then
//     returns the results and the range pairs straight into the caller's arrays. Separate input
//     and output streams let the next launch's inputs cross while this launch runs.
// Launches run one after another on the compute stream, so every request's reads see all earlier
// requests' writes; copies of the next launch overlap the running one.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "mvbt.h"
#include "mvbt_device.cuh"

using mvbt::device_tree;

extern "C" int mvbt_internal_view(mvbt_tree* t, device_tree* view, int* tile_width, int* block_size,
                                  int* num_sms, uint32_t* blocks_per_sm, uint32_t* max_blocks,
                                  void** control);
extern "C" void mvbt_internal_set_error(const char* msg);
extern "C" uint64_t* mvbt_internal_plan_staging(mvbt_batch_plan* p);
extern "C" int mvbt_internal_batch_enqueue(mvbt_batch_plan* p, uint32_t num_batches, const uint32_t* type,
                                           const uint32_t* key, const uint32_t* arg, const uint64_t* out_off,
                                           const uint32_t* range_cap, uint32_t* result, mvbt_pair* range_out,
                                           void* stream);

namespace {

int fail(int code, const std::string& msg) {
  mvbt_internal_set_error(msg.c_str());
  return code;
}

// Node usage after a launch: [0] bump pointer, [1] reclaimed nodes waiting for reuse, [2] epoch,
// [3] reclamation lag: version copies retired and not yet freed (retire-log entries).
__global__ void k_usage(const mvbt::control_block* c, unsigned long long* out) {
  if (threadIdx.x == 0) {
    const long long avail = (long long)c->free_avail;
    out[0] = c->bump;
    out[1] = c->reclaim_cap && avail > 0 ? (unsigned long long)avail : 0ull;
    out[2] = c->epoch;
    out[3] = c->reclaim_cap ? c->retire_tail - c->retire_head : 0ull;
  }
}

struct slot_t {
  mvbt_batch_plan* plan = nullptr;
  uint32_t *type = nullptr, *key = nullptr, *arg = nullptr, *cap = nullptr, *result = nullptr;
  uint64_t* off     = nullptr;
  mvbt_pair* range  = nullptr;
  cudaEvent_t h2d   = nullptr, kdone = nullptr, done = nullptr;
  unsigned long long* usage     = nullptr;  // mapped host memory [3]
  unsigned long long* usage_dev = nullptr;
  uint32_t r0 = 0, r1 = 0;
  uint64_t reserve = 0;
  bool busy        = false;
};

struct session {
  std::vector<slot_t> slots;
  cudaStream_t cs = nullptr, xs = nullptr, ys = nullptr;  // compute, inputs, outputs
  ~session() {
    if (cs) cudaStreamSynchronize(cs);
    if (xs) cudaStreamSynchronize(xs);
    if (ys) cudaStreamSynchronize(ys);
    for (auto& s : slots) {
      if (s.plan) mvbt_batch_plan_destroy(s.plan);
      for (void* p : {(void*)s.type, (void*)s.key, (void*)s.arg, (void*)s.cap, (void*)s.result, (void*)s.off,
                      (void*)s.range})
        if (p) cudaFree(p);
      for (cudaEvent_t e : {s.h2d, s.kdone, s.done})
        if (e) cudaEventDestroy(e);
      if (s.usage) cudaFreeHost(s.usage);
    }
    if (cs) cudaStreamDestroy(cs);
    if (xs) cudaStreamDestroy(xs);
    if (ys) cudaStreamDestroy(ys);
  }
};

#define SERVE_TRY(expr)                                                                              \
  do {                                                                                               \
    cudaError_t e_ = (expr);                                                                         \
    if (e_ != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

extern "C" {

void mvbt_serve_config_init(mvbt_serve_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->max_ops_per_launch      = 1ull << 21;
  cfg->max_range_pairs         = 32ull << 21;
  cfg->max_requests_per_launch = 1024;
  cfg->pipeline_depth          = 2;
  cfg->mode                    = MVBT_BATCH_PERSISTENT;
  cfg->reclaim_every           = 0;
  cfg->nodes_per_write         = 3;
  cfg->reserve_nodes           = 1ull << 16;
}

int mvbt_serve_trace(mvbt_tree* tree, const mvbt_serve_config* cfg_in, uint32_t R, const uint64_t* req_off,
                     const uint64_t* arrival, const uint32_t* type, const uint32_t* key, const uint32_t* arg,
                     const uint64_t* out_off, const uint32_t* range_cap, uint32_t* result, mvbt_pair* range_out,
                     uint64_t* done_ns, uint32_t* snapshot, mvbt_serve_stats* stats) {
  if (!tree || !req_off || !arrival || !done_ns) return fail(MVBT_ERR_BAD_ARG, "null argument");
  mvbt_serve_config cfg;
  mvbt_serve_config_init(&cfg);
  if (cfg_in) {
    cfg = *cfg_in;
    if (!cfg.max_ops_per_launch) cfg.max_ops_per_launch = 1ull << 21;
    if (!cfg.max_range_pairs) cfg.max_range_pairs = 32 * cfg.max_ops_per_launch;
    if (!cfg.max_requests_per_launch) cfg.max_requests_per_launch = 1024;
    if (!cfg.pipeline_depth) cfg.pipeline_depth = 2;
    if (!cfg.nodes_per_write) cfg.nodes_per_write = 3;
    if (!cfg.reserve_nodes) cfg.reserve_nodes = 1ull << 16;
  }
  if (cfg.snapshots > MVBT_SERVE_SNAPSHOT_PER_REQUEST) return fail(MVBT_ERR_BAD_ARG, "unknown snapshots mode");
  if (cfg.mode != MVBT_BATCH_PERSISTENT && cfg.mode != MVBT_BATCH_PER_LAUNCH)
    return fail(MVBT_ERR_BAD_ARG, "serving mode must be MVBT_BATCH_PERSISTENT or MVBT_BATCH_PER_LAUNCH");
  if (cfg.pipeline_depth > 8) return fail(MVBT_ERR_BAD_ARG, "pipeline_depth is at most 8");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (R == 0) return MVBT_OK;
  const uint64_t total_ops = req_off[R];
  if (total_ops && (!type || !key || !arg || !result)) return fail(MVBT_ERR_BAD_ARG, "null op array");

  int kind = 0, W = 0, dev = 0;
  int st = mvbt_get_info(tree, &kind, &W, &dev);
  if (st) return st;
  if (kind != MVBT_KIND_VERSIONED)
    return fail(MVBT_ERR_NOT_SUPPORTED, "serving needs the versioned tree (one snapshot per request)");
  SERVE_TRY(cudaSetDevice(dev));
  // The engine's streams do not synchronise with the legacy default stream, so work the caller
  // queued on any stream (the tree's build, say) must finish before the first launch: writes in
  // an older epoch may not run beside the session's.
  SERVE_TRY(cudaDeviceSynchronize());
  device_tree view;
  int block = 0, sms = 0;
  uint32_t bps = 0, maxb = 0;
  void* ctl = nullptr;
  st = mvbt_internal_view(tree, &view, &W, &block, &sms, &bps, &maxb, &ctl);
  if (st) return st;
  if ((cfg.reclaim_every || cfg.reclaim_in_launch || cfg.max_reclaim_lag) && !view.reclaim)
    return fail(MVBT_ERR_NOT_SUPPORTED, "reclamation needs a tree created with config.reclaim = 1");
  const uint32_t max_req = cfg.mode == MVBT_BATCH_PER_LAUNCH ? 1u : cfg.max_requests_per_launch;
  // batches per launch: one per request, or the whole admitted group as one batch
  const bool per_request = cfg.snapshots == MVBT_SERVE_SNAPSHOT_PER_REQUEST;

  // per request: write count and range-output region [rp0, rp1) (slots increase in op order)
  std::vector<uint64_t> rp0(R), rp1(R), writes(R);
  uint64_t range_end = 0;
  bool have_range    = false;
  for (uint32_t r = 0; r < R; ++r) {
    if (req_off[r + 1] < req_off[r]) return fail(MVBT_ERR_BAD_ARG, "req_off must not decrease");
    if (r && arrival[r] < arrival[r - 1]) return fail(MVBT_ERR_BAD_ARG, "arrival_ns must not decrease");
    if (req_off[r + 1] - req_off[r] > cfg.max_ops_per_launch)
      return fail(MVBT_ERR_BAD_ARG, "a request has more ops than max_ops_per_launch");
    uint64_t w = 0, first = UINT64_MAX;
    for (uint64_t i = req_off[r]; i < req_off[r + 1]; ++i) {
      const uint32_t t = type[i];
      if (t == MVBT_OP_INSERT || t == MVBT_OP_ERASE) ++w;
      if (t == MVBT_OP_RANGE) {
        if (!out_off || !range_cap || !range_out) return fail(MVBT_ERR_BAD_ARG, "range ops need out_off, range_cap and range_out");
        if (have_range && out_off[i] < range_end)
          return fail(MVBT_ERR_BAD_ARG, "range slots must be disjoint and increasing in op order");
        if (first == UINT64_MAX) first = out_off[i];
        range_end  = out_off[i] + range_cap[i];
        have_range = true;
      }
    }
    writes[r] = w;
    rp0[r]    = first == UINT64_MAX ? range_end : first;
    rp1[r]    = range_end;
    if (rp1[r] - rp0[r] > cfg.max_range_pairs)
      return fail(MVBT_ERR_BAD_ARG, "a request needs more range pairs than max_range_pairs");
  }

  session S;
  SERVE_TRY(cudaStreamCreateWithFlags(&S.cs, cudaStreamNonBlocking));
  SERVE_TRY(cudaStreamCreateWithFlags(&S.xs, cudaStreamNonBlocking));
  SERVE_TRY(cudaStreamCreateWithFlags(&S.ys, cudaStreamNonBlocking));
  S.slots.resize(cfg.pipeline_depth);
  const uint64_t mo = cfg.max_ops_per_launch, mp = cfg.max_range_pairs;
  for (auto& s : S.slots) {
    st = mvbt_batch_plan_create(tree, mo, per_request ? max_req : 1u, &s.plan);
    if (st) return st;
    // every snapshot of the session is taken and read inside its launch: none is held outside
    if (cfg.reclaim_in_launch && cfg.mode == MVBT_BATCH_PERSISTENT) {
      st = mvbt_batch_plan_set_reclaim(s.plan, 1, MVBT_RECLAIM_ALL);
      if (st) return st;
    }
    SERVE_TRY(cudaMalloc(&s.type, mo * 4));
    SERVE_TRY(cudaMalloc(&s.key, mo * 4));
    SERVE_TRY(cudaMalloc(&s.arg, mo * 4));
    SERVE_TRY(cudaMalloc(&s.cap, mo * 4));
    SERVE_TRY(cudaMalloc(&s.result, mo * 4));
    SERVE_TRY(cudaMalloc(&s.off, mo * 8));
    SERVE_TRY(cudaMalloc(&s.range, std::max<uint64_t>(mp, 1) * sizeof(mvbt_pair)));
    SERVE_TRY(cudaEventCreateWithFlags(&s.h2d, cudaEventDisableTiming));
    SERVE_TRY(cudaEventCreateWithFlags(&s.kdone, cudaEventDisableTiming));
    SERVE_TRY(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
    SERVE_TRY(cudaHostAlloc(&s.usage, 4 * sizeof(unsigned long long), cudaHostAllocMapped));
    SERVE_TRY(cudaHostGetDevicePointer(&s.usage_dev, s.usage, 0));
  }
  auto* cb = static_cast<const mvbt::control_block*>(ctl);
  // node usage and epoch now
  k_usage<<<1, 32, 0, S.cs>>>(cb, S.slots[0].usage_dev);
  SERVE_TRY(cudaStreamSynchronize(S.cs));
  const uint64_t capacity = view.capacity;
  uint64_t in_use         = S.slots[0].usage[0] - S.slots[0].usage[1];
  uint32_t epoch          = (uint32_t)S.slots[0].usage[2];
  uint64_t lag            = S.slots[0].usage[3];
  uint64_t max_lag = lag, lag_waits = 0, high_water = in_use;

  using clk      = std::chrono::steady_clock;
  const auto t0  = clk::now();
  auto now_ns    = [&]() { return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(clk::now() - t0).count(); };
  uint32_t next = 0, ndone = 0, arrived = 0;
  uint64_t reserved = 0, launches = 0, reclaims = 0, since_reclaim = 0, max_waiting = 0, mem_waits = 0,
           max_launch_ops = 0;
  bool force_reclaim = false;
  std::deque<int> inflight;

  auto launch = [&](int si, uint32_t r0, uint32_t r1, uint64_t reserve) -> int {
    slot_t& s        = S.slots[si];
    const uint64_t o0 = req_off[r0], n = req_off[r1] - o0;
    const uint64_t p0 = rp0[r0], p1 = rp1[r1 - 1];
    const uint32_t nb = r1 - r0;
    if (n) {
      SERVE_TRY(cudaMemcpyAsync(s.type, type + o0, n * 4, cudaMemcpyHostToDevice, S.xs));
      SERVE_TRY(cudaMemcpyAsync(s.key, key + o0, n * 4, cudaMemcpyHostToDevice, S.xs));
      SERVE_TRY(cudaMemcpyAsync(s.arg, arg + o0, n * 4, cudaMemcpyHostToDevice, S.xs));
      if (out_off && range_cap) {
        SERVE_TRY(cudaMemcpyAsync(s.cap, range_cap + o0, n * 4, cudaMemcpyHostToDevice, S.xs));
        SERVE_TRY(cudaMemcpyAsync(s.off, out_off + o0, n * 8, cudaMemcpyHostToDevice, S.xs));
      }
    }
    SERVE_TRY(cudaEventRecord(s.h2d, S.xs));
    SERVE_TRY(cudaStreamWaitEvent(S.cs, s.h2d, 0));
    if (view.reclaim && ((cfg.reclaim_every && since_reclaim >= cfg.reclaim_every) || force_reclaim)) {
      // every snapshot of the earlier launches is finished (stream order): free their copies
      int rs = mvbt_reclaim(tree, MVBT_RECLAIM_ALL, S.cs);
      if (rs) return rs;
      ++reclaims;
      since_reclaim = 0;
      force_reclaim = false;
    }
    // range slots are addressed by the trace's out_off: shift the slot's base by p0 pairs
    mvbt_pair* shifted = reinterpret_cast<mvbt_pair*>(reinterpret_cast<uintptr_t>(s.range) - p0 * sizeof(mvbt_pair));
    if (n) {
      if (cfg.mode == MVBT_BATCH_PERSISTENT) {
        uint64_t* stage = mvbt_internal_plan_staging(s.plan);
        const uint32_t lb = per_request ? nb : 1u;
        if (per_request)
          for (uint32_t b = 0; b <= nb; ++b) stage[b] = req_off[r0 + b] - o0;
        else
          stage[0] = 0, stage[1] = n;
        int es = mvbt_internal_batch_enqueue(s.plan, lb, s.type, s.key, s.arg, s.off, s.cap, s.result, shifted, S.cs);
        if (es) return es;
      } else {
        const uint64_t one[2] = {0, n};
        int es = mvbt_batch_run(s.plan, 1, one, s.type, s.key, s.arg, s.off, s.cap, s.result, shifted,
                                MVBT_BATCH_PER_LAUNCH, S.cs);
        if (es) return es;
      }
    }
    k_usage<<<1, 32, 0, S.cs>>>(cb, s.usage_dev);
    SERVE_TRY(cudaGetLastError());
    SERVE_TRY(cudaEventRecord(s.kdone, S.cs));
    SERVE_TRY(cudaStreamWaitEvent(S.ys, s.kdone, 0));
    if (n) SERVE_TRY(cudaMemcpyAsync(result + o0, s.result, n * 4, cudaMemcpyDeviceToHost, S.ys));
    if (p1 > p0)
      SERVE_TRY(cudaMemcpyAsync(range_out + p0, s.range, (p1 - p0) * sizeof(mvbt_pair), cudaMemcpyDeviceToHost, S.ys));
    SERVE_TRY(cudaEventRecord(s.done, S.ys));
    // an empty request still takes its snapshot in the persistent path; the per-launch path
    // takes one per launch
    const bool own = per_request || cfg.mode == MVBT_BATCH_PER_LAUNCH;  // a snapshot per request
    for (uint32_t b = 0; b < nb; ++b)
      if (snapshot) snapshot[r0 + b] = own ? epoch + b : epoch;
    epoch += n ? (own ? nb : 1u) : 0u;
    s.r0 = r0;
    s.r1 = r1;
    s.reserve = reserve;
    s.busy    = true;
    reserved += reserve;
    inflight.push_back(si);
    ++launches;
    ++since_reclaim;
    max_launch_ops = std::max(max_launch_ops, n);
    return MVBT_OK;
  };

  while (ndone < R) {
    bool progress = false;
    // completions, oldest first
    while (!inflight.empty()) {
      slot_t& s       = S.slots[inflight.front()];
      cudaError_t q   = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) return fail(MVBT_ERR_CUDA, std::string("serving launch: ") + cudaGetErrorString(q));
      const uint64_t t = now_ns();
      for (uint32_t r = s.r0; r < s.r1; ++r) done_ns[r] = t;
      ndone += s.r1 - s.r0;
      reserved -= s.reserve;
      in_use     = s.usage[0] - s.usage[1];
      lag        = s.usage[3];
      max_lag    = std::max(max_lag, lag);
      high_water = std::max(high_water, in_use);
      s.busy = false;
      inflight.pop_front();
      progress = true;
    }
    const uint64_t tnow = now_ns();
    while (arrived < R && arrival[arrived] <= tnow) ++arrived;
    max_waiting = std::max<uint64_t>(max_waiting, arrived - next);
    // admission by reclamation lag: too many copies wait in the retire log -- reclaim first
    if (cfg.max_reclaim_lag && lag > cfg.max_reclaim_lag && next < arrived && inflight.size() < S.slots.size()) {
      ++lag_waits;
      if (inflight.empty()) {
        int rs = mvbt_reclaim(tree, MVBT_RECLAIM_ALL, S.cs);
        if (rs) return rs;
        ++reclaims;
        since_reclaim = 0;
        k_usage<<<1, 32, 0, S.cs>>>(cb, S.slots[0].usage_dev);
        SERVE_TRY(cudaStreamSynchronize(S.cs));
        in_use        = S.slots[0].usage[0] - S.slots[0].usage[1];
        lag           = S.slots[0].usage[3];
        force_reclaim = false;
        progress      = true;
      } else {
        force_reclaim = true;  // the next launch starts with a pass
      }
    }
    // admission into a free slot
    if (next < arrived && inflight.size() < S.slots.size() &&
        !(cfg.max_reclaim_lag && lag > cfg.max_reclaim_lag && force_reclaim)) {
      int si = 0;
      while (S.slots[si].busy) ++si;
      const uint64_t gstart = rp0[next];
      uint64_t ops = 0, nodes = 0;
      uint32_t r1 = next;
      bool mem_limited = false;
      while (r1 < arrived && r1 - next < max_req) {
        const uint64_t o = req_off[r1 + 1] - req_off[r1];
        const uint64_t need = writes[r1] * cfg.nodes_per_write;
        if (r1 > next && (ops + o > cfg.max_ops_per_launch || rp1[r1] - gstart > cfg.max_range_pairs)) break;
        if (in_use + reserved + nodes + need + cfg.reserve_nodes > capacity) {
          mem_limited = true;
          break;
        }
        ops += o;
        nodes += need;
        ++r1;
      }
      if (r1 > next) {
        int ls = launch(si, next, r1, nodes);
        if (ls) return ls;
        next     = r1;
        progress = true;
      } else if (mem_limited) {
        ++mem_waits;
        if (inflight.empty()) {
          if (!view.reclaim || force_reclaim)
            return fail(MVBT_ERR_POOL_EXHAUSTED, "serving: the node pool cannot hold the next request");
          // reclaim alone, then read the usage again
          force_reclaim = true;
          int rs        = mvbt_reclaim(tree, MVBT_RECLAIM_ALL, S.cs);
          if (rs) return rs;
          ++reclaims;
          since_reclaim = 0;
          k_usage<<<1, 32, 0, S.cs>>>(cb, S.slots[si].usage_dev);
          SERVE_TRY(cudaStreamSynchronize(S.cs));
          const uint64_t after = S.slots[si].usage[0] - S.slots[si].usage[1];
          if (after >= in_use) return fail(MVBT_ERR_POOL_EXHAUSTED, "serving: reclamation freed no nodes");
          in_use        = after;
          force_reclaim = false;
          progress      = true;
        } else if (view.reclaim) {
          force_reclaim = true;  // the next launch frees what the finished launches left behind
        }
      }
    }
    if (!progress) {
      if (inflight.empty() && next < R && arrival[next] > now_ns() + 20000) {
        std::this_thread::sleep_for(std::chrono::microseconds(5));
      } else {
        std::this_thread::yield();
      }
    }
  }
  SERVE_TRY(cudaStreamSynchronize(S.cs));
  SERVE_TRY(cudaStreamSynchronize(S.xs));
  SERVE_TRY(cudaStreamSynchronize(S.ys));
  if (stats) {
    stats->requests       = R;
    stats->ops            = total_ops;
    stats->launches       = launches;
    stats->reclaims       = reclaims;
    stats->span_ns        = done_ns[R - 1];
    for (uint32_t r = 0; r < R; ++r) stats->span_ns = std::max(stats->span_ns, done_ns[r]);
    stats->max_waiting    = max_waiting;
    stats->memory_waits   = mem_waits;
    stats->max_launch_ops = max_launch_ops;
    stats->max_reclaim_lag  = max_lag;
    stats->lag_waits        = lag_waits;
    stats->nodes_high_water = high_water;
  }
  return MVBT_OK;
}

}  // extern "C"
