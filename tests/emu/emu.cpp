// CPU emulation harness for the device tree (test infrastructure).
//
// Compiles include/mvbt_device.cuh for the host (MVBT_HOST_EMULATION) and runs every W-lane tile
// as W host threads: shfl / ballot / sync go through a per-tile exchange buffer and a barrier,
// atomics are GCC atomics on the shared pool. Several tiles run at once, so the lock, split and
// versioning protocols are exercised concurrently on the CPU before any GPU run.
#define MVBT_HOST_EMULATION 1
#include <barrier>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

#include "mvbt.h"
#include "mvbt_device.cuh"

namespace {

struct tile_shared {
  std::barrier<> bar;
  uint64_t slot[32];
  explicit tile_shared(int w) : bar(w) {}
};

// Emulated cooperative-groups tile of W lanes.
struct emu_tile {
  int rank;
  int W;
  tile_shared* sh;
  int thread_rank() const { return rank; }
  void sync() const { sh->bar.arrive_and_wait(); }
  template <class T>
  T shfl(T v, int src) const {
    sh->slot[rank] = (uint64_t)v;
    sync();
    T r = (T)sh->slot[((src % W) + W) % W];
    sync();
    return r;
  }
  unsigned ballot(int p) const {
    sh->slot[rank] = p ? 1u : 0u;
    sync();
    unsigned m = 0;
    for (int i = 0; i < W; ++i)
      if (sh->slot[i]) m |= 1u << i;
    sync();
    return m;
  }
};

struct emu_tree {
  std::vector<uint32_t> pool;
  std::vector<uint32_t> retire_log, free_ring;  // reclamation on
  mvbt::control_block ctl;
  uint32_t capacity;
  int versioned;
  mvbt::device_tree view() {
    mvbt::device_tree t;
    t.pool      = pool.data();
    t.ctl       = &ctl;
    t.versioned = (uint32_t)versioned;
    t.capacity  = capacity;
    t.reclaim   = retire_log.empty() ? 0u : 1u;
    return t;
  }
};

// Runs op(i, tile) for i in [0, n) over `tiles` concurrent tiles of W threads (grid-stride).
void run(uint64_t n, int tiles, int W, const std::function<void(uint64_t, const emu_tile&)>& op) {
  if (n == 0) return;
  if (tiles < 1) tiles = 1;
  std::vector<std::unique_ptr<tile_shared>> sh;
  for (int t = 0; t < tiles; ++t) sh.emplace_back(new tile_shared(W));
  std::vector<std::thread> th;
  for (int t = 0; t < tiles; ++t) {
    for (int l = 0; l < W; ++l) {
      th.emplace_back([&, t, l] {
        mvbt::emu::sm = (uint32_t)t;
        emu_tile tile{l, W, sh[t].get()};
        for (uint64_t i = (uint64_t)t; i < n; i += (uint64_t)tiles) op(i, tile);
      });
    }
  }
  for (auto& x : th) x.join();
}

// Runs fn(warp, tile) on `warps` emulated warps of 32 threads, each split into tiles of W lanes.
void run_warps(int warps, int W, const std::function<void(const emu_tile&, const emu_tile&)>& fn) {
  if (warps < 1) warps = 1;
  const int tpw = 32 / W;
  std::vector<std::unique_ptr<tile_shared>> wsh, tsh;
  for (int w = 0; w < warps; ++w) {
    wsh.emplace_back(new tile_shared(32));
    for (int j = 0; j < tpw; ++j) tsh.emplace_back(new tile_shared(W));
  }
  std::vector<std::thread> th;
  for (int w = 0; w < warps; ++w) {
    for (int l = 0; l < 32; ++l) {
      th.emplace_back([&, w, l] {
        mvbt::emu::sm = (uint32_t)w;
        emu_tile warp{l, 32, wsh[w].get()};
        emu_tile tile{l % W, W, tsh[w * tpw + l / W].get()};
        fn(warp, tile);
      });
    }
  }
  for (auto& x : th) x.join();
}

}  // namespace

extern "C" {

void* emu_create(int versioned, uint32_t capacity, uint32_t spin_limit, uint32_t chunk, int reclaim) {
  auto* t      = new emu_tree();
  t->capacity  = capacity;
  t->versioned = versioned;
  t->pool.assign((size_t)capacity * 32, 0xA5A5A5A5u);  // garbage, as fresh cudaMalloc memory
  for (int i = 0; i < 32 * mvbt::kInitialNodes; ++i) t->pool[i] = mvbt::initial_tree_word(i);
  chunk             = chunk ? chunk : 8;
  uint32_t log_cap  = 0, ring_cap = 0;
  if (reclaim) {  // the same power-of-two sizes as the library
    auto pow2 = [](uint64_t x) {
      uint64_t p = 1;
      while (p < x) p <<= 1;
      return (uint32_t)p;
    };
    log_cap  = pow2(capacity);
    ring_cap = pow2((uint64_t)capacity + (uint64_t)mvbt::kMaxSmSlots * chunk);
    t->retire_log.assign(log_cap, 0xFFFFFFFFu);  // both start empty, as mvbt_create fills them
    t->free_ring.assign(ring_cap, 0xFFFFFFFFu);
  }
  mvbt::init_control(t->ctl, capacity, chunk, spin_limit ? spin_limit : (1u << 20), 4000u * 1000u * 1000u,
                     reclaim ? (unsigned long long)t->retire_log.data() : 0ull,
                     reclaim ? (unsigned long long)t->free_ring.data() : 0ull, log_cap, ring_cap);
  return t;
}

// A reclaim pass, as mvbt_reclaim runs it (k_reclaim + k_reclaim_finish), single-threaded.
void emu_reclaim(void* h, uint32_t M) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  auto& c = t->ctl;
  if (M == mvbt::kReclaimAll) M = c.epoch;
  const unsigned long long head = c.retire_head;
  const unsigned long long n    = std::min<unsigned long long>(c.retire_tail - head, c.reclaim_cap);
  uint32_t* ring                = reinterpret_cast<uint32_t*>(c.free_ring);
  for (unsigned long long i = 0; i < n; ++i) {
    uint32_t idx = 0;
    const int r  = v.reclaim_entry(head + i, M, idx);
    if (r == 1) {  // the ring push of one lane: reserve, write, publish
      ring[c.free_tail++ & (c.ring_cap - 1u)] = idx;
      c.free_avail += 1;
      c.stat_reclaimed += 1;
    }
    if (r == 2) c.rc_first_kept = std::min<uint32_t>(c.rc_first_kept, (uint32_t)i);
  }
  v.reclaim_publish();
}

void emu_destroy(void* h) { delete static_cast<emu_tree*>(h); }

uint32_t emu_errors(void* h) { return static_cast<emu_tree*>(h)->ctl.error; }
uint32_t emu_bump(void* h) { return static_cast<emu_tree*>(h)->ctl.bump; }
void emu_stats(void* h, uint64_t* out) {
  auto& c = static_cast<emu_tree*>(h)->ctl;
  out[0] = mvbt::stat_total(c, 0);
  out[1] = mvbt::stat_total(c, 1);
  out[2] = c.stat_max_hops;
  out[3] = c.stat_max_steps;
  for (int i = 0; i < 16; ++i) out[4 + i] = c.err_site[i];
  out[20] = c.stat_restarts;
  out[21] = c.reclaim_cap ? c.retire_tail : mvbt::stat_total(c, 0);
  out[22] = c.stat_reclaimed;
  out[23] = c.reclaim_cap ? (uint64_t)std::max<long long>(0, (long long)c.free_avail) : 0;
  out[24] = mvbt::stat_total(c, 2);
  out[25] = c.stat_log_dropped;
}

uint32_t emu_snapshot(void* h) {
  auto* t = static_cast<emu_tree*>(h);
  return __atomic_fetch_add(&t->ctl.epoch, 1u, __ATOMIC_SEQ_CST);
}

#define EMU_DISPATCH(W, BODY)                    \
  if (W == 8) {                                  \
    constexpr int kW = 8;                        \
    BODY;                                        \
  } else {                                       \
    constexpr int kW = 16;                       \
    BODY;                                        \
  }

void emu_insert(void* h, const uint32_t* keys, const uint32_t* vals, uint64_t n, int tiles, int W) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  EMU_DISPATCH(W, run(n, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
    uint32_t E = v.versioned ? v.current_epoch() : 0u;
    v.cooperative_insert<kW>(keys[i], vals[i], tile, E);
  }));
}

void emu_erase(void* h, const uint32_t* keys, uint64_t n, int tiles, int W) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  EMU_DISPATCH(W, run(n, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
    uint32_t E = v.versioned ? v.current_epoch() : 0u;
    v.cooperative_erase<kW>(keys[i], tile, E);
  }));
}

// quiescent != 0: the lookup of a tree no writer changes meanwhile (find_quiescent).
void emu_find(void* h, const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t ts, int tiles, int W,
              int quiescent) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  if (!v.versioned) ts = mvbt::kLatest;
  EMU_DISPATCH(W, run(n, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
    uint32_t r = quiescent ? v.find_quiescent<kW>(keys[i], tile, ts) : v.cooperative_find<kW>(keys[i], tile, ts, true);
    if (tile.thread_rank() == 0) out[i] = r;
  }));
}

// quiescent != 0: the range query of a tree no writer changes meanwhile (range_quiescent).
void emu_range(void* h, const uint32_t* lo, const uint32_t* hi, uint32_t* pairs, uint32_t* counts,
               uint32_t avg_len, uint64_t n, uint32_t ts, int tiles, int W, int quiescent) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  if (!v.versioned) ts = mvbt::kLatest;
  EMU_DISPATCH(W, run(n, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
    uint2* o   = pairs ? reinterpret_cast<uint2*>(pairs) + i * (uint64_t)avg_len : nullptr;
    uint32_t c = quiescent ? v.range_quiescent<kW>(lo[i], hi[i], tile, ts, o, avg_len)
                           : v.cooperative_range_query<kW>(lo[i], hi[i], tile, ts, o, avg_len, true);
    if (counts && tile.thread_rank() == 0) counts[i] = c;
  }));
}

// One run mixing inserts and range queries; queries read snapshot S, inserts land in S + 1.
void emu_insert_range(void* h, const uint32_t* keys, const uint32_t* vals, uint64_t n_ins,
                      const uint32_t* lo, const uint32_t* hi, uint64_t n_rq, uint32_t* pairs,
                      uint32_t* counts, uint32_t avg_len, int tiles, int W) {
  auto* t          = static_cast<emu_tree*>(h);
  auto v           = t->view();
  const uint32_t S = v.versioned ? emu_snapshot(h) : mvbt::kLatest;
  const uint32_t E = v.versioned ? S + 1 : 0u;
  const uint64_t total = n_ins + n_rq;
  EMU_DISPATCH(W, run(total, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
    uint64_t a = (i * n_ins) / total, b = ((i + 1) * n_ins) / total;
    if (b > a) {
      v.cooperative_insert<kW>(keys[a], vals[a], tile, E);
    } else {
      uint64_t r = i - a;
      uint2* o   = pairs ? reinterpret_cast<uint2*>(pairs) + r * (uint64_t)avg_len : nullptr;
      uint32_t c = v.cooperative_range_query<kW>(lo[r], hi[r], tile, S, o, avg_len, true);
      if (counts && tile.thread_rank() == 0) counts[r] = c;
    }
  }));
}

// Sorted runs (the sorted batch front-end): keys[0, n) ascending, pos[i] = the input position of
// keys[i]; each of `tiles` tiles takes one contiguous share of the run and keeps its path memory
// (mvbt::finger, one per lane, as registers are on the GPU). kind: 0 find, 1 range, 2 insert (a
// repeated key: its last occurrence wins; the keys of one leaf under one lock), 3 erase, 4 find and
// 5 range of a tree no writer changes meanwhile.
void emu_sorted_run(void* h, int kind, const uint32_t* keys, const uint32_t* pos, const uint32_t* arg,
                    uint32_t* out, uint32_t* pairs, uint32_t avg_len, uint64_t n, uint32_t ts, int tiles, int W) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  if (!v.versioned) ts = mvbt::kLatest;
  if (n == 0) return;
  if (tiles < 1) tiles = 1;
  const uint64_t per = (n + tiles - 1) / tiles;
  EMU_DISPATCH(W, {
    std::vector<std::unique_ptr<tile_shared>> sh;
    for (int x = 0; x < tiles; ++x) sh.emplace_back(new tile_shared(kW));
    std::vector<std::thread> th;
    for (int x = 0; x < tiles; ++x) {
      for (int l = 0; l < kW; ++l) {
        th.emplace_back([&, x, l] {
          mvbt::emu::sm = (uint32_t)x;
          emu_tile tile{l, kW, sh[x].get()};
          mvbt::finger<kW> f;
          const uint32_t E = v.versioned ? v.current_epoch() : 0u;
          const uint64_t b = (uint64_t)x * per, e = std::min<uint64_t>(n, b + per);
          for (uint64_t i = b; i < e; ++i) {
            const uint32_t k = keys[i];
            if (kind == 2) {
              while (i < e) {
                if (i + 1 < n && keys[i + 1] == keys[i]) {
                  ++i;
                  continue;
                }
                v.insert_run_group<kW>(keys, pos, arg, i, e, n, tile, E, f);
              }
              break;
            }
            if (kind == 4) {
              const uint32_t r = v.find_quiescent<kW>(k, tile, ts, f.start_for(k, tile), &f);
              if (tile.thread_rank() == 0) out[pos[i]] = r;
            } else if (kind == 5) {
              uint2* o = pairs ? reinterpret_cast<uint2*>(pairs) + pos[i] * (uint64_t)avg_len : nullptr;
              const uint32_t c = v.range_quiescent<kW>(k, arg[pos[i]], tile, ts, o, avg_len, f.start_for(k, tile), &f);
              if (out && tile.thread_rank() == 0) out[pos[i]] = c;
            } else if (kind == 0) {
              const uint32_t r = v.cooperative_find<kW>(k, tile, ts, true, f.start_for(k, tile), &f);
              if (tile.thread_rank() == 0) out[pos[i]] = r;
            } else if (kind == 1) {
              uint2* o = pairs ? reinterpret_cast<uint2*>(pairs) + pos[i] * (uint64_t)avg_len : nullptr;
              const uint32_t c = v.cooperative_range_query<kW>(k, arg[pos[i]], tile, ts, o, avg_len, true,
                                                               f.start_for(k, tile), &f);
              if (out && tile.thread_rank() == 0) out[pos[i]] = c;
            } else {
              v.erase_in_run<kW>(k, tile, E, f);
            }
          }
        });
      }
    }
    for (auto& y : th) y.join();
  });
}

// One run mixing finds of the newest state and erases (the plain tree's concurrent_find_erase).
void emu_find_erase(void* h, const uint32_t* fkeys, uint32_t* out, uint64_t n_find,
                    const uint32_t* ekeys, uint64_t n_erase, int tiles, int W) {
  auto* t              = static_cast<emu_tree*>(h);
  auto v               = t->view();
  const uint64_t total = n_find + n_erase;
  EMU_DISPATCH(W, run(total, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
    uint64_t a = (i * n_erase) / total, b = ((i + 1) * n_erase) / total;
    if (b > a) {
      v.cooperative_erase<kW>(ekeys[a], tile, 0u);
    } else {
      uint32_t r = v.cooperative_find<kW>(fkeys[i - a], tile, mvbt::kLatest, true);
      if (tile.thread_rank() == 0) out[i - a] = r;
    }
  }));
}

// Mixed batches. mode 0: the persistent worker loop (claim order writes-first per batch, batch b
// waits for the writes of batch b - 1); mode 1: one snapshot + one run per batch.
// reclaim = 1: reclamation inside the persistent run (mvbt_batch_plan_set_reclaim) with external
// watermark ext; series (nullable) receives 4 values per batch as mvbt_batch_plan_memory_series.
void emu_batch_run(void* h, uint32_t nb, const uint64_t* off, const uint32_t* type, const uint32_t* key,
                   const uint32_t* arg, const uint64_t* out_off, const uint32_t* cap, uint32_t* result,
                   uint32_t* range_out, int mode, int tiles, int W, int reclaim, uint32_t ext,
                   uint64_t* series) {
  auto* t = static_cast<emu_tree*>(h);
  auto v  = t->view();
  mvbt::batch_view B{type, key, arg, out_off, cap, result, reinterpret_cast<uint2*>(range_out)};
  if (mode == 1) {
    for (uint32_t b = 0; b < nb; ++b) {
      uint32_t S = emu_snapshot(h);
      uint64_t lo = off[b], n = off[b + 1] - off[b];
      EMU_DISPATCH(W, run(n, tiles, kW, [&](uint64_t i, const emu_tile& tile) {
        mvbt::run_batch_op<kW>(v, B, lo + i, S, S + 1, tile);
      }));
    }
    return;
  }
  std::vector<uint32_t> perm(off[nb]), n_writes(nb, 0), writes_done(nb, 0);
  std::vector<uint64_t> wpre(nb + 1, 0), rpre(nb + 1, 0);
  for (uint32_t b = 0; b < nb; ++b) {  // claim order: writes | finds | ranges
    uint64_t pos = off[b];
    for (uint64_t i = off[b]; i < off[b + 1]; ++i)
      if (mvbt::is_write_op(type[i])) perm[pos++] = (uint32_t)i, ++n_writes[b];
    for (uint64_t i = off[b]; i < off[b + 1]; ++i)
      if (type[i] == mvbt::kOpFind) perm[pos++] = (uint32_t)i;
    for (uint64_t i = off[b]; i < off[b + 1]; ++i)
      if (type[i] == mvbt::kOpRange) perm[pos++] = (uint32_t)i;
    wpre[b + 1] = wpre[b] + n_writes[b];
    rpre[b + 1] = rpre[b] + (off[b + 1] - off[b]) - n_writes[b];
  }
  unsigned long long cursors[2] = {0, 0};
  uint32_t done                 = 0;
  uint32_t params[3]            = {nb, t->ctl.epoch, ext};
  mvbt::batch_sched sc{off, perm.data(), n_writes.data(), wpre.data(), rpre.data(), writes_done.data(),
                       &done, &cursors[0], &cursors[1], params};
  std::vector<uint32_t> reads_done(nb, 0);
  std::vector<unsigned long long> tail_at(nb, ~0ull), ser(4ull * nb, 0);
  uint32_t full_done           = 0;
  unsigned long long rc_limit  = 0;
  if (reclaim && t->ctl.reclaim_cap) {  // as k_batch_begin_reclaim
    const uint32_t S0 = params[1];
    rc_limit      = (ext == mvbt::kReclaimAll || S0 <= ext) ? t->ctl.retire_tail : t->ctl.retire_head;
    sc.reads_done = reads_done.data();
    sc.full_done  = &full_done;
    sc.tail_at    = tail_at.data();
    sc.rc_limit   = &rc_limit;
    sc.series     = ser.data();
  }
  EMU_DISPATCH(W, run_warps(std::max(1, tiles * kW / 32), kW, [&](const emu_tile& warp, const emu_tile& tile) {
    mvbt::batched_worker<kW>(v, B, sc, warp, tile);
  }));
  t->ctl.epoch = params[1] + nb;
  if (series && sc.series) std::memcpy(series, ser.data(), ser.size() * sizeof(uint64_t));
}

int emu_validate(void* h, uint32_t ts, mvbt_report* rep) {
  auto* t     = static_cast<emu_tree*>(h);
  uint64_t nn = std::min<uint64_t>(t->ctl.bump, t->capacity);
  return mvbt_validate_image(t->pool.data(), nn, t->versioned, ts, rep);
}

}  // extern "C"
