// Device-side multiversion B-link tree for sm_100a.
//
// This header is the device half of the library. Its kernels (mvgpubtree_b200/csrc) and user
// kernels call the same tile-cooperative operations, the counterparts of the reference's
// device methods:
//   cooperative_find          <- gpu_blink_tree::cooperative_find (include/gpu_blink_tree.hpp:277-303)
//                                gpu_versioned_btree::cooperative_find(key, tile, alloc, ts, ...)
//                                (include/gpu_versioned_blink_tree.hpp:438-474)
//   cooperative_insert        <- cooperative_insert_blink (include/gpu_blink_tree.hpp:522-733) and
//                                cooperative_insert_versioned_in_place
//                                (include/gpu_versioned_blink_tree.hpp:824-1086)
//   cooperative_erase         <- cooperative_erase (include/gpu_blink_tree.hpp:357-390,
//                                include/gpu_versioned_blink_tree.hpp:393-436)
//   cooperative_range_query   <- cooperative_range_query (include/gpu_blink_tree.hpp:306-355) and
//                                concurrent_cooperative_range_query
//                                (include/gpu_versioned_blink_tree.hpp:504-559)
//   take_snapshot             <- take_snapshot(tile) (include/gpu_versioned_blink_tree.hpp:332-344)
//
// Node format (128 bytes, 128-byte aligned, 32 words):
//   pairs 0..12  {key, value}  leaf: key/value, interior: {separator, child index}; sorted by key,
//                              unused pairs are {0xFFFFFFFF, 0xFFFFFFFF}
//   pair 13      {low fence, mod}     low fence = smallest key the node may hold (fixed for the
//                                     node's life); mod = bit31 lock | bits 0..30 modification
//                                     count, bumped by the release that follows a change
//   pair 14      {high key, link}     high key = exclusive upper fence (0xFFFFFFFF on the
//                                     rightmost node of a level); link = bits 0..27 right-sibling
//                                     index (0x0FFFFFFF = none)
//   pair 15      {ts, older|level}    ts = epoch of this version; bits 28..31 level (0 = leaf),
//                                     bits 0..27 index of the next older version (none = 0x0FFFFFFF)
// A tile of W threads (W = 8 or 16) holds one node in registers: lane l owns pairs
// [l*16/W, (l+1)*16/W), so an 8-lane tile reads a node as eight 16-byte vector loads and a
// 16-lane tile as sixteen 8-byte loads -- one 128-byte line either way.
//
// A node is read as several vector loads that are not one atomic access, so a node read while a
// writer stores it can mix two versions, even inside one lane. Every visit therefore checks
// low <= key (a mixed parent can route one child too far right; the visit then restarts from the
// anchor) and key < high (too far left: follow the right link), and a reader that uses the data of
// a leaf validates it (see recheck_version / read_leaf_latest).
//
// Concurrency protocol (B-link, Lehman-Yao style):
//   * readers never lock; a reader whose key is >= a node's high key follows the right link;
//   * a writer locks one leaf (atomicOr on the lock bit of the mod word, bounded spin with
//     __nanosleep backoff; the release that follows a change clears the bit and bumps the count
//     in one exchange, so the mod word is a sequence lock for readers of the newest state),
//     moves right under lock coupling, and applies its change; a full node splits into itself
//     and a new right sibling (right written first, then left, each followed by a fence), then
//     the writer releases the node and inserts the separator into the parent recorded on its
//     way down (moving right there as needed); node 0 is a fixed anchor whose single entry points
//     at the top of the tree, and the tree grows by building a new top node and re-pointing the
//     anchor, so no node ever changes its level or role (a reader that sees a mix of two
//     versions of a node still follows a valid route);
//   * versioning (versioned trees): a writer in epoch E that first touches a node whose ts < E
//     copies it to a fresh node O and publishes the header {ts = E, older = O} once O is complete,
//     and nodes created by splits in epoch E point to the same O. A reader at snapshot S follows
//     `older` while ts > S, so the version it uses is immutable; a reader under writers validates
//     the leaf it uses with its mod word and header read again after it (recheck_version).
//   * every wait is bounded; on a limit the operation gives up, records an error bit in the
//     control block and returns (no trap, no unbounded loop).
#pragma once

#include <cstdint>

#if defined(MVBT_HOST_EMULATION)
// Host build of this header for the CPU emulation harness (tests/emu): each W-lane tile runs as W
// host threads and the CUDA primitives below map to GCC atomics. The sm_100a build never sees
// this branch.
#include <atomic>
#include <chrono>
#include <thread>
#define MVBT_DEV inline
#define MVBT_COLD static inline
#define MVBT_OUTLINE inline
struct uint2 {
  uint32_t x, y;
};
inline uint2 make_uint2(uint32_t x, uint32_t y) { return uint2{x, y}; }
inline int __popc(uint32_t x) { return __builtin_popcount(x); }
inline int __ffs(uint32_t x) { return __builtin_ffs((int)x); }
inline int __clz(uint32_t x) { return x ? __builtin_clz(x) : 32; }
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void __nanosleep(unsigned) { std::this_thread::yield(); }
template <class T, class U>
inline T atomicOr(T* p, U v) { return __atomic_fetch_or(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U>
inline T atomicAnd(T* p, U v) { return __atomic_fetch_and(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U>
inline T atomicAdd(T* p, U v) { return __atomic_fetch_add(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U>
inline T atomicExch(T* p, U v) { return __atomic_exchange_n(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U, class V>
inline T atomicCAS(T* p, U expected, V desired) {
  T e = (T)expected;
  __atomic_compare_exchange_n(p, &e, (T)desired, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return e;
}
template <class T, class U>
inline T atomicMin(T* p, U v) {
  T cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (cur > (T)v && !__atomic_compare_exchange_n(p, &cur, (T)v, false, __ATOMIC_SEQ_CST, __ATOMIC_RELAXED)) {}
  return cur;
}
template <class T, class U>
inline T atomicMax(T* p, U v) {
  T cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (cur < (T)v && !__atomic_compare_exchange_n(p, &cur, (T)v, false, __ATOMIC_SEQ_CST, __ATOMIC_RELAXED)) {}
  return cur;
}
namespace mvbt {
namespace emu {
inline thread_local uint32_t sm = 0;  // emulated SM id of the calling lane
}
}  // namespace mvbt
#else
#include <cooperative_groups.h>
#ifndef MVBT_DEV
#define MVBT_DEV __device__ __forceinline__
#endif
// Rarely taken paths (chunk refills, the retire log). Inlined: an out-of-line call raises the
// register count of the persistent kernels past the three-blocks-per-SM limit.
#ifndef MVBT_COLD
#define MVBT_COLD __device__ __forceinline__
#endif
// The separator push of a split (taken by a minority of writes). Inlined by default, as the
// persistent kernels need; a translation unit whose kernels are not register-bound defines it as
// __device__ __noinline__ so that one copy of that code is shared by every call site and the hot
// loop of a write stays small in the instruction cache.
#ifndef MVBT_OUTLINE
#define MVBT_OUTLINE __device__ __forceinline__
#endif
#endif

namespace mvbt {
#if !defined(MVBT_HOST_EMULATION)
namespace cg = cooperative_groups;
#endif

// ----------------------------------------------------------------------------------------------
// Constants
// ----------------------------------------------------------------------------------------------
constexpr int kNodeWords      = 32;
constexpr int kDataPairs      = 13;
constexpr int kSplitLeft      = 7;  // a full node plus one entry (14) splits 7 | 7
constexpr uint32_t kEmptyKey  = 0xFFFFFFFFu;
constexpr uint32_t kNotFound  = 0xFFFFFFFFu;
constexpr uint32_t kLatest    = 0xFFFFFFFFu;  // read the newest version
constexpr uint32_t kNone      = 0x0FFFFFFFu;  // "no node" in 28-bit index fields
constexpr uint32_t kIndexMask = 0x0FFFFFFFu;
// Mod word (node word 27): bit 31 lock; bits 0..28 modification count of a live node. A version
// copy is never locked or changed again, so its mod word records instead that it is retired and
// the epoch E it was made in (it is read only at snapshots below E); a node that reclamation
// freed carries kFreeBit until it is reused.
constexpr uint32_t kLockBit    = 0x80000000u;
constexpr uint32_t kRetiredBit = 0x40000000u;
constexpr uint32_t kFreeBit    = 0x20000000u;
constexpr uint32_t kCountMask  = 0x1FFFFFFFu;  // count (live node) or epoch (retired copy)
constexpr int kModWord         = 27;
constexpr uint32_t kRingChunk  = 0x80000000u;  // per-SM chunk base: positions in the free ring
constexpr uint32_t kRingEmpty  = 0xFFFFFFFFu;  // a free-ring slot not written yet (or read already)
constexpr uint32_t kReclaimAll = 0xFFFFFFFFu;  // reclaim watermark: the current epoch
constexpr uint32_t kAnchor    = 0;  // fixed entry node: one entry {0 -> top}, level = top + 1
constexpr uint32_t kFirstLeaf = 1;  // the initial leaf (holds the tombstone {0, 0})
constexpr int kMaxLevels      = 16;
constexpr int kMaxSmSlots     = 256;
constexpr uint32_t kMaxSteps  = 1u << 16;  // node visits per operation before giving up
constexpr uint32_t kCoupledHops  = 4;       // right moves taken while holding a lock
constexpr uint32_t kChaseRestart = 16;      // unlocked right moves before restarting at the anchor

// Sticky error bits in control_block::error.
enum : uint32_t {
  kErrPoolExhausted = 1u,
  kErrSpinLimit     = 2u,
  kErrCorrupt       = 4u,
  kErrStepLimit     = 8u,
};

// Device-resident tree state (one per tree).
struct control_block {
  uint32_t epoch;       // current write epoch == id the next take_snapshot returns
  uint32_t error;       // sticky error bits
  uint32_t bump;        // first never-allocated node index
  uint32_t capacity;    // pool capacity in nodes
  uint32_t chunk;       // nodes per per-SM allocation chunk
  uint32_t spin_limit;  // lock / wait attempts before giving up
  uint32_t wait_ns;     // wall-clock limit of one bounded wait (ns)
  uint32_t reserved;
  unsigned long long stat_cow;    // copy-on-write versions created
  unsigned long long stat_split;  // node splits
  unsigned long long stat_max_hops;   // longest move-right walk under locks
  unsigned long long stat_max_steps;  // longest unlocked descent of a writer (node visits)
  unsigned long long stat_restarts;   // locked approaches abandoned for an unlocked re-approach
  uint32_t err_site[32];              // errors per raising site (diagnostics; 16 = the
                                      // offsets check of mvbt_batch_run_noalloc, 17 = a
                                      // bulk load that did not fit the pool)
  unsigned long long sm_pool[kMaxSmSlots];  // per-SM chunk cursor: (base << 32) | used
  // Reclamation of version copies (off when reclaim_cap == 0). The retire log holds the index of
  // every copy not yet reclaimed, in the order the copies were made (which is epoch order); the
  // free ring the nodes reclamation freed. Allocation refills a per-SM chunk from the free ring
  // before the bump pointer. Both run while kernels run: a copy reserves a log position
  // (retire_tail) and writes it; a reclaimer claims log positions below a limit it knows to be
  // safe (retire_head), frees the copies, reserves ring positions (free_tail), writes them and
  // then counts them in free_avail; an allocation takes free_avail first, then ring positions
  // (free_head), waits for each slot to be written and clears it again (kRingEmpty) as it reads it.
  unsigned long long retire_log;   // device address of uint32_t[reclaim_cap]
  unsigned long long free_ring;    // device address of uint32_t[ring_cap]
  unsigned long long retire_head, retire_tail;  // log positions (monotonic; slot = pos % cap)
  unsigned long long free_head, free_tail;      // ring positions (monotonic; slot = pos % cap)
  unsigned long long free_avail;                // ring entries written and not yet taken (signed)
  uint32_t reclaim_cap;     // retire log entries: a power of two >= pool capacity
  uint32_t rc_first_kept;   // first log entry (relative to retire_head) a pass had to keep
  uint32_t ring_cap;        // free ring slots: a power of two >= capacity + kMaxSmSlots * chunk
  uint32_t reserved2;
  unsigned long long stat_reclaimed;    // nodes freed (passes between kernels and reclamation in them)
  unsigned long long stat_log_dropped;  // copies not logged because the log was full (never freed)
  // Per-SM shares of counters, one 128-B line per SM slot ([slot][0] copies, [slot][1] splits,
  // [slot][2] freed nodes handed out again): the counting atomics of different SMs land on
  // different lines instead of all on one word. stat_cow / stat_split stay 0; a count is its
  // slots' sum (stat_total).
  unsigned long long sm_stats[kMaxSmSlots][16];
};


#if defined(MVBT_HOST_EMULATION)
#define MVBT_HD inline
#else
#define MVBT_HD __host__ __device__ __forceinline__
#endif

// Total of per-SM counter k (0 copies, 1 splits, 2 freed nodes reused) plus the unsharded field.
MVBT_HD unsigned long long stat_total(const control_block& c, int k) {
  unsigned long long s = k == 0 ? c.stat_cow : (k == 1 ? c.stat_split : 0ull);
  for (int i = 0; i < kMaxSmSlots; ++i) s += c.sm_stats[i][k];
  return s;
}

// Word t (0..63) of the initial tree. Node 0 is the anchor: an interior node whose only entry
// {0 -> 1} points at the top of the tree, level 1. Node 1 is a leaf holding the tombstone {0, 0}.
// Both have high key 0xFFFFFFFF, no sibling, ts 0 and no older version. The anchor's single
// entry is the only pointer that changes when the tree grows, and no node ever changes level, so
// a reader that sees a mix of two versions of any node still finds a valid route.
MVBT_HD uint32_t initial_tree_word(int t) {
  const int node = t >> 5, w = t & 31;
  if (w == 26 || w == 27) return 0u;                 // low fence 0, modification count 0
  if (w < 26) {
    if (w == 0) return 0u;                           // first key: 0
    if (w == 1) return node == 0 ? kFirstLeaf : 0u;  // anchor -> leaf 1; tombstone value 0
    return kEmptyKey;
  }
  if (w == 28) return kEmptyKey;                     // high key
  if (w == 29) return kNone;                         // link
  if (w == 30) return 0u;                            // ts
  return (node == 0 ? (1u << 28) : 0u) | kNone;      // level | no older version
}
constexpr int kInitialNodes = 2;

// retire_log / free_ring: device addresses of uint32_t[reclaim_cap] and uint32_t[ring_cap]
// (powers of two), or 0 with reclaim_cap 0 (reclamation off).
MVBT_HD void init_control(control_block& c, uint32_t capacity, uint32_t chunk, uint32_t spin_limit,
                          uint32_t wait_ns, unsigned long long retire_log = 0,
                          unsigned long long free_ring = 0, uint32_t reclaim_cap = 0,
                          uint32_t ring_cap = 0) {
  c.epoch         = 0;
  c.error         = 0;
  c.bump          = kInitialNodes;  // nodes 0 (anchor) and 1 (first leaf)
  c.capacity      = capacity;
  c.chunk         = chunk;
  c.spin_limit    = spin_limit;
  c.wait_ns       = wait_ns;
  c.reserved      = 0;
  c.stat_cow      = 0;
  c.stat_split    = 0;
  c.stat_max_hops  = 0;
  c.stat_restarts  = 0;
  c.stat_max_steps = 0;
  for (int i = 0; i < 32; ++i) c.err_site[i] = 0;
  // used == chunk: the first allocation on each SM refills its chunk from the bump pointer
  for (int i = 0; i < kMaxSmSlots; ++i) c.sm_pool[i] = chunk;
  for (int i = 0; i < kMaxSmSlots; ++i)
    for (int j = 0; j < 16; ++j) c.sm_stats[i][j] = 0;
  c.retire_log       = retire_log;
  c.free_ring        = free_ring;
  c.retire_head      = 0;
  c.retire_tail      = 0;
  c.free_head        = 0;
  c.free_tail        = 0;
  c.free_avail       = 0;
  c.reclaim_cap      = reclaim_cap;
  c.rc_first_kept    = 0xFFFFFFFFu;
  c.ring_cap         = ring_cap;
  c.reserved2        = 0;
  c.stat_reclaimed   = 0;
  c.stat_log_dropped = 0;
}

// ----------------------------------------------------------------------------------------------
// Low-level memory access
// ----------------------------------------------------------------------------------------------
template <int W>
struct node_regs {
  static constexpr int P = 16 / W;  // pairs per lane
  uint32_t k[P];
  uint32_t v[P];
};

#if defined(MVBT_HOST_EMULATION)
MVBT_DEV uint32_t sm_id() { return emu::sm; }
template <class Tile>
MVBT_DEV uint32_t tile_ordinal(const Tile&) { return emu::sm; }
MVBT_DEV unsigned long long global_ns() {
  return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
MVBT_DEV uint32_t ld_relaxed_u32(const uint32_t* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
MVBT_DEV void st_relaxed_u32(uint32_t* p, uint32_t v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
MVBT_DEV unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  return __atomic_load_n(p, __ATOMIC_RELAXED);
}
template <int W>
MVBT_DEV void ld_lane(const uint32_t* p, node_regs<W>& n, bool) {
  for (int j = 0; j < 16 / W; ++j) {
    n.k[j] = __atomic_load_n(p + 2 * j, __ATOMIC_RELAXED);
    n.v[j] = __atomic_load_n(p + 2 * j + 1, __ATOMIC_RELAXED);
  }
}
template <int W>
MVBT_DEV void st_lane(uint32_t* p, const node_regs<W>& n) {
  for (int j = 0; j < 16 / W; ++j) {
    __atomic_store_n(p + 2 * j, n.k[j], __ATOMIC_RELAXED);
    __atomic_store_n(p + 2 * j + 1, n.v[j], __ATOMIC_RELAXED);
  }
}
#else
// Ordinal of the calling tile among the tiles of the launch.
template <class Tile>
MVBT_DEV uint32_t tile_ordinal(const Tile& t) {
  return (blockIdx.x * blockDim.x + threadIdx.x) / t.num_threads();
}
MVBT_DEV uint32_t sm_id() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
}

MVBT_DEV unsigned long long global_ns() {
  unsigned long long r;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(r));
  return r;
}

MVBT_DEV uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t r;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(r) : "l"(p) : "memory");
  return r;
}
MVBT_DEV unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long r;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(r) : "l"(p) : "memory");
  return r;
}
MVBT_DEV void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" : : "l"(p), "r"(v) : "memory");
}

// Loads this lane's share of a node. strong = L2-coherent relaxed loads (needed while writers
// may run in the same kernel); otherwise read-only cached loads.
template <int W>
MVBT_DEV void ld_lane(const uint32_t* p, node_regs<W>& n, bool strong) {
  if constexpr (W == 8) {
    if (strong) {
      asm volatile("ld.relaxed.gpu.global.v4.u32 {%0,%1,%2,%3}, [%4];"
                   : "=r"(n.k[0]), "=r"(n.v[0]), "=r"(n.k[1]), "=r"(n.v[1])
                   : "l"(p)
                   : "memory");
    } else {
      asm("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
          : "=r"(n.k[0]), "=r"(n.v[0]), "=r"(n.k[1]), "=r"(n.v[1])
          : "l"(p));
    }
  } else {
    if (strong) {
      asm volatile("ld.relaxed.gpu.global.v2.u32 {%0,%1}, [%2];"
                   : "=r"(n.k[0]), "=r"(n.v[0])
                   : "l"(p)
                   : "memory");
    } else {
      asm("ld.global.nc.v2.u32 {%0,%1}, [%2];" : "=r"(n.k[0]), "=r"(n.v[0]) : "l"(p));
    }
  }
}

template <int W>
MVBT_DEV void st_lane(uint32_t* p, const node_regs<W>& n) {
  if constexpr (W == 8) {
    asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1,%2,%3,%4};"
                 :
                 : "l"(p), "r"(n.k[0]), "r"(n.v[0]), "r"(n.k[1]), "r"(n.v[1])
                 : "memory");
  } else {
    asm volatile("st.relaxed.gpu.global.v2.u32 [%0], {%1,%2};"
                 :
                 : "l"(p), "r"(n.k[0]), "r"(n.v[0])
                 : "memory");
  }
}

#endif  // MVBT_HOST_EMULATION

// ----------------------------------------------------------------------------------------------
// Register-resident node helpers (all are tile-collective: every lane must call them)
// ----------------------------------------------------------------------------------------------
template <int W>
struct layout {
  static constexpr int P          = 16 / W;
  static constexpr int kFenceLane = 13 / P;  // lane owning pair 13 {low, mod}
  static constexpr int kFenceSlot = 13 % P;
  static constexpr int kLinkLane  = 14 / P;  // lane owning pair 14 {high, link}
  static constexpr int kLinkSlot  = 14 % P;
  static constexpr int kVerLane   = 15 / P;  // lane owning pair 15 {ts, older|level}
  static constexpr int kVerSlot   = 15 % P;
};

struct header {
  uint32_t high;
  uint32_t link;
  uint32_t ts;
  uint32_t ol;   // older | level << 28
  uint32_t low;  // low fence: every key of the node is >= low (fixed for the life of the node)
  uint32_t mod;  // modification count, published before every change of the node
  MVBT_DEV uint32_t level() const { return ol >> 28; }
  MVBT_DEV uint32_t older() const { return ol & kIndexMask; }
  MVBT_DEV uint32_t sibling() const { return link & kIndexMask; }
  MVBT_DEV bool is_leaf() const { return level() == 0; }
};

// Every lane loads the header words (26..31) of the node at p itself: read-only cached loads, for
// readers that run with no writer in flight. They read the 128-byte line the lane's own share
// comes from, so they cost two L1 accesses where get_header costs six shuffles.
#if defined(MVBT_HOST_EMULATION)
MVBT_DEV header ld_header_words(const uint32_t* p) {
  header h;
  h.low  = __atomic_load_n(p + 26, __ATOMIC_RELAXED);
  h.mod  = __atomic_load_n(p + 27, __ATOMIC_RELAXED);
  h.high = __atomic_load_n(p + 28, __ATOMIC_RELAXED);
  h.link = __atomic_load_n(p + 29, __ATOMIC_RELAXED);
  h.ts   = __atomic_load_n(p + 30, __ATOMIC_RELAXED);
  h.ol   = __atomic_load_n(p + 31, __ATOMIC_RELAXED);
  return h;
}
#else
MVBT_DEV header ld_header_words(const uint32_t* p) {
  header h;
  asm("ld.global.nc.v2.u32 {%0,%1}, [%2];" : "=r"(h.low), "=r"(h.mod) : "l"(p + 26));
  asm("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
      : "=r"(h.high), "=r"(h.link), "=r"(h.ts), "=r"(h.ol)
      : "l"(p + 28));
  return h;
}
#endif

MVBT_DEV header make_header(uint32_t low, uint32_t mod, uint32_t high, uint32_t link, uint32_t ts,
                            uint32_t ol) {
  header h;
  h.low  = low;
  h.mod  = mod;
  h.high = high;
  h.link = link;
  h.ts   = ts;
  h.ol   = ol;
  return h;
}

template <int W, class Tile>
MVBT_DEV header get_header(const node_regs<W>& n, const Tile& t) {
  using L = layout<W>;
  header h;
  h.low  = t.shfl(n.k[L::kFenceSlot], L::kFenceLane);
  h.mod  = t.shfl(n.v[L::kFenceSlot], L::kFenceLane);
  h.high = t.shfl(n.k[L::kLinkSlot], L::kLinkLane);
  h.link = t.shfl(n.v[L::kLinkSlot], L::kLinkLane);
  h.ts   = t.shfl(n.k[L::kVerSlot], L::kVerLane);
  h.ol   = t.shfl(n.v[L::kVerSlot], L::kVerLane);
  return h;
}

template <int W, class Tile>
MVBT_DEV void set_header(node_regs<W>& n, const header& h, const Tile& t) {
  using L      = layout<W>;
  const int r  = t.thread_rank();
  if (r == L::kFenceLane) {
    n.k[L::kFenceSlot] = h.low;
    n.v[L::kFenceSlot] = h.mod;
  }
  if (r == L::kLinkLane) {
    n.k[L::kLinkSlot] = h.high;
    n.v[L::kLinkSlot] = h.link;
  }
  if (r == L::kVerLane) {
    n.k[L::kVerSlot] = h.ts;
    n.v[L::kVerSlot] = h.ol;
  }
}

// Pair index of slot j in this lane.
template <int W, class Tile>
MVBT_DEV int pair_index(const Tile& t, int j) {
  return t.thread_rank() * (16 / W) + j;
}

// Number of valid data pairs.
template <int W, class Tile>
MVBT_DEV int count_valid(const node_regs<W>& n, const Tile& t) {
  int c = 0;
#pragma unroll
  for (int j = 0; j < 16 / W; ++j) {
    bool valid = pair_index<W>(t, j) < kDataPairs && n.k[j] != kEmptyKey;
    c += __popc(t.ballot(valid));
  }
  return c;
}

// Number of valid data pairs whose key is < key (= insertion position).
template <int W, class Tile>
MVBT_DEV int count_less(const node_regs<W>& n, uint32_t key, const Tile& t) {
  int c = 0;
#pragma unroll
  for (int j = 0; j < 16 / W; ++j) {
    bool less = pair_index<W>(t, j) < kDataPairs && n.k[j] != kEmptyKey && n.k[j] < key;
    c += __popc(t.ballot(less));
  }
  return c;
}

// Interior search: child of the last pair whose separator is <= key. Returns kNone if no
// separator is <= key (only possible on a corrupt route).
template <int W, class Tile>
MVBT_DEV uint32_t child_for(const node_regs<W>& n, uint32_t key, const Tile& t) {
  constexpr int P = 16 / W;
  int cnt         = 0;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    bool le = pair_index<W>(t, j) < kDataPairs && n.k[j] != kEmptyKey && n.k[j] <= key;
    cnt += le ? 1 : 0;
  }
  uint32_t mask = t.ballot(cnt > 0);
  uint32_t cand = n.v[0];
  if constexpr (P == 2) cand = (cnt == 2) ? n.v[1] : n.v[0];
  int src        = mask ? (31 - __clz(mask)) : 0;
  uint32_t child = t.shfl(cand, src);
  return mask ? child : kNone;
}

// Leaf search: value stored for key, or kNotFound.
template <int W, class Tile>
MVBT_DEV uint32_t leaf_value(const node_regs<W>& n, uint32_t key, const Tile& t) {
  constexpr int P = 16 / W;
  bool hit        = false;
  uint32_t val    = kNotFound;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    if (pair_index<W>(t, j) < kDataPairs && n.k[j] == key) {
      hit = true;
      val = n.v[j];
    }
  }
  uint32_t mask = t.ballot(hit);
  uint32_t r    = t.shfl(val, mask ? (__ffs(mask) - 1) : 0);
  return (mask && key != kEmptyKey) ? r : kNotFound;
}

// Range-query step on one leaf: writes the pairs of n with lo <= key < hi ascending at
// out[count...] (those below cap; out nullable) and returns how many there are. Collective.
template <int W, class Tile>
MVBT_DEV uint32_t leaf_collect(const node_regs<W>& n, uint32_t lo, uint32_t hi, uint2* out, uint32_t cap,
                               uint32_t count, const Tile& t) {
  constexpr int P = 16 / W;
  int first = -1, inr = 0;
  bool in[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int q = pair_index<W>(t, j);
    in[j]       = q < kDataPairs && n.k[j] != kEmptyKey && n.k[j] >= lo && n.k[j] < hi;
    const uint32_t m = t.ballot(in[j]);
    inr += __popc(m);
    if (m) {
      const int f = (__ffs(m) - 1) * P + j;
      first       = (first < 0 || f < first) ? f : first;
    }
  }
  if (out != nullptr) {
#pragma unroll
    for (int j = 0; j < P; ++j) {
      if (in[j]) {
        const uint32_t o = count + (uint32_t)(pair_index<W>(t, j) - first);
        if (o < cap) out[o] = make_uint2(n.k[j], n.v[j]);
      }
    }
  }
  return (uint32_t)inr;
}

// Fetches pair `src` (per-lane index, 0..15) of node n. Collective.
template <int W, class Tile>
MVBT_DEV void fetch_pair(const node_regs<W>& n, int src, uint32_t& k, uint32_t& v, const Tile& t) {
  constexpr int P = 16 / W;
  src             = src < 0 ? 0 : (src > 15 ? 15 : src);
  if constexpr (P == 1) {
    k = t.shfl(n.k[0], src);
    v = t.shfl(n.v[0], src);
  } else {
    int lane    = src >> 1;
    uint32_t k0 = t.shfl(n.k[0], lane), k1 = t.shfl(n.k[1], lane);
    uint32_t v0 = t.shfl(n.v[0], lane), v1 = t.shfl(n.v[1], lane);
    k           = (src & 1) ? k1 : k0;
    v           = (src & 1) ? v1 : v0;
  }
}

// Data pairs of the merged sequence "n's valid pairs with {key, val} inserted at pos":
// entry e < pos -> old e, e == pos -> new, e > pos -> old e - 1. Entries past `total` are empty.
// Output pair q of `out` takes merged entry q + first (q < take), else empty. Header pairs of
// `out` are copied from n.
template <int W, class Tile>
MVBT_DEV void build_from_merged(const node_regs<W>& n,
                                int pos,
                                uint32_t key,
                                uint32_t val,
                                int first,
                                int take,
                                node_regs<W>& out,
                                const Tile& t) {
  constexpr int P = 16 / W;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int q = pair_index<W>(t, j);
    const int e = q + first;
    int src     = (e < pos) ? e : e - 1;
    uint32_t fk, fv;
    fetch_pair<W>(n, src, fk, fv, t);
    if (q >= kDataPairs) {
      out.k[j] = n.k[j];
      out.v[j] = n.v[j];
    } else if (q >= take) {
      out.k[j] = kEmptyKey;
      out.v[j] = kEmptyKey;
    } else if (e == pos) {
      out.k[j] = key;
      out.v[j] = val;
    } else {
      out.k[j] = fk;
      out.v[j] = fv;
    }
  }
}

// Removes data pair pos (shifting the rest down).
template <int W, class Tile>
MVBT_DEV void remove_at(node_regs<W>& n, int pos, const Tile& t) {
  constexpr int P = 16 / W;
  node_regs<W> out;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int q = pair_index<W>(t, j);
    int src     = (q < pos) ? q : q + 1;
    uint32_t fk, fv;
    fetch_pair<W>(n, src, fk, fv, t);
    if (q >= kDataPairs) {
      out.k[j] = n.k[j];
      out.v[j] = n.v[j];
    } else if (src >= kDataPairs) {
      out.k[j] = kEmptyKey;
      out.v[j] = kEmptyKey;
    } else {
      out.k[j] = fk;
      out.v[j] = fv;
    }
  }
  n = out;
}

// Pair index of the data pair holding key, or -1.
template <int W, class Tile>
MVBT_DEV int find_pos(const node_regs<W>& n, uint32_t key, const Tile& t) {
  constexpr int P = 16 / W;
  int pos         = -1;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    uint32_t mask = t.ballot(pair_index<W>(t, j) < kDataPairs && n.k[j] == key);
    int p         = mask ? (__ffs(mask) - 1) * P + j : -1;
    pos           = (pos < 0) ? p : ((p >= 0 && p < pos) ? p : pos);
  }
  return key == kEmptyKey ? -1 : pos;
}

// ----------------------------------------------------------------------------------------------
// The tree view: a plain struct passed to kernels by value.
// ----------------------------------------------------------------------------------------------
// ---- allocation and retirement slow paths (free functions: no copy of the tree view) ----
// Whether the bounded wait that started at t0 (lane 0's clock) has run past `limit` ns, decided by
// lane 0 for the whole tile or warp. Every lane of a group that runs warp-synchronous operations
// inside a wait loop must leave the loop together: a lane that left alone would make the next
// shuffle or ballot of the others name a lane that no longer takes part.
template <class Group>
MVBT_DEV bool wait_expired(unsigned long long t0, unsigned long long limit, const Group& g) {
  uint32_t late = 0;
  if (g.thread_rank() == 0) late = global_ns() - t0 > limit ? 1u : 0u;
  return g.shfl(late, 0) != 0;
}

// Node `used` of the chunk that starts at `base`: consecutive nodes of the bump range, or the node
// stored at consecutive free-ring positions (kRingChunk set). A ring slot is read once: the reader
// waits (bounded) for its pusher to have written it and clears it (kRingEmpty) for the ring's next
// lap. Returns kNone (and records kErrSpinLimit) if the slot stays empty past the wait limit. The
// ring and the retire log start filled with kRingEmpty (all bits set).
MVBT_DEV uint32_t chunk_node(control_block* c, uint32_t base, uint32_t used) {
  if (!(base & kRingChunk)) return base + used;
  uint32_t* slot = reinterpret_cast<uint32_t*>(c->free_ring) +
                   (((unsigned long long)(base & ~kRingChunk) + used) & (c->ring_cap - 1u));
  uint32_t v                  = ld_relaxed_u32(slot);
  const unsigned long long t0 = v == kRingEmpty ? global_ns() : 0;
  while (v == kRingEmpty) {
    if (global_ns() - t0 > c->wait_ns) {
      atomicOr(&c->error, kErrSpinLimit);
      atomicAdd(&c->err_site[18], 1u);
      return kNone;
    }
    __nanosleep(64);
    v = ld_relaxed_u32(slot);
  }
  st_relaxed_u32(slot, kRingEmpty);
  atomicAdd(&c->sm_stats[sm_id() % kMaxSmSlots][2], 1ull);  // a freed node handed out again
  return v;
}
// Takes C free-ring entries for a chunk: one atomic on free_avail (undone if fewer are there),
// then one on the ring head for their positions. False: allocate from the bump pointer instead.
MVBT_DEV bool take_free_chunk(control_block* c, uint32_t C, uint32_t& base) {
  if ((long long)ld_relaxed_u64(&c->free_avail) < (long long)C) return false;
  const long long a = (long long)atomicAdd(&c->free_avail, (unsigned long long)(-(long long)C));
  if (a < (long long)C) {
    atomicAdd(&c->free_avail, (unsigned long long)C);
    return false;
  }
  const unsigned long long h = atomicAdd(&c->free_head, (unsigned long long)C);
  base                       = kRingChunk | (uint32_t)(h & (c->ring_cap - 1u));
  return true;
}
// Appends the nodes of the lanes with `freed` set to the free ring (warp-collective, every lane of
// `warp` calls it): one reservation per warp, the slots written (waiting, bounded, for a slot the
// ring's previous lap has not yet read), then one fence and the count published in free_avail.
// ring_cap >= capacity + kMaxSmSlots * chunk: the entries written and not yet read (free nodes,
// and the rest of per-SM chunks taken from the ring) never fill the ring, so a pusher meets a
// slot of the previous lap only while its reader is about to clear it.
template <class Warp>
MVBT_DEV void ring_push(control_block* c, bool freed, uint32_t node, const Warp& warp) {
  const uint32_t m = warp.ballot(freed);
  if (!m) return;
  const uint32_t lane = warp.thread_rank();
  const int lead      = __ffs(m) - 1;
  unsigned long long base = 0;
  if ((int)lane == lead) base = atomicAdd(&c->free_tail, (unsigned long long)__popc(m));
  base = warp.shfl(base, lead);
  if (freed) {
    uint32_t* slot = reinterpret_cast<uint32_t*>(c->free_ring) +
                     ((base + __popc(m & ((1u << lane) - 1u))) & (c->ring_cap - 1u));
    const unsigned long long t0 = global_ns();
    while (ld_relaxed_u32(slot) != kRingEmpty && global_ns() - t0 <= c->wait_ns) __nanosleep(64);
    st_relaxed_u32(slot, node);
  }
  __threadfence();
  warp.sync();
  if ((int)lane == lead) {
    atomicAdd(&c->free_avail, (unsigned long long)__popc(m));
    atomicAdd(&c->stat_reclaimed, (unsigned long long)__popc(m));
  }
}
// Records a version copy in the retire log. A copy the full log cannot take is never freed
// (counted in stat_log_dropped).
MVBT_COLD void retire_logged(control_block* c, uint32_t copy) {
  const uint32_t cap           = c->reclaim_cap;
  const unsigned long long pos = atomicAdd(&c->retire_tail, 1ull);
  if (pos - ld_relaxed_u64(&c->retire_head) < cap)
    reinterpret_cast<uint32_t*>(c->retire_log)[pos & (cap - 1u)] = copy;
  else
    atomicAdd(&c->stat_log_dropped, 1ull);
}

// Path memory of a tile that runs ops in ascending key order (the sorted batch front-end): lane l
// remembers the node it last passed at level l and that node's fences [low, high). The next op
// starts at the lowest remembered node whose fences cover its key instead of at the anchor, so a
// run of nearby keys shares the upper levels and often the leaf. Any node whose low fence is <= the
// key is a valid start (low fences never change; a split that lowered the high fence since the
// node was read is repaired by the right-link chase), and a remembered version is the one a
// snapshot read resolved to, so its children route that snapshot. Levels >= W are not kept.
template <int W>
struct finger {
  uint32_t idx  = kNone;
  uint32_t low  = 0;
  uint32_t high = 0;
  // Lowest remembered node covering key, or the anchor. level (nullable): that node's level, or
  // kNone for the anchor.
  template <class Tile>
  MVBT_DEV uint32_t start_for(uint32_t key, const Tile& t, uint32_t* level = nullptr) const {
    const uint32_t m = t.ballot(idx != kNone && low <= key && key < high);
    if (level) *level = m ? (uint32_t)(__ffs(m) - 1) : kNone;
    return m ? t.shfl(idx, __ffs(m) - 1) : kAnchor;
  }
  template <class Tile>
  MVBT_DEV void record(uint32_t level, uint32_t node, uint32_t lo, uint32_t hi, const Tile& t) {
    if (t.thread_rank() == (int)level) {
      idx  = node;
      low  = lo;
      high = hi;
    }
  }
  // The interior node remembered at `level` (kNone if none): the parent hint of insert_at.
  template <class Tile>
  MVBT_DEV uint32_t at(uint32_t level, const Tile& t) const {
    return level < (uint32_t)W ? t.shfl(idx, (int)level) : kNone;
  }
};

struct device_tree {
  uint32_t* pool;       // node words; node i starts at pool + 32 * i
  control_block* ctl;   // device control block
  uint32_t versioned;   // 1 = multiversion tree, 0 = plain B-link tree
  uint32_t capacity;    // pool size in nodes: every index read from memory is checked against it
  uint32_t reclaim = 0; // 1: version copies go to the retire log (the tree was made with reclaim)

  MVBT_DEV uint32_t* node_ptr(uint32_t idx) const { return pool + (size_t)idx * kNodeWords; }
  // An index is dereferenced only after this check; a bad one records kErrCorrupt instead.
  template <class Tile>
  MVBT_DEV bool valid(uint32_t idx, const Tile& t) const {
    if (idx < capacity) return true;
    if (t.thread_rank() == 0) set_error(kErrCorrupt, 1);
    return false;
  }

  template <int W, class Tile>
  MVBT_DEV void load(uint32_t idx, node_regs<W>& n, bool strong, const Tile& t) const {
    ld_lane<W>(node_ptr(idx) + t.thread_rank() * (32 / W), n, strong);
  }
  template <int W, class Tile>
  MVBT_DEV void store(uint32_t idx, const node_regs<W>& n, const Tile& t) const {
    st_lane<W>(node_ptr(idx) + t.thread_rank() * (32 / W), n);
  }
  // Stores only the lanes that own header pairs.
  template <int W, class Tile>
  MVBT_DEV void store_header(uint32_t idx, const node_regs<W>& n, const Tile& t) const {
    using L     = layout<W>;
    const int r = t.thread_rank();
    if (r == L::kFenceLane || r == L::kLinkLane || r == L::kVerLane)
      st_lane<W>(node_ptr(idx) + r * (32 / W), n);
  }

  // Records error bits and counts the site that raised them (control_block::err_site).
  // Orders every lane's earlier stores before any lane's later ones. A fence orders only the
  // calling thread's own accesses; the warp barrier after it carries that order across the lanes
  // of the tile, so a store that publishes a node (a link, a header) is never visible before the
  // stores of other lanes that wrote what it points to.
  template <class Tile>
  MVBT_DEV void publish_fence(const Tile& t) const {
    __threadfence();
    t.sync();
  }

  MVBT_DEV void set_error(uint32_t bits, uint32_t site = 0) const {
    atomicOr(&ctl->error, bits);
    atomicAdd(&ctl->err_site[site & 31], 1u);
  }
  MVBT_DEV uint32_t current_epoch() const { return ld_relaxed_u32(&ctl->epoch); }

  // ---- allocation: per-SM chunks, refilled from the free ring or the global bump pointer ----
  // Returns a node index, or a free-ring position tagged kRingChunk that alloc() resolves.
  MVBT_DEV uint32_t alloc_one() const {
    control_block* c              = ctl;
    unsigned long long* slot      = &c->sm_pool[sm_id() % kMaxSmSlots];
    const uint32_t C              = c->chunk;
    const uint32_t limit          = c->spin_limit;
    const unsigned long long t0 = global_ns();
    for (uint32_t tries = 0; tries < limit; ++tries) {
      if (tries && (ld_relaxed_u32(&c->error) & kErrPoolExhausted)) return kNone;
      unsigned long long old = atomicAdd(slot, 1ull);
      uint32_t base = (uint32_t)(old >> 32), used = (uint32_t)old;
      if (used < C) return base + used;
      if (used == C) {  // this thread refills the chunk
        uint32_t rb = 0;
        if (reclaim && take_free_chunk(c, C, rb)) {
          atomicExch(slot, ((unsigned long long)rb << 32) | 1ull);
          return rb;
        }
        uint32_t nb = atomicAdd(&c->bump, C);
        if ((unsigned long long)nb + C > c->capacity) {
          atomicOr(&c->error, kErrPoolExhausted);
          atomicAdd(&c->err_site[15], 1u);
          return kNone;
        }
        atomicExch(slot, ((unsigned long long)nb << 32) | 1ull);
        return nb;
      }
      // another thread is refilling: wait (bounded) for the chunk base to change
      for (uint32_t w = 0; w < limit; ++w) {
        __nanosleep(64);
        unsigned long long cur = ld_relaxed_u64(slot);
        if ((uint32_t)(cur >> 32) != base || (uint32_t)cur < C) break;
        if (ld_relaxed_u32(&c->error) & kErrPoolExhausted) return kNone;
        if (global_ns() - t0 > c->wait_ns) break;
      }
      if (global_ns() - t0 > c->wait_ns) break;
    }
    atomicOr(&c->error, kErrSpinLimit);
    atomicAdd(&c->err_site[0], 1u);
    return kNone;
  }
  template <class Tile>
  MVBT_DEV uint32_t alloc(const Tile& t) const {
    uint32_t idx = kNone;
    if (t.thread_rank() == 0) {
      idx = alloc_one();
      // a position in the free ring (a chunk of reclaimed nodes): the node stored there, read
      // once (reading clears the slot), by this lane alone
      if (idx != kNone && (idx & kRingChunk)) idx = chunk_node(ctl, idx, 0);
    }
    return t.shfl(idx, 0);
  }

  // ---- locks on the mod word ----
  template <class Tile>
  MVBT_DEV bool lock(uint32_t idx, const Tile& t) const {
    if (!valid(idx, t)) return false;
    uint32_t* word               = node_ptr(idx) + kModWord;
    uint32_t backoff             = 32;
    const uint32_t lim           = ctl->spin_limit;
    const unsigned long long t0  = global_ns();
    const unsigned long long lns = ctl->wait_ns;
    for (uint32_t i = 0; i < lim; ++i) {
      uint32_t old = 0;
      if (t.thread_rank() == 0) old = atomicOr(word, kLockBit);
      old = t.shfl(old, 0);
      if (!(old & kLockBit)) {
        __threadfence();
        t.sync();
        return true;
      }
      // wait until the lock looks free before the next atomic
      for (uint32_t w = 0; w < 64; ++w) {
        __nanosleep(backoff);
        uint32_t cur = 0;
        if (t.thread_rank() == 0) cur = ld_relaxed_u32(word);
        cur = t.shfl(cur, 0);
        if (!(cur & kLockBit)) break;
        backoff = backoff < 1024 ? backoff * 2 : 1024;
      }
      if (wait_expired(t0, lns, t)) break;
    }
    if (t.thread_rank() == 0) set_error(kErrSpinLimit, 2);
    return false;
  }
  // Releases a node this tile locked and left unchanged (the count stays).
  template <class Tile>
  MVBT_DEV void unlock(uint32_t idx, const Tile& t) const {
    __threadfence();
    t.sync();
    if (t.thread_rank() == 0) atomicAnd(node_ptr(idx) + kModWord, ~kLockBit);
  }
  // Releases a node this tile locked and changed: after every lane's stores are ordered (fence +
  // warp barrier), one exchange clears the lock bit and bumps the count. h.mod is the mod word
  // read under the lock; while the lock is held only failing lock attempts (atomicOr of a bit
  // that is already set) touch the word, so the exchange loses nothing.
  template <class Tile>
  MVBT_DEV void release(uint32_t idx, const header& h, const Tile& t) const {
    __threadfence();
    t.sync();
    if (t.thread_rank() == 0)
      atomicExch(node_ptr(idx) + kModWord, ((h.mod & kCountMask) + 1u) & kCountMask);
  }

  // ---- versioning ----
  // Makes the version visible to older snapshots immutable before node idx (locked, content n)
  // is changed in epoch E. On a versioned tree the first change in epoch E copies the node to a
  // fresh node O and publishes {ts = E, older = O} before any data changes, so a snapshot reader
  // that re-reads ts after reading the data sees that it must use O. Readers of the newest state
  // need nothing here: the lock bit and the count bumped by release() cover them.
  template <int W, class Tile>
  MVBT_DEV bool prepare_write(uint32_t idx, node_regs<W>& n, header& h, uint32_t E, const Tile& t) const {
    if (versioned && h.ts != E) {
      uint32_t copy = alloc(t);
      if (copy == kNone) return false;
      node_regs<W> c = n;
      header hc      = h;
      hc.mod         = kRetiredBit | (E & kCountMask);  // immutable; read only at snapshots < E
      set_header<W>(c, hc, t);
      store<W>(copy, c, t);
      publish_fence(t);  // the copy is complete before the header names it
      h.ts = E;
      h.ol = (h.ol & ~kIndexMask) | copy;
      set_header<W>(n, h, t);
      store_header<W>(idx, n, t);
      // No fence between the header and the data change: a snapshot reader that saw data of this
      // change before the header finds the mod word changed (the lock preceded every store here)
      // and reads the leaf again (recheck_version); the release's fence publishes both.
      if (t.thread_rank() == 0) retire(copy);
    }
    return true;
  }

  // ---- reclamation of version copies ----
  // Records a version copy in the retire log (reclamation on), else counts it.
  MVBT_DEV void retire(uint32_t copy) const {
    if (reclaim)
      retire_logged(ctl, copy);
    else
      atomicAdd(&ctl->sm_stats[sm_id() % kMaxSmSlots][0], 1ull);
  }
  // One retire-log entry at position pos. A copy made in epoch E is read only at snapshots below
  // E, so with no live snapshot below the watermark M it is unreachable once E <= M (compared in a
  // window of 2^28 epochs). Returns 1 if the entry's copy is now marked free (the caller appends
  // idx to the free ring), 2 if it must be kept, 0 if the entry holds nothing (consumed, or a copy
  // the full log dropped). A consumed or freed entry's slot is cleared. check_epoch = false: the
  // caller knows the position holds a reclaimable copy (reclaim_online).
  MVBT_DEV int reclaim_entry(unsigned long long pos, uint32_t M, uint32_t& idx, bool check_epoch = true) const {
    control_block* c = ctl;
    uint32_t* slot   = reinterpret_cast<uint32_t*>(c->retire_log) + (pos & (c->reclaim_cap - 1u));
    idx              = ld_relaxed_u32(slot);
    if (idx >= capacity) return 0;
    uint32_t* mod    = node_ptr(idx) + kModWord;
    const uint32_t m = ld_relaxed_u32(mod);
    if (!(m & kRetiredBit)) {
      st_relaxed_u32(slot, kNone);
      return 0;
    }
    if (check_epoch && ((M - m) & kCountMask) > (kCountMask >> 1)) return 2;  // made after the watermark
    st_relaxed_u32(mod, kFreeBit);
    st_relaxed_u32(slot, kNone);
    return 1;
  }
  // End of a reclaim pass between kernels (one thread, after every entry): moves the log head
  // past the consumed entries, up to the first copy the pass had to keep. retire_tail stays the
  // count of every copy made. Positions beyond head + capacity were never written (those copies
  // were dropped); they alias slots this pass cleared, so a later pass passes over them.
  MVBT_DEV void reclaim_publish() const {
    control_block* c              = ctl;
    const unsigned long long head = c->retire_head;
    unsigned long long n          = c->retire_tail - head;
    if (n > c->reclaim_cap) n = c->reclaim_cap;
    const uint32_t keep = c->rc_first_kept;
    c->retire_head      = head + (keep == 0xFFFFFFFFu ? n : keep);
    c->rc_first_kept    = 0xFFFFFFFFu;
  }
  // Reclamation while kernels run (warp-collective): claims up to 32 retire-log positions below
  // `limit` -- positions the caller knows hold only copies that no live snapshot reads -- frees
  // their copies and appends them to the free ring. Returns the number of positions claimed.
  template <class Warp>
  MVBT_DEV uint32_t reclaim_online(unsigned long long limit, const Warp& warp) const {
    control_block* c       = ctl;
    unsigned long long h   = 0;
    uint32_t n             = 0;
    if (warp.thread_rank() == 0) {
      h = ld_relaxed_u64(&c->retire_head);
      const unsigned long long tail = ld_relaxed_u64(&c->retire_tail);
      if (limit > tail) limit = tail;  // never past the entries reserved so far
      if (h < limit) {
        n = (uint32_t)(limit - h < 32 ? limit - h : 32);
        if (atomicCAS(&c->retire_head, h, h + n) != h) n = 0;  // another warp took them
      }
    }
    h = warp.shfl(h, 0);
    n = warp.shfl(n, 0);
    if (n == 0) return 0;
    __threadfence();  // the copies' last readers finished before `limit` was published
    const uint32_t lane = warp.thread_rank();
    uint32_t idx        = kNone;
    const bool freed    = lane < n && reclaim_entry(h + lane, 0, idx, false) == 1;
    ring_push(c, freed, idx, warp);
    return n;
  }

  // Moves from node idx to the version visible at ts (snapshot readers only). Sets `copy` when it
  // followed at least one older pointer: such a version is never written again.
  template <int W, class Tile>
  MVBT_DEV bool to_version(uint32_t& idx, node_regs<W>& n, header& h, uint32_t ts, bool strong,
                           bool& copy, const Tile& t) const {
    uint32_t hops = 0;
    while (h.ts > ts) {
      uint32_t older = h.older();
      if (older == kNone || ++hops > kMaxSteps) {
        if (t.thread_rank() == 0) set_error(kErrCorrupt, 3);
        return false;
      }
      idx = older;
      if (!valid(idx, t)) return false;
      load<W>(idx, n, strong, t);
      h    = get_header<W>(n, t);
      copy = true;
    }
    return true;
  }

  // Reads leaf idx for a reader of the newest state while writers may run: a sequence lock on
  // the mod word (lock bit | count). A writer holds the lock bit while it changes a reachable
  // leaf and clears it with a bumped count in one exchange after its stores, so the data is
  // consistent when the mod word is unlocked in a read ordered before the data (fence) and
  // unchanged in a re-read ordered after it (fence). Lock and count share one word on purpose:
  // two words read separately could show the state before a writer's lock in one and after its
  // change in the other. Each lane reads the word itself, so its own fences order it around its
  // own share of the node; the read counts only if it held in every lane. Bounded: gives up
  // after the wait limit (kErrSpinLimit) and returns false.
  template <int W, class Tile>
  MVBT_DEV bool read_leaf_latest(uint32_t idx, node_regs<W>& n, const Tile& t) const {
    const uint32_t* p             = node_ptr(idx);
    const unsigned long long t0   = global_ns();
    const unsigned long long lim  = ctl->wait_ns;
    uint32_t backoff              = 32;
    for (;;) {
      const uint32_t mod0 = ld_relaxed_u32(p + kModWord);
      __threadfence();
      ld_lane<W>(p + t.thread_rank() * (32 / W), n, true);
      __threadfence();
      const uint32_t mod1 = ld_relaxed_u32(p + kModWord);
      const bool torn     = (mod0 & kLockBit) != 0 || mod0 != mod1;
      if (t.ballot(torn) == 0) return true;
      if (wait_expired(t0, lim, t)) break;
      __nanosleep(backoff);
      backoff = backoff < 1024 ? backoff * 2 : 1024;
    }
    if (t.thread_rank() == 0) set_error(kErrSpinLimit, 2);
    return false;
  }

  // A concurrent snapshot reader that is about to use the data of a leaf version it read with
  // ts <= snapshot re-reads the leaf's mod word and header after a fence (mod0 = the mod word of
  // the read itself). Returns the immutable copy to read instead if the header now shows a version
  // newer than the snapshot (a writer publishes {ts = E, older = copy} only after the copy is
  // complete). Otherwise sets retry if the mod word was locked or has changed: a writer locked the
  // leaf before any of its stores, so data of a change the header does not show yet can only have
  // been read while the word differs. Returns kNone with retry false if the data read is the
  // version at ts: no writer changed the leaf since before the read, or one did and released it
  // before the mod word was read, whose release fence also published its header (then ts2 > ts).
  template <class Tile>
  MVBT_DEV uint32_t recheck_version(uint32_t idx, uint32_t ts, uint32_t mod0, bool& retry,
                                    const Tile& t) const {
    __threadfence();
    t.sync();
    unsigned long long v = 0;
    uint32_t mod1        = 0;
    if (t.thread_rank() == 0) {
      mod1 = ld_relaxed_u32(node_ptr(idx) + kModWord);
      v    = ld_relaxed_u64(reinterpret_cast<const unsigned long long*>(node_ptr(idx) + 30));
    }
    v            = t.shfl(v, 0);
    mod1         = t.shfl(mod1, 0);
    uint32_t ts2 = (uint32_t)v, ol2 = (uint32_t)(v >> 32);
    retry        = false;
    if (ts2 > ts) return ol2 & kIndexMask;
    retry = (mod0 & kLockBit) != 0 || mod1 != mod0;
    return kNone;
  }

  // ------------------------------------------------------------------------------------------
  // Point lookup at snapshot ts (kLatest = newest). concurrent = writers may run meanwhile.
  // ------------------------------------------------------------------------------------------
  // f (nullable): path memory of a sorted run; every node the lookup passes on key's route is
  // recorded in it (the version a snapshot read resolved to).
  template <int W, class Tile>
  MVBT_DEV uint32_t cooperative_find(uint32_t key, const Tile& t, uint32_t ts = kLatest,
                                     bool concurrent = false, uint32_t start = kAnchor,
                                     finger<W>* f = nullptr) const {
    const bool snap   = versioned && ts != kLatest;
    const bool seqlk  = !snap && concurrent;  // newest state under writers: read leaves locked-free
    uint32_t idx      = start;  // the anchor, or a node on key's route found earlier
    bool via_older    = false;  // idx was reached through an older-version pointer
    bool leaf_next    = false;  // idx is a leaf (child of a level-1 node, or a leaf's sibling)
    node_regs<W> n;
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
      if (!valid(idx, t)) return kNotFound;
      const bool stable = seqlk && leaf_next;
      if (stable) {
        if (!read_leaf_latest<W>(idx, n, t)) return kNotFound;
      } else {
        load<W>(idx, n, concurrent, t);
      }
      header h  = get_header<W>(n, t);
      bool copy = via_older;
      via_older = false;
      if (snap && !to_version<W>(idx, n, h, ts, concurrent, copy, t)) return kNotFound;
      if (key < h.low) {  // routed too far right by a torn read upstream: start over
        idx       = kAnchor;
        leaf_next = false;
        continue;
      }
      if (key >= h.high && h.sibling() != kNone) {
        idx       = h.sibling();
        leaf_next = h.is_leaf();
        continue;
      }
      if (h.is_leaf()) {
        if (snap && concurrent && !copy) {
          bool retry     = false;
          uint32_t older = recheck_version(idx, ts, h.mod, retry, t);
          if (older != kNone) {  // changed under us: use the immutable copy instead
            idx       = older;
            via_older = true;
            continue;
          }
          if (retry) {  // a writer is changing it: read it again (bounded by the step limit)
            __nanosleep(64);
            continue;
          }
        } else if (seqlk && !stable) {
          leaf_next = true;  // reached without knowing it was a leaf: read it again, consistently
          continue;
        }
        if (f) f->record(0, idx, h.low, h.high, t);
        return leaf_value<W>(n, key, t);
      }
      if (f) f->record(h.level(), idx, h.low, h.high, t);
      leaf_next = h.level() == 1;
      idx       = child_for<W>(n, key, t);
      if (idx == kNone) {
        idx       = kAnchor;
        leaf_next = false;
      }
    }
    if (t.thread_rank() == 0) set_error(kErrStepLimit, 4);
    return kNotFound;
  }

  // The point lookup of a tree no writer changes meanwhile (concurrent = false): the same route
  // and result as cooperative_find(key, t, ts, false, start, f), but every lane loads the header
  // words itself (ld_header_words) beside its share of the node instead of receiving them by
  // shuffle, and the versions a snapshot read passes over are read as headers alone.
  template <int W, class Tile>
  MVBT_DEV uint32_t find_quiescent(uint32_t key, const Tile& t, uint32_t ts = kLatest, uint32_t start = kAnchor,
                                   finger<W>* f = nullptr) const {
    const bool snap = versioned && ts != kLatest;
    uint32_t idx    = start;
    node_regs<W> n;
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
      if (!valid(idx, t)) return kNotFound;
      const header h = ld_header_words(node_ptr(idx));
      load<W>(idx, n, false, t);  // issued with the header loads: one round trip per visit
      if (snap && h.ts > ts) {  // a newer version: move to the older one
        idx = h.older();
        if (idx == kNone) {
          if (t.thread_rank() == 0) set_error(kErrCorrupt, 3);
          return kNotFound;
        }
        continue;
      }
      if (key < h.low) {
        idx = kAnchor;
        continue;
      }
      if (key >= h.high && h.sibling() != kNone) {
        idx = h.sibling();
        continue;
      }
      if (h.is_leaf()) {
        if (f) f->record(0, idx, h.low, h.high, t);
        return leaf_value<W>(n, key, t);
      }
      if (f) f->record(h.level(), idx, h.low, h.high, t);
      idx = child_for<W>(n, key, t);
      if (idx == kNone) idx = kAnchor;
    }
    if (t.thread_rank() == 0) set_error(kErrStepLimit, 4);
    return kNotFound;
  }

  // ------------------------------------------------------------------------------------------
  // Range query [lo, hi) at snapshot ts. Writes at most cap pairs {key, value} ascending at out
  // (nullable) and returns the full count.
  // ------------------------------------------------------------------------------------------
  // f (nullable): path memory of a sorted run (as in cooperative_find), recorded along lo's route.
  template <int W, class Tile>
  MVBT_DEV uint32_t cooperative_range_query(uint32_t lo, uint32_t hi, const Tile& t, uint32_t ts,
                                            uint2* out, uint32_t cap, bool concurrent = false,
                                            uint32_t start = kAnchor, finger<W>* f = nullptr) const {
    if (hi <= lo) return 0;
    const bool snap  = versioned && ts != kLatest;
    const bool seqlk = !snap && concurrent;  // newest state under writers (read_leaf_latest)
    uint32_t idx     = start;  // the anchor, or a node on lo's route found earlier
    bool via_older   = false;
    bool leaf_next   = false;
    node_regs<W> n;
    header h;
    // descend to the leaf that holds lo and settle on a consistent version of it
    for (uint32_t step = 0;; ++step) {
      if (step >= kMaxSteps) {
        if (t.thread_rank() == 0) set_error(kErrStepLimit, 5);
        return 0;
      }
      if (!valid(idx, t)) return 0;
      const bool stable = seqlk && leaf_next;
      if (stable) {
        if (!read_leaf_latest<W>(idx, n, t)) return 0;
      } else {
        load<W>(idx, n, concurrent, t);
      }
      h         = get_header<W>(n, t);
      bool copy = via_older;
      via_older = false;
      if (snap && !to_version<W>(idx, n, h, ts, concurrent, copy, t)) return 0;
      if (lo < h.low) {
        idx       = kAnchor;
        leaf_next = false;
        continue;
      }
      if (lo >= h.high && h.sibling() != kNone) {
        idx       = h.sibling();
        leaf_next = h.is_leaf();
        continue;
      }
      if (h.is_leaf()) {
        if (snap && concurrent && !copy) {
          bool retry     = false;
          uint32_t older = recheck_version(idx, ts, h.mod, retry, t);
          if (older != kNone) {
            idx       = older;
            via_older = true;
            continue;
          }
          if (retry) {
            __nanosleep(64);
            continue;
          }
        } else if (seqlk && !stable) {
          leaf_next = true;
          continue;
        }
        if (f) f->record(0, idx, h.low, h.high, t);
        break;
      }
      if (f) f->record(h.level(), idx, h.low, h.high, t);
      leaf_next = h.level() == 1;
      idx       = child_for<W>(n, lo, t);
      if (idx == kNone) {
        idx       = kAnchor;
        leaf_next = false;
      }
    }
    // scan leaves to the right (a sibling chain is never longer than the pool)
    uint32_t count = 0;
    for (uint32_t leaves = 0;; ++leaves) {
      count += leaf_collect<W>(n, lo, hi, out, cap, count, t);
      if (!(hi > h.high && h.sibling() != kNone)) break;
      if (leaves >= capacity) {
        if (t.thread_rank() == 0) set_error(kErrStepLimit, 6);
        break;
      }
      // next leaf: load, resolve the snapshot version, validate before its data is used
      idx           = h.sibling();
      bool settled  = false;
      for (uint32_t tries = 0; tries < kMaxSteps && !settled; ++tries) {
        if (!valid(idx, t)) return count;
        if (seqlk) {
          if (!read_leaf_latest<W>(idx, n, t)) return count;
        } else {
          load<W>(idx, n, concurrent, t);
        }
        h         = get_header<W>(n, t);
        bool copy = via_older;
        via_older = false;
        if (snap && !to_version<W>(idx, n, h, ts, concurrent, copy, t)) return count;
        if (snap && concurrent && !copy) {
          bool retry     = false;
          uint32_t older = recheck_version(idx, ts, h.mod, retry, t);
          if (older != kNone) {
            idx       = older;
            via_older = true;
            continue;
          }
          if (retry) {
            __nanosleep(64);
            continue;
          }
        }
        settled = true;
      }
      if (!settled) {
        if (t.thread_rank() == 0) set_error(kErrStepLimit, 7);
        return count;
      }
    }
    return count;
  }

  // The range query of a tree no writer changes meanwhile (concurrent = false): the same route
  // and result as cooperative_range_query(lo, hi, t, ts, out, cap, false, start, f), with every
  // lane loading the header words itself (as find_quiescent) on the descent and along the leaf
  // chain, and the versions a snapshot read passes over read as headers alone.
  template <int W, class Tile>
  MVBT_DEV uint32_t range_quiescent(uint32_t lo, uint32_t hi, const Tile& t, uint32_t ts, uint2* out,
                                    uint32_t cap, uint32_t start = kAnchor, finger<W>* f = nullptr) const {
    if (hi <= lo) return 0;
    const bool snap = versioned && ts != kLatest;
    uint32_t idx    = start;
    node_regs<W> n;
    header h;
    for (uint32_t step = 0;; ++step) {  // descend to the leaf that holds lo
      if (step >= kMaxSteps) {
        if (t.thread_rank() == 0) set_error(kErrStepLimit, 5);
        return 0;
      }
      if (!valid(idx, t)) return 0;
      h = ld_header_words(node_ptr(idx));
      load<W>(idx, n, false, t);  // issued with the header loads
      if (snap && h.ts > ts) {    // a newer version: move to the older one
        idx = h.older();
        if (idx == kNone) {
          if (t.thread_rank() == 0) set_error(kErrCorrupt, 3);
          return 0;
        }
        continue;
      }
      if (lo < h.low) {
        idx = kAnchor;
        continue;
      }
      if (lo >= h.high && h.sibling() != kNone) {
        idx = h.sibling();
        continue;
      }
      if (h.is_leaf()) {
        if (f) f->record(0, idx, h.low, h.high, t);
        break;
      }
      if (f) f->record(h.level(), idx, h.low, h.high, t);
      idx = child_for<W>(n, lo, t);
      if (idx == kNone) idx = kAnchor;
    }
    uint32_t count = 0;
    for (uint32_t leaves = 0;; ++leaves) {  // scan leaves to the right
      count += leaf_collect<W>(n, lo, hi, out, cap, count, t);
      if (!(hi > h.high && h.sibling() != kNone)) break;
      if (leaves >= capacity) {
        if (t.thread_rank() == 0) set_error(kErrStepLimit, 6);
        break;
      }
      idx = h.sibling();
      for (uint32_t hops = 0;; ++hops) {  // the next leaf, at ts
        if (!valid(idx, t)) return count;
        h = ld_header_words(node_ptr(idx));
        load<W>(idx, n, false, t);
        if (!(snap && h.ts > ts)) break;
        idx = h.older();
        if (idx == kNone || hops >= kMaxSteps) {
          if (t.thread_rank() == 0) set_error(kErrCorrupt, 3);
          return count;
        }
      }
    }
    return count;
  }

  // ------------------------------------------------------------------------------------------
  // Writers
  // ------------------------------------------------------------------------------------------
  // Descent of a writer in a sorted run: like descend_for_write, but it starts at the lowest node
  // of f covering key and records every interior node it passes in f, which then serves as the
  // path of parent hints (insert_at with path0 = f's per-lane nodes). The leaf is recorded by the
  // caller once it has read it under its lock.
  template <int W, class Tile>
  MVBT_DEV uint32_t descend_with_finger(uint32_t key, finger<W>& f, const Tile& t) const {
    uint32_t start_level;
    uint32_t idx = f.start_for(key, t, &start_level);
    if (start_level == 0) return idx;  // the leaf of the previous op covers key
    node_regs<W> n;
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
      if (!valid(idx, t)) return kNone;
      load<W>(idx, n, true, t);
      header h = get_header<W>(n, t);
      if (key < h.low) {  // a torn read upstream routed too far right: start over from the anchor
        idx = kAnchor;
        continue;
      }
      if (key >= h.high && h.sibling() != kNone) {
        idx = h.sibling();
        continue;
      }
      f.record(h.level(), idx, h.low, h.high, t);
      if (h.is_leaf()) return idx;  // reached through a sibling link or a misrouted read
      const uint32_t child = child_for<W>(n, key, t);
      if (child == kNone) {
        idx = kAnchor;
        continue;
      }
      if (h.level() == 1) return child;  // a leaf: read under the lock, not before it
      idx = child;
    }
    if (t.thread_rank() == 0) set_error(kErrStepLimit, 8);
    return kNone;
  }

  // Insert / erase of one key of a sorted run (the sorted batch front-end): the descent starts
  // from the run's path memory f instead of the anchor.
  template <int W, class Tile>
  MVBT_DEV bool insert_in_run(uint32_t key, uint32_t value, const Tile& t, uint32_t E, finger<W>& f) const {
    if (key == kEmptyKey) return false;
    const uint32_t leaf = descend_with_finger<W>(key, f, t);
    if (leaf == kNone) return false;
    return insert_at<W>(key, value, t, E, leaf, f.idx, kNone, (uint32_t)W - 1, &f);
  }

  // Inserts the keys of a sorted run that land in one leaf under a single lock (the sorted batch
  // front-end): skeys[i] ascending, its value at values[spos[i]]. The leaf of skeys[i] is locked
  // and prepared for epoch E once; then that key and each following key of the run below the
  // leaf's high fence is merged into the node in registers while the leaf has room, and the leaf
  // is stored and released once. A key that finds the leaf full splits it (split_insert), its
  // separators go up as in insert_at, and the group ends there. Keys repeated in the run count at
  // their last occurrence only (i + 1 < n_all with the same key: skipped); the caller starts a
  // group at such a last occurrence. Advances i past every key the group consumed (at least one).
  template <int W, class Tile>
  MVBT_DEV void insert_run_group(const uint32_t* skeys, const uint32_t* spos, const uint32_t* values,
                                 uint64_t& i, uint64_t end, uint64_t n_all, const Tile& t, uint32_t E,
                                 finger<W>& f) const {
    uint32_t key = skeys[i];
    if (key == kEmptyKey) {  // not a key; the run is sorted, so every later one is the same
      i = end;
      return;
    }
    node_regs<W> n;
    header h;
    uint32_t leaf = descend_with_finger<W>(key, f, t);
    if (leaf != kNone) leaf = lock_covering<W>(leaf, 0, key, n, h, t, true);
    if (leaf == kNone) {
      ++i;
      return;
    }
    f.record(0, leaf, h.low, h.high, t);
    if (!prepare_write<W>(leaf, n, h, E, t)) {
      unlock(leaf, t);
      ++i;
      return;
    }
    int nvalid = count_valid<W>(n, t);
    for (;;) {
      const uint32_t value = values[spos[i]];
      ++i;
      const int pos = find_pos<W>(n, key, t);
      if (pos >= 0) {
#pragma unroll
        for (int j = 0; j < 16 / W; ++j)
          if (pair_index<W>(t, j) == pos) n.v[j] = value;
      } else if (nvalid < kDataPairs) {
        node_regs<W> out;
        build_from_merged<W>(n, count_less<W>(n, key, t), key, value, 0, nvalid + 1, out, t);
        n = out;
        ++nvalid;
      } else {  // full: split with this key (stores the node, releases it) and end the group
        uint32_t sep_key = 0, sep_child = kNone;
        if (split_insert<W>(leaf, n, h, key, value, E, sep_key, sep_child, t))
          push_up<W>(sep_key, sep_child, E, f.idx, kNone, (uint32_t)W - 1, t);
        return;
      }
      while (i < end && i + 1 < n_all && skeys[i + 1] == skeys[i]) ++i;
      if (i >= end) break;
      key = skeys[i];
      if (key >= h.high || key == kEmptyKey) break;
    }
    store<W>(leaf, n, t);
    release(leaf, h, t);
  }

  template <int W, class Tile>
  MVBT_DEV bool erase_in_run(uint32_t key, const Tile& t, uint32_t E, finger<W>& f) const {
    if (key == kEmptyKey) return false;
    const uint32_t leaf = descend_with_finger<W>(key, f, t);
    if (leaf == kNone) return false;
    return erase_at<W>(key, t, E, leaf, &f);
  }

  // Descends to the leaf for key (newest versions, strong loads), recording in `path` the
  // interior node visited at each level: lane l holds level l in path0 and level l + W in path1.
  // Returns the leaf its level-1 parent names without reading it: the writer reads it under its
  // lock (lock_covering with direct = true), one round trip instead of three.
  template <int W, class Tile>
  MVBT_DEV uint32_t descend_for_write(uint32_t key, uint32_t& path0, uint32_t& path1,
                                      uint32_t& top_level, const Tile& t) const {
    uint32_t idx = kAnchor;
    node_regs<W> n;
    top_level = 0;
    bool first = true;
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
      if (!valid(idx, t)) return kNone;
      load<W>(idx, n, true, t);
      header h = get_header<W>(n, t);
      if (first) {
        top_level = h.level();
        first     = false;
      }
      if (key < h.low) {  // routed too far right by a torn read: start over from the anchor
        idx   = kAnchor;
        first = true;
        path0 = kNone;
        path1 = kNone;
        continue;
      }
      if (key >= h.high && h.sibling() != kNone) {
        idx = h.sibling();
        continue;
      }
      uint32_t lvl = h.level();
      if (lvl == 0) {
        if (step > 16 && t.thread_rank() == 0) atomicMax(&ctl->stat_max_steps, (unsigned long long)step);
        return idx;
      }
      if (lvl < (uint32_t)W) {
        if (t.thread_rank() == (int)lvl) path0 = idx;
      } else {
        if (t.thread_rank() == (int)(lvl - W)) path1 = idx;
      }
      const uint32_t child = child_for<W>(n, key, t);
      if (child == kNone) {
        idx = kAnchor;
        continue;
      }
      if (lvl == 1) {
        if (step > 16 && t.thread_rank() == 0) atomicMax(&ctl->stat_max_steps, (unsigned long long)step);
        return child;
      }
      idx = child;
    }
    if (t.thread_rank() == 0) set_error(kErrStepLimit, 8);
    return kNone;
  }

  // Unlocked approach to the node at `level` whose range covers key, starting from idx (a node
  // at `level` or above on key's route): walks down along key and right along links. A long
  // chase to the right means the start is stale (many splits since it was read), so the walk
  // restarts from the anchor, which reaches the key in about height steps. Returns the index
  // with n/h loaded, or kNone on failure.
  template <int W, class Tile>
  MVBT_DEV uint32_t seek(uint32_t idx, uint32_t level, uint32_t key, node_regs<W>& n, header& h,
                         const Tile& t) const {
    uint32_t chase = 0;
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
      if (!valid(idx, t)) return kNone;
      load<W>(idx, n, true, t);
      h = get_header<W>(n, t);
      if (key < h.low) {
        idx   = kAnchor;
        chase = 0;
        continue;
      }
      if (key >= h.high && h.sibling() != kNone) {
        if (++chase > kChaseRestart) {
          idx   = kAnchor;
          chase = 0;
        } else {
          idx = h.sibling();
        }
        continue;
      }
      if (h.level() == level) return idx;
      if (h.level() < level) {
        if (t.thread_rank() == 0) set_error(kErrCorrupt, 9);
        return kNone;
      }
      idx   = child_for<W>(n, key, t);
      chase = 0;
      if (idx == kNone) idx = kAnchor;
    }
    if (t.thread_rank() == 0) set_error(kErrStepLimit, 12);
    return kNone;
  }

  // Locks the node at `level` that covers key, starting from idx (the node recorded on the way
  // down, or the anchor). Only a few lock-coupled hops to the right are taken while holding a
  // lock; a node further right is re-approached unlocked. direct: idx is a live node at `level`
  // named by its parent or recorded on the way down, locked before it is read (a stale or
  // misrouted one is released again unchanged and approached as above). Returns the locked index
  // with n/h loaded; kNone on failure.
  template <int W, class Tile>
  MVBT_DEV uint32_t lock_covering(uint32_t idx, uint32_t level, uint32_t key, node_regs<W>& n,
                                  header& h, const Tile& t, bool direct = false) const {
    for (uint32_t attempt = 0; attempt < kMaxSteps; ++attempt) {
      if (!direct || attempt > 0) {
        idx = seek<W>(idx, level, key, n, h, t);
        if (idx == kNone) return kNone;
      }
      if (!lock(idx, t)) return kNone;
      load<W>(idx, n, true, t);
      h = get_header<W>(n, t);
      if (h.level() != level || key < h.low) {  // the anchor grew, or the approach was misrouted
        unlock(idx, t);
        if (key < h.low || h.level() < level) idx = kAnchor;
        continue;
      }
      uint32_t hops = 0;
      while (key >= h.high && h.sibling() != kNone && hops < kCoupledHops) {
        uint32_t sib = h.sibling();
        if (!lock(sib, t)) {
          unlock(idx, t);
          return kNone;
        }
        unlock(idx, t);
        idx = sib;
        load<W>(idx, n, true, t);
        h = get_header<W>(n, t);
        ++hops;
        if (h.level() != level) {  // a right link always stays on its level
          unlock(idx, t);
          if (t.thread_rank() == 0) set_error(kErrCorrupt, 10);
          return kNone;
        }
      }
      if (hops > 2 && t.thread_rank() == 0) atomicMax(&ctl->stat_max_hops, (unsigned long long)hops);
      if (!(key >= h.high && h.sibling() != kNone)) return idx;
      unlock(idx, t);  // still far to the left: approach again without holding locks
      if (t.thread_rank() == 0) atomicAdd(&ctl->stat_restarts, 1ull);
    }
    if (t.thread_rank() == 0) set_error(kErrStepLimit, 11);
    return kNone;
  }

  // Splits locked node idx (content n, header h, already prepared for epoch E) while inserting
  // {key, val}: the left half stays in idx, the right half goes to a new node written first.
  // Outputs the separator and the new node for the parent; releases the lock on idx. New nodes
  // of epoch E point at the version of idx older snapshots read, so such a reader that reaches
  // one continues from a node that covers its key.
  template <int W, class Tile>
  MVBT_DEV bool split_insert(uint32_t idx, node_regs<W>& n, header& h, uint32_t key, uint32_t val,
                             uint32_t E, uint32_t& sep_key, uint32_t& sep_child, const Tile& t) const {
    const int pos     = count_less<W>(n, key, t);
    const uint32_t ts = versioned ? E : 0u;
    uint32_t r = alloc(t);
    if (r == kNone) {
      unlock(idx, t);
      return false;
    }
    node_regs<W> left, right;
    build_from_merged<W>(n, pos, key, val, 0, kSplitLeft, left, t);
    build_from_merged<W>(n, pos, key, val, kSplitLeft, kDataPairs + 1 - kSplitLeft, right, t);
    uint32_t rmin = t.shfl(right.k[0], 0);
    header hr = make_header(rmin, 0u, h.high, h.sibling(), ts,
                            (h.level() << 28) | (versioned ? h.older() : kNone));
    header hl = make_header(h.low, h.mod, rmin, r, h.ts, h.ol);
    set_header<W>(right, hr, t);
    set_header<W>(left, hl, t);
    store<W>(r, right, t);
    publish_fence(t);
    store<W>(idx, left, t);
    if (t.thread_rank() == 0) atomicAdd(&ctl->sm_stats[sm_id() % kMaxSmSlots][1], 1ull);
    release(idx, h, t);
    sep_key   = rmin;
    sep_child = r;
    return true;
  }

  // The split node was the top: build a new top {0 -> old top, sep -> new node} one level up and
  // point the (locked, prepared) anchor at it. Releases the anchor.
  template <int W, class Tile>
  MVBT_DEV bool grow(node_regs<W>& n, header& h, uint32_t sep_key, uint32_t sep_child, uint32_t E,
                     const Tile& t) const {
    const uint32_t old_top = t.shfl(n.v[0], 0);
    const uint32_t top     = alloc(t);
    if (top == kNone) {
      unlock(kAnchor, t);
      return false;
    }
    const uint32_t lvl   = h.level();  // level of the new top
    const uint32_t older = versioned ? h.older() : kNone;
    node_regs<W> x;
#pragma unroll
    for (int j = 0; j < 16 / W; ++j) {
      const int q = pair_index<W>(t, j);
      x.k[j]      = q == 0 ? 0u : (q == 1 ? sep_key : kEmptyKey);
      x.v[j]      = q == 0 ? old_top : (q == 1 ? sep_child : kEmptyKey);
    }
    header hx = make_header(0u, 0u, kEmptyKey, kNone, versioned ? E : 0u, (lvl << 28) | older);
    set_header<W>(x, hx, t);
    store<W>(top, x, t);
    publish_fence(t);
#pragma unroll
    for (int j = 0; j < 16 / W; ++j)
      if (pair_index<W>(t, j) == 0) n.v[j] = top;
    h.ol = ((lvl + 1) << 28) | (h.ol & kIndexMask);
    set_header<W>(n, h, t);
    store<W>(kAnchor, n, t);
    if (t.thread_rank() == 0) atomicAdd(&ctl->sm_stats[sm_id() % kMaxSmSlots][1], 1ull);
    release(kAnchor, h, t);
    return true;
  }

  // Insert or update key -> value in write epoch E. Returns true on success.
  template <int W, class Tile>
  MVBT_DEV bool cooperative_insert(uint32_t key, uint32_t value, const Tile& t, uint32_t E) const {
    if (key == kEmptyKey) return false;
    uint32_t path0 = kNone, path1 = kNone, top = 0;
    const uint32_t leaf = descend_for_write<W>(key, path0, path1, top, t);
    if (leaf == kNone) return false;
    return insert_at<W>(key, value, t, E, leaf, path0, path1, top);
  }

  // The insert after its descent: `leaf` and the path (path0 / path1 / top, as descend_for_write
  // records them) may have been found before other writers changed the tree; lock_covering moves
  // right as far as needed and a stale path entry only lengthens the approach to a parent.
  // f (nullable): path memory of a sorted run, which records the leaf as read under the lock.
  template <int W, class Tile>
  MVBT_DEV bool insert_at(uint32_t key, uint32_t value, const Tile& t, uint32_t E, uint32_t leaf,
                          uint32_t path0, uint32_t path1, uint32_t top, finger<W>* f = nullptr) const {
    if (key == kEmptyKey) return false;
    {
      node_regs<W> n;
      header h;
      leaf = lock_covering<W>(leaf, 0, key, n, h, t, true);
      if (leaf == kNone) return false;
      if (f) f->record(0, leaf, h.low, h.high, t);
      // update in place if present
      int pos = find_pos<W>(n, key, t);
      if (pos >= 0) {
        if (!prepare_write<W>(leaf, n, h, E, t)) {
          unlock(leaf, t);
          return false;
        }
#pragma unroll
        for (int j = 0; j < 16 / W; ++j)
          if (pair_index<W>(t, j) == pos) n.v[j] = value;
        store<W>(leaf, n, t);
        release(leaf, h, t);
        return true;
      }
      if (!prepare_write<W>(leaf, n, h, E, t)) {
        unlock(leaf, t);
        return false;
      }
      int nvalid = count_valid<W>(n, t);
      if (nvalid < kDataPairs) {
        int ipos = count_less<W>(n, key, t);
        node_regs<W> out;
        build_from_merged<W>(n, ipos, key, value, 0, nvalid + 1, out, t);
        store<W>(leaf, out, t);
        release(leaf, h, t);
        return true;
      }
      // full leaf: split, then push separators up
      uint32_t sep_key = 0, sep_child = kNone;
      if (!split_insert<W>(leaf, n, h, key, value, E, sep_key, sep_child, t)) return false;
      return push_up<W>(sep_key, sep_child, E, path0, path1, top, t);
    }
  }

  // Inserts the separator {sep_key -> sep_child} of a leaf split into the level above, splitting
  // full interior nodes in turn and growing the tree at the anchor. path0 / path1 / top are the
  // parent hints as descend_for_write records them.
  template <int W, class Tile>
  MVBT_OUTLINE bool push_up(uint32_t sep_key, uint32_t sep_child, uint32_t E, uint32_t path0, uint32_t path1,
                        uint32_t top, const Tile& t) const {
    node_regs<W> n;
    header h;
    int nvalid;
    uint32_t level = 1;
    while (sep_child != kNone) {
      uint32_t start;
      if (level <= top) {
        start = (level < (uint32_t)W) ? t.shfl(path0, level) : t.shfl(path1, level - W);
        if (start == kNone) start = kAnchor;
      } else {
        start = kAnchor;
      }
      if (level >= (uint32_t)kMaxLevels) {
        if (t.thread_rank() == 0) set_error(kErrCorrupt, 13);
        return false;
      }
      uint32_t p = lock_covering<W>(start, level, sep_key, n, h, t, start != kAnchor);
      if (p == kNone) return false;
      if (!prepare_write<W>(p, n, h, E, t)) {
        unlock(p, t);
        return false;
      }
      if (p == kAnchor) return grow<W>(n, h, sep_key, sep_child, E, t);
      nvalid = count_valid<W>(n, t);
      if (nvalid < kDataPairs) {
        int ipos = count_less<W>(n, sep_key, t);
        node_regs<W> out;
        build_from_merged<W>(n, ipos, sep_key, sep_child, 0, nvalid + 1, out, t);
        store<W>(p, out, t);
        release(p, h, t);
        return true;
      }
      uint32_t k2 = sep_key, c2 = sep_child;
      if (!split_insert<W>(p, n, h, k2, c2, E, sep_key, sep_child, t)) return false;
      ++level;
    }
    return true;
  }

  // Erase key in write epoch E. Returns true if the key was present.
  template <int W, class Tile>
  MVBT_DEV bool cooperative_erase(uint32_t key, const Tile& t, uint32_t E) const {
    if (key == kEmptyKey) return false;
    uint32_t path0 = kNone, path1 = kNone, top = 0;
    const uint32_t leaf = descend_for_write<W>(key, path0, path1, top, t);
    if (leaf == kNone) return false;
    return erase_at<W>(key, t, E, leaf);
  }

  // The erase after its descent (the leaf may be stale: lock_covering moves right). f (nullable):
  // as in insert_at.
  template <int W, class Tile>
  MVBT_DEV bool erase_at(uint32_t key, const Tile& t, uint32_t E, uint32_t leaf, finger<W>* f = nullptr) const {
    if (key == kEmptyKey) return false;
    node_regs<W> n;
    header h;
    leaf = lock_covering<W>(leaf, 0, key, n, h, t, true);
    if (leaf == kNone) return false;
    if (f) f->record(0, leaf, h.low, h.high, t);
    int pos = find_pos<W>(n, key, t);
    if (pos < 0) {
      unlock(leaf, t);
      return false;
    }
    if (!prepare_write<W>(leaf, n, h, E, t)) {
      unlock(leaf, t);
      return false;
    }
    remove_at<W>(n, pos, t);
    store<W>(leaf, n, t);
    release(leaf, h, t);
    return true;
  }

  // Snapshot: returns the id of the new snapshot (the pre-increment epoch).
  template <class Tile>
  MVBT_DEV uint32_t take_snapshot(const Tile& t) const {
    __threadfence();
    uint32_t s = 0;
    if (t.thread_rank() == 0) s = atomicAdd(&ctl->epoch, 1u);
    return t.shfl(s, 0);
  }
};

// ----------------------------------------------------------------------------------------------
// Mixed operation batches
//
// A batch is a list of ops {type, key, arg}: find (arg unused), insert (arg = value), erase, and
// range query (arg = exclusive upper bound, output slot at range_out + out_off[i] holding at most
// cap[i] pairs). One snapshot per batch: batch b reads at snapshot S0 + b and writes in epoch
// S0 + b + 1, so every result is that of the batch applied after all earlier batches. The
// reference issues each op kind of a batch as its own host launch
// (include/gpu_versioned_blink_tree.hpp:106-216); here a batch is one launch, or many batches
// are one persistent launch.
// ----------------------------------------------------------------------------------------------
enum : uint32_t { kOpFind = 0, kOpInsert = 1, kOpErase = 2, kOpRange = 3 };

struct batch_view {
  const uint32_t* type;
  const uint32_t* key;
  const uint32_t* arg;
  const uint64_t* out_off;  // range output offset, pairs
  const uint32_t* cap;      // range output capacity, pairs
  uint32_t* result;         // find value or range count (0 for writes)
  uint2* range_out;
};

MVBT_DEV bool is_write_op(uint32_t type) { return type == kOpInsert || type == kOpErase; }

// Runs op i of a batch; returns true if it was a write.
template <int W, class Tile>
MVBT_DEV bool run_batch_op(const device_tree& T, const batch_view& B, uint64_t i, uint32_t S,
                           uint32_t E, const Tile& t) {
  const uint32_t ty = B.type[i], k = B.key[i];
  uint32_t r        = 0;
  bool write        = false;
  if (ty == kOpFind) {
    r = T.cooperative_find<W>(k, t, S, true);
  } else if (ty == kOpRange) {
    uint2* out = B.range_out ? B.range_out + B.out_off[i] : nullptr;
    r          = T.cooperative_range_query<W>(k, B.arg[i], t, S, out, B.cap[i], true);
  } else if (ty == kOpInsert) {
    T.cooperative_insert<W>(k, B.arg[i], t, E);
    write = true;
  } else if (ty == kOpErase) {
    T.cooperative_erase<W>(k, t, E);
    write = true;
  }
  if (t.thread_rank() == 0) B.result[i] = r;
  return write;
}

// An op whose batch is not ready yet does its descent first (routing at the newest state; nothing
// it returns depends on the batches still running), then waits, then finishes from the leaf it
// found: run_batch_op_at. Readers start their snapshot read at that leaf -- its low fence is fixed
// for life, a node made after the snapshot leads to the version the snapshot reads through its
// older pointer, and the fence checks move right or restart as needed -- and writers lock the
// covering leaf from it. Returns the leaf (kNone: fall back to the whole op).
template <int W, class Tile>
MVBT_DEV uint32_t batch_op_descend(const device_tree& T, const batch_view& B, uint64_t i, uint32_t& path0,
                                   uint32_t& path1, uint32_t& top, const Tile& t) {
  const uint32_t k = B.key[i];
  if (k == kEmptyKey) return kNone;
  return T.descend_for_write<W>(k, path0, path1, top, t);
}

template <int W, class Tile>
MVBT_DEV bool run_batch_op_at(const device_tree& T, const batch_view& B, uint64_t i, uint32_t S, uint32_t E,
                              const Tile& t, uint32_t leaf, uint32_t path0, uint32_t path1, uint32_t top) {
  if (leaf == kNone) return run_batch_op<W>(T, B, i, S, E, t);
  const uint32_t ty = B.type[i], k = B.key[i];
  uint32_t r        = 0;
  bool write        = false;
  if (ty == kOpFind) {
    r = T.cooperative_find<W>(k, t, S, true, leaf);
  } else if (ty == kOpRange) {
    uint2* out = B.range_out ? B.range_out + B.out_off[i] : nullptr;
    r          = T.cooperative_range_query<W>(k, B.arg[i], t, S, out, B.cap[i], true, leaf);
  } else if (ty == kOpInsert) {
    T.insert_at<W>(k, B.arg[i], t, E, leaf, path0, path1, top);
    write = true;
  } else if (ty == kOpErase) {
    T.erase_at<W>(k, t, E, leaf);
    write = true;
  }
  if (t.thread_rank() == 0) B.result[i] = r;
  return write;
}

// Schedule of the persistent batched launch. Within each batch the claim order puts writes first
// (perm maps a claim position to an op index). Writes of batch b may start once every write of
// the batches before b has finished, reads of batch b likewise (they read the state after those
// writes; writes of b and later batches go into newer versions, so the reads may lag behind).
// Two device queues hand out work: write ordinals (the critical path, small claims, served first)
// and read ordinals (larger claims, taken when no write is ready). done_batches counts the leading
// batches whose writes are all finished.
struct batch_sched {
  const uint64_t* batch_off;     // [nb + 1] claim positions of each batch
  const uint32_t* perm;          // claim position -> op index
  const uint32_t* n_writes;      // [nb] writes per batch
  const uint64_t* wpre;          // [nb + 1] first write ordinal of each batch
  const uint64_t* rpre;          // [nb + 1] first read ordinal of each batch
  uint32_t* writes_done;         // [nb] finished writes (zero at launch)
  uint32_t* done_batches;        // zero at launch
  unsigned long long* wcursor;   // next write ordinal (zero at launch)
  unsigned long long* rcursor;   // next read ordinal (zero at launch)
  const uint32_t* params;        // [0] num_batches, [1] snapshot of batch 0, [2] external watermark
  // Reclamation inside the launch (all null: off). A copy made in epoch E is read only at
  // snapshots below E; batch b writes in epoch S0 + b + 1 and reads at S0 + b. So once batches
  // 0..b have finished their writes and their reads, the copies batch b and earlier made (all at
  // retire-log positions below the log tail read when batch b's writes had finished) are read by
  // no snapshot of this launch; params[2] is the caller's watermark: the oldest snapshot it still
  // reads outside the launch (copies made in later epochs are kept; kReclaimAll: none held).
  uint32_t* reads_done            = nullptr;  // [nb] finished reads (zero at launch)
  uint32_t* full_done             = nullptr;  // leading batches with writes and reads all finished
  unsigned long long* tail_at     = nullptr;  // [nb] log tail once batch b's writes finished (~0: not yet)
  unsigned long long* rc_limit    = nullptr;  // log positions below it are reclaimable
  unsigned long long* series      = nullptr;  // [nb][4] when batch b's writes finished: epoch, bump,
                                              // free_avail, stat_reclaimed (memory over time)
};

constexpr uint32_t kWriteClaim   = 1;   // writes per tile per claim
constexpr uint32_t kAdvancers    = 16;  // one waiting tile in 16 advances the batch chain each poll
constexpr uint32_t kAdvanceEvery = 8;   // the others on every 8th poll
constexpr uint32_t kReadClaim    = 4;   // reads per tile per claim

// Largest b in [lo, nb) with pre[b] <= x (pre is non-decreasing), starting from the hint lo.
MVBT_DEV uint32_t batch_of_ordinal(const uint64_t* pre, uint32_t nb, uint64_t x, uint32_t lo) {
  if (lo >= nb) lo = 0;
  if (pre[lo] > x) lo = 0;
  if (lo + 1 < nb && pre[lo + 1] > x) return lo;
  uint32_t hi = nb;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (pre[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Advances done_batches past every leading batch whose writes are all finished (lane 0 only). With
// reclamation on, the thread that advances past batch d records the retire-log tail (read after
// d's writes finished and before any write of d + 1 can start) and a memory sample.
MVBT_DEV void advance_done(const batch_sched& sc, uint32_t nb, control_block* ctl = nullptr) {
  uint32_t d = ld_relaxed_u32(sc.done_batches);
  while (d < nb) {
    if (ld_relaxed_u32(&sc.writes_done[d]) < sc.n_writes[d]) break;
    __threadfence();
    const unsigned long long tail = (sc.tail_at && ctl) ? ld_relaxed_u64(&ctl->retire_tail) : 0ull;
    uint32_t prev = atomicCAS(sc.done_batches, d, d + 1);
    if (prev == d && sc.tail_at && ctl) {
      if (sc.series) {
        unsigned long long* e = sc.series + 4ull * d;
        e[0] = ld_relaxed_u32(sc.params + 1) + d + 1u;
        e[1] = ld_relaxed_u32(&ctl->bump);
        // a chunk taker's reservation on free_avail is undone when fewer entries are there, so
        // the word can dip below zero for a moment: recorded as none free
        const unsigned long long fa = ld_relaxed_u64(&ctl->free_avail);
        e[2] = (long long)fa < 0 ? 0ull : fa;
        e[3] = ld_relaxed_u64(&ctl->stat_reclaimed);
      }
      atomicExch(&sc.tail_at[d], tail);
    }
    d = (prev == d) ? d + 1 : prev;
  }
}

// Reclamation on: advances full_done past every leading batch whose writes and reads are all
// finished and raises rc_limit to the log tail recorded for it (lane 0 only).
MVBT_DEV void advance_full(const batch_sched& sc, uint32_t nb) {
  uint32_t f       = ld_relaxed_u32(sc.full_done);
  const uint32_t d = ld_relaxed_u32(sc.done_batches);
  const uint32_t S0 = ld_relaxed_u32(sc.params + 1), ext = ld_relaxed_u32(sc.params + 2);
  while (f < d && f < nb) {
    const uint32_t reads = (uint32_t)(sc.batch_off[f + 1] - sc.batch_off[f]) - sc.n_writes[f];
    if (ld_relaxed_u32(&sc.reads_done[f]) < reads) break;
    __threadfence();
    const unsigned long long t = ld_relaxed_u64(&sc.tail_at[f]);
    if (t == ~0ull) break;  // its writes' advancer has not recorded the tail yet
    const uint32_t prev = atomicCAS(sc.full_done, f, f + 1);
    if (prev == f) {
      // batch f's copies were made in epoch S0 + f + 1: free only at or below the watermark
      if (ext == kReclaimAll || S0 + f + 1u <= ext) atomicMax(sc.rc_limit, t);
      ++f;
    } else {
      f = prev;
    }
  }
}

// Waits (bounded) until the writes of every batch before b have finished; returns false on timeout.
template <class Tile>
MVBT_DEV bool wait_batch_ready(const device_tree& T, const batch_sched& sc, uint32_t nb, uint32_t b,
                               const Tile& t) {
  const unsigned long long t0 = global_ns();
  // Thousands of tiles can wait here at once, and every poll reads the same few words (the batch
  // counter and the finished batch's write count) on one L2 slice. One tile in kAdvancers tries
  // to advance the chain on every poll, the others on every kAdvanceEvery-th and otherwise only
  // read the counter, backing off longer, so the slice keeps up with the writers' own counting.
  const bool advancer = tile_ordinal(t) % kAdvancers == 0;
  for (uint32_t w = 0;; ++w) {
    uint32_t d = 0;
    if (t.thread_rank() == 0) {
      if (advancer || w % kAdvanceEvery == kAdvanceEvery - 1) advance_done(sc, nb, T.ctl);
      d = ld_relaxed_u32(sc.done_batches);
    }
    d = t.shfl(d, 0);
    if (d >= b) {
      __threadfence();
      t.sync();
      return true;
    }
    if (wait_expired(t0, T.ctl->wait_ns, t)) return false;
    __nanosleep(advancer ? 128 : (w < 4 ? 256 : 2048));
  }
}

// One step of reclamation inside the launch (warp-collective): advances full_done, then frees up
// to 32 copies below rc_limit. Returns true if it claimed any log position.
template <class Warp>
MVBT_DEV bool reclaim_step(const device_tree& T, const batch_sched& sc, uint32_t nb, const Warp& warp) {
  unsigned long long lim = 0;
  if (warp.thread_rank() == 0) {
    advance_full(sc, nb);
    lim = ld_relaxed_u64(sc.rc_limit);
  }
  lim = warp.shfl(lim, 0);
  return T.reclaim_online(lim, warp) > 0;
}
// At the end of a warp's work: one more reclamation step (at most 32 copies), then leave. The
// copies the last batches made become reclaimable only when their last reads finish, at the very
// end of the launch, when few warps are left; draining them there would stretch the launch, so
// they wait for the next launch, whose warps free them from its start while work runs.
template <class Warp>
MVBT_DEV void reclaim_drain(const device_tree& T, const batch_sched& sc, uint32_t nb, const Warp& warp) {
  if (warp.thread_rank() == 0) advance_done(sc, nb, T.ctl);
  reclaim_step(T, sc, nb, warp);
}

// Worker loop of one warp in the persistent batched launch. The warp claims consecutive claim
// positions and hands them to its tiles interleaved (tile j takes every (32/W)-th position), and
// the claim order inside a batch is writes | finds | ranges, so the tiles of a warp run the same
// kind of op side by side and their instructions issue together.
template <int W, class Warp, class Tile>
MVBT_DEV void batched_worker(const device_tree& T, const batch_view& B, const batch_sched& sc,
                             const Warp& warp, const Tile& t) {
  constexpr uint32_t kTiles = 32 / W;
  const uint32_t tid = warp.thread_rank() / W;
  const uint32_t nb  = ld_relaxed_u32(sc.params + 0);
  const uint32_t S0  = ld_relaxed_u32(sc.params + 1);
  const uint64_t TW = sc.wpre[nb], TR = sc.rpre[nb];
  uint32_t wb = 0, rb = 0;  // batch hints for the two queues
  unsigned long long idle_since = 0;
  for (uint32_t spin = 0;;) {
    warp.sync();
    uint32_t d = 0;
    unsigned long long g = 0, r = 0;
    if (warp.thread_rank() == 0) {
      d = ld_relaxed_u32(sc.done_batches);
      g = ld_relaxed_u64(sc.wcursor);
      r = ld_relaxed_u64(sc.rcursor);
    }
    d = warp.shfl(d, 0);
    g = warp.shfl(g, 0);
    r = warp.shfl(r, 0);
    if (g >= TW && r >= TR) {
      // all work is claimed: help reclaim what the finished batches no longer need, then leave
      if (sc.rc_limit) reclaim_drain(T, sc, nb, warp);
      break;
    }
    __threadfence();  // the batches counted in d are finished: see their writes
    warp.sync();
    bool did = false;
    // writes first: they gate every later batch. Work is taken up to one batch past the finished
    // ones; an op of a batch that is not ready does its descent, then waits (run_batch_op_at).
    if (g < TW) {
      wb = batch_of_ordinal(sc.wpre, nb, g, wb);
      if (wb <= d + 1) {
        unsigned long long g0 = 0;
        if (warp.thread_rank() == 0) g0 = atomicAdd(sc.wcursor, (unsigned long long)(kTiles * kWriteClaim));
        g0 = warp.shfl(g0, 0);
        did = g0 < TW;
        uint32_t b = wb, dd = d;
        for (uint32_t k = 0; k < kWriteClaim; ++k) {
          const unsigned long long x = g0 + k * kTiles + tid;
          if (x >= TW) break;
          b = batch_of_ordinal(sc.wpre, nb, x, b);
          const uint32_t i = sc.perm[sc.batch_off[b] + (x - sc.wpre[b])];
          if (b > dd) {
            uint32_t p0 = kNone, p1 = kNone, top = 0;
            const uint32_t leaf = batch_op_descend<W>(T, B, i, p0, p1, top, t);
            if (!wait_batch_ready(T, sc, nb, b, t) && t.thread_rank() == 0) T.set_error(kErrSpinLimit, 14);
            dd = b;
            run_batch_op_at<W>(T, B, i, S0 + b, S0 + b + 1, t, leaf, p0, p1, top);
          } else {
            run_batch_op<W>(T, B, i, S0 + b, S0 + b + 1, t);
          }
          // Counted without reading the sum back (a reduction the tile does not wait for): the
          // tiles that wait for a batch (wait_batch_ready) and the warps with nothing runnable
          // advance done_batches. No fence here: every write path ends with the fence of its
          // last release or unlock, which orders its stores before this count.
          t.sync();
          if (t.thread_rank() == 0) atomicAdd(&sc.writes_done[b], 1u);
        }
        // the writes just made copies: free as many older ones as there are reclaimable, so
        // that reclamation keeps pace with copying even when no warp is ever idle
        if (did && sc.rc_limit) reclaim_step(T, sc, nb, warp);
      }
    }
    if (!did && r < TR) {
      rb = batch_of_ordinal(sc.rpre, nb, r, rb);
      if (rb <= d + 1) {
        unsigned long long r0 = 0;
        if (warp.thread_rank() == 0) r0 = atomicAdd(sc.rcursor, (unsigned long long)(kTiles * kReadClaim));
        r0 = warp.shfl(r0, 0);
        did = r0 < TR;
        uint32_t b = rb, dd = d;
        uint32_t done_b[kReadClaim];  // batch of each read this tile ran (counted after a fence)
#pragma unroll
        for (uint32_t k = 0; k < kReadClaim; ++k) done_b[k] = 0xFFFFFFFFu;  // all set: the loop may stop early
        for (uint32_t k = 0; k < kReadClaim; ++k) {
          const unsigned long long x = r0 + k * kTiles + tid;
          if (x >= TR) break;
          b = batch_of_ordinal(sc.rpre, nb, x, b);
          const uint32_t i = sc.perm[sc.batch_off[b] + sc.n_writes[b] + (x - sc.rpre[b])];
          if (b > dd) {
            uint32_t p0 = kNone, p1 = kNone, top = 0;
            const uint32_t leaf = batch_op_descend<W>(T, B, i, p0, p1, top, t);
            if (!wait_batch_ready(T, sc, nb, b, t) && t.thread_rank() == 0) T.set_error(kErrSpinLimit, 14);
            dd = b;
            run_batch_op_at<W>(T, B, i, S0 + b, S0 + b + 1, t, leaf, p0, p1, top);
          } else {
            run_batch_op<W>(T, B, i, S0 + b, S0 + b + 1, t);
          }
          done_b[k] = b;
        }
        if (sc.reads_done) {  // the reads' loads are complete before they are counted
          __threadfence();
          t.sync();
          if (t.thread_rank() == 0)
            for (uint32_t k = 0; k < kReadClaim; ++k)
              if (done_b[k] < nb) atomicAdd(&sc.reads_done[done_b[k]], 1u);
        }
      }
    }
    if (did) {
      spin       = 0;
      idle_since = 0;
      continue;
    }
    // nothing runnable yet: help advance done_batches, reclaim, then back off (bounded)
    if (warp.thread_rank() == 0) advance_done(sc, nb, T.ctl);
    if (sc.rc_limit && reclaim_step(T, sc, nb, warp)) {
      spin       = 0;
      idle_since = 0;
      continue;
    }
    if (idle_since == 0) idle_since = global_ns();
    if (wait_expired(idle_since, T.ctl->wait_ns, warp)) {
      if (warp.thread_rank() == 0) T.set_error(kErrSpinLimit, 14);
      break;
    }
    __nanosleep(spin < 8 ? 256 : 2048);
    ++spin;
  }
}

}  // namespace mvbt
