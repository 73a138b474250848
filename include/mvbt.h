/*
 * mvbt.h -- C ABI of the B200 multiversion B-link tree (libmvbt.so).
 *
 * Plain pointers, sizes and status codes only, so any FFI (ctypes, cgo, JNI, N-API) can bind it.
 * Every array argument is a device pointer (or pinned, UVA-mapped host memory, as the
 * reference's own tests pass) unless the comment says "host". `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream). All operations are stream ordered and
 * asynchronous unless stated otherwise.
 *
 * Each entry point names the reference interface it replaces (owensgroup/MVGpuBTree, a header-only
 * C++ template library: GpuBTree::gpu_blink_tree and GpuBTree::gpu_versioned_btree in
 * include/gpu_blink_tree.hpp and include/gpu_versioned_blink_tree.hpp).
 *
 * Keys and values are uint32. Key 0xFFFFFFFF is reserved (an empty slot); 0xFFFFFFFF as a found
 * value is the not-found sentinel. Key 0 starts present with value 0 (the reference's root
 * tombstone). Range queries are half-open [lower, upper).
 *
 * Calls that write (insert, erase, the concurrent_* calls, batches, reclaim) must not overlap in
 * time on different streams: each write call stamps its own epoch, and a versioned tree's
 * copy-on-write order assumes epochs do not interleave. Readers and writers inside one call are
 * safe together; so are read-only calls beside anything. As with the reference's host API, the
 * caller orders the calls.
 */
#ifndef MVBT_H_
#define MVBT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MVBT_OK 0
#define MVBT_ERR_BAD_ARG 1        /* invalid argument (null handle, bad tile width, ...) */
#define MVBT_ERR_CUDA 2           /* a CUDA runtime call failed; see mvbt_last_error() */
#define MVBT_ERR_POOL_EXHAUSTED 3 /* the node pool is full (device error bit) */
#define MVBT_ERR_SPIN_LIMIT 4     /* a bounded wait gave up (device error bit) */
#define MVBT_ERR_CORRUPT 5        /* a structural invariant failed (device error bit) */
#define MVBT_ERR_NOT_SUPPORTED 6  /* operation not available for this tree kind */
#define MVBT_ERR_OUT_OF_MEMORY 7  /* cudaMalloc of the pool / buffers failed */

/* Device error bits reported by mvbt_check_errors(). */
#define MVBT_DEVERR_POOL_EXHAUSTED 1u
#define MVBT_DEVERR_SPIN_LIMIT 2u
#define MVBT_DEVERR_CORRUPT 4u
#define MVBT_DEVERR_STEP_LIMIT 8u

/* Tree kinds. */
#define MVBT_KIND_BLINK 0     /* GpuBTree::gpu_blink_tree */
#define MVBT_KIND_VERSIONED 1 /* GpuBTree::gpu_versioned_btree (alias gpu_versioned_blink_tree) */

/* Timestamp that reads the newest version (the reference's invalid_timestamp_). */
#define MVBT_LATEST 0xFFFFFFFFu
#define MVBT_NOT_FOUND 0xFFFFFFFFu

typedef struct mvbt_tree mvbt_tree;

/* A range-query result pair; layout of the reference's pair_type<uint32,uint32>
 * (include/pair_type.hpp:22-30). */
typedef struct mvbt_pair {
  uint32_t first;
  uint32_t second;
} mvbt_pair;

typedef struct mvbt_config {
  uint64_t pool_bytes;  /* node pool size in bytes (0 = 4 GiB); at most 2^28 nodes of 128 B */
  int32_t device;       /* CUDA device ordinal (-1 = current device) */
  int32_t tile_width;   /* threads per node tile for the bulk kernels: 8 or 16 (0 = 8) */
  int32_t block_size;   /* threads per block of the bulk kernels (0 = 256) */
  uint32_t spin_limit;  /* bounded-wait attempts before an op gives up (0 = 1<<20) */
  uint32_t chunk_nodes; /* nodes per per-SM allocation chunk (0 = 64) */
  uint32_t blocks_per_sm; /* resident blocks per SM of the bulk kernels (0 = full occupancy) */
  uint32_t max_blocks;  /* hard cap on the grid of the bulk kernels (0 = none) */
  uint32_t wait_ms;     /* wall-clock limit of one bounded wait, ms (0 = 2000); a lock queue of
                           every resident tile on one node drains in ~0.1 s */
  uint32_t reclaim;     /* 1 = version copies can be freed (mvbt_reclaim): a retire log and a free
                           ring of 4 bytes per pool node each, rounded up to powers of two (8 to
                           16 bytes per node); 0 = keep every version, as the reference's bump
                           allocator does */
  uint32_t frontend;    /* batch front-end of the bulk calls (MVBT_FRONTEND_*; 0 = AUTO) */
  uint32_t reserved[2];
} mvbt_config;

/* Batch front-end of the bulk calls (insert, find, erase, range_query). SORTED first sorts the
 * call's keys (a stable radix sort on the device: all 32 bits for writes, so a repeated key's last
 * occurrence in the array wins; the top 24 bits for reads, which only need locality) and gives
 * each tile a contiguous run of them; each op then starts its descent at the deepest node of the
 * previous op's path that covers its key, and results go back to the caller's positions. UNSORTED
 * runs the ops in the caller's order, each from the root. AUTO takes SORTED when the call is large
 * and dense against the tree (at least 2^16 ops and one op per 128 keys), where neighbouring ops
 * share nodes. Results are the same either way (for a repeated key in one insert call, UNSORTED
 * leaves which value wins unspecified, as the reference does). The sort's scratch (16 bytes per op)
 * comes from a stream-ordered memory pool of the library. No counterpart in the reference. */
#define MVBT_FRONTEND_AUTO 0u
#define MVBT_FRONTEND_UNSORTED 1u
#define MVBT_FRONTEND_SORTED 2u

/* Structural report of a host walk over a copy of the node pool (mvbt_validate). */
typedef struct mvbt_report {
  uint32_t height;          /* levels, leaves included */
  uint32_t reserved0;
  uint64_t keys;            /* visible keys (the tombstone key 0 included if present) */
  uint64_t leaves;          /* leaf nodes on the level-0 chain */
  uint64_t interior;        /* interior nodes */
  uint64_t nodes_allocated; /* nodes handed out by the allocator (all versions) */
  uint64_t key_checksum;    /* sum over visible pairs of (key * 0x9E3779B1 + value), mod 2^64 */
  uint32_t locked_nodes;    /* nodes left locked (must be 0 between kernels) */
  uint32_t violations;      /* failed invariants (order, fences, levels, links) */
} mvbt_report;

/* Device view for user kernels (see include/mvbt_device.cuh: mvbt::device_tree). */
typedef struct mvbt_device_view {
  void* pool;         /* node array, 128 B per node */
  void* control;      /* device control block */
  uint32_t versioned; /* 1 = multiversion tree */
  uint32_t capacity;  /* pool size in nodes */
  uint32_t reclaim;   /* 1 = the tree was created with config.reclaim (copies go to the retire log) */
  uint32_t reserved;
} mvbt_device_view;

void mvbt_config_init(mvbt_config* cfg);

/* Creates a tree with one root leaf holding the tombstone {0, 0}; synchronises the device.
 * Replaces: gpu_blink_tree() (include/gpu_blink_tree.hpp:77-81) and gpu_versioned_btree()
 * (include/gpu_versioned_blink_tree.hpp:88-93). */
int mvbt_create(int kind, const mvbt_config* cfg, mvbt_tree** out);

/* Frees the pool and all buffers. Replaces the shared_ptr teardown of the reference handles. */
int mvbt_destroy(mvbt_tree* tree);

/* Sets the batch front-end of the bulk calls (MVBT_FRONTEND_*), as config.frontend does at
 * creation. Host-side only; affects calls issued afterwards. No counterpart in the reference. */
int mvbt_set_frontend(mvbt_tree* tree, uint32_t frontend);

/* Upserts n pairs. in_place selects the reference's ViB (1) or VoB (0) insert; both keep every
 * version an older snapshot can read, so results are identical; blink trees ignore it. With the
 * sorted front-end (AUTO or SORTED), an insert of at least 4096 pairs into a pristine tree (created
 * by mvbt_create, with no write and no snapshot since) is a bulk load: the sorted pairs, each
 * key's last occurrence, are built bottom up into nodes 10 of 13 pairs full, in the write epoch
 * of the call, asynchronously like any insert; the contents are those of the pairs upserted in
 * order.
 * Replaces: gpu_blink_tree::insert (include/gpu_blink_tree.hpp:218-225),
 * gpu_versioned_btree::insert(..., in_place) (include/gpu_versioned_blink_tree.hpp:106-142). */
int mvbt_insert(mvbt_tree* tree, const uint32_t* keys, const uint32_t* values, uint32_t n,
                void* stream, int in_place);

/* values[i] = value of keys[i] at snapshot `timestamp` (MVBT_LATEST = newest), else
 * MVBT_NOT_FOUND. concurrent = 1 when writers may run on the tree at the same time.
 * Replaces: gpu_blink_tree::find (include/gpu_blink_tree.hpp:227-236),
 * gpu_versioned_btree::find (include/gpu_versioned_blink_tree.hpp:144-164). */
int mvbt_find(mvbt_tree* tree, const uint32_t* keys, uint32_t* values, uint32_t n,
              uint32_t timestamp, void* stream, int concurrent);

/* Erases n keys (missing keys are no-ops). On a versioned tree the erase is a new version, so
 * reads at older snapshots still see the key.
 * Replaces: gpu_blink_tree::erase (include/gpu_blink_tree.hpp:238-245),
 * gpu_versioned_btree::erase (include/gpu_versioned_blink_tree.hpp:166-173). */
int mvbt_erase(mvbt_tree* tree, const uint32_t* keys, uint32_t n, void* stream, int concurrent);

/* Range query i returns the pairs with lower[i] <= key < upper[i], ascending, written from
 * result + i * average_range_length; at most average_range_length pairs are written (the
 * reference writes past the slot), counts[i] (nullable) receives the full count.
 * Replaces: gpu_blink_tree::range_query (include/gpu_blink_tree.hpp:247-265),
 * gpu_versioned_btree::range_query(..., timestamp, ...) (include/gpu_versioned_blink_tree.hpp:195-216). */
int mvbt_range_query(mvbt_tree* tree, const uint32_t* lower, const uint32_t* upper,
                     mvbt_pair* result, uint32_t* counts, uint32_t average_range_length, uint32_t n,
                     uint32_t timestamp, void* stream, int concurrent);

/* One kernel mixing n_insert inserts with n_range range queries. A snapshot S is taken when the
 * call is issued; every range query reads at S and every insert lands after it, so results are
 * deterministic. counts (nullable) receives each query's full count.
 * Replaces: concurrent_insert_range (include/gpu_blink_tree.hpp:148-187,
 * include/gpu_versioned_blink_tree.hpp:252-294). */
int mvbt_concurrent_insert_range(mvbt_tree* tree, const uint32_t* keys, const uint32_t* values,
                                 uint32_t n_insert, const uint32_t* lower, const uint32_t* upper,
                                 uint32_t n_range, mvbt_pair* result,
                                 uint32_t average_range_length, uint32_t* counts, void* stream);

/* One kernel mixing n_find finds with n_erase erases; finds read at a snapshot taken when the
 * call is issued (versioned tree) or the newest state (blink tree).
 * Replaces: concurrent_find_erase (include/gpu_blink_tree.hpp:189-216,
 * include/gpu_versioned_blink_tree.hpp:218-250). */
int mvbt_concurrent_find_erase(mvbt_tree* tree, const uint32_t* find_keys, uint32_t* find_results,
                               uint32_t n_find, const uint32_t* erase_keys, uint32_t n_erase,
                               void* stream);

/* Takes a snapshot and returns its id in *snapshot_out (host); synchronises `stream`.
 * Replaces: gpu_versioned_btree::take_snapshot (include/gpu_versioned_blink_tree.hpp:297-302). */
int mvbt_take_snapshot(mvbt_tree* tree, void* stream, uint32_t* snapshot_out);

/* Stream-ordered snapshot: writes the id to the device word d_snapshot_out, no host sync. */
int mvbt_take_snapshot_async(mvbt_tree* tree, void* stream, uint32_t* d_snapshot_out);

/* Synchronises `stream` and returns the sticky device error bits (MVBT_DEVERR_*) in *bits;
 * the status is MVBT_OK when no bit is set, else the first matching MVBT_ERR_*. */
int mvbt_check_errors(mvbt_tree* tree, void* stream, uint32_t* bits);

/* Clears the sticky device error bits. */
int mvbt_clear_errors(mvbt_tree* tree, void* stream);

/* Allocator usage. Replaces: compute_memory_usage (include/gpu_blink_tree.hpp:1076-1080). */
int mvbt_memory_usage(mvbt_tree* tree, uint64_t* nodes_allocated, uint64_t* bytes_allocated,
                      uint64_t* pool_bytes);

/* Host walk of the tree as visible at `timestamp`: checks key order, fences, levels, links and
 * lock bits and fills *report. Synchronises the device.
 * Replaces: validate_tree_structure (include/gpu_blink_tree.hpp:742-900,
 * include/gpu_versioned_blink_tree.hpp:1098-1259). */
int mvbt_validate(mvbt_tree* tree, uint32_t timestamp, mvbt_report* report);

/* The same walk over a HOST image of the pool (nodes * 32 words, node i at word 32 * i), e.g. a
 * dump taken with cudaMemcpy; versioned selects snapshot resolution. Needs no GPU. */
int mvbt_validate_image(const uint32_t* image, uint64_t nodes, int versioned, uint32_t timestamp,
                        mvbt_report* report);

/* As mvbt_validate_image, and writes a text description of the first violations (NUL-terminated,
 * at most detail_len bytes) into the HOST buffer detail. */
int mvbt_validate_image_detail(const uint32_t* image, uint64_t nodes, int versioned,
                               uint32_t timestamp, mvbt_report* report, char* detail,
                               uint64_t detail_len);

/* Copies up to max_nodes allocated nodes (node i = 32 words) into the HOST buffer dst and
 * returns the number copied in *nodes; synchronises the device. The image can be checked with
 * mvbt_validate_image or stored as a dump of the tree. */
int mvbt_copy_pool(mvbt_tree* tree, void* dst, uint64_t max_nodes, uint64_t* nodes);

#define MVBT_RECLAIM_ALL 0xFFFFFFFFu

/* Frees the version copies that no snapshot id >= min_live_snapshot reads: copies made in write
 * epochs <= min_live_snapshot. MVBT_RECLAIM_ALL takes the current epoch, after which only the
 * newest state and snapshots taken later are readable. Freed nodes are reused by later writes.
 * Stream-ordered: no writer (insert, erase, batch) may run on the tree concurrently with it, and
 * no reader may use a snapshot below the watermark afterwards (validation at such a snapshot is
 * undefined too). Needs config.reclaim = 1 (else MVBT_ERR_NOT_SUPPORTED); a no-op on the plain
 * tree, which makes no copies. Replaces: the epoch-based reclaimer DEBR_device / DEBR_host
 * (include/memory_reclaimer.hpp:70-410), which frees retired nodes after about two epoch
 * advances whether or not a snapshot still reads them; here the caller states the oldest live
 * snapshot. */
int mvbt_reclaim(mvbt_tree* tree, uint32_t min_live_snapshot, void* stream);

/* Device counters (synchronises the device): out[0] versions copied, [1] node splits, [2] longest
 * locked move-right walk, [3] longest unlocked writer descent, [4] write epoch, [5] error bits,
 * [6..21] errors per raising site 0..15, [22] locked approaches restarted unlocked, [23] nodes
 * freed by mvbt_reclaim, [24] freed nodes waiting for reuse, [25] nodes handed out again, [26]
 * copies the full retire log could not record (never freed), [27..42] errors per raising site
 * 16..31 (16: rejected batch offsets of mvbt_batch_run_noalloc; 17: a bulk load into a pristine
 * tree that did not fit the pool, which leaves the tree empty). Writes min(n, 43) values. */
int mvbt_stats(mvbt_tree* tree, uint64_t* out, uint32_t n);

/* Device view for user kernels calling the cooperative_* device API. */
int mvbt_get_device_view(mvbt_tree* tree, mvbt_device_view* out);

/* ---------------------------------------------------------------------------------------------
 * Mixed operation batches (versioned trees). Batch b holds ops [batch_off[b], batch_off[b+1]);
 * op i is type[i] (MVBT_OP_*), key[i] and arg[i] (the value of an insert, the exclusive upper
 * bound of a range query). One snapshot per batch: batch b reads at the snapshot taken when it
 * starts and writes after it, so every result equals that of the batches applied one by one, in
 * order. result[i] receives a find's value (or MVBT_NOT_FOUND) or a range query's full count (0
 * for writes); range query i writes at most range_cap[i] pairs at range_out + out_off[i].
 * Writes inside one batch must touch distinct keys. No counterpart exists in the reference,
 * whose callers issue each op kind of a batch as its own launch
 * (include/gpu_versioned_blink_tree.hpp:106-216); MVBT_BATCH_PER_LAUNCH is that plain method
 * (one snapshot + one launch per batch).
 * ------------------------------------------------------------------------------------------- */
#define MVBT_OP_FIND 0u
#define MVBT_OP_INSERT 1u
#define MVBT_OP_ERASE 2u
#define MVBT_OP_RANGE 3u

#define MVBT_BATCH_PERSISTENT 0 /* one persistent launch fed by a device work queue */
#define MVBT_BATCH_PER_LAUNCH 1 /* one snapshot and one launch per batch */
#define MVBT_BATCH_GRAPH 2      /* the persistent launch captured once and replayed as a CUDA graph */

typedef struct mvbt_batch_plan mvbt_batch_plan;

/* Allocates the device scratch of the batched path for up to max_ops ops in max_batches batches. */
int mvbt_batch_plan_create(mvbt_tree* tree, uint64_t max_ops, uint32_t max_batches,
                           mvbt_batch_plan** out);
int mvbt_batch_plan_destroy(mvbt_batch_plan* plan);

/* Compact range output of a batch run (device arrays, stream-ordered, uses the plan's scratch,
 * which the first call allocates): the first min(result[i], range_cap[i]) pairs of every range
 * query i, in op order, packed into `compact` (room for the sum of the range caps), and the number
 * of pairs written to *total (a device uint64). Query i's pairs start at the sum of
 * min(count, cap) over the range queries before it, which the caller recomputes from result[] and
 * range_cap[]. A caller that copies results to the host then copies only the pairs that exist
 * instead of every fixed-size slot. */
int mvbt_batch_compact_ranges(mvbt_batch_plan* plan, uint64_t num_ops, const uint32_t* type,
                              const uint32_t* result, const uint64_t* out_off, const uint32_t* range_cap,
                              const mvbt_pair* range_out, mvbt_pair* compact, uint64_t* total, void* stream);

/* Launch shape of the plan's persistent path (the autotuner's knobs): tile width 8 or 16 (0 = the
 * tree's; the node format is the same for both) and resident blocks per SM (-1 = the tree's,
 * 0 = full occupancy, 4, 6 and 8 pick register-capped kernel variants). Drops a captured graph. */
int mvbt_batch_plan_set_launch(mvbt_batch_plan* plan, int tile_width, int blocks_per_sm);

/* Runs num_batches batches. batch_off is a HOST array of num_batches + 1 offsets; the op arrays
 * are device arrays. Stream ordered; the call waits (on the host) for the plan's own previous
 * persistent or graph run to finish before it reuses the plan's pinned staging memory, so a
 * caller can keep other plans and streams busy meanwhile. MVBT_BATCH_GRAPH re-captures when an
 * array pointer or the stream changes. */
int mvbt_batch_run(mvbt_batch_plan* plan, uint32_t num_batches, const uint64_t* batch_off,
                   const uint32_t* type, const uint32_t* key, const uint32_t* arg,
                   const uint64_t* out_off, const uint32_t* range_cap, uint32_t* result,
                   mvbt_pair* range_out, int mode, void* stream);

/* enable = 1 records CUDA events around the persistent kernel of each MVBT_BATCH_PERSISTENT run
 * (up to 64 runs are kept); mvbt_batch_plan_kernel_times waits for them, writes the kernel times
 * in ms of the runs since the last call (oldest first, at most max) and their number to *n. */
int mvbt_batch_plan_timing(mvbt_batch_plan* plan, int enable);

/* Reclamation inside the plan's persistent runs (MVBT_BATCH_PERSISTENT and MVBT_BATCH_GRAPH;
 * config.reclaim trees, else MVBT_ERR_NOT_SUPPORTED). While a run goes on, warps without work
 * free the version copies that no snapshot of the run reads any more -- those batch b and
 * earlier made, once batches 0..b have finished their writes and their reads -- together with the
 * copies made before the run, and append them to the free ring, from which the same run's writes
 * allocate. min_live_snapshot is the oldest snapshot the caller still reads outside the run, as in
 * mvbt_reclaim: copies made in later epochs are kept (MVBT_RECLAIM_ALL: none held).
 * Replaces: the reference's device-side epoch-based reclaimer DEBR_device (retire, leave_qstate,
 * enter_qstate; include/memory_reclaimer.hpp:146-410), which frees retired nodes about two
 * epoch advances after retirement whether or not a snapshot still reads them; here the batches'
 * own completion counters are the announcements, and a held snapshot stays exact. */
int mvbt_batch_plan_set_reclaim(mvbt_batch_plan* plan, int enable, uint32_t min_live_snapshot);

/* Memory over time of the plan's last persistent run with reclamation on: per batch b (up to
 * max_batches), 4 values sampled when its writes had finished: the write epoch, nodes ever taken
 * from the pool (bump pointer), freed nodes waiting in the free ring, and nodes freed so far; live
 * nodes = bump - waiting. *n = batches written. Waits for the run. Replaces the reference's
 * per-epoch reclaimer statistics (compute_reclaimer_stats, include/memory_reclaimer.hpp:114-133). */
int mvbt_batch_plan_memory_series(mvbt_batch_plan* plan, uint64_t* out, uint32_t max_batches, uint32_t* n);
int mvbt_batch_plan_kernel_times(mvbt_batch_plan* plan, float* ms, uint32_t max, uint32_t* n);

/* Mixed batches for callers that cannot allocate device memory on their call path: a serving
 * loop with a latency budget (cudaMalloc / cudaFree can block the device for milliseconds), or a
 * host application that owns every allocation and gives the library a fixed budget up front.
 * Same semantics and results as mvbt_batch_run in MVBT_BATCH_PERSISTENT mode, but its scratch
 * lives in one fixed-size device array inside the library (about 4.3 MB, held by every GPU that
 * loads the library until the process exits) instead of a batch plan: this call allocates
 * nothing. It has no counterpart in the reference.
 * batch_off is a DEVICE array of num_batches + 1 offsets with batch_off[num_batches] == num_ops;
 * at most MVBT_NOALLOC_MAX_BATCHES batches and MVBT_NOALLOC_MAX_OPS ops (larger requests return
 * MVBT_ERR_BAD_ARG without touching the GPU). Offsets that do not start at 0, decrease or end
 * elsewhere than num_ops are rejected on the device: nothing runs and mvbt_check_errors reports
 * MVBT_ERR_CORRUPT. Every call shares the array (it is cleared where it must start at zero), so
 * calls that overlap on the GPU (other streams, other threads) race: serialise them. The first
 * call on a device looks up the array's address; make that first call before any stream
 * capture. */
#define MVBT_NOALLOC_MAX_OPS (1u << 20)
#define MVBT_NOALLOC_MAX_BATCHES 1024u
int mvbt_batch_run_noalloc(mvbt_tree* tree, uint32_t num_batches, const uint64_t* batch_off,
                           uint64_t num_ops, const uint32_t* type, const uint32_t* key,
                           const uint32_t* arg, const uint64_t* out_off, const uint32_t* range_cap,
                           uint32_t* result, mvbt_pair* range_out, void* stream);

/* ---- Serving: a host request loop with continuous batching ----
 * mvbt_serve_trace replays a trace of requests (each a batch of mixed ops with an arrival time)
 * against the tree as a server would: from the session start it admits the requests that have
 * arrived, in arrival order, as launch slots and node memory allow, and runs every admitted
 * group as one persistent launch. With MVBT_SERVE_SNAPSHOT_PER_BATCH (the default) the group is
 * one batch with one snapshot: every read of the group sees the state after all earlier groups,
 * every write lands after them, so each query is linearizable at its group's snapshot (requests
 * admitted together were concurrent). With MVBT_SERVE_SNAPSHOT_PER_REQUEST each request is its
 * own batch with its own snapshot: reads also see the writes of earlier requests of the group
 * (sequential order; slower, as each batch's reads wait for the previous batch's writes).
 * While one launch runs, requests that arrive meanwhile are admitted into the next one (up to
 * pipeline_depth launches staged or running; copies overlap compute on two more streams).
 * Between launches a reclaim pass frees the version copies the finished snapshots read
 * (config.reclaim trees). Results and completion times come back per request. Requests of one
 * group must not write the same key (a trace from the workload generator,
 * workload/mvbt_workload.h, with erase_lag above max_requests_per_launch guarantees it). It has no counterpart in the reference, which has no
 * serving path. */
#define MVBT_SERVE_SNAPSHOT_PER_BATCH 0u
#define MVBT_SERVE_SNAPSHOT_PER_REQUEST 1u
typedef struct mvbt_serve_config {
  uint64_t max_ops_per_launch;      /* ops admitted into one launch (0 = 1 << 21) */
  uint64_t max_range_pairs;         /* range-output pairs of one launch (0 = 32 * max_ops) */
  uint32_t max_requests_per_launch; /* requests (batches) in one launch (0 = 1024) */
  uint32_t pipeline_depth;          /* launches staged or running at once (0 = 2) */
  uint32_t mode;                    /* MVBT_BATCH_PERSISTENT: continuous batching (default);
                                       MVBT_BATCH_PER_LAUNCH: one request per launch, the plain
                                       method, for comparison */
  uint32_t reclaim_every;           /* launches between reclaim passes; 0 = never (needs
                                       config.reclaim on the tree otherwise) */
  uint32_t nodes_per_write;         /* admission: nodes a write may allocate (0 = 3) */
  uint32_t snapshots;               /* MVBT_SERVE_SNAPSHOT_PER_BATCH (0) or _PER_REQUEST */
  uint64_t reserve_nodes;           /* admission: nodes kept free (0 = 1 << 16) */
  uint32_t reclaim_in_launch;       /* 1: reclamation inside every persistent launch
                                       (mvbt_batch_plan_set_reclaim; config.reclaim trees) */
  uint32_t pad0;
  uint64_t max_reclaim_lag;         /* admission: while more version copies than this wait in the
                                       retire log (retired, not yet freed), no request is admitted
                                       until a reclaim pass has run (0 = no limit) */
  uint64_t reserved[2];
} mvbt_serve_config;

typedef struct mvbt_serve_stats {
  uint64_t requests;      /* requests served */
  uint64_t ops;           /* ops served */
  uint64_t launches;      /* launches issued */
  uint64_t reclaims;      /* reclaim passes issued */
  uint64_t span_ns;       /* session start to the last completion */
  uint64_t max_waiting;   /* most requests arrived but not yet admitted at one time */
  uint64_t memory_waits;  /* admissions deferred until memory was freed */
  uint64_t max_launch_ops;
  uint64_t max_reclaim_lag;  /* most version copies seen waiting for reclamation after a launch */
  uint64_t lag_waits;        /* admissions deferred by max_reclaim_lag */
  uint64_t nodes_high_water; /* most nodes in use (taken from the pool, not free) after a launch */
  uint64_t reserved[5];
} mvbt_serve_stats;

void mvbt_serve_config_init(mvbt_serve_config* cfg);

/* All arrays are HOST arrays; pinned memory (cudaMallocHost) lets the copies run asynchronously.
 * Request r holds ops [req_off[r], req_off[r + 1]) of type/key/arg/range_cap (as in
 * mvbt_batch_run) and arrives arrival_ns[r] after the session start (non-decreasing). Range
 * query i writes at most range_cap[i] pairs at range_out + out_off[i]; the slots of all range
 * queries must be disjoint and increasing in op order (as the workload generator's
 * mvbt_wl_mix_copy produces them).
 * Outputs: result[i] per op, the range pairs (a query's slot past its count, and any gap between
 * slots, is unspecified), done_ns[r] (session clock when the request's results were on the host),
 * snapshot[r] (the snapshot its reads used: requests with the same one formed one group; may be
 * null), stats (may be null). Works on the versioned tree. Synchronises the device. */
int mvbt_serve_trace(mvbt_tree* tree, const mvbt_serve_config* cfg, uint32_t num_requests,
                     const uint64_t* req_off, const uint64_t* arrival_ns, const uint32_t* type,
                     const uint32_t* key, const uint32_t* arg, const uint64_t* out_off,
                     const uint32_t* range_cap, uint32_t* result, mvbt_pair* range_out,
                     uint64_t* done_ns, uint32_t* snapshot, mvbt_serve_stats* stats);

/* Builds a fresh tree (no writes or snapshots yet) from n pairs with keys sorted strictly
 * increasing (device arrays; key 0xFFFFFFFF is not allowed; a key 0 replaces the tombstone's
 * value). Every node is written once: leaves hold `fill` pairs and interior nodes `fill`
 * children (0 = 8, half full as the reference builds, so later inserts do not split at once;
 * at most 13). Checks the order on the device first (MVBT_ERR_BAD_ARG if unsorted); synchronises
 * the stream. Works for both tree kinds.
 * Replaces: the bulk-build constructor gpu_blink_tree(keys, values, n, sorted_input, stream)
 * (include/gpu_blink_tree.hpp:85-136, include/btree_kernels.hpp:915-1025). */
int mvbt_bulk_build(mvbt_tree* tree, const uint32_t* keys, const uint32_t* values, uint64_t n,
                    uint32_t fill, void* stream);

/* A copy of the tree (all versions, allocator and reclamation state) in a new tree with the same
 * configuration on the same device. Synchronises the device. The reference shares device
 * buffers between handle copies instead (include/gpu_versioned_blink_tree.hpp:94-102); a deep
 * copy has no counterpart there. */
int mvbt_clone(mvbt_tree* tree, mvbt_tree** out);

/* Checkpoint: writes the tree (configuration, control block, the allocated node prefix of the
 * pool and the reclamation rings) to a file, and loads such a file into a new tree on `device`
 * (-1 = current). Both synchronise the device. The reference's pool-image dump is
 * copy_buffer (include/device_bump_allocator.hpp:71-73), with no load. */
int mvbt_save(mvbt_tree* tree, const char* path);
int mvbt_load(const char* path, int device, mvbt_tree** out);

/* Tree kind, tile width and device of a handle. */
int mvbt_get_info(mvbt_tree* tree, int* kind, int* tile_width, int* device);

/* Last error message of this thread (host-side detail for MVBT_ERR_CUDA / BAD_ARG). */
const char* mvbt_last_error(void);
const char* mvbt_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* MVBT_H_ */
