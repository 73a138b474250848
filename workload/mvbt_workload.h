/*
 * mvbt_workload.h -- deterministic synthetic workloads for the tree (host-only libworkload.so).
 *
 * The harness counterpart of the reference's include/rkg.hpp (generate_keys,
 * prep_experiment_find_with_exist_ratio, prep_experiment_range_query). All arrays here are HOST
 * arrays. Keys are drawn from [1, 2^32 - 3]:
 *   distinct key i  = 1 + cw(F_seed(i)), F a keyed 4-round Feistel bijection on 32 bits and cw
 *                     cycle-walking into [0, 2^32 - 3), so disjoint index ranges give disjoint keys;
 *   uniform keys    = 1 + (splitmix64 >> 32) * (2^32 - 3) >> 32;
 *   values          = fmix32(key ^ salt) (the MurmurHash3 32-bit finalizer).
 * Index ranges [0, 2^31) are used for keys that get inserted and [2^31, 2^32 - 3) for keys that
 * are never inserted (find misses).
 */
#ifndef MVBT_WORKLOAD_H_
#define MVBT_WORKLOAD_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MVBT_OP_FIND 0u
#define MVBT_OP_INSERT 1u
#define MVBT_OP_ERASE 2u
#define MVBT_OP_RANGE 3u

#define MVBT_MISS_INDEX_BASE 0x80000000ull

uint64_t mvbt_wl_splitmix64(uint64_t* state);
uint32_t mvbt_wl_fmix32(uint32_t h);
void mvbt_wl_distinct_keys(uint64_t seed, uint64_t start, uint64_t n, uint32_t* out);
void mvbt_wl_values(const uint32_t* keys, uint64_t n, uint32_t salt, uint32_t* out);
void mvbt_wl_uniform_keys(uint64_t seed, uint64_t n, uint32_t* out);
void mvbt_wl_shuffle(uint64_t seed, uint32_t* a, uint64_t n);
/* out[i] = min(lower[i] + length * stride, 0xFFFFFFFF) in 64-bit arithmetic. */
void mvbt_wl_upper_bounds(const uint32_t* lower, uint64_t n, uint64_t length, uint64_t stride,
                          uint32_t* out);

/* Mixed batched workload (erase / insert / find / range per op). */
typedef struct mvbt_mix_params {
  double p_erase;       /* 0.10: erase of a key present at the batch snapshot */
  double p_insert;      /* 0.20: insert of a new key */
  double p_find;        /* 0.50: point find */
  double p_range;       /* 0.20: range query */
  double find_hit;      /* 0.50: fraction of finds that target a present key */
  double batch_median;  /* 16384 */
  double batch_sigma;   /* 1.5 (lognormal) */
  uint32_t batch_min;   /* 1024 */
  uint32_t batch_max;   /* 4 << 20 */
  double range_mean;    /* 32: geometric range length L */
  uint32_t range_min;   /* 1 */
  uint32_t range_max;   /* 1024 */
  uint32_t stride;      /* key distance per unit of L: upper = lower + L * stride */
  uint32_t value_salt;  /* values are fmix32(key ^ salt) */
  uint32_t fixed_batch; /* nonzero: every batch has exactly this many ops */
  uint32_t erase_lag;   /* batches before an inserted key can be erased or picked as a find hit
                           (0 = from the next batch on); a serving trace whose requests may share
                           one snapshot uses more than a launch's requests, so no request erases
                           a key another request of its launch inserts */
  uint32_t reserved[2];
} mvbt_mix_params;

void mvbt_wl_mix_default(mvbt_mix_params* p);

/* Generator over a present-key set that starts as distinct keys [0, initial_keys) of `seed`. */
void* mvbt_wl_mix_create(const mvbt_mix_params* p, uint64_t seed, uint64_t initial_keys);
void mvbt_wl_mix_destroy(void* h);
/* Generates the next num_batches batches; returns their total op count and the total range
 * output capacity in pairs (*range_pairs). The result is held until the next call. */
uint64_t mvbt_wl_mix_generate(void* h, uint32_t num_batches, uint64_t* range_pairs);
/* Copies the last generated batches: batch_off[num_batches + 1], per op type/key/arg, out_off
 * (range output offset in pairs) and range_cap (range output capacity in pairs). */
void mvbt_wl_mix_copy(void* h, uint64_t* batch_off, uint32_t* type, uint32_t* key, uint32_t* arg,
                      uint64_t* out_off, uint32_t* range_cap);
/* Number of keys present after all generated batches (key 0 excluded). */
uint64_t mvbt_wl_mix_present(void* h);

#ifdef __cplusplus
}
#endif

#endif /* MVBT_WORKLOAD_H_ */
