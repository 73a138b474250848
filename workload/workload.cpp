// Deterministic synthetic workloads (host-only library workload/libworkload.so).
//
// Counterpart of the reference's key generator include/rkg.hpp:77-97 (iota + std::shuffle with a
// seeded mt19937) and its query preparation helpers (include/rkg.hpp:36-73). Keys here are
// distinct uniform draws from [1, 2^32 - 3] instead of a dense iota, values are fmix32(key ^ salt).
#include <algorithm>
#include <cmath>
#include <deque>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "mvbt_workload.h"

namespace {

constexpr uint64_t kDomain = 0xFFFFFFFDull;  // 2^32 - 3 keys: [1, 2^32 - 3]

inline uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return h;
}

struct Feistel {
  uint32_t rk[4];
  explicit Feistel(uint64_t seed) {
    uint64_t s = seed ^ 0x5EEDF00DCAFEBABEull;
    for (int i = 0; i < 4; ++i) rk[i] = (uint32_t)splitmix(s);
  }
  uint32_t perm(uint32_t x) const {
    uint32_t l = x >> 16, r = x & 0xFFFFu;
    for (int i = 0; i < 4; ++i) {
      uint32_t f = fmix32(r ^ rk[i]) & 0xFFFFu;
      uint32_t t = l ^ f;
      l          = r;
      r          = t;
    }
    return (l << 16) | r;
  }
  // Bijection on [0, kDomain) by cycle walking.
  uint32_t key(uint64_t i) const {
    uint32_t y = perm((uint32_t)i);
    while (y >= kDomain) y = perm(y);
    return y + 1;
  }
};

inline uint32_t uniform_key(uint64_t& s) {
  uint64_t r = splitmix(s) >> 32;
  return (uint32_t)((r * kDomain) >> 32) + 1;
}

inline double uniform01(uint64_t& s) { return ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

inline double normal01(uint64_t& s) {
  double u1 = uniform01(s), u2 = uniform01(s);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

struct MixGen {
  mvbt_mix_params p;
  Feistel f;
  uint64_t rng;
  std::vector<uint32_t> present;
  // keys inserted in the last erase_lag batches (batch number, key): present in the tree, but
  // neither erased nor picked as find hits until they join `present`
  std::deque<std::pair<uint64_t, uint32_t>> young;
  uint64_t batch_no = 0;
  uint64_t next_insert;
  uint64_t next_miss = MVBT_MISS_INDEX_BASE;
  // last generated batches
  std::vector<uint64_t> batch_off;
  std::vector<uint32_t> type, key, arg, cap;
  std::vector<uint64_t> out_off;

  MixGen(const mvbt_mix_params& pp, uint64_t seed, uint64_t initial)
      : p(pp), f(seed), rng(seed * 0x2545F4914F6CDD1Dull + 17), next_insert(initial) {
    present.resize(initial);
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
      th.emplace_back([&, t] {
        for (uint64_t i = t; i < initial; i += nt) present[i] = f.key(i);
      });
    }
    for (auto& x : th) x.join();
  }

  uint32_t range_length() {
    // geometric on {1, 2, ...} with the given mean, clipped
    double m  = std::max(1.0, p.range_mean);
    double q  = 1.0 / m;
    double u  = uniform01(rng);
    double L  = (q >= 1.0) ? 1.0 : 1.0 + std::floor(std::log(u) / std::log1p(-q));
    L         = std::min<double>(std::max<double>(L, p.range_min), p.range_max);
    return (uint32_t)L;
  }

  uint64_t generate(uint32_t nb, uint64_t* range_pairs) {
    batch_off.assign(1, 0);
    type.clear();
    key.clear();
    arg.clear();
    cap.clear();
    out_off.clear();
    uint64_t pairs = 0;
    const double c1 = p.p_erase, c2 = c1 + p.p_insert, c3 = c2 + p.p_find;
    for (uint32_t b = 0; b < nb; ++b, ++batch_no) {
      while (!young.empty() && young.front().first + p.erase_lag <= batch_no) {
        present.push_back(young.front().second);
        young.pop_front();
      }
      uint64_t size;
      if (p.fixed_batch) {
        size = p.fixed_batch;
      } else {
        double ln = std::log(p.batch_median) + p.batch_sigma * normal01(rng);
        double sz = std::exp(ln);
        sz        = std::min<double>(std::max<double>(std::round(sz), p.batch_min), p.batch_max);
        size      = (uint64_t)sz;
      }
      const uint64_t base = type.size();
      type.resize(base + size);
      key.resize(base + size);
      arg.resize(base + size);
      cap.resize(base + size);
      out_off.resize(base + size);
      for (uint64_t i = 0; i < size; ++i) {
        double u = uniform01(rng);
        type[base + i] = u < c1 ? MVBT_OP_ERASE : (u < c2 ? MVBT_OP_INSERT : (u < c3 ? MVBT_OP_FIND : MVBT_OP_RANGE));
      }
      const uint64_t n_present = present.size();
      const double density     = (double)(n_present + young.size() + 1) / 4294967296.0;
      // pass 1: reads (they see the state at the batch snapshot: the present set as it is now)
      for (uint64_t i = 0; i < size; ++i) {
        const uint64_t o = base + i;
        if (type[o] == MVBT_OP_FIND) {
          bool hit = n_present > 0 && uniform01(rng) < p.find_hit;
          key[o]   = hit ? present[splitmix(rng) % n_present] : f.key(next_miss++);
          arg[o]   = 0;
          cap[o]   = 0;
          out_off[o] = 0;
        } else if (type[o] == MVBT_OP_RANGE) {
          uint32_t L   = range_length();
          uint32_t lo  = uniform_key(rng);
          uint64_t hi  = (uint64_t)lo + (uint64_t)L * p.stride;
          key[o]       = lo;
          arg[o]       = (uint32_t)std::min<uint64_t>(hi, 0xFFFFFFFFull);
          double lam   = (double)L * p.stride * density;
          uint64_t c   = (uint64_t)std::ceil(lam + 6.0 * std::sqrt(lam) + 16.0);
          c            = (c + 7) & ~7ull;
          cap[o]       = (uint32_t)c;
          out_off[o]   = pairs;
          pairs += c;
        }
      }
      // pass 2: erases of keys present at the snapshot (distinct within the batch)
      uint64_t live = n_present;
      for (uint64_t i = 0; i < size; ++i) {
        const uint64_t o = base + i;
        if (type[o] != MVBT_OP_ERASE) continue;
        if (live == 0) {  // nothing left to erase: erase a never-present key (a no-op)
          key[o] = f.key(next_miss++);
        } else {
          uint64_t j = splitmix(rng) % live;
          std::swap(present[j], present[live - 1]);
          --live;
          key[o] = present[live];
        }
        arg[o] = 0;
        cap[o] = 0;
        out_off[o] = 0;
      }
      present.resize(live);
      // pass 3: inserts of new keys
      for (uint64_t i = 0; i < size; ++i) {
        const uint64_t o = base + i;
        if (type[o] != MVBT_OP_INSERT) continue;
        uint32_t k = f.key(next_insert++);
        key[o]     = k;
        arg[o]     = fmix32(k ^ p.value_salt);
        cap[o]     = 0;
        out_off[o] = 0;
        if (p.erase_lag)
          young.emplace_back(batch_no, k);
        else
          present.push_back(k);
      }
      batch_off.push_back(type.size());
    }
    if (range_pairs) *range_pairs = pairs;
    return type.size();
  }
};

}  // namespace

extern "C" {

uint64_t mvbt_wl_splitmix64(uint64_t* state) { return splitmix(*state); }
uint32_t mvbt_wl_fmix32(uint32_t h) { return fmix32(h); }

void mvbt_wl_distinct_keys(uint64_t seed, uint64_t start, uint64_t n, uint32_t* out) {
  Feistel f(seed);
  const unsigned nt = (n > (1u << 20)) ? std::max(1u, std::min(16u, std::thread::hardware_concurrency())) : 1u;
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t) {
    th.emplace_back([&, t] {
      for (uint64_t i = t; i < n; i += nt) out[i] = f.key(start + i);
    });
  }
  for (auto& x : th) x.join();
}

void mvbt_wl_values(const uint32_t* keys, uint64_t n, uint32_t salt, uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i) out[i] = fmix32(keys[i] ^ salt);
}

void mvbt_wl_uniform_keys(uint64_t seed, uint64_t n, uint32_t* out) {
  uint64_t s = seed ^ 0xA5A5A5A5DEADBEEFull;
  for (uint64_t i = 0; i < n; ++i) out[i] = uniform_key(s);
}

void mvbt_wl_shuffle(uint64_t seed, uint32_t* a, uint64_t n) {
  uint64_t s = seed ^ 0x0123456789ABCDEFull;
  for (uint64_t i = n; i > 1; --i) {
    uint64_t j = splitmix(s) % i;
    std::swap(a[i - 1], a[j]);
  }
}

void mvbt_wl_upper_bounds(const uint32_t* lower, uint64_t n, uint64_t length, uint64_t stride,
                          uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t hi = (uint64_t)lower[i] + length * stride;
    out[i]      = (uint32_t)std::min<uint64_t>(hi, 0xFFFFFFFFull);
  }
}

void mvbt_wl_mix_default(mvbt_mix_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->p_erase      = 0.10;
  p->p_insert     = 0.20;
  p->p_find       = 0.50;
  p->p_range      = 0.20;
  p->find_hit     = 0.50;
  p->batch_median = 16384;
  p->batch_sigma  = 1.5;
  p->batch_min    = 1024;
  p->batch_max    = 4u << 20;
  p->range_mean   = 32;
  p->range_min    = 1;
  p->range_max    = 1024;
  p->stride       = 107;
  p->value_salt   = 0;
  p->fixed_batch  = 0;
}

void* mvbt_wl_mix_create(const mvbt_mix_params* p, uint64_t seed, uint64_t initial_keys) {
  return new MixGen(*p, seed, initial_keys);
}
void mvbt_wl_mix_destroy(void* h) { delete static_cast<MixGen*>(h); }

uint64_t mvbt_wl_mix_generate(void* h, uint32_t num_batches, uint64_t* range_pairs) {
  return static_cast<MixGen*>(h)->generate(num_batches, range_pairs);
}

void mvbt_wl_mix_copy(void* h, uint64_t* batch_off, uint32_t* type, uint32_t* key, uint32_t* arg,
                      uint64_t* out_off, uint32_t* range_cap) {
  auto* g = static_cast<MixGen*>(h);
  if (batch_off) std::memcpy(batch_off, g->batch_off.data(), g->batch_off.size() * 8);
  size_t n = g->type.size();
  if (type) std::memcpy(type, g->type.data(), n * 4);
  if (key) std::memcpy(key, g->key.data(), n * 4);
  if (arg) std::memcpy(arg, g->arg.data(), n * 4);
  if (out_off) std::memcpy(out_off, g->out_off.data(), n * 8);
  if (range_cap) std::memcpy(range_cap, g->cap.data(), n * 4);
}

uint64_t mvbt_wl_mix_present(void* h) {
  auto* g = static_cast<MixGen*>(h);
  return g->present.size() + g->young.size();
}

}  // extern "C"
