// CPU oracle for the multiversion B-link tree hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: tests, the smoke entry point and the
// CPU-baseline leg of the benchmark may load it; the product library never links or calls it.
//
// It restates, as a plain ordered map, the logical semantics of the reference trees
// (owensgroup/MVGpuBTree). The reference has no CPU tree; its own tests check GPU results
// against std::set / std::unordered_set built from the inputs, and this oracle follows those
// validators:
//   * point lookups: membership + value, sentinel 0xFFFFFFFF on a miss
//       (include/validation.hpp:41-104, include/node.hpp:235-239)
//   * range queries: std::set::lower_bound walk over [lower, upper), ascending, written from
//       result + query_index * average_range_length (include/validation.hpp:184-264,
//       include/btree_kernels.hpp:308-361)
//   * one std::set state per snapshot (test/unittest_versioning.cu:286-376)
// and the semantics those validators rely on:
//   * the root leaf starts with the tombstone pair {0, 0}, so key 0 is present with value 0
//       (include/gpu_blink_tree.hpp:1151-1168, include/gpu_versioned_blink_tree.hpp:1455-1470)
//   * insert is an upsert (include/node.hpp:252-283)
//   * the snapshot counter starts at 0; take_snapshot returns the pre-increment value S and a
//     read at S sees exactly the writes made before that call
//       (include/gpu_versioned_blink_tree.hpp:297-302, 332-344, 1577-1603)
//   * a plain (non-versioned) tree ignores timestamps.
// Erase on the versioned tree is applied at the current write epoch, i.e. it is snapshot
// preserving (the copy-on-write erase of include/gpu_versioned_blink_tree.hpp:393-436). On
// every stream-ordered call sequence the reference's tests use, this is identical to the
// reference's in-place host erase (reads at an older snapshot are issued before the erase).
//
// The batch runner applies one snapshot per batch: reads at the batch snapshot S, writes at
// epoch S + 1. A multi-threaded key-range-partitioned runner times the same workload on all
// host cores.

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <map>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t kNotFound = 0xFFFFFFFFu;
constexpr uint32_t kLatest   = 0xFFFFFFFFu;

struct Version {
  uint32_t epoch;
  uint32_t value;
  bool present;
};

// Versions of one key, oldest first. Most keys carry exactly one version.
struct Chain {
  std::vector<Version> v;
};

struct MVMap {
  std::map<uint32_t, Chain> m;
  uint32_t counter = 0;  // current write epoch == next snapshot id
  bool versioned   = true;

  MVMap(bool ver) : versioned(ver) { write(0, 0, true, 0); }

  void write(uint32_t key, uint32_t value, bool present, uint32_t epoch) {
    auto& c = m[key].v;
    if (!versioned) {
      c.assign(1, Version{0, value, present});
      return;
    }
    if (!c.empty() && c.back().epoch == epoch) {
      c.back().value   = value;
      c.back().present = present;
    } else {
      c.push_back(Version{epoch, value, present});
    }
  }

  // Visible version at snapshot ts (kLatest = newest).
  static const Version* visible(const Chain& c, uint32_t ts) {
    const Version* best = nullptr;
    for (auto it = c.v.rbegin(); it != c.v.rend(); ++it) {
      if (ts == kLatest || it->epoch <= ts) {
        best = &*it;
        break;
      }
    }
    return best;
  }

  uint32_t find(uint32_t key, uint32_t ts) const {
    auto it = m.find(key);
    if (it == m.end()) return kNotFound;
    const Version* v = visible(it->second, versioned ? ts : kLatest);
    return (v && v->present) ? v->value : kNotFound;
  }

  // Writes up to cap pairs at out, returns the full count of keys in [lo, hi).
  uint32_t range(uint32_t lo, uint32_t hi, uint32_t* out, uint32_t cap, uint32_t ts) const {
    uint32_t count = 0;
    if (hi <= lo) return 0;
    for (auto it = m.lower_bound(lo); it != m.end() && it->first < hi; ++it) {
      const Version* v = visible(it->second, versioned ? ts : kLatest);
      if (!v || !v->present) continue;
      if (out && count < cap) {
        out[2 * count]     = it->first;
        out[2 * count + 1] = v->value;
      }
      ++count;
    }
    return count;
  }
};

// Op codes of the batched workload format (shared with the product's batch layout).
enum : uint32_t { kOpFind = 0, kOpInsert = 1, kOpErase = 2, kOpRange = 3 };

// Applies one batch: reads at snapshot ts, then writes at epoch ts + 1.
void run_one_batch(MVMap& mv,
                   const uint32_t* type,
                   const uint32_t* key,
                   const uint32_t* arg,
                   const uint64_t* out_off,
                   uint64_t begin,
                   uint64_t end,
                   uint32_t* result,
                   uint32_t* range_out,
                   uint32_t range_cap_of_op_fallback,
                   const uint32_t* range_cap) {
  const uint32_t ts = mv.counter;
  for (uint64_t i = begin; i < end; ++i) {
    if (type[i] == kOpFind) {
      result[i] = mv.find(key[i], ts);
    } else if (type[i] == kOpRange) {
      uint32_t cap = range_cap ? range_cap[i] : range_cap_of_op_fallback;
      uint32_t* o  = range_out ? range_out + 2 * out_off[i] : nullptr;
      result[i]    = mv.range(key[i], arg[i], o, cap, ts);
    }
  }
  mv.counter = ts + 1;  // take_snapshot() returned ts; writes of this batch land in ts + 1
  for (uint64_t i = begin; i < end; ++i) {
    if (type[i] == kOpInsert) {
      mv.write(key[i], arg[i], true, mv.counter);
      result[i] = 0;
    } else if (type[i] == kOpErase) {
      auto it = mv.m.find(key[i]);
      if (it != mv.m.end()) {
        const Version* v = MVMap::visible(it->second, kLatest);
        if (v && v->present) mv.write(key[i], kNotFound, false, mv.counter);
      }
      result[i] = 0;
    }
  }
}

}  // namespace

extern "C" {

void* orc_create(int versioned) { return new MVMap(versioned != 0); }
void orc_destroy(void* h) { delete static_cast<MVMap*>(h); }

uint32_t orc_current_epoch(void* h) { return static_cast<MVMap*>(h)->counter; }

// Reference: gpu_versioned_btree::take_snapshot (include/gpu_versioned_blink_tree.hpp:297-302).
uint32_t orc_take_snapshot(void* h) { return static_cast<MVMap*>(h)->counter++; }

// Reference: insert kernels (include/btree_kernels.hpp:363-472, 877-913): upsert each pair.
void orc_insert(void* h, const uint32_t* keys, const uint32_t* values, uint64_t n) {
  auto* mv = static_cast<MVMap*>(h);
  for (uint64_t i = 0; i < n; ++i) mv->write(keys[i], values[i], true, mv->counter);
}

// Reference: erase_kernel (include/btree_kernels.hpp:628-665); missing keys are no-ops.
void orc_erase(void* h, const uint32_t* keys, uint64_t n) {
  auto* mv = static_cast<MVMap*>(h);
  for (uint64_t i = 0; i < n; ++i) {
    auto it = mv->m.find(keys[i]);
    if (it == mv->m.end()) continue;
    const Version* v = MVMap::visible(it->second, kLatest);
    if (v && v->present) mv->write(keys[i], kNotFound, false, mv->counter);
  }
}

// Reference: find_kernel (include/btree_kernels.hpp:480-574). ts = 0xFFFFFFFF reads the newest.
void orc_find(void* h, const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t ts) {
  auto* mv = static_cast<MVMap*>(h);
  for (uint64_t i = 0; i < n; ++i) out[i] = mv->find(keys[i], ts);
}

// Reference: range_query_kernel (include/btree_kernels.hpp:308-361, 575-626). Query i writes
// its pairs (key, value) ascending at out + i * avg_len (at most avg_len of them) and its full
// count at counts[i] (counts may be null, out may be null).
void orc_range(void* h,
               const uint32_t* lo,
               const uint32_t* hi,
               uint32_t* out,
               uint32_t* counts,
               uint32_t avg_len,
               uint64_t n,
               uint32_t ts) {
  auto* mv = static_cast<MVMap*>(h);
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t c = mv->range(lo[i], hi[i], out ? out + 2 * i * (uint64_t)avg_len : nullptr, avg_len, ts);
    if (counts) counts[i] = c;
  }
}

// Number of keys visible at ts (the tombstone key 0 included).
uint64_t orc_size(void* h, uint32_t ts) {
  auto* mv   = static_cast<MVMap*>(h);
  uint64_t c = 0;
  for (auto& kv : mv->m) {
    const Version* v = MVMap::visible(kv.second, mv->versioned ? ts : kLatest);
    if (v && v->present) ++c;
  }
  return c;
}

// Writes the visible (key, value) pairs at ts in key order into keys/values (capacity cap);
// returns the number of visible pairs.
uint64_t orc_dump(void* h, uint32_t ts, uint32_t* keys, uint32_t* values, uint64_t cap) {
  auto* mv   = static_cast<MVMap*>(h);
  uint64_t c = 0;
  for (auto& kv : mv->m) {
    const Version* v = MVMap::visible(kv.second, mv->versioned ? ts : kLatest);
    if (!v || !v->present) continue;
    if (c < cap) {
      keys[c]   = kv.first;
      values[c] = v->value;
    }
    ++c;
  }
  return c;
}

// Runs a batched workload: batch b holds ops [batch_off[b], batch_off[b+1]). Per op:
// type (0 find, 1 insert, 2 erase, 3 range), key (or lower bound), arg (value or upper bound).
// Finds write the value, ranges the count, into result[i]; range op i writes at most
// range_cap[i] pairs at range_out + 2 * out_off[i] (u32 words).
void orc_run_batches(void* h,
                     uint32_t num_batches,
                     const uint64_t* batch_off,
                     const uint32_t* type,
                     const uint32_t* key,
                     const uint32_t* arg,
                     const uint64_t* out_off,
                     const uint32_t* range_cap,
                     uint32_t* result,
                     uint32_t* range_out) {
  auto* mv = static_cast<MVMap*>(h);
  for (uint32_t b = 0; b < num_batches; ++b)
    run_one_batch(*mv, type, key, arg, out_off, batch_off[b], batch_off[b + 1], result, range_out,
                  0, range_cap);
}

// ---------------------------------------------------------------------------------------------
// Partitioned runner used only to time the CPU baseline on all host cores: the key space is
// split into `parts` equal ranges, each owned by one thread and one MVMap. Each thread walks the
// whole batch list and applies the ops whose key falls in its range; a range query is clipped to
// each partition and its pieces land in key order in the op's slot (pieces are counted per
// partition, then concatenated). Semantics are identical to orc_run_batches.
// ---------------------------------------------------------------------------------------------
struct PartitionedOracle {
  std::vector<MVMap*> parts;
  std::vector<uint32_t> lo_bound;  // partition p owns keys [lo_bound[p], lo_bound[p+1])
};

void* orc_part_create(int versioned, uint32_t num_parts) {
  auto* po = new PartitionedOracle;
  for (uint32_t p = 0; p < num_parts; ++p) po->parts.push_back(new MVMap(versioned != 0));
  // Each MVMap seeds the tombstone key 0; only partition 0 owns it, the rest ignore key 0.
  for (uint32_t p = 0; p < num_parts; ++p) {
    uint64_t b = ((uint64_t)p << 32) / num_parts;
    po->lo_bound.push_back((uint32_t)b);
  }
  return po;
}

void orc_part_destroy(void* h) {
  auto* po = static_cast<PartitionedOracle*>(h);
  for (auto* m : po->parts) delete m;
  delete po;
}

void orc_part_insert(void* h, const uint32_t* keys, const uint32_t* values, uint64_t n) {
  auto* po   = static_cast<PartitionedOracle*>(h);
  uint32_t P = (uint32_t)po->parts.size();
  std::vector<std::thread> th;
  for (uint32_t p = 0; p < P; ++p) {
    th.emplace_back([&, p] {
      uint64_t lo = po->lo_bound[p], hi = (p + 1 < P) ? po->lo_bound[p + 1] : (1ull << 32);
      MVMap& mv = *po->parts[p];
      for (uint64_t i = 0; i < n; ++i)
        if (keys[i] >= lo && keys[i] < hi) mv.write(keys[i], values[i], true, mv.counter);
    });
  }
  for (auto& t : th) t.join();
}

void orc_part_run_batches(void* h,
                          uint32_t num_batches,
                          const uint64_t* batch_off,
                          const uint32_t* type,
                          const uint32_t* key,
                          const uint32_t* arg,
                          const uint64_t* out_off,
                          const uint32_t* range_cap,
                          uint32_t* result,
                          uint32_t* range_out) {
  auto* po   = static_cast<PartitionedOracle*>(h);
  uint32_t P = (uint32_t)po->parts.size();
  uint64_t n = batch_off[num_batches];
  struct Spill {
    uint64_t op;
    std::vector<uint32_t> pairs;
  };
  // part_count[p][i]: pairs partition p found for range op i. The partition that owns the lower
  // bound (the head) writes its piece straight into the op's slot; other partitions spill theirs
  // and the pieces are appended in partition (= key) order after all threads join.
  std::vector<std::vector<uint32_t>> part_count(P);
  std::vector<std::vector<Spill>> spills(P);
  std::vector<std::thread> th;
  for (uint32_t p = 0; p < P; ++p) {
    th.emplace_back([&, p] {
      uint64_t plo = po->lo_bound[p], phi = (p + 1 < P) ? po->lo_bound[p + 1] : (1ull << 32);
      MVMap& mv = *po->parts[p];
      auto& pc  = part_count[p];
      pc.assign(n, 0);
      for (uint32_t b = 0; b < num_batches; ++b) {
        const uint32_t ts = mv.counter;
        for (uint64_t i = batch_off[b]; i < batch_off[b + 1]; ++i) {
          if (type[i] == kOpFind) {
            if (key[i] >= plo && key[i] < phi) result[i] = mv.find(key[i], ts);
          } else if (type[i] == kOpRange) {
            uint64_t lo = std::max<uint64_t>(key[i], plo), hi = std::min<uint64_t>(arg[i], phi);
            if (lo >= hi) continue;
            bool head    = key[i] >= plo && key[i] < phi;
            uint32_t cap = range_cap[i];
            if (head) {
              pc[i] = mv.range((uint32_t)lo, (uint32_t)hi, range_out ? range_out + 2 * out_off[i] : nullptr,
                               cap, ts);
            } else {
              Spill s{i, std::vector<uint32_t>(2 * (size_t)cap)};
              pc[i] = mv.range((uint32_t)lo, (uint32_t)hi, s.pairs.data(), cap, ts);
              if (pc[i]) spills[p].push_back(std::move(s));
            }
          }
        }
        mv.counter = ts + 1;
        for (uint64_t i = batch_off[b]; i < batch_off[b + 1]; ++i) {
          if (!(key[i] >= plo && key[i] < phi)) continue;
          if (type[i] == kOpInsert) {
            mv.write(key[i], arg[i], true, mv.counter);
          } else if (type[i] == kOpErase) {
            auto it = mv.m.find(key[i]);
            if (it != mv.m.end()) {
              const Version* v = MVMap::visible(it->second, kLatest);
              if (v && v->present) mv.write(key[i], kNotFound, false, mv.counter);
            }
          }
        }
      }
    });
  }
  for (auto& t : th) t.join();
  std::vector<uint32_t> filled(n, 0);
  for (uint64_t i = 0; i < n; ++i) {
    if (type[i] == kOpRange) {
      uint32_t c = 0;
      for (uint32_t p = 0; p < P; ++p) c += part_count[p][i];
      result[i] = c;
      for (uint32_t p = 0; p < P; ++p)
        if (key[i] >= po->lo_bound[p] && (p + 1 == P || key[i] < po->lo_bound[p + 1]))
          filled[i] = part_count[p][i];
    } else if (type[i] != kOpFind) {
      result[i] = 0;
    }
  }
  if (range_out) {
    for (uint32_t p = 0; p < P; ++p) {
      for (auto& s : spills[p]) {
        uint64_t i   = s.op;
        uint32_t cap = range_cap[i];
        uint32_t c   = part_count[p][i];
        for (uint32_t j = 0; j < c && filled[i] < cap; ++j, ++filled[i]) {
          range_out[2 * (out_off[i] + filled[i])]     = s.pairs[2 * j];
          range_out[2 * (out_off[i] + filled[i]) + 1] = s.pairs[2 * j + 1];
        }
      }
    }
  }
}

}  // extern "C"
