// gpu_btree.h -- C++ drop-in for the reference's host API, over the C ABI of libmvbt.so.
//
// The reference (owensgroup/MVGpuBTree) is included as <gpu_btree.h> and used through
// GpuBTree::gpu_blink_tree<uint32_t, uint32_t> (include/gpu_blink_tree.hpp:63-67) and
// GpuBTree::gpu_versioned_btree<uint32_t, uint32_t> (include/gpu_versioned_blink_tree.hpp:71-75).
// This header keeps those names, template parameters and host method signatures, so a caller
// switches by changing its include path and linking -lmvbt. Differences a caller can see:
//   * errors throw GpuBTree::mvbt_error instead of printing and calling std::terminate
//     (include/macros.hpp:23-30 of the reference);
//   * the allocator template parameter is accepted and ignored (the library has its own per-SM
//     node pool); B must be 16 (node = 16 pairs = 128 bytes);
//   * range queries write at most average_range_length pairs per query (the reference writes past
//     the slot) and report the full count in `counts`;
//   * erase on the versioned tree is a new version, so older snapshots keep the key.
// Handles are cheap shared copies, as in the reference (it shares device buffers through
// std::shared_ptr, include/gpu_versioned_blink_tree.hpp:94-102).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>

#include "mvbt.h"

namespace GpuBTree {

template <typename Key, typename Value>
struct pair_type {
  Key first;
  Value second;
};

class mvbt_error : public std::runtime_error {
 public:
  mvbt_error(int status, const std::string& where)
      : std::runtime_error(where + ": " + mvbt_status_string(status) + " (" + mvbt_last_error() + ")"),
        status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

namespace detail {

inline void check(int status, const char* where) {
  if (status != MVBT_OK) throw mvbt_error(status, where);
}

inline std::shared_ptr<mvbt_tree> make_tree(int kind, const mvbt_config* cfg) {
  mvbt_tree* t = nullptr;
  check(mvbt_create(kind, cfg, &t), "mvbt_create");
  return std::shared_ptr<mvbt_tree>(t, [](mvbt_tree* p) { mvbt_destroy(p); });
}

// Host methods shared by both trees.
template <typename Key, typename Value, int Kind>
class tree_base {
  static_assert(sizeof(Key) == 4 && sizeof(Value) == 4, "keys and values are 32-bit");

 public:
  using key_type                         = Key;
  using value_type                       = Value;
  using size_type                        = uint32_t;
  using pair_type                        = GpuBTree::pair_type<Key, Value>;
  static constexpr int branching_factor  = 16;
  static constexpr key_type invalid_key  = 0xFFFFFFFFu;
  static constexpr value_type invalid_value = 0xFFFFFFFFu;

  explicit tree_base(const mvbt_config* cfg = nullptr) : tree_(make_tree(Kind, cfg)) {}

  // reference: gpu_blink_tree.hpp:218-225 / gpu_versioned_blink_tree.hpp:106-142
  void insert(const Key* keys, const Value* values, size_type num_keys, cudaStream_t stream = 0) {
    check(mvbt_insert(tree_.get(), keys, values, num_keys, stream, 1), "insert");
  }
  // reference: gpu_blink_tree.hpp:227-236 / gpu_versioned_blink_tree.hpp:144-153
  void find(const Key* keys, Value* values, size_type num_keys, cudaStream_t stream = 0,
            bool concurrent = false) const {
    check(mvbt_find(tree_.get(), keys, values, num_keys, MVBT_LATEST, stream, concurrent), "find");
  }
  // reference: gpu_blink_tree.hpp:238-245 / gpu_versioned_blink_tree.hpp:166-173
  void erase(const Key* keys, size_type num_keys, cudaStream_t stream = 0, bool concurrent = false) {
    check(mvbt_erase(tree_.get(), keys, num_keys, stream, concurrent), "erase");
  }
  // reference: gpu_blink_tree.hpp:148-187 / gpu_versioned_blink_tree.hpp:252-294
  void concurrent_insert_range(const Key* keys, const Value* values, size_type num_insertion,
                               const Key* lower_bound, const Key* upper_bound,
                               size_type num_ranges, pair_type* result,
                               size_type average_range_length, cudaStream_t stream = 0) {
    check(mvbt_concurrent_insert_range(tree_.get(), keys, values, num_insertion, lower_bound,
                                       upper_bound, num_ranges, reinterpret_cast<mvbt_pair*>(result),
                                       average_range_length, nullptr, stream),
          "concurrent_insert_range");
  }
  // reference: gpu_blink_tree.hpp:189-216 / gpu_versioned_blink_tree.hpp:218-250
  void concurrent_find_erase(const Key* find_keys, Value* find_results, size_type num_finds,
                             const Key* erase_keys, size_type num_erasures, cudaStream_t stream = 0) {
    check(mvbt_concurrent_find_erase(tree_.get(), find_keys, find_results, num_finds, erase_keys,
                                     num_erasures, stream),
          "concurrent_find_erase");
  }
  // reference: compute_memory_usage (gpu_blink_tree.hpp:1076-1080), in GiB
  double compute_memory_usage() const {
    uint64_t nodes = 0, bytes = 0, pool = 0;
    check(mvbt_memory_usage(tree_.get(), &nodes, &bytes, &pool), "compute_memory_usage");
    return double(bytes) / double(1ull << 30);
  }
  // reference: validate_tree_structure (gpu_blink_tree.hpp:742-900); throws std::logic_error
  // on a broken invariant as the reference does.
  mvbt_report validate_tree_structure(uint32_t timestamp = MVBT_LATEST) const {
    mvbt_report r{};
    int st = mvbt_validate(tree_.get(), timestamp, &r);
    if (st == MVBT_ERR_CORRUPT) throw std::logic_error(std::string("tree structure: ") + mvbt_last_error());
    check(st, "validate_tree_structure");
    return r;
  }
  // Sticky device error bits (MVBT_DEVERR_*); throws when one is set.
  uint32_t check_errors(cudaStream_t stream = 0) const {
    uint32_t bits = 0;
    check(mvbt_check_errors(tree_.get(), stream, &bits), "check_errors");
    return bits;
  }
  mvbt_device_view device_view() const {
    mvbt_device_view v{};
    check(mvbt_get_device_view(tree_.get(), &v), "device_view");
    return v;
  }
  mvbt_tree* handle() const { return tree_.get(); }

 protected:
  static void check(int status, const char* where) { detail::check(status, where); }
  std::shared_ptr<mvbt_tree> tree_;
};

}  // namespace detail

// GpuBTree::gpu_blink_tree<Key, Value, B, Allocator> (reference include/gpu_blink_tree.hpp:63-67)
template <typename Key, typename Value, int B = 16, typename Allocator = void>
class gpu_blink_tree : public detail::tree_base<Key, Value, MVBT_KIND_BLINK> {
  static_assert(B == 16, "nodes hold 16 pairs");
  using base = detail::tree_base<Key, Value, MVBT_KIND_BLINK>;

 public:
  using typename base::pair_type;
  using typename base::size_type;
  explicit gpu_blink_tree(const mvbt_config* cfg = nullptr) : base(cfg) {}
  // reference: the bulk-build constructor (gpu_blink_tree.hpp:85-136): sorted input only, a
  // half-full tree; unsorted input throws (the reference prints and terminates)
  gpu_blink_tree(const Key* keys, const Value* values, size_type num_keys, bool sorted_input = false,
                 cudaStream_t stream = 0, const mvbt_config* cfg = nullptr)
      : base(cfg) {
    if (!sorted_input) throw mvbt_error(MVBT_ERR_BAD_ARG, "bulk build: only sorted input is supported");
    base::check(mvbt_bulk_build(this->tree_.get(), keys, values, num_keys, 8, stream), "bulk_build");
  }
  // reference: range_query (gpu_blink_tree.hpp:247-265)
  void range_query(const Key* lower_bound, const Key* upper_bound, pair_type* result,
                   size_type* counts, size_type average_range_length, size_type num_keys,
                   cudaStream_t stream = 0, bool concurrent = false) {
    base::check(mvbt_range_query(this->tree_.get(), lower_bound, upper_bound,
                                 reinterpret_cast<mvbt_pair*>(result), counts, average_range_length,
                                 num_keys, MVBT_LATEST, stream, concurrent),
                "range_query");
  }
};

// GpuBTree::gpu_versioned_btree<Key, Value, B, Allocator>
// (reference include/gpu_versioned_blink_tree.hpp:71-75)
template <typename Key, typename Value, int B = 16, typename Allocator = void>
class gpu_versioned_btree : public detail::tree_base<Key, Value, MVBT_KIND_VERSIONED> {
  static_assert(B == 16, "nodes hold 16 pairs");
  using base = detail::tree_base<Key, Value, MVBT_KIND_VERSIONED>;

 public:
  using typename base::pair_type;
  using typename base::size_type;
  using base::find;
  explicit gpu_versioned_btree(const mvbt_config* cfg = nullptr) : base(cfg) {}
  // reference: insert(..., in_place) (gpu_versioned_blink_tree.hpp:106-142)
  void insert(const Key* keys, const Value* values, size_type num_keys, cudaStream_t stream = 0,
              bool in_place = true) {
    base::check(mvbt_insert(this->tree_.get(), keys, values, num_keys, stream, in_place), "insert");
  }
  // reference: find(..., timestamp, ...) (gpu_versioned_blink_tree.hpp:154-164)
  void find(const Key* keys, Value* values, size_type num_keys, size_type timestamp,
            cudaStream_t stream = 0, bool concurrent = false) const {
    base::check(mvbt_find(this->tree_.get(), keys, values, num_keys, timestamp, stream, concurrent),
                "find");
  }
  // reference: range_query(..., timestamp, ...) (gpu_versioned_blink_tree.hpp:195-216)
  void range_query(const Key* lower_bound, const Key* upper_bound, pair_type* result,
                   size_type* counts, size_type average_range_length, size_type num_keys,
                   size_type timestamp, cudaStream_t stream = 0, bool concurrent = false) {
    base::check(mvbt_range_query(this->tree_.get(), lower_bound, upper_bound,
                                 reinterpret_cast<mvbt_pair*>(result), counts, average_range_length,
                                 num_keys, timestamp, stream, concurrent),
                "range_query");
  }
  // reference: take_snapshot (gpu_versioned_blink_tree.hpp:297-302); synchronises the stream
  size_type take_snapshot(cudaStream_t stream = 0) {
    uint32_t ts = 0;
    base::check(mvbt_take_snapshot(this->tree_.get(), stream, &ts), "take_snapshot");
    return ts;
  }
};

// The north-star name of the versioned tree.
template <typename Key, typename Value, int B = 16, typename Allocator = void>
using gpu_versioned_blink_tree = gpu_versioned_btree<Key, Value, B, Allocator>;

template <typename Key, typename Value, int B = 16>
using node_type = pair_type<Key, Value>[B];

}  // namespace GpuBTree
