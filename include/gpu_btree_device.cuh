// gpu_btree_device.cuh -- the device half of the reference's API surface, for user kernels.
//
// The reference lets user kernels call tile-cooperative methods on the tree object they receive
// by value: cooperative_find / cooperative_insert / cooperative_erase / take_snapshot /
// concurrent_cooperative_range_query on GpuBTree::gpu_versioned_btree
// (include/gpu_versioned_blink_tree.hpp:304-559) and cooperative_insert / cooperative_find /
// cooperative_erase / cooperative_range_query on GpuBTree::gpu_blink_tree
// (include/gpu_blink_tree.hpp:268-390), each taking a cooperative-groups tile and a
// device_allocator_context built from the tree's allocator. This header keeps those names,
// argument orders and return values over mvbt::device_tree (include/mvbt_device.cuh):
//
//   auto dtree = GpuBTree::device_versioned_view(host_tree.handle());  // host: a by-value handle
//   ...
//   __global__ void k(GpuBTree::device_versioned_btree<uint32_t, uint32_t> tree, ...) {
//     auto tile = cg::tiled_partition<16>(cg::this_thread_block());   // 8 or 16 threads
//     using alloc_t = typename decltype(tree)::device_allocator_context_type;
//     alloc_t allocator{tree.allocator(), tile};
//     auto v = tree.cooperative_find(key, tile, allocator, snapshot, /*concurrent=*/true);
//   }
//
// Differences a caller sees: the allocator context carries nothing (the allocator's state lives
// in the tree's control block, per-SM chunks and the free ring), and user kernels need no friend
// access to build it; the reclaimer argument of the out-of-place forms is accepted and ignored
// (version copies go to the tree's retire log, freed by mvbt_reclaim or inside batch runs); a
// range query writes every hit from `buffer` on, as the reference does, so the caller sizes the
// buffer for the largest possible count. Writes stamp the tree's current write epoch, as the
// reference's writes read its current snapshot counter.
#pragma once

#include <cooperative_groups.h>

#include <cstdint>

#include "mvbt.h"
#include "mvbt_device.cuh"

namespace GpuBTree {

// Stand-ins for the reference's allocator context and device reclaimer.
struct device_allocator_handle {};
struct device_allocator_context {
  template <class Tile>
  __device__ device_allocator_context(const device_allocator_handle&, const Tile&) {}
};
struct device_reclaimer {};

namespace detail_device {
namespace cg = cooperative_groups;

template <unsigned W>
__device__ __forceinline__ void check_width() {
  static_assert(W == 8 || W == 16, "a node tile has 8 or 16 threads");
}

// Shared by both tree kinds: the view and the plain operations.
template <typename Key, typename Value, int B>
struct device_tree_base {
  static_assert(sizeof(Key) == 4 && sizeof(Value) == 4, "keys and values are 32-bit");
  static_assert(B == 16, "a node holds 16 pairs");
  using key_type                      = Key;
  using value_type                    = Value;
  using size_type                     = uint32_t;
  using pair_type                     = mvbt_pair;
  using device_allocator_context_type = device_allocator_context;
  static constexpr int branching_factor       = B;
  static constexpr Value invalid_value        = static_cast<Value>(MVBT_NOT_FOUND);
  static constexpr size_type invalid_timestamp = MVBT_LATEST;

  mvbt::device_tree tree;

  __host__ __device__ device_allocator_handle allocator() const { return {}; }

  template <unsigned W, class P, class DeviceAllocator>
  __device__ bool cooperative_insert(const Key& key, const Value& value, const cg::thread_block_tile<W, P>& tile,
                                     DeviceAllocator&) const {
    check_width<W>();
    const uint32_t E = tree.versioned ? tree.current_epoch() : 0u;
    return tree.template cooperative_insert<W>((uint32_t)key, (uint32_t)value, tile, E);
  }
  template <unsigned W, class P, class DeviceAllocator>
  __device__ bool cooperative_erase(const Key& key, const cg::thread_block_tile<W, P>& tile, DeviceAllocator&,
                                    bool /*concurrent*/ = false) const {
    check_width<W>();
    const uint32_t E = tree.versioned ? tree.current_epoch() : 0u;
    return tree.template cooperative_erase<W>((uint32_t)key, tile, E);
  }
};

}  // namespace detail_device

// The reference's gpu_blink_tree seen from a kernel.
template <typename Key, typename Value, int B = 16>
struct device_blink_tree : detail_device::device_tree_base<Key, Value, B> {
  using base = detail_device::device_tree_base<Key, Value, B>;
  using base::tree;

  // reference: cooperative_find(key, tile, allocator, concurrent) (gpu_blink_tree.hpp:277-303)
  template <unsigned W, class P, class DeviceAllocator>
  __device__ Value cooperative_find(const Key& key, const cooperative_groups::thread_block_tile<W, P>& tile,
                                    DeviceAllocator&, bool concurrent = false) const {
    detail_device::check_width<W>();
    return (Value)tree.template cooperative_find<W>((uint32_t)key, tile, mvbt::kLatest, concurrent);
  }
  // reference: cooperative_range_query(lower, upper, tile, allocator, buffer, concurrent)
  // (gpu_blink_tree.hpp:306-355); returns the number of keys in [lower, upper)
  template <unsigned W, class P, class DeviceAllocator>
  __device__ uint32_t cooperative_range_query(const Key& lower, const Key& upper,
                                              const cooperative_groups::thread_block_tile<W, P>& tile,
                                              DeviceAllocator&, mvbt_pair* buffer = nullptr,
                                              bool concurrent = false) const {
    detail_device::check_width<W>();
    return tree.template cooperative_range_query<W>((uint32_t)lower, (uint32_t)upper, tile, mvbt::kLatest,
                                                    reinterpret_cast<uint2*>(buffer), 0xFFFFFFFFu, concurrent);
  }
};

// The reference's gpu_versioned_btree (alias gpu_versioned_blink_tree) seen from a kernel.
template <typename Key, typename Value, int B = 16>
struct device_versioned_btree : detail_device::device_tree_base<Key, Value, B> {
  using base = detail_device::device_tree_base<Key, Value, B>;
  using base::cooperative_erase;
  using base::cooperative_insert;
  using base::tree;
  using size_type = typename base::size_type;

  // reference: take_snapshot(tile) (gpu_versioned_blink_tree.hpp:332-344): the pre-increment epoch
  template <unsigned W, class P>
  __device__ size_type take_snapshot(const cooperative_groups::thread_block_tile<W, P>& tile) const {
    return tree.take_snapshot(tile);
  }
  // reference: cooperative_find(key, tile, allocator, timestamp, concurrent) (:438-474)
  template <unsigned W, class P, class DeviceAllocator>
  __device__ Value cooperative_find(const Key& key, const cooperative_groups::thread_block_tile<W, P>& tile,
                                    DeviceAllocator&, const size_type& timestamp, bool concurrent = false) const {
    detail_device::check_width<W>();
    return (Value)tree.template cooperative_find<W>((uint32_t)key, tile, timestamp, concurrent);
  }
  // reference: cooperative_find(key, tile, allocator, concurrent): the newest state (:346-353)
  template <unsigned W, class P, class DeviceAllocator>
  __device__ Value cooperative_find(const Key& key, const cooperative_groups::thread_block_tile<W, P>& tile,
                                    DeviceAllocator& allocator, bool concurrent = false) const {
    const size_type latest = MVBT_LATEST;  // a local: the timestamp overload takes a reference
    return cooperative_find(key, tile, allocator, latest, concurrent);
  }
  // reference: concurrent_cooperative_range_query(lower, upper, tile, allocator, timestamp, buffer)
  // (:504-559); returns the number of keys in [lower, upper) at the snapshot
  template <unsigned W, class P, class DeviceAllocator>
  __device__ size_type concurrent_cooperative_range_query(const Key& lower, const Key& upper,
                                                          const cooperative_groups::thread_block_tile<W, P>& tile,
                                                          DeviceAllocator&, const size_type& timestamp,
                                                          mvbt_pair* buffer = nullptr) const {
    detail_device::check_width<W>();
    return tree.template cooperative_range_query<W>((uint32_t)lower, (uint32_t)upper, tile, timestamp,
                                                    reinterpret_cast<uint2*>(buffer), 0xFFFFFFFFu, true);
  }
  // reference: cooperative_insert_in_place / _out_of_place / cooperative_insert with a reclaimer
  // (:304-330): one copy-on-write scheme serves all three
  template <unsigned W, class P, class DeviceAllocator>
  __device__ bool cooperative_insert_in_place(const Key& key, const Value& value,
                                              const cooperative_groups::thread_block_tile<W, P>& tile,
                                              DeviceAllocator& allocator) const {
    return cooperative_insert(key, value, tile, allocator);
  }
  template <unsigned W, class P, class DeviceAllocator, class DeviceReclaimer>
  __device__ bool cooperative_insert_out_of_place(const Key& key, const Value& value,
                                                  const cooperative_groups::thread_block_tile<W, P>& tile,
                                                  DeviceAllocator& allocator, DeviceReclaimer&) const {
    return cooperative_insert(key, value, tile, allocator);
  }
  template <unsigned W, class P, class DeviceAllocator, class DeviceReclaimer>
  __device__ bool cooperative_insert(const Key& key, const Value& value,
                                     const cooperative_groups::thread_block_tile<W, P>& tile,
                                     DeviceAllocator& allocator, DeviceReclaimer&) const {
    return cooperative_insert(key, value, tile, allocator);
  }
  // reference: cooperative_erase(key, tile, allocator, reclaimer) (:393-436): a snapshot-preserving
  // erase (the in-place form, :355-390, is the base class's and preserves snapshots too)
  template <unsigned W, class P, class DeviceAllocator>
  __device__ bool cooperative_erase(const Key& key, const cooperative_groups::thread_block_tile<W, P>& tile,
                                    DeviceAllocator& allocator, device_reclaimer&) const {
    return cooperative_erase(key, tile, allocator, false);
  }
};

// Host: the by-value device handle of a tree created through the C ABI (mvbt_create, or the
// C++ classes of gpu_btree.h via their handle()). Kind and tile width are the caller's to match.
inline mvbt::device_tree device_tree_of(mvbt_tree* handle) {
  mvbt_device_view v{};
  mvbt::device_tree t{};
  if (mvbt_get_device_view(handle, &v) != MVBT_OK) return t;
  t.pool      = static_cast<uint32_t*>(v.pool);
  t.ctl       = static_cast<mvbt::control_block*>(v.control);
  t.versioned = v.versioned;
  t.capacity  = v.capacity;
  t.reclaim   = v.reclaim;
  return t;
}
template <typename Key = uint32_t, typename Value = uint32_t, int B = 16>
inline device_versioned_btree<Key, Value, B> device_versioned_view(mvbt_tree* handle) {
  device_versioned_btree<Key, Value, B> d;
  d.tree = device_tree_of(handle);
  return d;
}
template <typename Key = uint32_t, typename Value = uint32_t, int B = 16>
inline device_blink_tree<Key, Value, B> device_blink_view(mvbt_tree* handle) {
  device_blink_tree<Key, Value, B> d;
  d.tree = device_tree_of(handle);
  return d;
}

}  // namespace GpuBTree
