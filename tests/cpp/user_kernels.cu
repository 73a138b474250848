// User kernels written the way a reference user writes them (one key per thread; each tile of 8 or
// 16 threads serves its threads' keys one after another through the tile-cooperative methods),
// compiled against include/ only: gpu_btree_device.cuh (the reference's device method names) over
// mvbt_device.cuh, with the tree handle from the C ABI. Test infrastructure: the GPU tier drives
// these kernels through ctypes and checks their results against the oracle.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "gpu_btree_device.cuh"
#include "mvbt.h"

namespace cg = cooperative_groups;
using vtree = GpuBTree::device_versioned_btree<uint32_t, uint32_t>;
using btree = GpuBTree::device_blink_tree<uint32_t, uint32_t>;

namespace {

constexpr int kBlock = 128;

template <int W, class Tree>
__global__ void insert_kernel(Tree tree, const uint32_t* keys, const uint32_t* values, uint32_t n) {
  auto tile           = cg::tiled_partition<W>(cg::this_thread_block());
  const uint64_t tid  = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active   = tid < n;
  const uint32_t key  = active ? keys[tid] : 0u;
  const uint32_t val  = active ? values[tid] : 0u;
  typename Tree::device_allocator_context_type allocator{tree.allocator(), tile};
  for (uint32_t work = tile.ballot(active); work; work &= work - 1) {
    const int lane = __ffs(work) - 1;
    tree.cooperative_insert(tile.shfl(key, lane), tile.shfl(val, lane), tile, allocator);
  }
}

template <int W, class Tree>
__global__ void erase_kernel(Tree tree, const uint32_t* keys, uint32_t n) {
  auto tile          = cg::tiled_partition<W>(cg::this_thread_block());
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active  = tid < n;
  const uint32_t key = active ? keys[tid] : 0u;
  typename Tree::device_allocator_context_type allocator{tree.allocator(), tile};
  for (uint32_t work = tile.ballot(active); work; work &= work - 1) {
    const int lane = __ffs(work) - 1;
    tree.cooperative_erase(tile.shfl(key, lane), tile, allocator, true);
  }
}

template <int W>
__global__ void vfind_kernel(vtree tree, const uint32_t* keys, uint32_t* values, uint32_t n, uint32_t ts,
                             bool concurrent) {
  auto tile          = cg::tiled_partition<W>(cg::this_thread_block());
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active  = tid < n;
  const uint32_t key = active ? keys[tid] : 0u;
  vtree::device_allocator_context_type allocator{tree.allocator(), tile};
  for (uint32_t work = tile.ballot(active); work; work &= work - 1) {
    const int lane   = __ffs(work) - 1;
    const uint32_t v = ts == vtree::invalid_timestamp
                           ? tree.cooperative_find(tile.shfl(key, lane), tile, allocator, concurrent)
                           : tree.cooperative_find(tile.shfl(key, lane), tile, allocator, ts, concurrent);
    if ((int)tile.thread_rank() == lane) values[tid] = v;
  }
}

template <int W>
__global__ void vrange_kernel(vtree tree, const uint32_t* lo, const uint32_t* hi, mvbt_pair* out,
                              uint32_t* counts, uint32_t slot, uint32_t n, uint32_t ts) {
  auto tile          = cg::tiled_partition<W>(cg::this_thread_block());
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active  = tid < n;
  const uint32_t l = active ? lo[tid] : 0u, h = active ? hi[tid] : 0u;
  vtree::device_allocator_context_type allocator{tree.allocator(), tile};
  for (uint32_t work = tile.ballot(active); work; work &= work - 1) {
    const int lane     = __ffs(work) - 1;
    const uint64_t q   = tid - (uint64_t)tile.thread_rank() + lane;  // the query of that lane
    const uint32_t c   = tree.concurrent_cooperative_range_query(tile.shfl(l, lane), tile.shfl(h, lane), tile,
                                                                 allocator, ts, out + q * slot);
    if ((int)tile.thread_rank() == lane) counts[tid] = c;
  }
}

template <int W>
__global__ void bfind_kernel(btree tree, const uint32_t* keys, uint32_t* values, uint32_t n, bool concurrent) {
  auto tile          = cg::tiled_partition<W>(cg::this_thread_block());
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active  = tid < n;
  const uint32_t key = active ? keys[tid] : 0u;
  btree::device_allocator_context_type allocator{tree.allocator(), tile};
  for (uint32_t work = tile.ballot(active); work; work &= work - 1) {
    const int lane   = __ffs(work) - 1;
    const uint32_t v = tree.cooperative_find(tile.shfl(key, lane), tile, allocator, concurrent);
    if ((int)tile.thread_rank() == lane) values[tid] = v;
  }
}

template <int W>
__global__ void brange_kernel(btree tree, const uint32_t* lo, const uint32_t* hi, mvbt_pair* out, uint32_t* counts,
                              uint32_t slot, uint32_t n) {
  auto tile          = cg::tiled_partition<W>(cg::this_thread_block());
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active  = tid < n;
  const uint32_t l = active ? lo[tid] : 0u, h = active ? hi[tid] : 0u;
  btree::device_allocator_context_type allocator{tree.allocator(), tile};
  for (uint32_t work = tile.ballot(active); work; work &= work - 1) {
    const int lane   = __ffs(work) - 1;
    const uint64_t q = tid - (uint64_t)tile.thread_rank() + lane;
    const uint32_t c = tree.cooperative_range_query(tile.shfl(l, lane), tile.shfl(h, lane), tile, allocator,
                                                    out + q * slot, true);
    if ((int)tile.thread_rank() == lane) counts[tid] = c;
  }
}

template <int W>
__global__ void snapshot_kernel(vtree tree, uint32_t* out) {
  auto tile = cg::tiled_partition<W>(cg::this_thread_block());
  if (threadIdx.x < W) {
    const uint32_t s = tree.take_snapshot(tile);
    if (threadIdx.x == 0) *out = s;
  }
}

unsigned grid(uint32_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }
int done() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

}  // namespace

// W = 8 or 16; every entry point returns 0 after a successful launch.
extern "C" {

int uk_insert(mvbt_tree* h, int versioned, int W, const uint32_t* keys, const uint32_t* values, uint32_t n) {
  if (n == 0) return 0;
  if (versioned) {
    auto t = GpuBTree::device_versioned_view(h);
    if (W == 8) insert_kernel<8><<<grid(n), kBlock>>>(t, keys, values, n);
    else insert_kernel<16><<<grid(n), kBlock>>>(t, keys, values, n);
  } else {
    auto t = GpuBTree::device_blink_view(h);
    if (W == 8) insert_kernel<8><<<grid(n), kBlock>>>(t, keys, values, n);
    else insert_kernel<16><<<grid(n), kBlock>>>(t, keys, values, n);
  }
  return done();
}

int uk_erase(mvbt_tree* h, int versioned, int W, const uint32_t* keys, uint32_t n) {
  if (n == 0) return 0;
  if (versioned) {
    auto t = GpuBTree::device_versioned_view(h);
    if (W == 8) erase_kernel<8><<<grid(n), kBlock>>>(t, keys, n);
    else erase_kernel<16><<<grid(n), kBlock>>>(t, keys, n);
  } else {
    auto t = GpuBTree::device_blink_view(h);
    if (W == 8) erase_kernel<8><<<grid(n), kBlock>>>(t, keys, n);
    else erase_kernel<16><<<grid(n), kBlock>>>(t, keys, n);
  }
  return done();
}

int uk_find(mvbt_tree* h, int versioned, int W, const uint32_t* keys, uint32_t* values, uint32_t n, uint32_t ts,
            int concurrent) {
  if (n == 0) return 0;
  if (versioned) {
    auto t = GpuBTree::device_versioned_view(h);
    if (W == 8) vfind_kernel<8><<<grid(n), kBlock>>>(t, keys, values, n, ts, concurrent != 0);
    else vfind_kernel<16><<<grid(n), kBlock>>>(t, keys, values, n, ts, concurrent != 0);
  } else {
    auto t = GpuBTree::device_blink_view(h);
    if (W == 8) bfind_kernel<8><<<grid(n), kBlock>>>(t, keys, values, n, concurrent != 0);
    else bfind_kernel<16><<<grid(n), kBlock>>>(t, keys, values, n, concurrent != 0);
  }
  return done();
}

// out holds n * slot pairs; slot must be at least the largest count (the reference's contract).
int uk_range(mvbt_tree* h, int versioned, int W, const uint32_t* lo, const uint32_t* hi, mvbt_pair* out,
             uint32_t* counts, uint32_t slot, uint32_t n, uint32_t ts) {
  if (n == 0) return 0;
  if (versioned) {
    auto t = GpuBTree::device_versioned_view(h);
    if (W == 8) vrange_kernel<8><<<grid(n), kBlock>>>(t, lo, hi, out, counts, slot, n, ts);
    else vrange_kernel<16><<<grid(n), kBlock>>>(t, lo, hi, out, counts, slot, n, ts);
  } else {
    auto t = GpuBTree::device_blink_view(h);
    if (W == 8) brange_kernel<8><<<grid(n), kBlock>>>(t, lo, hi, out, counts, slot, n);
    else brange_kernel<16><<<grid(n), kBlock>>>(t, lo, hi, out, counts, slot, n);
  }
  return done();
}

int uk_take_snapshot(mvbt_tree* h, int W, uint32_t* d_out) {
  auto t = GpuBTree::device_versioned_view(h);
  if (W == 8) snapshot_kernel<8><<<1, 32>>>(t, d_out);
  else snapshot_kernel<16><<<1, 32>>>(t, d_out);
  return done();
}

}  // extern "C"
