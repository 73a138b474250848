// A reference-style caller: the unittest_versioning.cu flow (two batches with a snapshot between,
// finds and range queries at both snapshots) written against GpuBTree:: names from gpu_btree.h.
// Exits 0 when every result matches the expected values, 1 otherwise.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "gpu_btree.h"

#define CK(x)                                                              \
  do {                                                                     \
    cudaError_t e = (x);                                                   \
    if (e != cudaSuccess) {                                                \
      std::printf("%s: %s\n", #x, cudaGetErrorString(e));                 \
      return 1;                                                            \
    }                                                                      \
  } while (0)

int main() {
  using tree_t = GpuBTree::gpu_versioned_blink_tree<uint32_t, uint32_t>;
  const uint32_t n = 1024, half = n / 2, rq = 32;
  std::vector<uint32_t> keys(n), vals(n), lo(n), hi(n);
  for (uint32_t i = 0; i < n; ++i) {
    keys[i] = 2 * (i + 1);
    vals[i] = keys[i];
    lo[i]   = keys[i];
    hi[i]   = keys[i] + 2 * rq;
  }
  uint32_t *dk, *dv, *dlo, *dhi, *dout, *dcnt;
  tree_t::pair_type* dpairs;
  CK(cudaMalloc(&dk, n * 4));
  CK(cudaMalloc(&dv, n * 4));
  CK(cudaMalloc(&dlo, n * 4));
  CK(cudaMalloc(&dhi, n * 4));
  CK(cudaMalloc(&dout, n * 4));
  CK(cudaMalloc(&dcnt, n * 4));
  CK(cudaMalloc(&dpairs, n * rq * sizeof(tree_t::pair_type)));
  CK(cudaMemcpy(dk, keys.data(), n * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dv, vals.data(), n * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dlo, lo.data(), n * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dhi, hi.data(), n * 4, cudaMemcpyHostToDevice));
  int bad = 0;
  try {
    tree_t tree;
    tree.insert(dk, dv, half, 0, false);
    uint32_t s0 = tree.take_snapshot();
    tree.insert(dk + half, dv + half, n - half, 0, false);
    uint32_t s1 = tree.take_snapshot();
    std::vector<uint32_t> out(n), cnt(n);
    for (uint32_t ts : {s0, s1}) {
      tree.find(dk, dout, n, ts);
      CK(cudaMemcpy(out.data(), dout, n * 4, cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i < n; ++i) {
        uint32_t expect = (ts == s1 || i < half) ? vals[i] : 0xFFFFFFFFu;
        bad += out[i] != expect;
      }
      tree.range_query(dlo, dhi, dpairs, dcnt, rq, n, ts);
      CK(cudaMemcpy(cnt.data(), dcnt, n * 4, cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i < n; ++i) {
        uint32_t present = ts == s1 ? n : half;  // keys 2, 4, ..., 2 * present
        uint32_t first = i + 1, last = std::min(i + rq, present);
        uint32_t expect = last >= first ? last - first + 1 : 0;
        bad += cnt[i] != expect;
      }
    }
    tree.validate_tree_structure();
    tree.check_errors();
  } catch (const std::exception& e) {
    std::printf("error: %s\n", e.what());
    return 1;
  }
  std::printf(bad ? "FAILED %d mismatches\n" : "OK\n", bad);
  return bad ? 1 : 0;
}
