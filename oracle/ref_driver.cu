// ref_driver.cu -- runs the reference implementation (owensgroup/MVGpuBTree, its unmodified
// headers) through the reference's own public host API, on workloads from this repository's
// generator (workload/mvbt_workload.h), and prints one JSON line with throughput and checksums of
// every result. It is test and baseline infrastructure: oracle/ref_build.py compiles it, and only
// the tests and bench.py's reference arm run it.
//
// Modes:
//   c1 --n N --seed S [--warmup W] [--reps R]
//      Plain B-link tree, GpuBTree::gpu_blink_tree<uint32_t, uint32_t> (reference
//      include/gpu_blink_tree.hpp:63-67): insert N distinct keys of seed S with values
//      fmix32(key ^ S), then N finds shuffled from N/2 inserted keys and N - N/2 keys that were
//      never inserted (include/gpu_blink_tree.hpp:218-236).
//   c2 --initial N --updates U --seed S [--warmup W] [--reps R]
//      Versioned tree: insert, snapshot S0, update U keys in place, snapshot S1, the queries of c1
//      at S0 and at S1; each phase timed alone (run_c2).
//   c3 --initial N --seed S [--stride D] --combos I:R:L:Q[,...] [--warmup W] [--reps R]
//      [--checksums 0|1] [--dump PREFIX]
//      Versioned tree: per combination, inserts and range queries at the snapshot taken before
//      them, timed on a fresh tree, and a deterministic insert / snapshot / insert / range_query
//      sequence checked (run_c3).
//   c4 --initial N --batches B --steps K --warmup W --seed S [--stride D] [--median M]
//      [--batch-min A] [--batch-max Z] [--final-chunks C] [--checksums 0|1]
//      Versioned tree, GpuBTree::gpu_versioned_btree<uint32_t, uint32_t>
//      (include/gpu_versioned_blink_tree.hpp:71-75), N distinct keys of seed S with values
//      fmix32(key ^ 0), then W + K steps of B mixed batches each, issued one batch at a time in
//      the reference's plain form (include/gpu_versioned_blink_tree.hpp:106-216, 297-302):
//        S_b = take_snapshot(); find(keys, S_b); range_query(lo, hi, S_b); insert(in_place); erase
//      Reads see the state after every earlier batch; the batch's own writes follow them. Only the
//      K later steps are timed (CUDA events on the launching stream). With --final-chunks C the
//      whole key space [1, 2^32 - 1) is read at a final snapshot as C consecutive range queries.
//
// Checksums (the tests compute the same sums from this library's outputs): with
// mix(x) = the SplitMix64 finalizer of x + 0x9E3779B97F4A7C15 and i an op's index in its step,
//   find  = sum over finds of mix(i << 32 | value)
//   count = sum over range queries of mix((i << 32 | count) ^ 0xC3A5C85C97CB3127)
//   pairs = sum over range queries and j < min(count, capacity_i) of
//           mix(mix((i << 20 | j) ^ 0xB492B66FBE98F273) ^ (key_j << 32 | value_j))
// all modulo 2^64. The range slot of a batch holds as many pairs as the largest capacity among
// its queries; the reference writes every hit (it has no bound), so the buffer carries a tail of
// 1024 * stride pairs, more than any query [lo, lo + L * stride) with L <= 1024 can return.
#include <gpu_btree.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../workload/mvbt_workload.h"

namespace {

using key_t   = uint32_t;
using value_t = uint32_t;
using pair_t  = pair_type<key_t, value_t>;
using vnode_t = GpuBTree::node_type<key_t, value_t, 16>;
// 2^29 nodes (64 GiB of the B200's 180 GB): room for a 40M-key tree and the versions of 25 steps
// of 256 mixed batches (about 180M nodes by the estimate below; the reference's tree measured
// about 1 node per write). The reference's bump allocator does not check its bound
// (include/device_bump_allocator.hpp:46-54), so the driver refuses workloads whose estimate could
// come near it (pool_estimate_ok) and reads the allocator's count between steps (untimed), stopping
// with an error before a step could reach the bound.
using valloc_t  = device_bump_allocator<vnode_t, (1ull << 29)>;
using vtree_t   = GpuBTree::gpu_versioned_btree<key_t, value_t, 16, valloc_t>;
using btree_t   = GpuBTree::gpu_blink_tree<key_t, value_t, 16>;
constexpr uint64_t kPoolNodes = 1ull << 29;

// Generous node estimate of a versioned workload: the initial tree at half-full leaves (two nodes
// per 7 keys, interior levels included) plus 2 nodes per write (a version copy, a split now and
// then; measured about 1).
bool pool_estimate_ok(uint64_t initial, uint64_t writes) {
  const uint64_t bound = 2 * (initial / 7 + 1) + 2 * writes + 4096;
  if (bound <= kPoolNodes) return true;
  std::fprintf(stderr, "ref_driver: workload could exceed the %llu-node pool (estimate %llu)\n",
               (unsigned long long)kPoolNodes, (unsigned long long)bound);
  return false;
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ref_driver: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

uint64_t mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
uint64_t find_term(uint64_t i, uint32_t v) { return mix(i << 32 | v); }
uint64_t count_term(uint64_t i, uint32_t c) { return mix((i << 32 | c) ^ 0xC3A5C85C97CB3127ull); }
uint64_t pair_term(uint64_t i, uint64_t j, uint32_t k, uint32_t v) {
  return mix(mix((i << 20 | j) ^ 0xB492B66FBE98F273ull) ^ ((uint64_t)k << 32 | v));
}

struct args_t {
  std::string mode;
  uint64_t n = 1 << 20, initial = 1 << 20, seed = 1, updates = 0;
  uint32_t batches = 16, steps = 1, warmup = 0, final_chunks = 0, checksums = 1, reps = 1;
  uint64_t stride = 0;
  double median = 0;
  uint32_t batch_min = 0, batch_max = 0;
  std::string combos, dump;
};

args_t parse(int argc, char** argv) {
  args_t a;
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_driver c1|c2|c3|c4 [--key value]...\n");
    std::exit(2);
  }
  a.mode = argv[1];
  for (int i = 2; i + 1 < argc; i += 2) {
    std::string k = argv[i];
    const char* v = argv[i + 1];
    if (k == "--n") a.n = std::strtoull(v, nullptr, 10);
    else if (k == "--initial") a.initial = std::strtoull(v, nullptr, 10);
    else if (k == "--seed") a.seed = std::strtoull(v, nullptr, 10);
    else if (k == "--batches") a.batches = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--steps") a.steps = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--warmup") a.warmup = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--final-chunks") a.final_chunks = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--checksums") a.checksums = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--stride") a.stride = std::strtoull(v, nullptr, 10);
    else if (k == "--median") a.median = std::strtod(v, nullptr);
    else if (k == "--batch-min") a.batch_min = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--batch-max") a.batch_max = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--updates") a.updates = std::strtoull(v, nullptr, 10);
    else if (k == "--reps") a.reps = (uint32_t)std::strtoul(v, nullptr, 10);
    else if (k == "--combos") a.combos = v;
    else if (k == "--dump") a.dump = v;
    else {
      std::fprintf(stderr, "ref_driver: unknown option %s\n", k.c_str());
      std::exit(2);
    }
  }
  return a;
}

template <class T>
T* dev_alloc(uint64_t n) {
  T* p = nullptr;
  check(cudaMalloc(&p, std::max<uint64_t>(n, 1) * sizeof(T)), "cudaMalloc");
  return p;
}
template <class T>
T* dev_copy(const std::vector<T>& h) {
  T* p = dev_alloc<T>(h.size());
  if (!h.empty()) check(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
  return p;
}
template <class T>
std::vector<T> host_copy(const T* d, uint64_t n) {
  std::vector<T> h(n);
  if (n) check(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost), "download");
  return h;
}

float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  check(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
  return ms;
}

// Point queries of configs 1 and 2: n/2 inserted keys (a shuffle of seed + 1) and n - n/2 keys
// that were never inserted, shuffled together with seed + 2.
std::vector<uint32_t> hit_miss_queries(uint64_t seed, const std::vector<uint32_t>& keys) {
  const uint64_t n = keys.size(), nh = n / 2;
  std::vector<uint32_t> hits(keys), q(n);
  mvbt_wl_shuffle(seed + 1, hits.data(), n);
  std::copy(hits.begin(), hits.begin() + nh, q.begin());
  mvbt_wl_distinct_keys(seed, MVBT_MISS_INDEX_BASE, n - nh, q.data() + nh);
  mvbt_wl_shuffle(seed + 2, q.data(), n);
  return q;
}

uint64_t find_checksum(const uint32_t* d, uint64_t n) {
  auto out   = host_copy(d, n);
  uint64_t s = 0;
  for (uint64_t i = 0; i < n; ++i) s += find_term(i, out[i]);
  return s;
}

int run_c1(const args_t& a) {
  const uint64_t n = a.n;
  std::vector<uint32_t> keys(n), vals(n);
  mvbt_wl_distinct_keys(a.seed, 0, n, keys.data());
  mvbt_wl_values(keys.data(), n, (uint32_t)a.seed, vals.data());
  std::vector<uint32_t> q = hit_miss_queries(a.seed, keys);

  uint32_t *dk = dev_copy(keys), *dv = dev_copy(vals), *dq = dev_copy(q), *dr = dev_alloc<uint32_t>(n);
  cudaEvent_t e0, e1, e2;
  check(cudaEventCreate(&e0), "event");
  check(cudaEventCreate(&e1), "event");
  check(cudaEventCreate(&e2), "event");
  const uint32_t reps = std::max(1u, a.reps);
  double ins_ms = 0, find_ms = 0;
  for (uint32_t r = 0; r < a.warmup + reps; ++r) {  // fresh tree per experiment
    btree_t tree;
    check(cudaDeviceSynchronize(), "setup");
    check(cudaEventRecord(e0, 0), "record");
    tree.insert(dk, dv, (uint32_t)n, 0);
    check(cudaEventRecord(e1, 0), "record");
    tree.find(dq, dr, (uint32_t)n, 0, false);
    check(cudaEventRecord(e2, 0), "record");
    check(cudaEventSynchronize(e2), "sync");
    check(cudaGetLastError(), "kernels");
    if (r >= a.warmup) {
      ins_ms += elapsed_ms(e0, e1) / reps;
      find_ms += elapsed_ms(e1, e2) / reps;
    }
  }
  const uint64_t cs = find_checksum(dr, n);
  std::printf(
      "{\"mode\": \"c1\", \"n\": %llu, \"seed\": %llu, \"reps\": %u, \"insert_ms\": %.4f, \"find_ms\": %.4f, "
      "\"insert_mops\": %.3f, \"find_mops\": %.3f, \"find_checksum\": %llu}\n",
      (unsigned long long)n, (unsigned long long)a.seed, reps, ins_ms, find_ms, n / (ins_ms * 1e3),
      n / (find_ms * 1e3), (unsigned long long)cs);
  cudaFree(dk);
  cudaFree(dv);
  cudaFree(dq);
  cudaFree(dr);
  return 0;
}

// Config 2: versioned tree, N keys of seed S (values fmix32(key ^ S)), snapshot S0, U of them
// updated (a shuffle of seed S + 3, values fmix32(key ^ S ^ 1)), snapshot S1, then the N queries
// of hit_miss_queries at S0 and at S1. Writes in place (the reference's ViB form,
// include/gpu_versioned_blink_tree.hpp:106-142). Each phase is timed alone; the experiment runs
// W untimed and R timed times on fresh trees and the timed phases are averaged.
int run_c2(const args_t& a) {
  const uint64_t n = a.initial, u = a.updates ? std::min(a.updates, n) : n / 8;
  std::vector<uint32_t> keys(n), vals(n), upd, uvals(u);
  mvbt_wl_distinct_keys(a.seed, 0, n, keys.data());
  mvbt_wl_values(keys.data(), n, (uint32_t)a.seed, vals.data());
  upd = keys;
  mvbt_wl_shuffle(a.seed + 3, upd.data(), n);
  upd.resize(u);
  mvbt_wl_values(upd.data(), u, (uint32_t)a.seed ^ 1u, uvals.data());
  std::vector<uint32_t> q = hit_miss_queries(a.seed, keys);
  uint32_t *dk = dev_copy(keys), *dv = dev_copy(vals), *du = dev_copy(upd), *duv = dev_copy(uvals);
  uint32_t *dq = dev_copy(q), *dr0 = dev_alloc<uint32_t>(n), *dr1 = dev_alloc<uint32_t>(n);
  cudaEvent_t ev[7];
  for (auto& e : ev) check(cudaEventCreate(&e), "event");
  double ms[4] = {0, 0, 0, 0};
  uint64_t cs0 = 0, cs1 = 0;
  const uint32_t reps = std::max(1u, a.reps);
  for (uint32_t r = 0; r < a.warmup + reps; ++r) {  // fresh tree per experiment
    vtree_t tree;
    check(cudaDeviceSynchronize(), "setup");
    check(cudaEventRecord(ev[0], 0), "record");
    tree.insert(dk, dv, (uint32_t)n, 0, true);
    check(cudaEventRecord(ev[1], 0), "record");
    const uint32_t S0 = tree.take_snapshot();  // a blocking copy, outside the timed phases
    check(cudaEventRecord(ev[2], 0), "record");
    tree.insert(du, duv, (uint32_t)u, 0, true);
    check(cudaEventRecord(ev[3], 0), "record");
    const uint32_t S1 = tree.take_snapshot();
    check(cudaEventRecord(ev[4], 0), "record");
    tree.find(dq, dr0, (uint32_t)n, S0, 0, false);
    check(cudaEventRecord(ev[5], 0), "record");
    tree.find(dq, dr1, (uint32_t)n, S1, 0, false);
    check(cudaEventRecord(ev[6], 0), "record");
    check(cudaEventSynchronize(ev[6]), "sync");
    check(cudaGetLastError(), "kernels");
    if (r < a.warmup) continue;
    ms[0] += elapsed_ms(ev[0], ev[1]);
    ms[1] += elapsed_ms(ev[2], ev[3]);
    ms[2] += elapsed_ms(ev[4], ev[5]);
    ms[3] += elapsed_ms(ev[5], ev[6]);
    if (r + 1 == a.warmup + reps) {
      cs0 = find_checksum(dr0, n);
      cs1 = find_checksum(dr1, n);
    }
  }
  for (double& m : ms) m /= reps;
  std::printf(
      "{\"mode\": \"c2\", \"initial\": %llu, \"updates\": %llu, \"seed\": %llu, \"reps\": %u, "
      "\"insert_ms\": %.4f, \"update_ms\": %.4f, \"find0_ms\": %.4f, \"find1_ms\": %.4f, "
      "\"insert_mops\": %.3f, \"update_mops\": %.3f, \"find0_mops\": %.3f, \"find1_mops\": %.3f, "
      "\"find_checksums\": [%llu, %llu]}\n",
      (unsigned long long)n, (unsigned long long)u, (unsigned long long)a.seed, reps, ms[0], ms[1], ms[2], ms[3],
      n / (ms[0] * 1e3), u / (ms[1] * 1e3), n / (ms[2] * 1e3), n / (ms[3] * 1e3), (unsigned long long)cs0,
      (unsigned long long)cs1);
  for (auto& e : ev) cudaEventDestroy(e);
  for (uint32_t* p : {dk, dv, du, duv, dq, dr0, dr1}) cudaFree(p);
  return 0;
}

// Config 3: versioned tree of N keys of seed S (values fmix32(key ^ S)); per combination I:R:L:Q,
// I new keys (distinct_keys(S, N, I), values fmix32(key ^ S)) and R range queries with uniform
// lower bounds (seed S + 1) and upper = lower + L * stride, Q pairs of output per query.
//   timed: on a fresh tree, S0 = take_snapshot, then the I inserts in place and the R range
//          queries at S0 as two host calls (include/gpu_versioned_blink_tree.hpp:106-142,
//          195-216): the reference's plain form of the workload. Its one-kernel form,
//          concurrent_insert_range (include/gpu_versioned_blink_tree.hpp:252-294), raised an
//          illegal memory access on a B200 with inputs whose buffers are in bounds (1 of 2 runs of
//          262144 keys, 54000 inserts, 6000 queries of L = 128, then in 2 of 2), so it is not run.
//   checked (--checksums 1): insert, S0 = take_snapshot, insert of the new keys, S1 =
//          take_snapshot, range_query at S0 and at S1 with 4L + 64 pairs per query; counts and
//          pairs checksums, once with the second insert in place ("checksums") and once out of
//          place ("checksums_out_of_place"); --dump P writes each count array to P_<form>_s<v>.u32.
// The reference writes every hit of a query with no bound; each pair buffer carries a tail of
// L * stride pairs, more than the last query's range [lo, lo + L * stride) can hold.
struct c3_combo {
  uint64_t inserts, ranges, length, slot;
};

std::vector<c3_combo> parse_combos(const std::string& s) {
  std::vector<c3_combo> out;
  size_t p = 0;
  while (p < s.size()) {
    size_t e = s.find(',', p);
    if (e == std::string::npos) e = s.size();
    c3_combo c{};
    unsigned long long i = 0, r = 0, l = 0, q = 0;
    if (std::sscanf(s.substr(p, e - p).c_str(), "%llu:%llu:%llu:%llu", &i, &r, &l, &q) != 4 || l == 0 || q == 0) {
      std::fprintf(stderr, "ref_driver: bad combination '%s' (inserts:ranges:length:slot)\n",
                   s.substr(p, e - p).c_str());
      std::exit(2);
    }
    c = {i, r, l, q};
    out.push_back(c);
    p = e + 1;
  }
  return out;
}

void range_checksums(const std::vector<uint32_t>& cnt, const pair_t* dpairs, uint64_t slot, uint64_t& cs_c,
                     uint64_t& cs_p, uint64_t& max_count) {
  auto pairs = host_copy(dpairs, cnt.size() * slot);
  cs_c = cs_p = max_count = 0;
  for (uint64_t i = 0; i < cnt.size(); ++i) {
    cs_c += count_term(i, cnt[i]);
    max_count = std::max<uint64_t>(max_count, cnt[i]);
    const uint64_t m = std::min<uint64_t>(cnt[i], slot);
    for (uint64_t j = 0; j < m; ++j) cs_p += pair_term(i, j, pairs[i * slot + j].first, pairs[i * slot + j].second);
  }
}

int run_c3(const args_t& a) {
  const uint64_t n      = a.initial;
  const uint64_t stride = a.stride ? a.stride : 0xFFFFFFFDull / std::max<uint64_t>(n, 1);
  const auto combos     = parse_combos(a.combos);
  std::vector<uint32_t> keys(n), vals(n);
  mvbt_wl_distinct_keys(a.seed, 0, n, keys.data());
  mvbt_wl_values(keys.data(), n, (uint32_t)a.seed, vals.data());
  for (const auto& c : combos)
    if (!pool_estimate_ok(n, c.inserts)) return 2;
  uint32_t *dk = dev_copy(keys), *dv = dev_copy(vals);
  cudaEvent_t e0, e1, e2, e3;
  check(cudaEventCreate(&e0), "event");
  check(cudaEventCreate(&e1), "event");
  check(cudaEventCreate(&e2), "event");
  check(cudaEventCreate(&e3), "event");
  const uint32_t reps = std::max(1u, a.reps);
  std::printf("{\"mode\": \"c3\", \"initial\": %llu, \"seed\": %llu, \"stride\": %llu, \"reps\": %u, \"runs\": [",
              (unsigned long long)n, (unsigned long long)a.seed, (unsigned long long)stride, reps);
  for (size_t ci = 0; ci < combos.size(); ++ci) {
    const c3_combo& c = combos[ci];
    std::vector<uint32_t> ins(c.inserts), ivals(c.inserts), lo(c.ranges), hi(c.ranges);
    mvbt_wl_distinct_keys(a.seed, n, c.inserts, ins.data());
    mvbt_wl_values(ins.data(), c.inserts, (uint32_t)a.seed, ivals.data());
    mvbt_wl_uniform_keys(a.seed + 1, c.ranges, lo.data());
    mvbt_wl_upper_bounds(lo.data(), c.ranges, c.length, stride, hi.data());
    uint32_t *di = dev_copy(ins), *div = dev_copy(ivals), *dlo = dev_copy(lo), *dhi = dev_copy(hi);
    const uint64_t tail = c.length * stride;
    pair_t* dp          = dev_alloc<pair_t>(c.ranges * c.slot + tail);
    uint32_t* dcnt_t    = dev_alloc<uint32_t>(c.ranges);
    double ins_ms = 0, ops_ms = 0;
    for (uint32_t r = 0; r < a.warmup + reps; ++r) {  // fresh tree per experiment
      vtree_t tree;
      check(cudaDeviceSynchronize(), "setup");
      check(cudaEventRecord(e0, 0), "record");
      tree.insert(dk, dv, (uint32_t)n, 0, true);
      check(cudaEventRecord(e1, 0), "record");
      const uint32_t S0 = tree.take_snapshot();  // a blocking copy, before the timed calls start
      check(cudaEventRecord(e3, 0), "record");
      tree.insert(di, div, (uint32_t)c.inserts, 0, true);
      tree.range_query(dlo, dhi, dp, dcnt_t, (uint32_t)c.slot, (uint32_t)c.ranges, S0, 0, false);
      check(cudaEventRecord(e2, 0), "record");
      check(cudaEventSynchronize(e2), "sync");
      check(cudaGetLastError(), "insert + range_query");
      if (r < a.warmup) continue;
      ins_ms += elapsed_ms(e0, e1);
      ops_ms += elapsed_ms(e3, e2);
    }
    cudaFree(dp);
    cudaFree(dcnt_t);
    ins_ms /= reps;
    ops_ms /= reps;
    // sums[f][4]: f = 0 second insert in place (ViB), f = 1 out of place (VoB)
    uint64_t sums[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, maxc = 0;
    const uint64_t cslot = 4 * c.length + 64;
    if (a.checksums) {
      pair_t* dq     = dev_alloc<pair_t>(c.ranges * cslot + tail);
      uint32_t* dcnt = dev_alloc<uint32_t>(c.ranges);
      for (int f = 0; f < 2; ++f) {
        vtree_t tree;
        tree.insert(dk, dv, (uint32_t)n, 0, true);
        const uint32_t S0 = tree.take_snapshot();
        tree.insert(di, div, (uint32_t)c.inserts, 0, f == 0);
        const uint32_t S1 = tree.take_snapshot();
        const uint32_t S[2] = {S0, S1};
        for (int v = 0; v < 2; ++v) {
          check(cudaMemset(dq, 0xFF, (c.ranges * cslot + tail) * sizeof(pair_t)), "memset");
          tree.range_query(dlo, dhi, dq, dcnt, (uint32_t)cslot, (uint32_t)c.ranges, S[v], 0, false);
          check(cudaDeviceSynchronize(), "range_query");
          check(cudaGetLastError(), "range_query");
          const auto cnt = host_copy(dcnt, c.ranges);
          uint64_t m = 0;
          range_checksums(cnt, dq, cslot, sums[f][2 * v], sums[f][2 * v + 1], m);
          maxc = std::max(maxc, m);
          if (!a.dump.empty()) {  // raw uint32 counts, one file per insert form and snapshot
            const std::string path = a.dump + (f ? "_vob_s" : "_vib_s") + std::to_string(v) + ".u32";
            FILE* fp = std::fopen(path.c_str(), "wb");
            if (fp) {
              std::fwrite(cnt.data(), sizeof(uint32_t), cnt.size(), fp);
              std::fclose(fp);
            }
          }
        }
      }
      cudaFree(dq);
      cudaFree(dcnt);
    }
    std::printf("%s{\"inserts\": %llu, \"ranges\": %llu, \"length\": %llu, \"slot\": %llu, \"insert_ms\": %.4f, "
                "\"ops_ms\": %.4f, \"insert_mops\": %.3f, \"ops_mops\": %.3f, \"check_slot\": %llu, "
                "\"max_count\": %llu, \"checksums\": [%llu, %llu, %llu, %llu], "
                "\"checksums_out_of_place\": [%llu, %llu, %llu, %llu]}",
                ci ? ", " : "", (unsigned long long)c.inserts, (unsigned long long)c.ranges,
                (unsigned long long)c.length, (unsigned long long)c.slot, ins_ms, ops_ms, n / (ins_ms * 1e3),
                (c.inserts + c.ranges) / (ops_ms * 1e3), (unsigned long long)cslot, (unsigned long long)maxc,
                (unsigned long long)sums[0][0], (unsigned long long)sums[0][1], (unsigned long long)sums[0][2],
                (unsigned long long)sums[0][3], (unsigned long long)sums[1][0], (unsigned long long)sums[1][1],
                (unsigned long long)sums[1][2], (unsigned long long)sums[1][3]);
    std::fflush(stdout);
    for (uint32_t* p : {di, div, dlo, dhi}) cudaFree(p);
  }
  std::printf("]}\n");
  cudaFree(dk);
  cudaFree(dv);
  return 0;
}

// One step of batches split per op kind, in the order the reference's plain form issues them.
struct step_t {
  uint32_t nb = 0;
  std::vector<uint64_t> batch_off;
  std::vector<uint32_t> type, key, arg, cap;
  // per batch: [begin, end) in the per-kind arrays, and the range slot size
  std::vector<uint64_t> f0, r0, i0, e0, p0;
  std::vector<uint32_t> slot;
  std::vector<uint32_t> fkeys, lo, hi, ikeys, ivals, ekeys;
  std::vector<uint64_t> fop, rop;  // op index of each find / range query
  uint64_t pairs = 0, num_ops = 0;
};

step_t split(void* gen, uint32_t batches, uint64_t stride) {
  step_t s;
  s.nb      = batches;
  uint64_t range_pairs = 0;
  s.num_ops = mvbt_wl_mix_generate(gen, batches, &range_pairs);
  const uint64_t n = s.num_ops;
  s.batch_off.resize(batches + 1);
  s.type.resize(n);
  s.key.resize(n);
  s.arg.resize(n);
  s.cap.resize(n);
  std::vector<uint64_t> out_off(n);
  mvbt_wl_mix_copy(gen, s.batch_off.data(), s.type.data(), s.key.data(), s.arg.data(), out_off.data(),
                   s.cap.data());
  for (uint32_t b = 0; b < batches; ++b) {
    s.f0.push_back(s.fkeys.size());
    s.r0.push_back(s.lo.size());
    s.i0.push_back(s.ikeys.size());
    s.e0.push_back(s.ekeys.size());
    s.p0.push_back(s.pairs);
    uint32_t slot = 8;
    for (uint64_t i = s.batch_off[b]; i < s.batch_off[b + 1]; ++i) {
      switch (s.type[i]) {
        case MVBT_OP_FIND: s.fkeys.push_back(s.key[i]); s.fop.push_back(i); break;
        case MVBT_OP_RANGE:
          s.lo.push_back(s.key[i]);
          s.hi.push_back(s.arg[i]);
          s.rop.push_back(i);
          slot = std::max(slot, s.cap[i]);
          break;
        case MVBT_OP_INSERT: s.ikeys.push_back(s.key[i]); s.ivals.push_back(s.arg[i]); break;
        default: s.ekeys.push_back(s.key[i]); break;
      }
    }
    s.slot.push_back(slot);
    s.pairs += (uint64_t)(s.lo.size() - s.r0.back()) * slot;
  }
  s.f0.push_back(s.fkeys.size());
  s.r0.push_back(s.lo.size());
  s.i0.push_back(s.ikeys.size());
  s.e0.push_back(s.ekeys.size());
  s.p0.push_back(s.pairs);
  s.pairs += 1024 * stride;  // tail: no query can write past it
  return s;
}

struct dstep_t {
  uint32_t *fk, *fr, *lo, *hi, *cnt, *ik, *iv, *ek;
  pair_t* pairs;
};

dstep_t upload(const step_t& s) {
  dstep_t d;
  d.fk    = dev_copy(s.fkeys);
  d.fr    = dev_alloc<uint32_t>(s.fkeys.size());
  d.lo    = dev_copy(s.lo);
  d.hi    = dev_copy(s.hi);
  d.cnt   = dev_alloc<uint32_t>(s.lo.size());
  d.ik    = dev_copy(s.ikeys);
  d.iv    = dev_copy(s.ivals);
  d.ek    = dev_copy(s.ekeys);
  d.pairs = dev_alloc<pair_t>(s.pairs);
  check(cudaMemset(d.pairs, 0xFF, s.pairs * sizeof(pair_t)), "memset");
  return d;
}
void release(dstep_t& d) {
  for (uint32_t* p : {d.fk, d.fr, d.lo, d.hi, d.cnt, d.ik, d.iv, d.ek}) cudaFree(p);
  cudaFree(d.pairs);
}

// The reference's plain form, one batch at a time, on the default stream.
void run_step(vtree_t& tree, const step_t& s, const dstep_t& d) {
  for (uint32_t b = 0; b < s.nb; ++b) {
    const uint32_t S  = tree.take_snapshot();
    const uint64_t nf = s.f0[b + 1] - s.f0[b], nr = s.r0[b + 1] - s.r0[b];
    const uint64_t ni = s.i0[b + 1] - s.i0[b], ne = s.e0[b + 1] - s.e0[b];
    if (nf) tree.find(d.fk + s.f0[b], d.fr + s.f0[b], (uint32_t)nf, S, 0, false);
    if (nr)
      tree.range_query(d.lo + s.r0[b], d.hi + s.r0[b], d.pairs + s.p0[b], d.cnt + s.r0[b], s.slot[b],
                       (uint32_t)nr, S, 0, false);
    if (ni) tree.insert(d.ik + s.i0[b], d.iv + s.i0[b], (uint32_t)ni, 0, true);
    if (ne) tree.erase(d.ek + s.e0[b], (uint32_t)ne, 0, false);
  }
}

void step_checksums(const step_t& s, const dstep_t& d, uint64_t out[3]) {
  auto fr    = host_copy(d.fr, s.fkeys.size());
  auto cnt   = host_copy(d.cnt, s.lo.size());
  auto pairs = host_copy(d.pairs, s.pairs);
  uint64_t f = 0, c = 0, p = 0;
  for (uint64_t x = 0; x < fr.size(); ++x) f += find_term(s.fop[x], fr[x]);
  for (uint32_t b = 0; b < s.nb; ++b) {
    for (uint64_t x = s.r0[b]; x < s.r0[b + 1]; ++x) {
      const uint64_t i = s.rop[x];
      c += count_term(i, cnt[x]);
      const uint64_t m    = std::min<uint64_t>(cnt[x], s.cap[i]);
      const pair_t* slot  = pairs.data() + s.p0[b] + (x - s.r0[b]) * s.slot[b];
      for (uint64_t j = 0; j < m; ++j) p += pair_term(i, j, slot[j].first, slot[j].second);
    }
  }
  out[0] = f;
  out[1] = c;
  out[2] = p;
}

int run_c4(const args_t& a) {
  mvbt_mix_params p;
  mvbt_wl_mix_default(&p);
  const uint64_t stride = a.stride ? a.stride : (0xFFFFFFFDull / 40000000ull);
  p.stride = (uint32_t)stride;
  if (a.median > 0) p.batch_median = a.median;
  if (a.batch_min) p.batch_min = a.batch_min;
  if (a.batch_max) p.batch_max = a.batch_max;

  std::vector<uint32_t> keys(a.initial), vals(a.initial);
  mvbt_wl_distinct_keys(a.seed, 0, a.initial, keys.data());
  mvbt_wl_values(keys.data(), a.initial, 0u, vals.data());
  void* gen = mvbt_wl_mix_create(&p, a.seed, a.initial);

  // Generate every step first (untimed). Reads allocate nothing; a write adds about one node on
  // average (a version copy per node and epoch, a split now and then).
  std::vector<step_t> steps;
  uint64_t writes = 0, max_step_writes = 0;
  for (uint32_t k = 0; k < a.warmup + a.steps; ++k) {
    steps.push_back(split(gen, a.batches, stride));
    const uint64_t w = steps.back().ikeys.size() + steps.back().ekeys.size();
    writes += w;
    max_step_writes = std::max(max_step_writes, w);
  }
  if (!pool_estimate_ok(a.initial, writes)) return 2;

  uint32_t *dk = dev_copy(keys), *dv = dev_copy(vals);
  vtree_t tree;
  tree.insert(dk, dv, (uint32_t)a.initial, 0, true);
  check(cudaDeviceSynchronize(), "initial insert");
  check(cudaGetLastError(), "initial insert");
  cudaFree(dk);
  cudaFree(dv);

  cudaEvent_t e0, e1;
  check(cudaEventCreate(&e0), "event");
  check(cudaEventCreate(&e1), "event");
  double timed_ms = 0;
  uint64_t timed_ops = 0;
  std::vector<std::vector<uint64_t>> sums;
  for (uint32_t k = 0; k < a.warmup + a.steps; ++k) {
    dstep_t d = upload(steps[k]);
    check(cudaDeviceSynchronize(), "upload");
    check(cudaEventRecord(e0, 0), "record");
    run_step(tree, steps[k], d);
    check(cudaEventRecord(e1, 0), "record");
    check(cudaEventSynchronize(e1), "step");
    check(cudaGetLastError(), "step kernels");
    if (k >= a.warmup) {
      timed_ms += elapsed_ms(e0, e1);
      timed_ops += steps[k].num_ops;
    }
    // the allocator's count (a blocking copy, outside the timed region): stop before the next
    // step could pass the unchecked bound (4 nodes per write of the largest step as margin)
    const uint64_t used = tree.get_num_tree_node();  // public (include/gpu_versioned_blink_tree.hpp:1096)
    if (used + 4 * max_step_writes + 4096 > kPoolNodes) {
      std::fprintf(stderr, "ref_driver: the pool holds %llu of %llu nodes after step %u\n",
                   (unsigned long long)used, (unsigned long long)kPoolNodes, k);
      return 2;
    }
    if (a.checksums) {
      uint64_t cs[3];
      step_checksums(steps[k], d, cs);
      sums.push_back({cs[0], cs[1], cs[2]});
    }
    release(d);
  }

  // final state: the whole key space as consecutive range queries at a final snapshot
  uint64_t final_c = 0, final_p = 0;
  if (a.final_chunks) {
    const uint32_t C      = a.final_chunks;
    const uint64_t live   = mvbt_wl_mix_present(gen);
    const uint64_t span   = (0xFFFFFFFFull - 1 + C - 1) / C;
    const uint32_t slot   = (uint32_t)std::min<uint64_t>((live / C) * 2 + 1024, 1u << 24);
    std::vector<uint32_t> lo(C), hi(C);
    for (uint32_t c = 0; c < C; ++c) {
      lo[c] = (uint32_t)(1 + c * span);
      hi[c] = (uint32_t)std::min<uint64_t>(1 + (uint64_t)(c + 1) * span, 0xFFFFFFFFull);
    }
    uint32_t *dlo = dev_copy(lo), *dhi = dev_copy(hi), *dcnt = dev_alloc<uint32_t>(C);
    const uint64_t np = (uint64_t)C * slot + live + 1;  // tail: a chunk returns at most `live` keys
    pair_t* dp = dev_alloc<pair_t>(np);
    const uint32_t S = tree.take_snapshot();
    tree.range_query(dlo, dhi, dp, dcnt, slot, C, S, 0, false);
    check(cudaDeviceSynchronize(), "final range");
    check(cudaGetLastError(), "final range");
    auto cnt   = host_copy(dcnt, C);
    auto pairs = host_copy(dp, np);
    for (uint32_t c = 0; c < C; ++c) {
      final_c += count_term(c, cnt[c]);
      const uint64_t m = std::min<uint64_t>(cnt[c], slot);
      for (uint64_t j = 0; j < m; ++j) final_p += pair_term(c, j, pairs[(uint64_t)c * slot + j].first,
                                                           pairs[(uint64_t)c * slot + j].second);
    }
    cudaFree(dlo);
    cudaFree(dhi);
    cudaFree(dcnt);
    cudaFree(dp);
  }
  mvbt_wl_mix_destroy(gen);

  std::printf("{\"mode\": \"c4\", \"initial\": %llu, \"batches\": %u, \"steps\": %u, \"warmup\": %u, "
              "\"seed\": %llu, \"stride\": %llu, \"ops_timed\": %llu, \"ms\": %.4f, \"mops\": %.3f, "
              "\"final\": [%llu, %llu], \"step_checksums\": [",
              (unsigned long long)a.initial, a.batches, a.steps, a.warmup, (unsigned long long)a.seed,
              (unsigned long long)stride, (unsigned long long)timed_ops, timed_ms,
              timed_ms > 0 ? timed_ops / (timed_ms * 1e3) : 0.0, (unsigned long long)final_c,
              (unsigned long long)final_p);
  for (size_t k = 0; k < sums.size(); ++k)
    std::printf("%s[%llu, %llu, %llu]", k ? ", " : "", (unsigned long long)sums[k][0],
                (unsigned long long)sums[k][1], (unsigned long long)sums[k][2]);
  std::printf("]}\n");
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  args_t a = parse(argc, argv);
  if (a.mode == "c1") return run_c1(a);
  if (a.mode == "c2") return run_c2(a);
  if (a.mode == "c3") return run_c3(a);
  if (a.mode == "c4") return run_c4(a);
  std::fprintf(stderr, "ref_driver: unknown mode %s\n", a.mode.c_str());
  return 2;
}
