// Internal interface of the sort stage of the sorted batch front-end (mvbt_sort.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mvbt_sort {

// Scratch words (uint32) sort_pairs needs for n keys (digit counts and scan sums).
uint64_t scratch_words(uint32_t n);

// Stable sort of keys[0, n) by their bits [low_bit, 32) (low_bit in {0, 8, 16, 24}: 0 = a full
// sort, larger = a bucketing by the top bits that keeps input order inside a bucket). Writes the
// keys in order to k_out and each one's input position to v_out; k_tmp / v_tmp hold n words each
// between passes, scratch holds scratch_words(n). Stream-ordered; returns 0, or non-zero if a
// launch failed or low_bit is invalid.
int sort_pairs(const uint32_t* keys, uint32_t n, int low_bit, uint32_t* k_out, uint32_t* v_out, uint32_t* k_tmp,
               uint32_t* v_tmp, uint32_t* scratch, cudaStream_t s);

// Exclusive prefix sum of a[0, n) in place (uint32, total < 2^32); sums holds
// scan_scratch_words(n). Stream-ordered; returns 0, or non-zero if a launch failed.
uint64_t scan_scratch_words(uint64_t n);
int exclusive_scan(uint32_t* a, uint64_t n, uint32_t* sums, cudaStream_t s);

}  // namespace mvbt_sort
