// The library's own device sort and scans: a stable LSD radix sort of
// (key, value) pairs with 8-bit digits, and exclusive / inclusive prefix sums.
//
// The sort reads every key once for the digit histograms of all its passes,
// then runs one kernel per pass: each block takes the next tile of 1024 keys
// (tiles numbered in the order blocks start), ranks them stably among the
// tile's keys of the same digit (warp match in index order, per-warp digit
// counts across warps), publishes the tile's digit counts and adds its
// predecessors' counts by looking back through their published words
// (decoupled look-back), then scatters. A block only ever waits on blocks
// that started before it, and each wait is bounded: a look-back that gives
// up sets an error bit in the caller's error word instead of hanging.
// Stability keeps equal keys in input order, so the passes order by the whole
// key; the inputs are left untouched.
#pragma once
#include "common.cuh"

namespace cc {

struct NoValue {};  // the value type of a keys-only sort

class RadixSorter {
   public:
    // keys_out/vals_out[i] = the pairs of keys_in/vals_in ordered by the low
    // `bits` bits of the key (stable). K: uint16_t, uint32_t or uint64_t;
    // V: uint32_t or double. Returns the number of kernels launched.
    // `err` (device, may be null) receives `err_bit` if a look-back wait gave up.
    template <class K, class V>
    int sort_pairs(const K* keys_in, K* keys_out, const V* vals_in, V* vals_out, size_t n, int bits,
                   cudaStream_t s, unsigned int* err = nullptr, unsigned int err_bit = 1u);
    // The same for keys alone (K: uint64_t).
    template <class K>
    int sort_keys(const K* keys_in, K* keys_out, size_t n, int bits, cudaStream_t s, unsigned int* err = nullptr,
                  unsigned int err_bit = 1u);

   private:
    template <class K, class V>
    int sort_impl(const K* keys_in, K* keys_out, const V* vals_in, V* vals_out, size_t n, int bits, cudaStream_t s,
                  unsigned int* err, unsigned int err_bit);
    DBuf<uint32_t> hist_;
    DBuf<unsigned int> err_;
    DBuf<unsigned char> keys_tmp_, vals_tmp_;
};

// out[i] = sum of in[0..i) (exclusive) or in[0..i] (inclusive); T: uint32_t or
// double (summed in a fixed order: per thread, per tile, then over tiles).
// `scratch` holds the per-tile partials. Returns the kernels launched.
template <class T>
int exclusive_sum(const T* in, T* out, size_t n, DBuf<T>& scratch, cudaStream_t s);
template <class T>
int inclusive_sum(const T* in, T* out, size_t n, DBuf<T>& scratch, cudaStream_t s);

}  // namespace cc
