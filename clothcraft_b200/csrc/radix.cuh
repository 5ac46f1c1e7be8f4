// The library's own device sort and scans: a stable LSD radix sort of
// (key, value) pairs with 8-bit digits, and exclusive / inclusive prefix sums.
//
// Each radix pass is three kernels and needs no block to wait on another:
//   upsweep   - per tile of 2048 keys, the histogram of the pass's digit,
//               stored digit-major ([digit][tile]);
//   scan      - one block turns the histograms into exclusive global offsets
//               (digit-major order = where each tile's keys of a digit go);
//   downsweep - per tile, the stable rank of every key among the tile's keys
//               of the same digit (warp match + per-warp digit counts, in
//               index order), then the scatter to offset + rank.
// The sort is stable, so an LSD sequence of passes orders by the whole key
// and keeps equal keys in input order; the inputs are left untouched.
#pragma once
#include "common.cuh"

namespace cc {

class RadixSorter {
   public:
    // keys_out/vals_out[i] = the pairs of keys_in/vals_in ordered by the low
    // `bits` bits of the key (stable). K: uint16_t, uint32_t or uint64_t;
    // V: uint32_t or double. Returns the number of kernels launched.
    template <class K, class V>
    int sort_pairs(const K* keys_in, K* keys_out, const V* vals_in, V* vals_out, size_t n, int bits,
                   cudaStream_t s);

   private:
    DBuf<uint32_t> hist_;
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
