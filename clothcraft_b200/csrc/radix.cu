// Stable LSD radix sort and prefix sums (see radix.cuh).
#include <algorithm>
#include <type_traits>

#include "radix.cuh"

namespace cc {

namespace {

constexpr int kBlock = 256;              // threads per tile
constexpr int kItems = 4;                // keys per thread
constexpr int kTile = kBlock * kItems;   // 1024 keys per tile
constexpr int kRadix = 256;              // 8-bit digits
constexpr int kScanBlock = 1024;

// Exclusive scan of one value per thread over a block of NT threads (NT a
// multiple of 32, at most 1024); returns the thread's exclusive prefix and
// the block total in `total`.
template <class T, int NT>
__device__ __forceinline__ T block_exclusive_scan(T v, T& total) {
    __shared__ T warp_tot[NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < NT / 32 ? warp_tot[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        if (lane < NT / 32) warp_tot[lane] = wi - w;  // exclusive warp prefixes
    }
    __syncthreads();
    T prefix = warp_tot[warp] + inc - v;
    __shared__ T tot_sh;
    if (threadIdx.x == NT - 1) tot_sh = prefix + v;
    __syncthreads();
    total = tot_sh;
    __syncthreads();
    return prefix;
}

// In-place exclusive scan of a[0..total) by one block: each thread sums a
// contiguous chunk, the chunk sums are scanned, each chunk is rewritten.
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_single(T* a, size_t total, T base) {
    size_t per = (total + kScanBlock - 1) / kScanBlock;
    size_t b = threadIdx.x * per;
    size_t e = b + per < total ? b + per : total;
    T s = T(0);
    for (size_t i = b; i < e; ++i) s += a[i];
    T tot;
    T run = block_exclusive_scan<T, kScanBlock>(s, tot) + base;
    for (size_t i = b; i < e; ++i) {
        T v = a[i];
        a[i] = run;
        run += v;
    }
}

// ------------------------------------------------------------ radix sort
// One-pass-per-digit LSD sort (the decoupled look-back scheme of Merrill and
// Garland's "Single-pass Parallel Prefix Scan with Decoupled Look-back" and
// Adinets and Merrill's "Onesweep"): the global digit counts of every pass
// come from one histogram kernel; each pass then ranks a tile's keys locally,
// publishes the tile's digit counts, adds up its predecessors' counts by
// looking back through their published words, and scatters.

constexpr int kMaxPasses = 8;
constexpr uint32_t kFlagAgg = 1u << 30;   // status word: this tile's own count
constexpr uint32_t kFlagInc = 2u << 30;   // status word: count of tiles 0..this
constexpr uint32_t kCountMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;  // polls before a look-back gives up

template <class K>
__global__ void __launch_bounds__(kBlock) k_onesweep_hist(const K* __restrict__ keys, size_t n, int passes, int bits,
                                                          uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kMaxPasses * kRadix];
    for (int i = threadIdx.x; i < passes * kRadix; i += kBlock) h[i] = 0;
    __syncthreads();
    for (size_t i = blockIdx.x * (size_t)kBlock + threadIdx.x; i < n; i += (size_t)gridDim.x * kBlock) {
        K k = keys[i];
        for (int p = 0; p < passes; ++p) {
            int shift = 8 * p;
            int width = bits - shift < 8 ? bits - shift : 8;
            atomicAdd(&h[p * kRadix + ((uint32_t)(k >> shift) & ((1u << width) - 1u))], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += kBlock)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// hist[p][d] -> exclusive prefix over d (one block of kRadix threads)
__global__ void __launch_bounds__(kRadix) k_onesweep_offsets(uint32_t* hist, int passes) {
    for (int p = 0; p < passes; ++p) {
        uint32_t v = hist[p * kRadix + threadIdx.x];
        uint32_t tot;
        uint32_t ex = block_exclusive_scan<uint32_t, kRadix>(v, tot);
        hist[p * kRadix + threadIdx.x] = ex;
    }
}

template <class K, class V>
__global__ void __launch_bounds__(kBlock) k_onesweep_pass(const K* __restrict__ kin, K* __restrict__ kout,
                                                          const V* __restrict__ vin, V* __restrict__ vout, size_t n,
                                                          int shift, uint32_t mask,
                                                          const uint32_t* __restrict__ digit_off,
                                                          uint32_t* status, uint32_t* tile_counter,
                                                          unsigned int* err, unsigned int err_bit) {
    __shared__ uint32_t cnt[kBlock / 32][kRadix];  // this row's per-warp digit counts
    __shared__ uint32_t run[kRadix];               // keys of each digit in earlier rows
    __shared__ uint32_t goff[kRadix];              // global start of this tile's keys of each digit
    __shared__ uint32_t tile_sh;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned lt = (1u << lane) - 1u;
    if (tid == 0) tile_sh = atomicAdd(tile_counter, 1u);  // tiles in the order blocks start
    run[tid] = 0;
#pragma unroll
    for (int w = 0; w < kBlock / 32; ++w) cnt[w][tid] = 0;
    __syncthreads();
    const uint32_t tile = tile_sh;
    const size_t base = (size_t)tile * kTile;
    K key[kItems];
    uint32_t dig[kItems], rank[kItems];
    // local stable ranks, row by row (index order: row, warp, lane)
    for (int j = 0; j < kItems; ++j) {
        const size_t i = base + (size_t)j * kBlock + tid;
        const bool live = i < n;
        key[j] = live ? kin[i] : K(0);
        dig[j] = live ? ((uint32_t)(key[j] >> shift) & mask) : (uint32_t)kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, dig[j]);
        uint32_t wrank = __popc(peers & lt);
        if (live && wrank == 0) cnt[warp][dig[j]] = __popc(peers);
        __syncthreads();
        rank[j] = 0;
        if (live) {
            uint32_t before = run[dig[j]];
            for (uint32_t w = 0; w < warp; ++w) before += cnt[w][dig[j]];
            rank[j] = before + wrank;
        }
        __syncthreads();
        uint32_t add = 0;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) {
            add += cnt[w][tid];
            cnt[w][tid] = 0;
        }
        run[tid] += add;
        __syncthreads();
    }
    // publish this tile's count of digit `tid`, then look back for the
    // predecessors' (bounded: a predecessor that never publishes ends the
    // wait with an error bit instead of a hang)
    const uint32_t own = run[tid];
    volatile uint32_t* st = status;
    st[(size_t)tile * kRadix + tid] = (tile == 0 ? kFlagInc : kFlagAgg) | own;
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t t = (int64_t)tile - 1;
        uint32_t polls = 0;
        while (t >= 0) {
            uint32_t w = st[(size_t)t * kRadix + tid];
            uint32_t flag = w & ~kCountMask;
            if (flag == 0) {
                if (++polls > kSpinLimit) {
                    atomicOr(err, err_bit);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            excl += w & kCountMask;
            if (flag == kFlagInc) break;
            --t;
        }
        __threadfence();
        st[(size_t)tile * kRadix + tid] = kFlagInc | (excl + own);
    }
    goff[tid] = digit_off[tid] + excl;
    __syncthreads();
    for (int j = 0; j < kItems; ++j) {
        const size_t i = base + (size_t)j * kBlock + tid;
        if (i < n) {
            uint32_t pos = goff[dig[j]] + rank[j];
            kout[pos] = key[j];
            if constexpr (!std::is_same<V, NoValue>::value) vout[pos] = vin[i];
        }
    }
}

// ------------------------------------------------------------ prefix sums
template <class T>
__global__ void __launch_bounds__(kBlock) k_tile_reduce(const T* __restrict__ in, size_t n, T* __restrict__ partial) {
    const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kItems;
    T s = T(0);
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        if (base + j < n) s += in[base + j];
    T tot;
    block_exclusive_scan<T, kBlock>(s, tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

template <class T, bool INCLUSIVE>
__global__ void __launch_bounds__(kBlock) k_tile_scan(const T* __restrict__ in, T* __restrict__ out, size_t n,
                                                      const T* __restrict__ prefix) {
    const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kItems;
    T v[kItems];
    T s = T(0);
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        v[j] = base + j < n ? in[base + j] : T(0);
        s += v[j];
    }
    T tot;
    T run = block_exclusive_scan<T, kBlock>(s, tot) + (prefix ? prefix[blockIdx.x] : T(0));
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        if (INCLUSIVE) run += v[j];
        if (base + j < n) out[base + j] = run;
        if (!INCLUSIVE) run += v[j];
    }
}

template <class T, bool INCLUSIVE>
int prefix_sum(const T* in, T* out, size_t n, DBuf<T>& scratch, cudaStream_t s) {
    if (n == 0) return 0;
    const size_t tiles = (n + kTile - 1) / kTile;
    if (tiles == 1) {
        k_tile_scan<T, INCLUSIVE><<<1, kBlock, 0, s>>>(in, out, n, nullptr);
        CC_CUDA(cudaGetLastError());
        return 1;
    }
    scratch.reserve(tiles);
    k_tile_reduce<T><<<(unsigned)tiles, kBlock, 0, s>>>(in, n, scratch.ptr);
    k_scan_single<T><<<1, kScanBlock, 0, s>>>(scratch.ptr, tiles, T(0));
    k_tile_scan<T, INCLUSIVE><<<(unsigned)tiles, kBlock, 0, s>>>(in, out, n, scratch.ptr);
    CC_CUDA(cudaGetLastError());
    return 3;
}

}  // namespace

template <class K, class V>
int RadixSorter::sort_impl(const K* keys_in, K* keys_out, const V* vals_in, V* vals_out, size_t n, int bits,
                           cudaStream_t s, unsigned int* err, unsigned int err_bit) {
    constexpr bool kVals = !std::is_same<V, NoValue>::value;
    if (n == 0) return 0;
    if (bits <= 0) {
        CC_CUDA(cudaMemcpyAsync(keys_out, keys_in, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        if constexpr (kVals) CC_CUDA(cudaMemcpyAsync(vals_out, vals_in, n * sizeof(V), cudaMemcpyDeviceToDevice, s));
        return 0;
    }
    if (n > kCountMask) throw Failure{CC_ERR_INVALID_ARGUMENT, "radix sort: more than 2^30 keys"};
    if (bits > 8 * kMaxPasses) throw Failure{CC_ERR_INVALID_ARGUMENT, "radix sort: more than 64 key bits"};
    const int passes = (bits + 7) / 8;
    const uint32_t tiles = (uint32_t)((n + kTile - 1) / kTile);
    // per pass: kRadix digit offsets, a tile counter, tiles x kRadix status words
    const size_t per_pass = (size_t)kRadix + 1 + (size_t)tiles * kRadix;
    hist_.reserve((size_t)passes * per_pass + 1);
    err_.reserve(1);
    uint32_t* offs = hist_.ptr;                          // [passes][kRadix]
    uint32_t* counters = hist_.ptr + passes * kRadix;    // [passes]
    uint32_t* status = counters + passes;                // [passes][tiles][kRadix]
    CC_CUDA(cudaMemsetAsync(hist_.ptr, 0, ((size_t)passes * per_pass) * sizeof(uint32_t), s));
    unsigned int* errp = err ? err : err_.ptr;
    K* ktmp = nullptr;
    V* vtmp = nullptr;
    if (passes > 1) {
        keys_tmp_.reserve(n * sizeof(K));
        ktmp = reinterpret_cast<K*>(keys_tmp_.ptr);
        if constexpr (kVals) {
            vals_tmp_.reserve(n * sizeof(V));
            vtmp = reinterpret_cast<V*>(vals_tmp_.ptr);
        }
    }
    unsigned hist_grid = (unsigned)std::min<size_t>(tiles, 148 * 4);
    k_onesweep_hist<K><<<hist_grid, kBlock, 0, s>>>(keys_in, n, passes, bits, offs);
    k_onesweep_offsets<<<1, kRadix, 0, s>>>(offs, passes);
    const K* ksrc = keys_in;
    const V* vsrc = vals_in;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        const int width = bits - shift < 8 ? bits - shift : 8;
        const uint32_t mask = (1u << width) - 1u;
        const bool to_out = ((passes - 1 - p) % 2) == 0;  // the last pass lands in the output
        K* kd = to_out ? keys_out : ktmp;
        V* vd = to_out ? vals_out : vtmp;
        k_onesweep_pass<K, V><<<tiles, kBlock, 0, s>>>(ksrc, kd, vsrc, vd, n, shift, mask, offs + p * kRadix,
                                                       status + (size_t)p * tiles * kRadix, counters + p, errp,
                                                       err_bit);
        ksrc = kd;
        vsrc = vd;
    }
    CC_CUDA(cudaGetLastError());
    return 2 + passes;
}

template <class K, class V>
int RadixSorter::sort_pairs(const K* keys_in, K* keys_out, const V* vals_in, V* vals_out, size_t n, int bits,
                            cudaStream_t s, unsigned int* err, unsigned int err_bit) {
    return sort_impl<K, V>(keys_in, keys_out, vals_in, vals_out, n, bits, s, err, err_bit);
}

template <class K>
int RadixSorter::sort_keys(const K* keys_in, K* keys_out, size_t n, int bits, cudaStream_t s, unsigned int* err,
                           unsigned int err_bit) {
    return sort_impl<K, NoValue>(keys_in, keys_out, nullptr, nullptr, n, bits, s, err, err_bit);
}

template int RadixSorter::sort_pairs<uint16_t, uint32_t>(const uint16_t*, uint16_t*, const uint32_t*, uint32_t*,
                                                          size_t, int, cudaStream_t, unsigned int*, unsigned int);
template int RadixSorter::sort_pairs<unsigned long long, uint32_t>(const unsigned long long*, unsigned long long*,
                                                                    const uint32_t*, uint32_t*, size_t, int,
                                                                    cudaStream_t, unsigned int*, unsigned int);
template int RadixSorter::sort_pairs<unsigned long long, double>(const unsigned long long*, unsigned long long*,
                                                                  const double*, double*, size_t, int, cudaStream_t,
                                                                  unsigned int*, unsigned int);
template int RadixSorter::sort_keys<unsigned long long>(const unsigned long long*, unsigned long long*, size_t, int,
                                                         cudaStream_t, unsigned int*, unsigned int);

template <class T>
int exclusive_sum(const T* in, T* out, size_t n, DBuf<T>& scratch, cudaStream_t s) {
    return prefix_sum<T, false>(in, out, n, scratch, s);
}
template <class T>
int inclusive_sum(const T* in, T* out, size_t n, DBuf<T>& scratch, cudaStream_t s) {
    return prefix_sum<T, true>(in, out, n, scratch, s);
}
template int exclusive_sum<uint32_t>(const uint32_t*, uint32_t*, size_t, DBuf<uint32_t>&, cudaStream_t);
template int inclusive_sum<double>(const double*, double*, size_t, DBuf<double>&, cudaStream_t);

}  // namespace cc
