// Stable LSD radix sort and prefix sums (see radix.cuh).
#include "radix.cuh"

namespace cc {

namespace {

constexpr int kBlock = 256;              // threads per tile
constexpr int kItems = 8;                // keys per thread
constexpr int kTile = kBlock * kItems;   // 2048 keys per tile
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

// ------------------------------------------------------------ radix sort
template <class K>
__global__ void __launch_bounds__(kBlock) k_radix_upsweep(const K* __restrict__ keys, size_t n, int shift,
                                                          uint32_t mask, uint32_t tiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kTile;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        size_t i = base + (size_t)j * kBlock + threadIdx.x;
        if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & mask], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
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

template <class K, class V>
__global__ void __launch_bounds__(kBlock) k_radix_downsweep(const K* __restrict__ kin, K* __restrict__ kout,
                                                            const V* __restrict__ vin, V* __restrict__ vout, size_t n,
                                                            int shift, uint32_t mask, uint32_t tiles,
                                                            const uint32_t* __restrict__ offs) {
    __shared__ uint32_t cnt[kBlock / 32][kRadix];  // this row's per-warp digit counts
    __shared__ uint32_t run[kRadix];               // keys of each digit in earlier rows
    __shared__ uint32_t goff[kRadix];              // the tile's global start of each digit
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned lt = (1u << lane) - 1u;
    run[tid] = 0;
    goff[tid] = offs[(size_t)tid * tiles + blockIdx.x];
#pragma unroll
    for (int w = 0; w < kBlock / 32; ++w) cnt[w][tid] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kTile;
    for (int j = 0; j < kItems; ++j) {
        const size_t i = base + (size_t)j * kBlock + tid;
        const bool live = i < n;
        K key = live ? kin[i] : K(0);
        uint32_t dig = live ? ((uint32_t)(key >> shift) & mask) : (uint32_t)kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, dig);
        uint32_t wrank = __popc(peers & lt);
        if (live && wrank == 0) cnt[warp][dig] = __popc(peers);
        __syncthreads();
        uint32_t pos = 0;
        if (live) {
            uint32_t before = run[dig];
            for (uint32_t w = 0; w < warp; ++w) before += cnt[w][dig];
            pos = goff[dig] + before + wrank;
        }
        __syncthreads();
        {
            uint32_t add = 0;
#pragma unroll
            for (int w = 0; w < kBlock / 32; ++w) {
                add += cnt[w][tid];
                cnt[w][tid] = 0;
            }
            run[tid] += add;
        }
        __syncthreads();
        if (live) {
            kout[pos] = key;
            vout[pos] = vin[i];
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
int RadixSorter::sort_pairs(const K* keys_in, K* keys_out, const V* vals_in, V* vals_out, size_t n, int bits,
                            cudaStream_t s) {
    if (n == 0) return 0;
    if (bits <= 0) {
        CC_CUDA(cudaMemcpyAsync(keys_out, keys_in, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        CC_CUDA(cudaMemcpyAsync(vals_out, vals_in, n * sizeof(V), cudaMemcpyDeviceToDevice, s));
        return 0;
    }
    if (n > 0xffffffffull) throw Failure{CC_ERR_INVALID_ARGUMENT, "radix sort: more than 2^32 keys"};
    const int passes = (bits + 7) / 8;
    const uint32_t tiles = (uint32_t)((n + kTile - 1) / kTile);
    hist_.reserve((size_t)kRadix * tiles);
    K* ktmp = nullptr;
    V* vtmp = nullptr;
    if (passes > 1) {
        keys_tmp_.reserve(n * sizeof(K));
        vals_tmp_.reserve(n * sizeof(V));
        ktmp = reinterpret_cast<K*>(keys_tmp_.ptr);
        vtmp = reinterpret_cast<V*>(vals_tmp_.ptr);
    }
    const K* ksrc = keys_in;
    const V* vsrc = vals_in;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        const int width = bits - shift < 8 ? bits - shift : 8;
        const uint32_t mask = (1u << width) - 1u;
        const bool to_out = ((passes - 1 - p) % 2) == 0;  // the last pass lands in the output
        K* kd = to_out ? keys_out : ktmp;
        V* vd = to_out ? vals_out : vtmp;
        k_radix_upsweep<K><<<tiles, kBlock, 0, s>>>(ksrc, n, shift, mask, tiles, hist_.ptr);
        k_scan_single<uint32_t><<<1, kScanBlock, 0, s>>>(hist_.ptr, (size_t)kRadix * tiles, 0u);
        k_radix_downsweep<K, V><<<tiles, kBlock, 0, s>>>(ksrc, kd, vsrc, vd, n, shift, mask, tiles, hist_.ptr);
        ksrc = kd;
        vsrc = vd;
    }
    CC_CUDA(cudaGetLastError());
    return 3 * passes;
}

template int RadixSorter::sort_pairs<uint16_t, uint32_t>(const uint16_t*, uint16_t*, const uint32_t*, uint32_t*,
                                                          size_t, int, cudaStream_t);
template int RadixSorter::sort_pairs<unsigned long long, uint32_t>(const unsigned long long*, unsigned long long*,
                                                                    const uint32_t*, uint32_t*, size_t, int,
                                                                    cudaStream_t);
template int RadixSorter::sort_pairs<unsigned long long, double>(const unsigned long long*, unsigned long long*,
                                                                  const double*, double*, size_t, int, cudaStream_t);

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
