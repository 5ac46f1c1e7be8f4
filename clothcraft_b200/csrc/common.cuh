// Shared host/device helpers of the B200 ClothCraft library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/clothcraft.h"

namespace cc {

// ------------------------------------------------------------------ errors
struct Failure {
    int code;
    std::string message;
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof buf, "CUDA failure in %s: %s", what, cudaGetErrorString(e));
        throw Failure{CC_ERR_CUDA, buf};
    }
}
#define CC_CUDA(call) ::cc::cuda_check((call), #call)

// Records the message returned by cc_global_last_error (defined with the C ABI).
int record_global_error(int code, const std::string& message);

// Device error word bits (set with atomicOr; read by the host once per phase).
enum DeviceError : uint32_t {
    DERR_NONFINITE_STATE = 1u << 0,
    DERR_DEGENERATE_FACE = 1u << 1,
    DERR_FIXED_MOVED = 1u << 2,
    DERR_STACK_OVERFLOW = 1u << 3,
    DERR_NONFINITE_RESULT = 1u << 4,
    DERR_TRUST_REGION = 1u << 5,
    DERR_COLOR_LIMIT = 1u << 6,
    DERR_INTERSECTION = 1u << 7,
    DERR_SORT_WAIT = 1u << 8,  // a radix-sort look-back wait gave up
};

// ------------------------------------------------------------ device buffer
template <class T>
struct DBuf {
    T* ptr = nullptr;
    size_t cap = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
    // Ensure room for n elements; contents are not preserved on growth.
    // Growth is geometric (x1.5) so that buffers sized by data-dependent
    // counts (contacts, pairs) reallocate - and synchronise - rarely.
    void reserve(size_t n) {
        if (n <= cap) return;
        size_t grown = cap + cap / 2;
        if (cap && grown > n) n = grown;
        release();
        size_t bytes = (n ? n : 1) * sizeof(T);
        CC_CUDA(cudaMalloc(&ptr, bytes));
        cap = n;
    }
    void upload(const T* src, size_t n, cudaStream_t s) {
        reserve(n);
        if (n) CC_CUDA(cudaMemcpyAsync(ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
    void zero(size_t n, cudaStream_t s) {
        if (n) CC_CUDA(cudaMemsetAsync(ptr, 0, n * sizeof(T), s));
    }
};

// Pinned host scalar block used for small device->host reads.
template <class T>
struct Pinned {
    T* ptr = nullptr;
    size_t cap = 0;
    Pinned() = default;
    Pinned(const Pinned&) = delete;
    Pinned& operator=(const Pinned&) = delete;
    ~Pinned() {
        if (ptr) cudaFreeHost(ptr);
    }
    void reserve(size_t n) {
        if (n <= cap) return;
        if (ptr) cudaFreeHost(ptr);
        CC_CUDA(cudaMallocHost(&ptr, (n ? n : 1) * sizeof(T)));
        cap = n;
    }
};

// --------------------------------------------------------------- double3
struct d3 {
    double x, y, z;
};
__host__ __device__ inline d3 mk(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 operator-(d3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ inline d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline d3 operator/(d3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline d3 cross(d3 a, d3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__host__ __device__ inline double len2(d3 a) { return dot(a, a); }
__device__ inline double len(d3 a) { return sqrt(dot(a, a)); }
__device__ inline bool isfin(d3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// Positions are stored as double4 (32-byte aligned, w unused) so a vertex is
// one aligned 32-byte sector.
__device__ inline d3 ld3(const double4* p, uint32_t i) {
    double4 q = p[i];
    return {q.x, q.y, q.z};
}
__device__ inline void st3(double4* p, uint32_t i, d3 v) { p[i] = make_double4(v.x, v.y, v.z, 0.0); }

// Monotone mapping of non-negative doubles to uint64 (for atomicMin).
__device__ inline unsigned long long dbits(double d) { return (unsigned long long)__double_as_longlong(d); }
__device__ inline double bitsd(unsigned long long b) { return __longlong_as_double((long long)b); }
// Order-preserving key for any finite double (used for scene bounds).
__host__ __device__ inline unsigned long long order_key(double d) {
    unsigned long long b;
    std::memcpy(&b, &d, 8);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double from_order_key(unsigned long long k) {
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}

// CUDA keeps a kernel's dynamic shared-memory limit per device, so the limit
// is raised before every launch that needs more than 48 KB (a host call of a
// few microseconds) instead of once per process: a process that switches
// devices with cc_set_device then finds it raised on each device it uses.
template <class K>
inline void allow_dynamic_smem(K* kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        CC_CUDA(cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// The same for a kernel launched many times per step: `raised` records, one
// bit per device (ids below 64), where the limit is already raised, so the
// attribute is set once per device instead of before every launch.
template <class K>
inline void allow_dynamic_smem_once(K* kernel, size_t bytes, std::atomic<uint64_t>& raised) {
    int dev = 0;
    CC_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = dev >= 0 && dev < 64 ? (1ull << dev) : 0ull;
    if (bit && (raised.load(std::memory_order_acquire) & bit)) return;
    allow_dynamic_smem(kernel, bytes);
    if (bit) raised.fetch_or(bit, std::memory_order_acq_rel);
}

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;  // grid-stride loops cover the rest
    return (int)g;
}

}  // namespace cc
