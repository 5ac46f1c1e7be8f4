// MLP inference on the 5th-generation tensor cores (sm_100a tcgen05).
//
// One CTA of 128 threads owns a 128-column TMEM allocation and walks tiles of
// 128 samples. Per layer: the samples' activations (FP16, K-major canonical
// core-matrix layout, no swizzle) and the layer's weights (FP16, same layout,
// staged once per CTA) sit in shared memory; one thread issues the
// `tcgen05.mma.cta_group::1.kind::f16` instructions (M = 128, N = 64 or 16,
// K = 16 each) accumulating in FP32 in TMEM, commits them to an mbarrier, and
// every thread reads its sample's row back with `tcgen05.ld.32x32b`, adds the
// bias, applies GELU and writes the next layer's FP16 operand. Every wait is
// bounded; a timeout sets an error word, skips the remaining work and still
// frees the TMEM.
#include <cuda_fp16.h>

#include "learned.cuh"

namespace cc {

namespace {
constexpr int kTcM = 128;       // samples per tile = TMEM lanes
constexpr int kK1 = 32;         // layer-1 K (24 features padded)
constexpr int kN4 = 16;         // output layer N (3 outputs padded; M = 128 needs N % 16 == 0)
constexpr int kTmemCols = 128;  // [0,64) hidden accumulator, [64,80) output accumulator
constexpr uint64_t kWaitNs = 500ull * 1000 * 1000;  // bound of every mbarrier wait (0.5 s)

// Byte offset of element (row r, k) in a K-major, no-swizzle operand whose
// rows hold `ktot` elements: 8x8 core matrices of 128 contiguous bytes,
// K-adjacent core matrices 128 B apart (LBO), 8-row groups ktot*16 B apart (SBO).
__host__ __device__ constexpr uint32_t cm_offset(uint32_t r, uint32_t k, uint32_t ktot) {
    return (r >> 3) * (ktot * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// FP16 weights in the operand layout: W1 [64 x 32], W2, W3 [64 x 64], W4 [16 x 64].
constexpr uint32_t kW1Bytes = kMlpHidden * kK1 * 2;
constexpr uint32_t kW2Bytes = kMlpHidden * kMlpHidden * 2;
constexpr uint32_t kW4Bytes = kN4 * kMlpHidden * 2;
constexpr uint32_t kOffW1h = 0;
constexpr uint32_t kOffW2h = kOffW1h + kW1Bytes;
constexpr uint32_t kOffW3h = kOffW2h + kW2Bytes;
constexpr uint32_t kOffW4h = kOffW3h + kW2Bytes;
constexpr uint32_t kWBytes = kOffW4h + kW4Bytes;  // 22,528
constexpr uint32_t kXBytes = kTcM * kK1 * 2;        // 8 KB
constexpr uint32_t kHBytes = kTcM * kMlpHidden * 2;  // 16 KB
// shared memory map (1 KB aligned pieces)
constexpr uint32_t kSmW = 0;
constexpr uint32_t kSmX = kSmW + kWBytes;
constexpr uint32_t kSmH = kSmX + kXBytes;
constexpr uint32_t kSmBar = kSmH + kHBytes;
constexpr uint32_t kSmTmem = kSmBar + 8;
constexpr uint32_t kSmBytes = kSmTmem + 8;
// Dynamic shared memory requested per CTA: at least 57 KB so that no more
// than 3 CTAs (384 TMEM columns of 512) share an SM.
constexpr uint32_t kSmRequest = kSmBytes > 58 * 1024 ? kSmBytes : 58 * 1024;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (tcgen05): start >> 4 in [0,14), LBO >> 4
// in [16,30), SBO >> 4 in [32,46), version 1 in [46,48), base offset 0,
// LBO mode 0, layout type 0 (no swizzle) in [61,64).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A and B F16
// (formats 0), both K-major, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t instr_desc(uint32_t m, uint32_t n) {
    return (1u << 4) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the mbarrier phase with the given parity for at most `ns`.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t ns) {
    uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > ns) return false;
    return true;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float gelu_t(float z) {  // tanh form, as the FP32 path
    const float c0 = 0.7978845608028654f, c1 = 0.044715f;
    return 0.5f * z * (1.0f + tanhf(c0 * (z + c1 * z * z * z)));
}

// Write 8 consecutive K values of row r as one 16-byte store.
__device__ __forceinline__ void store8(unsigned char* base, uint32_t r, uint32_t k0, uint32_t ktot, const float* v) {
    __half2 h[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2half2_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(base + cm_offset(r, k0, ktot)) = *reinterpret_cast<uint4*>(h);
}
}  // namespace

// FP16 weight image in the operand layout (zero padding), from FP32 params.
__global__ void k_pack_half(const float* __restrict__ P, unsigned char* __restrict__ out) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < kWBytes / 2; e += gridDim.x * blockDim.x) {
        uint32_t byte = e * 2;
        float v = 0.0f;
        // locate (matrix, row, k) of this half by inverting cm_offset per matrix
        uint32_t off, ktot, rows, woff, in;
        if (byte < kOffW2h) {
            off = byte - kOffW1h, ktot = kK1, rows = kMlpHidden, woff = kOffW1, in = kMlpIn;
        } else if (byte < kOffW3h) {
            off = byte - kOffW2h, ktot = kMlpHidden, rows = kMlpHidden, woff = kOffW2, in = kMlpHidden;
        } else if (byte < kOffW4h) {
            off = byte - kOffW3h, ktot = kMlpHidden, rows = kMlpHidden, woff = kOffW3, in = kMlpHidden;
        } else {
            off = byte - kOffW4h, ktot = kMlpHidden, rows = kMlpOut, woff = kOffW4, in = kMlpHidden;
        }
        uint32_t rg = off / (ktot * 16u), rem = off % (ktot * 16u);
        uint32_t kb = rem / 128u, rem2 = rem % 128u;
        uint32_t r = rg * 8u + rem2 / 16u, k = kb * 8u + (rem2 % 16u) / 2u;
        if (r < rows && k < in) v = P[woff + r * in + k];
        reinterpret_cast<__half*>(out)[e] = __float2half_rn(v);
    }
}

__global__ void __launch_bounds__(128, 1) k_mlp_forward_tc(const float* __restrict__ P,
                                                           const unsigned char* __restrict__ Wh,
                                                           const float* __restrict__ F, uint64_t n,
                                                           float* __restrict__ out, unsigned int* err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sW = sm + kSmW;
    unsigned char* sX = sm + kSmX;
    unsigned char* sH = sm + kSmH;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kSmTmem);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;

    for (uint32_t i = tid; i < kWBytes / 16; i += 128)
        reinterpret_cast<uint4*>(sW)[i] = reinterpret_cast<const uint4*>(Wh)[i];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (warp * 32u) << 16;  // this warp's TMEM lanes
    const uint32_t barrier = smem_u32(bar);
    const uint32_t aX = smem_u32(sX), aH = smem_u32(sH), aW = smem_u32(sW);
    const uint32_t id_hidden = instr_desc(kTcM, kMlpHidden), id_out = instr_desc(kTcM, kN4);
    uint32_t phase = 0;
    bool failed = false;

    // issue one layer (thread 0) and wait for it (all threads)
    auto run_layer = [&](uint32_t a_addr, uint32_t a_ktot, uint32_t b_addr, uint32_t d_col, uint32_t idesc) {
        if (tid == 0) {
            for (uint32_t ks = 0; ks < a_ktot / 16; ++ks) {
                uint64_t da = smem_desc(a_addr + ks * 256u, 128u, a_ktot * 16u);
                uint64_t db = smem_desc(b_addr + ks * 256u, 128u, a_ktot * 16u);
                mma_f16(tmem + d_col, da, db, idesc, ks > 0 ? 1u : 0u);
            }
            mma_commit(barrier);
        }
        if (!mbar_wait_bounded(barrier, phase, kWaitNs)) {
            failed = true;
            // the MMAs of this layer may still be in flight: give them one more
            // bounded wait before the TMEM is released. A layer is at most four
            // K=16 MMAs on a 128x64 tile (microseconds of tensor work), so a
            // commit that has not arrived after 0.6 s was never going to; the
            // columns are still freed because a CTA must not exit holding TMEM.
            mbar_wait_bounded(barrier, phase, kWaitNs / 5);
        }
        phase ^= 1u;
        fence_after();
    };

    const uint64_t tiles = (n + kTcM - 1) / kTcM;
    for (uint64_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const uint64_t s = tile * kTcM + tid;
        const bool live = s < n;
        // layer-1 operand: features as FP16, K padded to 32 with zeros
        {
            float v[kK1];
#pragma unroll
            for (int j = 0; j < kK1; ++j) v[j] = (live && j < kMlpIn) ? F[s * kMlpIn + j] : 0.0f;
#pragma unroll
            for (int k0 = 0; k0 < kK1; k0 += 8) store8(sX, tid, k0, kK1, v + k0);
        }
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        const uint32_t wofs[3] = {kOffW1h, kOffW2h, kOffW3h};
        const float* bias[3] = {P + kOffB1, P + kOffB2, P + kOffB3};
#pragma unroll
        for (int layer = 0; layer < 3; ++layer) {
            if (layer == 0) run_layer(aX, kK1, aW + wofs[0], 0, id_hidden);
            else run_layer(aH, kMlpHidden, aW + wofs[layer], 0, id_hidden);
            if (__syncthreads_or(failed ? 1 : 0)) {
                failed = true;
                break;
            }
            // epilogue: row `tid` of the accumulator -> bias, GELU -> FP16 operand
#pragma unroll
            for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
                float acc[16];
                tmem_ld16(tmem + lane_base + (uint32_t)c0, acc);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[i] = gelu_t(acc[i] + bias[layer][c0 + i]);
                store8(sH, tid, c0, kMlpHidden, acc);
                store8(sH, tid, c0 + 8, kMlpHidden, acc + 8);
            }
            fence_async_smem();
            fence_before();
            __syncthreads();
            fence_after();
        }
        if (failed) break;
        run_layer(aH, kMlpHidden, aW + kOffW4h, 64, id_out);
        if (__syncthreads_or(failed ? 1 : 0)) {
            failed = true;
            break;
        }
        {
            float acc[16];
            tmem_ld16(tmem + lane_base + 64u, acc);
            tmem_wait_ld();
            if (live) {
#pragma unroll
                for (int k = 0; k < kMlpOut; ++k) out[s * kMlpOut + k] = acc[k] + P[kOffB4 + k];
            }
        }
        fence_before();
        __syncthreads();
        fence_after();
    }
    if (failed && tid == 0) atomicOr(err, 1u);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols)
                     : "memory");
}

void Mlp::refresh_half(cudaStream_t st) {
    if (w16_valid_) return;
    w16_.reserve(kWBytes / 2);
    k_pack_half<<<(kWBytes / 2 + 255) / 256, 256, 0, st>>>(p_.ptr, reinterpret_cast<unsigned char*>(w16_.ptr));
    CC_CUDA(cudaGetLastError());
    w16_valid_ = true;
}

void Mlp::forward_tc(const float* features, uint64_t n, float* out, cudaStream_t st) {
    refresh_half(st);
    err_.reserve(1);
    CC_CUDA(cudaMemsetAsync(err_.ptr, 0, sizeof(unsigned int), st));
    allow_dynamic_smem(k_mlp_forward_tc, kSmRequest);
    uint64_t tiles = (n + kTcM - 1) / kTcM;
    unsigned grid = (unsigned)std::min<uint64_t>(tiles, 148ull * 2ull);
    k_mlp_forward_tc<<<grid, 128, kSmRequest, st>>>(p_.ptr, reinterpret_cast<const unsigned char*>(w16_.ptr), features,
                                                     n, out, err_.ptr);
    CC_CUDA(cudaGetLastError());
}

unsigned int Mlp::read_error(cudaStream_t st) {
    if (!err_.ptr) return 0;
    unsigned int e = 0;
    CC_CUDA(cudaMemcpyAsync(&e, err_.ptr, sizeof e, cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    return e;
}

}  // namespace cc
