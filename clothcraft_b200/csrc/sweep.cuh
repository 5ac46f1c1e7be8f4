// VBD colour-sweep data layout and kernel entry points.
#pragma once
#include "world.cuh"

namespace cc {

struct MatParams {  // per material, membrane part (src/energy.rs:10-29)
    double warp, weft, shear, c, delta;
};
struct MatParams32 {  // the same, rounded to FP32 for the FP32-assembly sweep
    float warp, weft, shear, c, delta;
};

// Packed incidence entry: type (2 bits) | slot (2 bits) | index (28 bits).
enum TermType : uint32_t { TERM_TRI = 0, TERM_HINGE = 1, TERM_STITCH = 2 };
__host__ __device__ inline uint32_t pack_term(uint32_t type, uint32_t slot, uint32_t idx) {
    return (type << 30) | (slot << 28) | idx;
}

struct GrabDev {
    int active;
    uint32_t v[3];
    double w[3];
    double target[3];
    double k;
};

struct SweepView {
    uint32_t n;                 // moving vertices
    double4* x;                 // [n_all] positions (moving part written)
    const double4* target;      // [n]
    const double* inertia;      // [n]
    const uint8_t* pinned;      // [n]
    const uint32_t* inc_off;    // [n+1] static incidence
    const uint2* inc_mid;       // [n] first hinge entry, first stitch entry (entries grouped by type)
    const uint32_t* inc;
    const int4* tri_v;          // v0, v1, v2, material
    const double4* tri_coef;    // w = ds0*c.x + ds1*c.y ; v = ds0*c.z + ds1*c.w (grain-rotated inv_dm)
    const double* tri_area;
    const MatParams* mats;
    const MatParams32* mats32;
    const uint4* hinge_v;
    const double* hinge_k;      // 0.5 * weight * (bend_warp aw^2 + bend_weft af^2)
    const uint32_t* st_off;
    const uint32_t* st_v;
    const double* st_w;
    const double* st_k;
    ContactsView contacts;
    double contact_r, contact_k;
    GrabDev grab;
    double* residual;           // [n] |g|^2 of the vertex's last solve
    unsigned int* clipped;      // counter
    const unsigned int* skip_at;  // sweeps of iterations >= *skip_at exit at once (null: never)
    uint32_t iteration;
    unsigned char* clipped_flag;  // [n]
    // Sweep-span stamps of the iteration (null: off): the first colour's
    // launch lowers *stamp_start to its blocks' start times and the last
    // colour's raises *stamp_end to their end times (%globaltimer, ns).
    unsigned long long* stamp_start;
    unsigned long long* stamp_end;
    uint32_t stamp_first, stamp_last;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// the block's start (first colour) and, after all its threads are done, its
// end (last colour); every thread of the block calls both
__device__ __forceinline__ void stamp_block_start(const SweepView& s) {
    if (s.stamp_start && s.stamp_first && threadIdx.x == 0) atomicMin(s.stamp_start, global_ns());
}
__device__ __forceinline__ void stamp_block_end(const SweepView& s) {
    if (s.stamp_end && s.stamp_last) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(s.stamp_end, global_ns());
    }
}

// Term counts of the step objective (k_term_energy items).
struct ObjectiveCounts {
    uint64_t triangles, hinges, stitches, contacts;
};
__host__ __device__ inline uint64_t objective_items(const ObjectiveCounts& c) {
    return c.triangles + c.hinges + c.stitches + c.contacts + 1;  // + grab; the n vertex items come first
}
constexpr int kSumBlocks = 296;  // 2 x 148 SMs

// Sweep variant (an int): lanes per vertex (bits 0-7) | cap (bits 8-15: resident
// 128-thread blocks per SM the registers are budgeted for) | kVariantPersistent
// (bit 16: a grid of at most the resident blocks, each block looping over the
// colour's vertices) | block-size code << 17 (0: 128 threads, 1: 64, 2: 256;
// the register budget per thread stays that of `cap` 128-thread blocks).
constexpr int kVariantPersistent = 1 << 16;
struct SweepVariant {
    int lanes, cap, block;
    bool persistent;
};
inline SweepVariant decode_variant(int v) {
    int code = (v >> 17) & 3;
    return {v & 0xff, (v >> 8) & 0xff, code == 1 ? 64 : (code == 2 ? 256 : 128), (v & kVariantPersistent) != 0};
}
// valid variants of the FP64 (fp32 = false) and FP32-assembly sweeps
bool sweep_variant_valid(int v, bool fp32);

// launch helpers (sweep.cu); grid_cap > 0 limits the grid (persistent variants)
void launch_sweep(const SweepView& s, const uint32_t* order, uint32_t count, int variant, cudaStream_t st,
                  unsigned grid_cap = 0);
// FP32 element assembly (sweep32.cu); lanes 4, 8, 16 or 32
void launch_sweep32(const SweepView& s, const uint32_t* order, uint32_t count, int variant, cudaStream_t st,
                    unsigned grid_cap = 0);
// resident blocks of a variant's kernel on the current device (all SMs)
unsigned sweep_resident_blocks(int variant);
unsigned sweep32_resident_blocks(int variant);
void launch_local_blocks(const SweepView& s, double* energy, double* grad, double* hess, cudaStream_t st);
// out[v] = |dE/dx_v|^2 over moving vertices (variant as launch_sweep); with
// `project`, the KKT residual of the OGC-ball constraints (sweep.cu)
void launch_grad_sq(const SweepView& s, double* out, const unsigned* skip_at, uint32_t iteration, int variant,
                    bool project, cudaStream_t st);
// out[i] = energy of objective item i; items = s.n + objective_items(c)
void launch_term_energy(const SweepView& s, const ObjectiveCounts& c, double* out, cudaStream_t st);
void launch_sum_partial(const double* v, uint64_t n, double* partial, const unsigned* skip_at, uint32_t iteration,
                        cudaStream_t st);
// Second pass of the deterministic sum, run by one block of 256 threads: the
// kSumBlocks partials added in a fixed order (valid in every thread).
__device__ __forceinline__ double block_sum_partials(const double* partial) {
    __shared__ double sh[256];
    double a = 0.0;
    for (int i = threadIdx.x; i < kSumBlocks; i += 256) a += partial[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

}  // namespace cc
