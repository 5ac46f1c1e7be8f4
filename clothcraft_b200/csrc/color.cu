// Graph colouring on the device (replaces coloring::colors,
// src/vbd/coloring.rs:5-43, which the reference runs serially on the CPU
// after every detection).
//
// The reference visits vertices 0..n in order and gives each the smallest
// colour not used by an already-coloured neighbour (material graph, contact
// co-vertices, grab). Already-coloured means lower index, so the result is
// the unique solution of  c(v) = mex { c(u) : u ~ v, u < v }.  A plain
// parallel fixed-point iteration of that system needs as many sweeps as the
// longest descending chain, and contact edges between folded layers make
// chains of length ~n; k_color_chunked below bounds the work by walking
// index-ordered chunks instead.

#include "color.cuh"

namespace cc {

__device__ __forceinline__ void mark(unsigned long long& mask, uint32_t c, bool& high) {
    if (c < 64) mask |= 1ull << c;
    else high = true;
}

// Greedy rule for one vertex: smallest colour not used by a lower-index
// neighbour (material graph, contact co-vertices, grab).
__device__ __forceinline__ uint32_t greedy_color(const ColorView& g, const uint16_t* cin, uint32_t v) {
    unsigned long long mask = 0;
    bool high = false;
    for (uint32_t k = g.lo_off[v]; k < g.lo_off[v + 1]; ++k) mark(mask, cin[g.lo[k]], high);
    for (uint32_t k = g.contacts.inc_off[v]; k < g.contacts.inc_off[v + 1]; ++k) {
        uint32_t c = g.contacts.inc[k];
        uint32_t kind = g.contacts.kind[c];
        uint4 cv = g.contacts.verts[c];
        uint32_t ids[4] = {cv.x, cv.y, cv.z, cv.w};
        uint32_t cnt = kind == 0 ? 2u : (kind == 1 ? 3u : 4u);
        for (uint32_t j = 0; j < cnt; ++j)
            if (ids[j] < v) mark(mask, cin[ids[j]], high);
    }
    bool in_grab = g.grab_active && (g.grab_v[0] == v || g.grab_v[1] == v || g.grab_v[2] == v);
    if (in_grab)
        for (int j = 0; j < 3; ++j)
            if (g.grab_v[j] < v) mark(mask, cin[g.grab_v[j]], high);
    if (~mask != 0ull) return (uint32_t)__ffsll((long long)~mask) - 1;
    for (uint32_t col = 64;; ++col) {  // more than 64 colours around v: linear search
        bool used = false;
        for (uint32_t k = g.lo_off[v]; k < g.lo_off[v + 1] && !used; ++k) used = cin[g.lo[k]] == col;
        for (uint32_t k = g.contacts.inc_off[v]; k < g.contacts.inc_off[v + 1] && !used; ++k) {
            uint32_t c = g.contacts.inc[k];
            uint32_t kind = g.contacts.kind[c];
            uint4 cv = g.contacts.verts[c];
            uint32_t ids[4] = {cv.x, cv.y, cv.z, cv.w};
            uint32_t cnt = kind == 0 ? 2u : (kind == 1 ? 3u : 4u);
            for (uint32_t j = 0; j < cnt; ++j) used = used || (ids[j] < v && cin[ids[j]] == col);
        }
        if (in_grab)
            for (int j = 0; j < 3; ++j) used = used || (g.grab_v[j] < v && cin[g.grab_v[j]] == col);
        if (!used || col >= kMaxColors - 1) return col;
    }
}

// Exact sequential-greedy colouring by one CTA: chunks of kChunk consecutive
// vertices are visited in index order, so every lower neighbour outside the
// current chunk is already final; inside the chunk the greedy rule is
// iterated Jacobi-style (read all, barrier, write changes) until no colour
// changes. A chunk converges in at most (its internal descending chain + 1)
// rounds <= kChunk + 1, so the loop is bounded; starting from the previous
// colouring a chunk usually settles in a few rounds.
//
// Per chunk each thread first folds the colours of its vertex's final lower
// neighbours (index below the chunk) into a 64-bit mask, and keeps the
// in-chunk lower neighbours (at most kInner, as chunk-local indices) in
// shared memory; the rounds then read only shared memory: the mask, those
// indices and the chunk's current colours. A vertex with more in-chunk lower
// neighbours, or with a colour >= 64 around it, takes the full rule
// (greedy_color) every round instead. Both give the rule's exact value.
//
// The walk starts at the chunk of `first[0]`, the lowest vertex whose rule
// does not hold for the previous colouring (k_color_probe): every vertex
// below it already satisfies the rule against final lower neighbours, so it
// is final too. When the whole colouring fits (n <= kSmemColors) it is kept
// in shared memory for the walk.
constexpr int kChunk = 1024;
constexpr int kInner = 16;
constexpr uint32_t kSmemColors = 90 * 1024;  // 180 KB of uint16 colours (+ 34 KB static)
__global__ void __launch_bounds__(kChunk) k_color_chunked(ColorView g, uint16_t* col_g, const unsigned int* first,
                                                         unsigned int* rounds_out, unsigned int* err) {
    extern __shared__ uint16_t col_s[];
    __shared__ uint16_t inner[kInner][kChunk];  // chunk-local indices of in-chunk lower neighbours
    __shared__ uint16_t chunk_col[kChunk];      // the chunk's current colours
    uint32_t start = *first;
    if (start >= g.n) {  // already a fixed point
        if (threadIdx.x == 0) *rounds_out = 0;
        return;
    }
    bool smem = g.n <= kSmemColors;
    uint16_t* col = col_g;
    if (smem) {
        for (uint32_t i = threadIdx.x; i < g.n; i += kChunk) col_s[i] = col_g[i];
        __syncthreads();
        col = col_s;
    }
    const uint32_t t = threadIdx.x;
    unsigned int rounds = 0;
    for (uint32_t base = (start / kChunk) * kChunk; base < g.n; base += kChunk) {
        const uint32_t v = base + t;
        const bool live = v < g.n;
        // set-up: final colours below the chunk into a mask, in-chunk lower
        // neighbours into shared memory
        unsigned long long outer = 0;
        bool slow = false;
        uint32_t ninner = 0;
        auto visit = [&](uint32_t u) {
            if (u >= v) return;
            if (u < base) {
                mark(outer, col[u], slow);
            } else if (ninner < kInner) {
                inner[ninner++][t] = (uint16_t)(u - base);
            } else {
                slow = true;
            }
        };
        if (live) {
            for (uint32_t k = g.lo_off[v]; k < g.lo_off[v + 1]; ++k) visit(g.lo[k]);
            for (uint32_t k = g.contacts.inc_off[v]; k < g.contacts.inc_off[v + 1]; ++k) {
                uint32_t c = g.contacts.inc[k];
                uint32_t kind = g.contacts.kind[c];
                uint4 cv = g.contacts.verts[c];
                uint32_t ids[4] = {cv.x, cv.y, cv.z, cv.w};
                uint32_t cnt = kind == 0 ? 2u : (kind == 1 ? 3u : 4u);
                for (uint32_t j = 0; j < cnt; ++j) visit(ids[j]);
            }
            if (g.grab_active && (g.grab_v[0] == v || g.grab_v[1] == v || g.grab_v[2] == v))
                for (int j = 0; j < 3; ++j) visit(g.grab_v[j]);
            chunk_col[t] = col[v];
        }
        __syncthreads();
        int r = 0;
        for (; r <= kChunk + 1; ++r) {
            uint32_t c = 0u;
            if (live) {
                unsigned long long mask = outer;
                bool high = slow;
                for (uint32_t j = 0; j < ninner; ++j) mark(mask, chunk_col[inner[j][t]], high);
                // colours >= 64 around v, or all of 0..63 taken: the full rule
                if (high || ~mask == 0ull) c = greedy_color(g, col, v);
                else c = (uint32_t)__ffsll((long long)~mask) - 1;
            }
            __syncthreads();
            int changed = (live && c != chunk_col[t]) ? 1 : 0;
            if (changed) {
                chunk_col[t] = (uint16_t)c;
                col[v] = (uint16_t)c;
            }
            ++rounds;
            if (!__syncthreads_or(changed)) break;
        }
        if (r > kChunk + 1 && t == 0) atomicOr(err, 1u);
    }
    if (smem) {
        __syncthreads();
        for (uint32_t i = (start / kChunk) * kChunk + threadIdx.x; i < g.n; i += kChunk) col_g[i] = col_s[i];
    }
    if (t == 0) *rounds_out = rounds;
}

// Lowest vertex whose greedy rule fails for the current colouring.
__global__ void k_color_probe(ColorView g, const uint16_t* col, unsigned int* first) {
    unsigned int lo = 0xffffffffu;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x)
        if (greedy_color(g, col, v) != col[v]) lo = min(lo, v);
    for (int o = 16; o > 0; o >>= 1) lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    if ((threadIdx.x & 31) == 0 && lo != 0xffffffffu) atomicMin(first, lo);
}

__global__ void k_color_count(uint32_t n, const uint16_t* col, uint32_t* counts) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        atomicAdd(&counts[col[v]], 1u);
}

__global__ void k_iota(uint32_t n, uint32_t* out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) out[v] = v;
}

void Coloring::init(uint32_t n, cudaStream_t s) {
    n_ = n;
    a_.reserve(n);
    b_.reserve(n);
    order_.reserve(n);
    iota_.reserve(n);
    counts_.reserve(kMaxColors);
    changed_.reserve(kBatch);
    changed_h_.reserve(kBatch);
    counts_h_.reserve(kMaxColors);
    CC_CUDA(cudaMemsetAsync(a_.ptr, 0, n * sizeof(uint16_t), s));
    if (n) k_iota<<<grid_for(n, 256), 256, 0, s>>>(n, iota_.ptr);
    CC_CUDA(cudaGetLastError());
    cur_ = a_.ptr;
}

void Coloring::compute(const ColorView& view, cudaStream_t s) {
    uint32_t n = n_;
    if (n == 0) {
        n_colors_ = 0;
        offsets_h_.assign(1, 0);
        return;
    }
    // the chunked walk updates the previous colouring in place, from the
    // first vertex the probe finds out of date
    CC_CUDA(cudaMemsetAsync(changed_.ptr, 0, 2 * sizeof(unsigned int), s));
    CC_CUDA(cudaMemsetAsync(changed_.ptr + 2, 0xff, sizeof(unsigned int), s));
    k_color_probe<<<grid_for(n, 256), 256, 0, s>>>(view, cur_, changed_.ptr + 2);
    size_t smem = n <= kSmemColors ? n * sizeof(uint16_t) : 0;
    allow_dynamic_smem(k_color_chunked, smem);
    k_color_chunked<<<1, kChunk, smem, s>>>(view, cur_, changed_.ptr + 2, changed_.ptr, changed_.ptr + 1);
    launches_ += 2;
    CC_CUDA(cudaGetLastError());
    CC_CUDA(cudaMemsetAsync(counts_.ptr, 0, kMaxColors * sizeof(uint32_t), s));
    k_color_count<<<grid_for(n, 256), 256, 0, s>>>(n, cur_, counts_.ptr);
    CC_CUDA(cudaMemcpyAsync(counts_h_.ptr, counts_.ptr, kMaxColors * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CC_CUDA(cudaMemcpyAsync(changed_h_.ptr, changed_.ptr, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    CC_CUDA(cudaStreamSynchronize(s));
    last_iterations_ = changed_h_.ptr[0];
    if (changed_h_.ptr[1]) throw Failure{CC_ERR_CUDA, "colouring rounds exceeded their bound"};
    n_colors_ = 0;
    for (uint32_t c = 0; c < kMaxColors; ++c)
        if (counts_h_.ptr[c]) n_colors_ = c + 1;
    if (n_colors_ >= kMaxColors) throw Failure{CC_ERR_CUDA, "colour limit exceeded"};
    offsets_h_.assign(n_colors_ + 1, 0);
    for (uint32_t c = 0; c < n_colors_; ++c) offsets_h_[c + 1] = offsets_h_[c] + counts_h_.ptr[c];
    // vertices grouped by colour, in index order within a colour (a stable
    // sort on the colour bits): a warp's vertices are neighbours in the mesh
    // order, so the sweep's gathers share cache lines. The order within a
    // colour does not change any result (no two vertices of a colour interact).
    int bits = 1;
    while ((1u << bits) < n_colors_) ++bits;
    launches_ += sorter_.sort_pairs(cur_, b_.ptr, iota_.ptr, order_.ptr, n, bits, s, error_word_, DERR_SORT_WAIT);
    CC_CUDA(cudaGetLastError());
}

void Coloring::download(std::vector<uint32_t>& colors) {
    std::vector<uint16_t> c(n_);
    if (n_) CC_CUDA(cudaMemcpy(c.data(), cur_, n_ * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    colors.assign(c.begin(), c.end());
}

}  // namespace cc
