// Graph colouring on the device (replaces coloring::colors,
// src/vbd/coloring.rs:5-43, which the reference runs serially on the CPU
// after every detection).
//
// The reference visits vertices 0..n in order and gives each the smallest
// colour not used by an already-coloured neighbour (material graph, contact
// co-vertices, grab). Already-coloured means lower index, so the result is
// the unique solution of  c(v) = mex { c(u) : u ~ v, u < v }.  That system is
// solved here by Jacobi fixed-point iteration: every vertex re-evaluates its
// rule from the previous iterate, in parallel. A vertex is final once all its
// lower neighbours are, so the iteration reaches the exact sequential result
// in at most (longest descending chain + 1) sweeps; starting from the previous
// detection's colouring it usually needs far fewer.
#include <cub/device/device_scan.cuh>

#include "color.cuh"

namespace cc {

__device__ __forceinline__ void mark(unsigned long long& mask, uint32_t c, bool& high) {
    if (c < 64) mask |= 1ull << c;
    else high = true;
}

__global__ void k_color_step(ColorView g, const uint16_t* cin, uint16_t* cout, unsigned int* changed) {
    unsigned int any = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
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
        uint32_t col;
        if (~mask != 0ull) {
            col = (uint32_t)__ffsll((long long)~mask) - 1;
        } else {
            // more than 64 colours in the neighbourhood: linear search
            col = 64;
            for (;; ++col) {
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
                if (!used || col >= kMaxColors - 1) break;
            }
        }
        (void)high;
        if (col != cin[v]) any = 1;
        cout[v] = (uint16_t)col;
    }
    if (any) atomicOr(changed, 1u);
}

__global__ void k_color_count(uint32_t n, const uint16_t* col, uint32_t* counts) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        atomicAdd(&counts[col[v]], 1u);
}

__global__ void k_color_scatter(uint32_t n, const uint16_t* col, const uint32_t* offsets, uint32_t* cursor,
                                uint32_t* order) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t c = col[v];
        order[offsets[c] + atomicAdd(&cursor[c], 1u)] = v;
    }
}

void Coloring::init(uint32_t n, cudaStream_t s) {
    n_ = n;
    a_.reserve(n);
    b_.reserve(n);
    order_.reserve(n);
    counts_.reserve(kMaxColors);
    offsets_.reserve(kMaxColors);
    cursor_.reserve(kMaxColors);
    changed_.reserve(kBatch);
    changed_h_.reserve(kBatch);
    counts_h_.reserve(kMaxColors);
    CC_CUDA(cudaMemsetAsync(a_.ptr, 0, n * sizeof(uint16_t), s));
    cur_ = a_.ptr;
}

void Coloring::compute(const ColorView& view, cudaStream_t s) {
    uint32_t n = n_;
    if (n == 0) {
        n_colors_ = 0;
        offsets_h_.assign(1, 0);
        return;
    }
    uint16_t* in = cur_;
    uint16_t* out = (in == a_.ptr) ? b_.ptr : a_.ptr;
    last_iterations_ = 0;
    size_t limit = (size_t)n + 2;
    bool done = false;
    while (!done) {
        CC_CUDA(cudaMemsetAsync(changed_.ptr, 0, kBatch * sizeof(unsigned int), s));
        for (int k = 0; k < kBatch; ++k) {
            k_color_step<<<grid_for(n, 256), 256, 0, s>>>(view, in, out, changed_.ptr + k);
            ++launches_;
            std::swap(in, out);
        }
        CC_CUDA(cudaGetLastError());
        CC_CUDA(cudaMemcpyAsync(changed_h_.ptr, changed_.ptr, kBatch * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                s));
        CC_CUDA(cudaStreamSynchronize(s));
        for (int k = 0; k < kBatch; ++k) {
            ++last_iterations_;
            if (changed_h_.ptr[k] == 0) {
                done = true;
                break;
            }
        }
        if (!done && last_iterations_ > limit)
            throw Failure{CC_ERR_CUDA, "colouring fixed point did not converge"};
    }
    cur_ = in;  // the last output (a fixed point: equal to every later iterate)
    CC_CUDA(cudaMemsetAsync(counts_.ptr, 0, kMaxColors * sizeof(uint32_t), s));
    CC_CUDA(cudaMemsetAsync(cursor_.ptr, 0, kMaxColors * sizeof(uint32_t), s));
    k_color_count<<<grid_for(n, 256), 256, 0, s>>>(n, cur_, counts_.ptr);
    CC_CUDA(cudaMemcpyAsync(counts_h_.ptr, counts_.ptr, kMaxColors * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CC_CUDA(cudaStreamSynchronize(s));
    n_colors_ = 0;
    for (uint32_t c = 0; c < kMaxColors; ++c)
        if (counts_h_.ptr[c]) n_colors_ = c + 1;
    if (n_colors_ >= kMaxColors) throw Failure{CC_ERR_CUDA, "colour limit exceeded"};
    offsets_h_.assign(n_colors_ + 1, 0);
    for (uint32_t c = 0; c < n_colors_; ++c) offsets_h_[c + 1] = offsets_h_[c] + counts_h_.ptr[c];
    CC_CUDA(cudaMemcpyAsync(offsets_.ptr, offsets_h_.data(), (n_colors_ + 1) * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s));
    k_color_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, cur_, offsets_.ptr, cursor_.ptr, order_.ptr);
    launches_ += 2;
    CC_CUDA(cudaGetLastError());
}

void Coloring::download(std::vector<uint32_t>& colors) {
    std::vector<uint16_t> c(n_);
    if (n_) CC_CUDA(cudaMemcpy(c.data(), cur_, n_ * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    colors.assign(c.begin(), c.end());
}

}  // namespace cc
