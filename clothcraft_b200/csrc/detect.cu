// OGC detection on the device (replaces OgcWorld::detect, src/ogc/world.rs:308-557,
// which the reference runs on the CPU every step).
//
// This translation unit is compiled with --fmad=false: every FP64 multiply and
// add is rounded separately, as Rust's f64 arithmetic is, so that distances,
// feasibility decisions, radii and contact keys are bit-identical to the CPU
// path for identical positions.
//
// Pipeline per detection: primitive boxes -> candidate-cache coverage ->
// (on a miss) Morton LBVH build + dual-tree-equivalent pair queries ->
// FP64 narrow phase -> radix sort + dedup of contact keys -> incidence CSR ->
// per-vertex minimum distance -> conservative radii.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <set>

#include <cooperative_groups.h>

#include "world.cuh"

namespace cg = cooperative_groups;

namespace cc {

// ------------------------------------------------------------------ boxes
__device__ __forceinline__ void box_of3(d3 a, d3 b, d3 c, Box& o) {
    // Bounds::points folds min/max from +inf/-inf (src/ogc/bvh.rs:9-20)
    o.lo[0] = fmin(fmin(a.x, b.x), c.x);
    o.lo[1] = fmin(fmin(a.y, b.y), c.y);
    o.lo[2] = fmin(fmin(a.z, b.z), c.z);
    o.hi[0] = fmax(fmax(a.x, b.x), c.x);
    o.hi[1] = fmax(fmax(a.y, b.y), c.y);
    o.hi[2] = fmax(fmax(a.z, b.z), c.z);
}
__device__ __forceinline__ void box_of2(d3 a, d3 b, Box& o) {
    o.lo[0] = fmin(a.x, b.x);
    o.lo[1] = fmin(a.y, b.y);
    o.lo[2] = fmin(a.z, b.z);
    o.hi[0] = fmax(a.x, b.x);
    o.hi[1] = fmax(a.y, b.y);
    o.hi[2] = fmax(a.z, b.z);
}
__device__ __forceinline__ void box_of1(d3 a, Box& o) {
    o.lo[0] = o.hi[0] = a.x;
    o.lo[1] = o.hi[1] = a.y;
    o.lo[2] = o.hi[2] = a.z;
}
// Bounds::distance_squared (src/ogc/bvh.rs:31-36), same operation order.
__device__ __forceinline__ double box_dist2(const Box& a, const Box& b) {
    double dx = fmax(fmax(a.lo[0] - b.hi[0], b.lo[0] - a.hi[0]), 0.0);
    double dy = fmax(fmax(a.lo[1] - b.hi[1], b.lo[1] - a.hi[1]), 0.0);
    double dz = fmax(fmax(a.lo[2] - b.hi[2], b.lo[2] - a.hi[2]), 0.0);
    return dx * dx + dy * dy + dz * dz;
}
// Bounds::overlaps (src/ogc/bvh.rs:27-29)
__device__ __forceinline__ bool box_overlap(const Box& a, const Box& b) {
    return a.lo[0] <= b.hi[0] && a.lo[1] <= b.hi[1] && a.lo[2] <= b.hi[2] && a.hi[0] >= b.lo[0] &&
           a.hi[1] >= b.lo[1] && a.hi[2] >= b.lo[2];
}
__device__ __forceinline__ Box box_union(const Box& a, const Box& b) {
    Box r;
    for (int k = 0; k < 3; ++k) {
        r.lo[k] = fmin(a.lo[k], b.lo[k]);
        r.hi[k] = fmax(a.hi[k], b.hi[k]);
    }
    return r;
}
// ------------------------------------------------------------------- LBVH
__global__ void k_bounds_init(unsigned long long* b) {
    if (threadIdx.x < 3) b[threadIdx.x] = ~0ull;
    else if (threadIdx.x < 6) b[threadIdx.x] = 0ull;
}

__global__ void k_centroid_bounds(const Box* box, const uint32_t* ids, uint32_t m, unsigned long long* b) {
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const Box& q = box[ids[i]];
        for (int k = 0; k < 3; ++k) {
            unsigned long long key = order_key(0.5 * (q.lo[k] + q.hi[k]));
            lo[k] = min(lo[k], key);
            hi[k] = max(hi[k], key);
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(&b[k], lo[k]);
            atomicMax(&b[3 + k], hi[k]);
        }
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned long long v) {
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

// 63-bit Morton code of a point in the centroid bounds, every axis scaled by
// the largest extent (a cube), so that a nearly flat set keeps its flat
// order: its thin axis then only reaches the low bits instead of being
// stretched over all 21.
__device__ __forceinline__ unsigned long long morton63(const double* c, const unsigned long long* b) {
    double lo[3], ext = 0.0;
    for (int k = 0; k < 3; ++k) {
        lo[k] = from_order_key(b[k]);
        ext = fmax(ext, from_order_key(b[3 + k]) - lo[k]);
    }
    unsigned long long code = 0;
    for (int k = 0; k < 3; ++k) {
        double t = ext > 0.0 ? (c[k] - lo[k]) / ext : 0.0;
        double s = t * 2097152.0;
        unsigned long long u = s <= 0.0 ? 0ull : (s >= 2097151.0 ? 2097151ull : (unsigned long long)s);
        code |= spread21(u) << (2 - k);
    }
    return code;
}

__global__ void k_morton(const Box* box, const uint32_t* ids, uint32_t m, const unsigned long long* b,
                         unsigned long long* code, uint32_t* vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        uint32_t id = ids[i];
        const Box& q = box[id];
        double c[3] = {0.5 * (q.lo[0] + q.hi[0]), 0.5 * (q.lo[1] + q.hi[1]), 0.5 * (q.lo[2] + q.hi[2])};
        code[i] = morton63(c, b);
        vals[i] = id;
    }
}

// Bounds and Morton codes of points (the VF query order).
__global__ void k_point_bounds(const double4* x, uint32_t n, unsigned long long* b) {
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double4 p = x[i];
        double c[3] = {p.x, p.y, p.z};
        for (int k = 0; k < 3; ++k) {
            unsigned long long key = order_key(c[k]);
            lo[k] = min(lo[k], key);
            hi[k] = max(hi[k], key);
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(&b[k], lo[k]);
            atomicMax(&b[3 + k], hi[k]);
        }
    }
}

__global__ void k_point_morton(const double4* x, uint32_t n, const unsigned long long* b, unsigned long long* code,
                               uint32_t* vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double4 p = x[i];
        double c[3] = {p.x, p.y, p.z};
        code[i] = morton63(c, b);
        vals[i] = i;
    }
}

__device__ __forceinline__ int lbvh_delta(const unsigned long long* code, int m, int i, int j) {
    if (j < 0 || j >= m) return -1;
    unsigned long long a = code[i], b = code[j];
    if (a == b) return 64 + __clz((unsigned)(i ^ j));
    return __clzll(a ^ b);
}

// Karras 2012, "Maximizing parallelism in the construction of BVHs". The
// children go into the node records (d.x, d.y); the boxes follow in
// k_lbvh_refit.
__global__ void k_karras(const unsigned long long* code, int m, LNode* node, int* parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m - 1; i += gridDim.x * blockDim.x) {
        int d = (lbvh_delta(code, m, i, i + 1) - lbvh_delta(code, m, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = lbvh_delta(code, m, i, i - d);
        int lmax = 2;
        while (lbvh_delta(code, m, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (lbvh_delta(code, m, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = lbvh_delta(code, m, i, j);
        int s = 0;
        int t = l;
        do {
            t = (t + 1) >> 1;
            if (lbvh_delta(code, m, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        int gamma = i + s * d + min(d, 0);
        int left, right;
        if (min(i, j) == gamma) {
            left = gamma | 0x80000000;
            parent[m - 1 + gamma] = i;
        } else {
            left = gamma;
            parent[gamma] = i;
        }
        if (max(i, j) == gamma + 1) {
            right = (gamma + 1) | 0x80000000;
            parent[m - 1 + gamma + 1] = i;
        } else {
            right = gamma + 1;
            parent[gamma + 1] = i;
        }
        *reinterpret_cast<int2*>(&node[i].d) = make_int2(left, right);
        if (i == 0) parent[0] = -1;
    }
}

__global__ void k_leaf_boxes(const Box* prim_box, const uint32_t* leaf_prim, int m, Box* leaf_box) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        leaf_box[i] = prim_box[leaf_prim[i]];
}

// Writes one child's box and largest id into its parent's record (slot 0 =
// left: floats 0..5 and d.z; slot 1 = right: floats 6..11 and d.w).
__device__ __forceinline__ void put_slot(LNode* node, int p, int slot, const float* lo, const float* hi, uint32_t mx) {
    float* f = reinterpret_cast<float*>(node + p) + 6 * slot;
    f[0] = lo[0];
    f[1] = lo[1];
    f[2] = lo[2];
    f[3] = hi[0];
    f[4] = hi[1];
    f[5] = hi[2];
    reinterpret_cast<int*>(&node[p].d)[2 + slot] = (int)mx;
}

// Bottom-up boxes: each leaf writes its outward-rounded box into its parent's
// slot; the second of a node's two children to arrive (atomic counter) forms
// the node's box from both slots and carries it one level up. FP32 min/max of
// outward-rounded boxes is exact, so every node box contains the exact boxes
// below it.
__global__ void k_lbvh_refit(const Box* leaf_box, const uint32_t* leaf_prim, int m, LNode* node, const int* parent,
                             unsigned* visits) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const Box& b = leaf_box[i];
        float lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = __double2float_rd(b.lo[k]);
            hi[k] = __double2float_ru(b.hi[k]);
        }
        uint32_t mx = leaf_prim[i];
        int code = i | 0x80000000;
        int p = parent[m - 1 + i];
        while (p >= 0) {
            int2 ch = *reinterpret_cast<const int2*>(&node[p].d);
            put_slot(node, p, ch.x == code ? 0 : 1, lo, hi, mx);
            __threadfence();
            if (atomicAdd(&visits[p], 1u) == 0u) break;
            __threadfence();
            const float* f = reinterpret_cast<const float*>(node + p);
            for (int k = 0; k < 3; ++k) {
                lo[k] = fminf(__ldcg(f + k), __ldcg(f + 6 + k));
                hi[k] = fmaxf(__ldcg(f + 3 + k), __ldcg(f + 9 + k));
            }
            const int* d = reinterpret_cast<const int*>(&node[p].d);
            mx = max((uint32_t)__ldcg(d + 2), (uint32_t)__ldcg(d + 3));
            code = p;
            p = parent[p];
        }
    }
}

int Lbvh::build(const Box* prim_box, const uint32_t* ids, uint32_t count, cudaStream_t s, unsigned int* err) {
    m = count;
    built = true;
    if (m == 0) return 0;
    leaf_prim.reserve(m);
    ids_tmp.reserve(m);
    morton.reserve(m);
    morton_tmp.reserve(m);
    bounds.reserve(6);
    node.reserve(m > 1 ? m - 1 : 1);
    parent.reserve(2 * m);
    visits.reserve(m);
    leaf_box.reserve(m);
    k_bounds_init<<<1, 32, 0, s>>>(bounds.ptr);
    k_centroid_bounds<<<grid_for(m, 256), 256, 0, s>>>(prim_box, ids, m, bounds.ptr);
    k_morton<<<grid_for(m, 256), 256, 0, s>>>(prim_box, ids, m, bounds.ptr, morton_tmp.ptr, ids_tmp.ptr);
    int sorts = sorter.sort_pairs(morton_tmp.ptr, morton.ptr, ids_tmp.ptr, leaf_prim.ptr, m, 63, s, err, DERR_SORT_WAIT);
    int n = 3 + sorts;
    if (m > 1) {
        k_karras<<<grid_for(m - 1, 256), 256, 0, s>>>(morton.ptr, (int)m, node.ptr, parent.ptr);
        ++n;
    }
    CC_CUDA(cudaGetLastError());
    return n + refit(prim_box, s);
}

int Lbvh::refit(const Box* prim_box, cudaStream_t s) {
    if (m == 0) return 0;
    k_leaf_boxes<<<grid_for(m, 256), 256, 0, s>>>(prim_box, leaf_prim.ptr, (int)m, leaf_box.ptr);
    if (m > 1) {
        CC_CUDA(cudaMemsetAsync(visits.ptr, 0, (m - 1) * sizeof(unsigned), s));
        k_lbvh_refit<<<grid_for(m, 256), 256, 0, s>>>(leaf_box.ptr, leaf_prim.ptr, (int)m, node.ptr, parent.ptr,
                                                      visits.ptr);
    }
    CC_CUDA(cudaGetLastError());
    return m > 1 ? 2 : 1;
}

// A query box rounded outward to FP32 for the node tests.
struct QBox {
    float lo[3], hi[3];
};
__device__ __forceinline__ QBox qbox(const Box& b) {
    QBox q;
    for (int k = 0; k < 3; ++k) {
        q.lo[k] = __double2float_rd(b.lo[k]);
        q.hi[k] = __double2float_ru(b.hi[k]);
    }
    return q;
}

// Node test for a distance query: false only if the exact distance between
// the query's and the child's FP64 boxes exceeds the search radius. The gaps
// and their squares are rounded down and the bound (r2_up) up, so the test
// never drops a child whose leaves pass the exact FP64 leaf test.
__device__ __forceinline__ bool near32(const QBox& q, float lx, float ly, float lz, float hx, float hy, float hz,
                                       float r2_up) {
    float gx = fmaxf(0.f, fmaxf(__fsub_rd(lx, q.hi[0]), __fsub_rd(q.lo[0], hx)));
    float gy = fmaxf(0.f, fmaxf(__fsub_rd(ly, q.hi[1]), __fsub_rd(q.lo[1], hy)));
    float gz = fmaxf(0.f, fmaxf(__fsub_rd(lz, q.hi[2]), __fsub_rd(q.lo[2], hz)));
    float d2 = __fadd_rd(__fadd_rd(__fmul_rd(gx, gx), __fmul_rd(gy, gy)), __fmul_rd(gz, gz));
    return d2 <= r2_up;
}
// the bound for near32: search^2 with a 1e-6 relative margin for the FP64
// rounding of the exact leaf test, rounded up to FP32
__device__ __forceinline__ float r2_bound(double search2) { return __double2float_ru(search2 * (1.0 + 1e-6)); }

// Node test for an overlap query (outward-rounded boxes overlap whenever the
// exact ones do).
__device__ __forceinline__ bool overlap32(const QBox& q, float lx, float ly, float lz, float hx, float hy, float hz) {
    return !(lx > q.hi[0] || ly > q.hi[1] || lz > q.hi[2] || hx < q.lo[0] || hy < q.lo[1] || hz < q.lo[2]);
}

// Depth-first traversal that goes down one passing child and stacks the
// other. near(lx, ly, lz, hx, hy, hz) tests a child's FP32 box; leaf_ok(box)
// is the exact FP64 primitive predicate; visit(prim) receives the accepted
// primitive id. With ABOVE, only primitives with id > above are visited and
// subtrees whose largest id is <= above are skipped unvisited (self-pair
// queries that keep the canonical order e < f). Returns false if the stack
// overflowed.
constexpr int kTraversalStack = 96;
template <bool ABOVE, class Near, class LeafOk, class Visit>
__device__ __forceinline__ bool lbvh_walk(const LbvhView& t, uint32_t above, Near near, LeafOk leaf_ok, Visit visit) {
    if (t.m == 0) return true;
    if (t.m == 1) {
        uint32_t p = t.leaf_prim[0];
        if ((!ABOVE || p > above) && leaf_ok(t.leaf_box[0])) visit(p);
        return true;
    }
    int stack[kTraversalStack];
    int sp = 0;
    int node = 0;
    while (true) {
        const float4* r = reinterpret_cast<const float4*>(t.node + node);
        const float4 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2);
        const int4 d = __ldg(reinterpret_cast<const int4*>(r + 3));
        bool go_l = (!ABOVE || (uint32_t)d.z > above) && near(a.x, a.y, a.z, a.w, b.x, b.y);
        bool go_r = (!ABOVE || (uint32_t)d.w > above) && near(b.z, b.w, c.x, c.y, c.z, c.w);
        if (go_l && d.x < 0) {
            uint32_t i = (uint32_t)d.x & 0x7fffffffu;
            if (leaf_ok(t.leaf_box[i])) visit(t.leaf_prim[i]);
            go_l = false;
        }
        if (go_r && d.y < 0) {
            uint32_t i = (uint32_t)d.y & 0x7fffffffu;
            if (leaf_ok(t.leaf_box[i])) visit(t.leaf_prim[i]);
            go_r = false;
        }
        if (go_l && go_r) {
            if (sp >= kTraversalStack) return false;
            stack[sp++] = d.y;
            node = d.x;
        } else if (go_l) {
            node = d.x;
        } else if (go_r) {
            node = d.y;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return true;
}

// ---------------------------------------------------------------- geometry
__device__ __forceinline__ bool adjacent(const WorldView& w, uint32_t a, uint32_t b) {  // world.rs:215-217
    if (a == b) return true;
    uint32_t lo = w.ex_off[a], hi = w.ex_off[a + 1];
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t v = w.ex[mid];
        if (v == b) return true;
        if (v < b) lo = mid + 1;
        else hi = mid;
    }
    return false;
}

__device__ bool vertex_feasible(const WorldView& w, d3 p, uint32_t v) {  // geometry.rs:13-17
    d3 xv = ld3(w.x, v);
    for (uint32_t k = w.nb_off[v]; k < w.nb_off[v + 1]; ++k) {
        d3 xj = ld3(w.x, w.nb[k]);
        if (!(dot(p - xv, xv - xj) >= -1e-14)) return false;
    }
    return true;
}

__device__ bool edge_feasible(const WorldView& w, d3 p, uint32_t e) {  // geometry.rs:18-29
    uint2 ev = w.edges[e];
    d3 a = ld3(w.x, ev.x), b = ld3(w.x, ev.y);
    d3 u = b - a;
    double t = dot(p - a, u) / len2(u);
    if (!(t > 0.0 && t < 1.0)) return false;
    int2 op = w.opposites[e];
    int ops[2] = {op.x, op.y};
    for (int k = 0; k < 2; ++k) {
        if (ops[k] < 0) continue;
        d3 c = ld3(w.x, (uint32_t)ops[k]);
        d3 q = a + u * (dot(c - a, u) / len2(u));
        if (!(dot(p - q, q - c) >= -1e-14)) return false;
    }
    return true;
}

// closest_triangle (geometry.rs:31-77) on explicit corners. kind: 0 vertex,
// 1 edge, 2 face; which: the corner (0..2) of a vertex feature, or the
// triangle-edge slot (0 = ab, 1 = bc, 2 = ca) of an edge feature.
__device__ d3 closest_on_triangle(d3 p, d3 a, d3 b, d3 c, int& kind, int& which) {
    d3 ab = b - a, ac = c - a, ap = p - a;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) {
        kind = 0;
        which = 0;
        return a;
    }
    d3 bp = p - b;
    double d3_ = dot(ab, bp), d4 = dot(ac, bp);
    if (d3_ >= 0.0 && d4 <= d3_) {
        kind = 0;
        which = 1;
        return b;
    }
    double vc = d1 * d4 - d3_ * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) {
        kind = 1;
        which = 0;
        return a + ab * (d1 / (d1 - d3_));
    }
    d3 cp = p - c;
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) {
        kind = 0;
        which = 2;
        return c;
    }
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        kind = 1;
        which = 2;
        return a + ac * (d2 / (d2 - d6));
    }
    double va = d3_ * d6 - d5 * d4;
    if (va <= 0.0 && d4 - d3_ >= 0.0 && d5 - d6 >= 0.0) {
        kind = 1;
        which = 1;
        return b + (c - b) * ((d4 - d3_) / ((d4 - d3_) + (d5 - d6)));
    }
    double denom = 1.0 / (va + vb + vc);
    kind = 2;
    which = 0;
    return a + ab * (vb * denom) + ac * (vc * denom);
}

// closest_triangle on world triangle t, returning the feature's id.
__device__ d3 closest_triangle(const WorldView& w, d3 p, uint32_t t, int& kind, uint32_t& fid) {
    uint3 ids = w.tri[t];
    int which;
    d3 q = closest_on_triangle(p, ld3(w.x, ids.x), ld3(w.x, ids.y), ld3(w.x, ids.z), kind, which);
    if (kind == 0) fid = which == 0 ? ids.x : (which == 1 ? ids.y : ids.z);
    else if (kind == 1) fid = which == 0 ? w.tri_edges[t].x : (which == 1 ? w.tri_edges[t].y : w.tri_edges[t].z);
    else fid = t;
    return q;
}

__device__ __forceinline__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

// closest_segments (geometry.rs:78-107)
__device__ void closest_segments(d3 a, d3 b, d3 c, d3 d, double& s_out, double& t_out) {
    d3 u = b - a;
    d3 v = d - c;
    d3 w = a - c;
    double aa = len2(u);
    double ee = len2(v);
    if (aa < 1e-24 || ee < 1e-24) {
        s_out = 0.0;
        t_out = 0.0;
        return;
    }
    double bb = dot(u, v);
    double cc = dot(u, w);
    double ff = dot(v, w);
    double den = aa * ee - bb * bb;
    double s = den > 1e-14 * aa * ee ? clamp01((bb * ff - cc * ee) / den) : 0.0;
    double t = (bb * s + ff) / ee;
    if (t < 0.0) {
        s = clamp01(-cc / aa);
        t = 0.0;
    } else if (t > 1.0) {
        s = clamp01((bb - cc) / aa);
        t = 1.0;
    }
    s_out = s;
    t_out = t;
}

// segment_triangle (geometry.rs:131-147)
__device__ bool segment_triangle(d3 a, d3 b, d3 p, d3 q, d3 r) {
    d3 e = q - p;
    d3 f = r - p;
    d3 d = b - a;
    d3 h = cross(d, f);
    double det = dot(e, h);
    if (fabs(det) < 1e-14) return false;
    d3 s = a - p;
    double u = dot(s, h) / det;
    d3 z = cross(s, e);
    double v = dot(d, z) / det;
    double k = dot(f, z) / det;
    return u >= -1e-10 && v >= -1e-10 && u + v <= 1.0 + 1e-10 && (k >= 1e-10 && k < 1.0 - 1e-10);
}

// ------------------------------------------------------------ refit/checks
__global__ void k_refit(WorldView w, const double4* fixed_x, int check_fixed, unsigned int* err) {
    unsigned int e = 0;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (size_t i = i0; i < w.n_all; i += stride) {
        d3 p = ld3(w.x, (uint32_t)i);
        if (!isfin(p)) e |= DERR_NONFINITE_STATE;
        if (check_fixed && i >= w.moving) {
            double4 f = fixed_x[i - w.moving];
            if (!(p.x == f.x && p.y == f.y && p.z == f.z)) e |= DERR_FIXED_MOVED;
        }
    }
    for (size_t t = i0; t < w.n_tri; t += stride) {
        uint3 ids = w.tri[t];
        d3 a = ld3(w.x, ids.x), b = ld3(w.x, ids.y), c = ld3(w.x, ids.z);
        Box bx;
        box_of3(a, b, c, bx);
        w.tri_box[t] = bx;
        if (ids.x < w.moving || ids.y < w.moving || ids.z < w.moving) {
            if (len2(cross(b - a, c - a)) < 1e-24) e |= DERR_DEGENERATE_FACE;
        }
    }
    for (size_t k = i0; k < w.n_edge; k += stride) {
        uint2 ev = w.edges[k];
        Box bx;
        box_of2(ld3(w.x, ev.x), ld3(w.x, ev.y), bx);
        w.edge_box[k] = bx;
    }
    if (e) atomicOr(err, e);
}

// max_i |x_i - c_i|^2 over moving vertices and max |x| component over all.
__global__ void k_cover_and_scale(WorldView w, const double4* centers, int have_centers,
                                  unsigned long long* max_move, unsigned long long* max_abs) {
    double mm = 0.0, ma = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < w.n_all; i += (size_t)gridDim.x * blockDim.x) {
        d3 p = ld3(w.x, (uint32_t)i);
        ma = fmax(ma, fmax(fmax(fabs(p.x), fabs(p.y)), fabs(p.z)));
        if (have_centers && i < w.moving) {
            d3 c = ld3(centers, (uint32_t)i);
            mm = fmax(mm, len2(p - c));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mm = fmax(mm, __shfl_xor_sync(0xffffffffu, mm, o));
        ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(max_move, dbits(mm));
        atomicMax(max_abs, dbits(ma));
    }
}

// ------------------------------------------------------------ pair queries
// Warp-aggregated append: the lanes that reach this call together take
// consecutive slots of an output list with one atomic per warp instead of
// one per lane (the candidate and raw-contact lists are order-free: pairs are
// consumed as a set, contacts are sorted canonically afterwards).
__device__ __forceinline__ unsigned long long append_slot(unsigned long long* count) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(count, (unsigned long long)g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

// VF candidates (candidates.rs:29-37): every point against triangles, pairs
// with box distance <= search, not both fixed, triangle not adjacent.
// Points are taken in `order` (a Morton order of the points), so that the
// lanes of a warp walk nearby points. (Walking a warp's 32 queries as one
// node sequence, the union of their walks, measured 4x slower for VF and
// 1.2x for EE on the fold: the union is several times the longest walk.)
__global__ void k_vf_query(WorldView w, const uint32_t* order, LbvhView tri_moving, LbvhView tri_fixed, double search2,
                           uint2* out, unsigned long long cap, unsigned long long* count, unsigned int* err) {
    const float r2 = r2_bound(search2);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < w.n_all; j += gridDim.x * blockDim.x) {
        const uint32_t v = order[j];
        Box q;
        box_of1(ld3(w.x, v), q);
        const QBox q32 = qbox(q);
        auto near = [&](float lx, float ly, float lz, float hx, float hy, float hz) {
            return near32(q32, lx, ly, lz, hx, hy, hz, r2);
        };
        auto leaf_ok = [&](const Box& b) { return box_dist2(q, b) <= search2; };
        auto visit = [&](uint32_t t) {
            uint3 ids = w.tri[t];
            if (adjacent(w, v, ids.x) || adjacent(w, v, ids.y) || adjacent(w, v, ids.z)) return;
            unsigned long long k = append_slot(count);
            if (k < cap) out[k] = make_uint2(v, t);
        };
        bool ok = lbvh_walk<false>(tri_moving, 0u, near, leaf_ok, visit);
        if (v < w.moving) ok = lbvh_walk<false>(tri_fixed, 0u, near, leaf_ok, visit) && ok;
        if (!ok) atomicOr(err, DERR_STACK_OVERFLOW);
    }
}

// EE candidates (candidates.rs:38-55): moving edges against moving edges
// (each unordered pair once, canonical e < f) and against fixed edges
// (moving edge first). `edge_moving` lists the moving edges in the moving
// edge tree's leaf order (a Morton order), so neighbouring lanes query
// neighbouring edges.
__global__ void k_ee_query(WorldView w, const uint32_t* edge_moving, uint32_t n_moving_edges, LbvhView edge_moving_t,
                           LbvhView edge_fixed_t, double search2, uint2* out, unsigned long long cap,
                           unsigned long long* count, unsigned int* err) {
    const float r2 = r2_bound(search2);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_moving_edges; k += gridDim.x * blockDim.x) {
        uint32_t e = edge_moving[k];
        Box q = w.edge_box[e];
        const QBox q32 = qbox(q);
        uint2 ids = w.edges[e];
        auto near = [&](float lx, float ly, float lz, float hx, float hy, float hz) {
            return near32(q32, lx, ly, lz, hx, hy, hz, r2);
        };
        auto leaf_ok = [&](const Box& b) { return box_dist2(q, b) <= search2; };
        auto filtered = [&](uint32_t f) {
            uint2 js = w.edges[f];
            return adjacent(w, ids.x, js.x) || adjacent(w, ids.x, js.y) || adjacent(w, ids.y, js.x) ||
                   adjacent(w, ids.y, js.y);
        };
        auto visit_moving = [&](uint32_t f) {
            if (f <= e || filtered(f)) return;
            unsigned long long i = append_slot(count);
            if (i < cap) out[i] = make_uint2(e, f);
        };
        auto visit_fixed = [&](uint32_t f) {
            if (filtered(f)) return;
            unsigned long long i = append_slot(count);
            if (i < cap) out[i] = make_uint2(e, f);
        };
        bool ok = lbvh_walk<true>(edge_moving_t, e, near, leaf_ok, visit_moving);
        ok = lbvh_walk<false>(edge_fixed_t, 0u, near, leaf_ok, visit_fixed) && ok;
        if (!ok) atomicOr(err, DERR_STACK_OVERFLOW);
    }
}

// ------------------------------------------------------------ narrow phase
// Contact keys. The reference orders contacts by (kind, v0, v1, v2, v3) with
// the vertices in canonical order (world.rs:435-452). Within a kind the
// trailing vertices always form a mesh edge (PE: v1 v2; EE: v0 v1 and v2 v3)
// or a triangle (PF: v1 v2 v3), so each such group is replaced by its rank
// among the mesh's distinct edges (or triangles) in lexicographic vertex
// order, which keeps the order:
//   PP (v0, v1)          -> (v0, v1)
//   PE (v0, v1, v2)      -> (v0, rank(v1 v2))
//   PF (v0, v1, v2, v3)  -> (v0, rank(v1 v2 v3))
//   EE (v0, v1, v2, v3)  -> (rank(v0 v1), rank(v2 v3))
// key = kind << 2W | A << W | B with 2^W above every vertex id and rank: one
// key of 2W + 2 bits, sorted in one keys-only radix sort.
struct NarrowOut {
    unsigned long long* key;
    unsigned long long cap;
    unsigned long long* count;
    unsigned long long* dist;  // [n_all] double bits
    unsigned long long* vf_count;
    unsigned long long* ee_count;
    unsigned long long* rejections;
    const uint32_t* edge_rank;  // [n_edge]
    const uint32_t* tri_rank;   // [n_tri]
    uint32_t w;                 // bits per key field
};

__device__ __forceinline__ void push_key(const NarrowOut& o, unsigned kind, uint32_t a, uint32_t b) {
    unsigned long long k = append_slot(o.count);
    if (k < o.cap)
        o.key[k] = ((unsigned long long)kind << (2 * o.w)) | ((unsigned long long)a << o.w) | (unsigned long long)b;
}
__device__ __forceinline__ void push_pp(const NarrowOut& o, uint32_t i, uint32_t j) {
    push_key(o, 0, min(i, j), max(i, j));
}
// point v against mesh edge e
__device__ __forceinline__ void push_pe(const NarrowOut& o, uint32_t v, uint32_t e) { push_key(o, 1, v, o.edge_rank[e]); }
// point v against triangle t
__device__ __forceinline__ void push_pf(const NarrowOut& o, uint32_t v, uint32_t t) { push_key(o, 2, v, o.tri_rank[t]); }
// edges e (vertices ids) and f (js), the canonical order putting first the
// edge with the smaller first vertex (world.rs:446-451)
__device__ __forceinline__ void push_ee(const NarrowOut& o, uint32_t e, uint2 ids, uint32_t f, uint2 js) {
    uint32_t re = o.edge_rank[e], rf = o.edge_rank[f];
    if (ids.x > js.x) push_key(o, 3, rf, re);
    else push_key(o, 3, re, rf);
}

__global__ void k_narrow(WorldView w, const uint2* vf, unsigned long long n_vf, const uint2* ee,
                         unsigned long long n_ee, double query_radius, const unsigned long long* max_abs_bits,
                         int prune, NarrowOut o) {
    double scale = fmax(query_radius, bitsd(*max_abs_bits));
    double pr = query_radius + 64.0 * 2.220446049250313e-16 * scale;
    double padded2 = pr * pr;
    unsigned long long nvf = 0, nee = 0, nrej = 0;
    unsigned long long total = n_vf + n_ee;
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        if (k < n_vf) {
            uint32_t v = vf[k].x, t = vf[k].y;
            d3 xv = ld3(w.x, v);
            if (prune) {
                Box pb;
                box_of1(xv, pb);
                if (box_dist2(pb, w.tri_box[t]) > padded2) {
                    ++nrej;
                    continue;
                }
            }
            uint3 ids = w.tri[t];
            int kind;
            uint32_t fid;
            d3 p = closest_triangle(w, xv, t, kind, fid);
            double d = len(xv - p);
            if (d >= query_radius) continue;
            ++nvf;
            unsigned long long db = dbits(d);
            atomicMin(&o.dist[v], db);
            atomicMin(&o.dist[ids.x], db);
            atomicMin(&o.dist[ids.y], db);
            atomicMin(&o.dist[ids.z], db);
            if (kind == 0) {
                if (vertex_feasible(w, xv, fid)) push_pp(o, v, fid);
            } else if (kind == 1) {
                if (edge_feasible(w, xv, fid)) push_pe(o, v, fid);
            } else {
                push_pf(o, v, t);
            }
        } else {
            unsigned long long kk = k - n_vf;
            uint32_t e = ee[kk].x, f = ee[kk].y;
            if (prune && box_dist2(w.edge_box[e], w.edge_box[f]) > padded2) {
                ++nrej;
                continue;
            }
            uint2 ids = w.edges[e], js = w.edges[f];
            d3 a = ld3(w.x, ids.x), b = ld3(w.x, ids.y), c = ld3(w.x, js.x), dd = ld3(w.x, js.y);
            double s, t;
            closest_segments(a, b, c, dd, s, t);
            d3 p = a + (b - a) * s;
            d3 q = c + (dd - c) * t;
            double dist = len(p - q);
            if (dist >= query_radius) continue;
            ++nee;
            unsigned long long db = dbits(dist);
            atomicMin(&o.dist[ids.x], db);
            atomicMin(&o.dist[ids.y], db);
            atomicMin(&o.dist[js.x], db);
            atomicMin(&o.dist[js.y], db);
            long end_a = s <= 0.0 ? (long)ids.x : (s >= 1.0 ? (long)ids.y : -1);
            long end_b = t <= 0.0 ? (long)js.x : (t >= 1.0 ? (long)js.y : -1);
            if ((end_a >= 0 && !vertex_feasible(w, q, (uint32_t)end_a)) ||
                (end_b >= 0 && !vertex_feasible(w, p, (uint32_t)end_b)))
                continue;
            if (end_a >= 0 && end_b >= 0) push_pp(o, (uint32_t)end_a, (uint32_t)end_b);
            else if (end_a >= 0) push_pe(o, (uint32_t)end_a, f);
            else if (end_b >= 0) push_pe(o, (uint32_t)end_b, e);
            else push_ee(o, e, ids, f, js);
        }
    }
    for (int s = 16; s > 0; s >>= 1) {
        nvf += __shfl_xor_sync(0xffffffffu, nvf, s);
        nee += __shfl_xor_sync(0xffffffffu, nee, s);
        nrej += __shfl_xor_sync(0xffffffffu, nrej, s);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nvf) atomicAdd(o.vf_count, nvf);
        if (nee) atomicAdd(o.ee_count, nee);
        if (nrej) atomicAdd(o.rejections, nrej);
    }
}

__global__ void k_fill_u64(unsigned long long* p, size_t n, unsigned long long v) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_unique_flags(const unsigned long long* key, size_t n, uint32_t* flag) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

__device__ __forceinline__ uint32_t kind_count(uint32_t kind) { return kind == 0 ? 2u : (kind == 1 ? 3u : 4u); }

// Contact::energy > 0 at the detection configuration (potential.rs:39-65):
// active iff d < r, and for EE the edges are not parallel (|n|^2 >= 1e-30).
__device__ bool contact_active(const WorldView& w, uint32_t kind, uint4 v, double r) {
    d3 p0 = ld3(w.x, v.x), p1 = ld3(w.x, v.y), p2 = ld3(w.x, v.z), p3 = ld3(w.x, v.w);
    double d;
    if (kind == 0) {
        d = len(p0 - p1);
    } else if (kind == 1) {
        d3 u = p2 - p1;
        d3 ww = p0 - p1;
        double q = dot(ww, u) / dot(u, u);
        d3 dd = ww - u * q;
        d = sqrt(dot(dd, dd));
    } else if (kind == 2) {
        d3 n = cross(p2 - p1, p3 - p1);
        double h = dot(p0 - p1, n) / sqrt(dot(n, n));
        d = h < 0.0 ? -h : h;
    } else {
        d3 n = cross(p1 - p0, p3 - p2);
        if (dot(n, n) < 1e-30) return false;
        double h = dot(p0 - p2, n) / sqrt(dot(n, n));
        d = h < 0.0 ? -h : h;
    }
    if (d >= r) return false;
    if (d <= 0.0) return true;  // infinite energy
    return true;
}

// Rank tables for decoding contact keys: the distinct edges and triangles in
// lexicographic vertex order.
struct RankTables {
    const uint2* edge_verts;    // [edge ranks] (v0 < v1)
    const uint32_t* edge_id;    // [edge ranks] the world edge of each rank
    const uint3* tri_verts;     // [triangle ranks] (v1 < v2 < v3)
};

// Unique keys back to (kind, vertices, epsilon). The EE mollifier epsilon is
// 1e-3 |e0|^2 |f0|^2 (world.rs:174-178) in the operand order of the candidate
// pair that found the contact: moving-moving pairs have e < f by edge id,
// moving-fixed pairs the moving edge first (k_ee_query); each unordered edge
// pair is a candidate once, so that order is a function of the two edges.
__global__ void k_compact(WorldView w, const unsigned long long* key, const uint32_t* flag, const uint32_t* pos,
                          size_t n, RankTables r, uint32_t bits, uint32_t* c_kind, uint4* c_verts, double* c_eps) {
    const unsigned long long m = (1ull << bits) - 1ull;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        const uint32_t j = pos[i];
        const unsigned long long k = key[i];
        const uint32_t kind = (uint32_t)(k >> (2 * bits));
        const uint32_t a = (uint32_t)((k >> bits) & m), b = (uint32_t)(k & m);
        uint4 v = make_uint4(0, 0, 0, 0);
        double eps = 0.0;
        if (kind == 0) {
            v = make_uint4(a, b, 0, 0);
        } else if (kind == 1) {
            uint2 e = r.edge_verts[b];
            v = make_uint4(a, e.x, e.y, 0);
        } else if (kind == 2) {
            uint3 t = r.tri_verts[b];
            v = make_uint4(a, t.x, t.y, t.z);
        } else {
            uint2 e = r.edge_verts[a], f = r.edge_verts[b];
            v = make_uint4(e.x, e.y, f.x, f.y);
            uint32_t ea = r.edge_id[a], eb = r.edge_id[b];
            bool ma = e.x < w.moving, mb = f.x < w.moving;  // an edge moves if its smaller vertex does
            uint32_t first = (ma && mb) ? min(ea, eb) : (ma ? ea : eb);
            uint32_t second = first == ea ? eb : ea;
            eps = 1e-3 * w.rest_len2[first] * w.rest_len2[second];
        }
        c_kind[j] = kind;
        c_verts[j] = v;
        c_eps[j] = eps;
    }
}

// The unique-contact count from the dedup scan: last position + last flag.
__global__ void k_unique_count(const uint32_t* flag, const uint32_t* pos, size_t n_raw, unsigned long long* out) {
    *out = (unsigned long long)pos[n_raw - 1] + flag[n_raw - 1];
}

// n_ptr: the unique-contact count on the device (grids are sized for the raw count)
__global__ void k_contact_finalize(WorldView w, const uint32_t* c_kind, const uint4* c_verts,
                                   const unsigned long long* n_ptr, double r, uint32_t* inc_count,
                                   unsigned long long* active) {
    const size_t n = (size_t)*n_ptr;
    unsigned long long a = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t kind = c_kind[i];
        uint4 v = c_verts[i];
        if (contact_active(w, kind, v, r)) ++a;
        uint32_t vs[4] = {v.x, v.y, v.z, v.w};
        uint32_t cnt = kind_count(kind);
        for (uint32_t k = 0; k < cnt; ++k)
            if (vs[k] < w.moving) atomicAdd(&inc_count[vs[k]], 1u);
    }
    for (int s = 16; s > 0; s >>= 1) a += __shfl_xor_sync(0xffffffffu, a, s);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(active, a);
}

// Incidence rows: every moving vertex's contacts in ascending contact order,
// as the reference's incidence lists are (world.rs:386-393). Contacts are dealt
// into their rows (offsets: the exclusive scan of the per-vertex counts) with
// one atomic cursor per row, then every row is sorted on its own; rows are
// short (one vertex's contacts), so an insertion sort per thread suffices.
__global__ void k_incidence_scatter(uint32_t moving, const uint32_t* c_kind, const uint4* c_verts,
                                    const unsigned long long* n_ptr, const uint32_t* off, uint32_t* cursor,
                                    uint32_t* inc) {
    const size_t n = (size_t)*n_ptr;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint4 v = c_verts[i];
        uint32_t vs[4] = {v.x, v.y, v.z, v.w};
        uint32_t cnt = kind_count(c_kind[i]);
        for (uint32_t k = 0; k < cnt; ++k)
            if (vs[k] < moving) inc[off[vs[k]] + atomicAdd(&cursor[vs[k]], 1u)] = (uint32_t)i;
    }
}

__global__ void k_incidence_sort_rows(uint32_t moving, const uint32_t* off, uint32_t* inc) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < moving; v += gridDim.x * blockDim.x) {
        const uint32_t a = off[v], b = off[v + 1];
        for (uint32_t i = a + 1; i < b; ++i) {
            uint32_t x = inc[i];
            uint32_t j = i;
            while (j > a && inc[j - 1] > x) {
                inc[j] = inc[j - 1];
                --j;
            }
            inc[j] = x;
        }
    }
}

__global__ void k_radii(WorldView w, const unsigned long long* dist, double relaxation, double query_radius,
                        double* radii, double4* centers, unsigned long long* min_bits) {
    unsigned long long m = dbits(query_radius);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.moving; i += gridDim.x * blockDim.x) {
        unsigned long long b = dist[i];
        m = min(m, b);
        radii[i] = relaxation * bitsd(b);
        centers[i] = w.x[i];
    }
    for (int s = 16; s > 0; s >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, s));
    if ((threadIdx.x & 31) == 0) atomicMin(min_bits, m);
}

// validate_start face-face segment tests (world.rs:242-292).
__global__ void k_intersections(WorldView w, LbvhView tri_moving, LbvhView tri_fixed, const uint32_t* ex_pairs_off,
                                unsigned long long* first_hit, unsigned int* err) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.n_tri; i += gridDim.x * blockDim.x) {
        uint3 t = w.tri[i];
        bool t_fixed = t.x >= w.moving && t.y >= w.moving && t.z >= w.moving;
        Box q = w.tri_box[i];
        for (int k = 0; k < 3; ++k) {
            q.lo[k] = q.lo[k] - 1e-10;
            q.hi[k] = q.hi[k] + 1e-10;
        }
        uint32_t tv[3] = {t.x, t.y, t.z};
        auto visit = [&](uint32_t j) {
            uint3 qq = w.tri[j];
            bool q_fixed = qq.x >= w.moving && qq.y >= w.moving && qq.z >= w.moving;
            if (j <= i || (t_fixed && q_fixed)) return;
            uint32_t qv[3] = {qq.x, qq.y, qq.z};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    if (tv[a] != qv[b] && adjacent(w, tv[a], qv[b])) return;
            auto contains = [](const uint32_t* s, uint32_t v) { return s[0] == v || s[1] == v || s[2] == v; };
            bool hit = false;
            for (int k = 0; k < 3; ++k) {
                bool h1 = !contains(qv, tv[k]) && !contains(qv, tv[(k + 1) % 3]) &&
                          segment_triangle(ld3(w.x, tv[k]), ld3(w.x, tv[(k + 1) % 3]), ld3(w.x, qv[0]),
                                           ld3(w.x, qv[1]), ld3(w.x, qv[2]));
                bool h2 = !contains(tv, qv[k]) && !contains(tv, qv[(k + 1) % 3]) &&
                          segment_triangle(ld3(w.x, qv[k]), ld3(w.x, qv[(k + 1) % 3]), ld3(w.x, tv[0]),
                                           ld3(w.x, tv[1]), ld3(w.x, tv[2]));
                hit = hit || h1 || h2;
            }
            if (hit) atomicMin(first_hit, ((unsigned long long)i << 32) | j);
        };
        const QBox q32 = qbox(q);
        auto near = [&](float lx, float ly, float lz, float hx, float hy, float hz) {
            return overlap32(q32, lx, ly, lz, hx, hy, hz);
        };
        auto leaf_ok = [&](const Box& b) { return box_overlap(b, q); };
        bool ok = lbvh_walk<false>(tri_moving, 0u, near, leaf_ok, visit);
        if (!t_fixed) ok = lbvh_walk<false>(tri_fixed, 0u, near, leaf_ok, visit) && ok;
        if (!ok) atomicOr(err, DERR_STACK_OVERFLOW);
    }
}

// ------------------------------------------------------------------- host
TopologyHost build_topology(size_t n, const std::vector<std::array<uint32_t, 3>>& tris) {  // topology.rs:13-52
    TopologyHost top;
    std::map<std::array<uint32_t, 2>, uint32_t> map;
    std::vector<std::set<uint32_t>> neighbors(n);
    std::vector<std::vector<uint32_t>> opp;
    for (const auto& t : tris) {
        if (t[0] >= n || t[1] >= n || t[2] >= n || t[0] == t[1] || t[1] == t[2] || t[0] == t[2])
            throw Failure{CC_ERR_INVALID_ARGUMENT, "OGC: invalid triangle indices"};
        std::array<uint32_t, 3> te{};
        for (int k = 0; k < 3; ++k) {
            uint32_t a = t[k], b = t[(k + 1) % 3], c = t[(k + 2) % 3];
            std::array<uint32_t, 2> key{std::min(a, b), std::max(a, b)};
            auto it = map.find(key);
            uint32_t e;
            if (it == map.end()) {
                top.edges.push_back(key);
                opp.emplace_back();
                e = (uint32_t)(top.edges.size() - 1);
                map.emplace(key, e);
            } else {
                e = it->second;
            }
            opp[e].push_back(c);
            neighbors[a].insert(b);
            neighbors[b].insert(a);
            te[k] = e;
        }
        top.tri_edges.push_back(te);
    }
    for (const auto& o : opp)
        if (o.size() > 2)
            throw Failure{CC_ERR_INVALID_ARGUMENT, "OGC requires manifold triangle edges (at most two incident faces)"};
    top.tri = tris;
    top.opposites.resize(opp.size());
    for (size_t e = 0; e < opp.size(); ++e)
        top.opposites[e] = {opp[e].size() > 0 ? (int32_t)opp[e][0] : -1, opp[e].size() > 1 ? (int32_t)opp[e][1] : -1};
    top.nb_off.assign(n + 1, 0);
    for (size_t i = 0; i < n; ++i) top.nb_off[i + 1] = top.nb_off[i] + (uint32_t)neighbors[i].size();
    top.nb.reserve(top.nb_off[n]);
    for (size_t i = 0; i < n; ++i) top.nb.insert(top.nb.end(), neighbors[i].begin(), neighbors[i].end());
    return top;
}

World::World(const double* x_all, size_t n_all, const std::vector<std::array<uint32_t, 3>>& tris, size_t moving,
             const std::vector<std::array<uint32_t, 2>>& excluded, cudaStream_t stream)
    : stream_(stream), n_all_(n_all), moving_(moving) {
    if (moving > n_all) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid OGC positions"};
    for (size_t i = 0; i < 3 * n_all; ++i)
        if (!std::isfinite(x_all[i])) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid OGC positions"};
    top_ = build_topology(n_all, tris);
    n_tri_ = top_.tri.size();
    n_edge_ = top_.edges.size();
    auto X = [&](uint32_t i) { return mk(x_all[3 * i], x_all[3 * i + 1], x_all[3 * i + 2]); };
    for (const auto& t : top_.tri) {
        d3 a = X(t[0]), b = X(t[1]), c = X(t[2]);
        if (len2(cross(b - a, c - a)) < 1e-24) throw Failure{CC_ERR_INVALID_ARGUMENT, "OGC degenerate initial face"};
    }
    // excluded neighbours, sorted (world.rs:183-197)
    std::set<std::array<uint32_t, 2>> ex;
    for (auto e : excluded) ex.insert({std::min(e[0], e[1]), std::max(e[0], e[1])});
    std::vector<std::vector<uint32_t>> exn(n_all);
    for (const auto& e : ex) {
        if (e[1] >= n_all) throw Failure{CC_ERR_INVALID_ARGUMENT, "OGC invalid excluded vertex"};
        exn[e[0]].push_back(e[1]);
        exn[e[1]].push_back(e[0]);
    }
    std::vector<uint32_t> ex_off(n_all + 1, 0), exv;
    for (size_t i = 0; i < n_all; ++i) {
        std::sort(exn[i].begin(), exn[i].end());
        ex_off[i + 1] = ex_off[i] + (uint32_t)exn[i].size();
        exv.insert(exv.end(), exn[i].begin(), exn[i].end());
    }
    std::vector<double> rl2(n_edge_);
    for (size_t e = 0; e < n_edge_; ++e) rl2[e] = len2(X(top_.edges[e][0]) - X(top_.edges[e][1]));
    // contact-key ranks: distinct edges and triangles (vertex sets) in
    // lexicographic order; equal sets share a rank
    std::vector<uint32_t> edge_rank(n_edge_), tri_rank(n_tri_), rank_edge_id;
    std::vector<uint2> rank_edge_verts;
    std::vector<uint3> rank_tri_verts;
    {
        std::vector<uint32_t> ord(n_edge_);
        for (size_t e = 0; e < n_edge_; ++e) ord[e] = (uint32_t)e;
        std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
            return top_.edges[a] < top_.edges[b] || (top_.edges[a] == top_.edges[b] && a < b);
        });
        for (size_t k = 0; k < n_edge_; ++k) {
            const auto& ev = top_.edges[ord[k]];
            if (k == 0 || ev != top_.edges[ord[k - 1]]) {
                rank_edge_verts.push_back(make_uint2(ev[0], ev[1]));
                rank_edge_id.push_back(ord[k]);
            }
            edge_rank[ord[k]] = (uint32_t)rank_edge_verts.size() - 1;
        }
        std::vector<std::array<uint32_t, 3>> sorted(n_tri_);
        for (size_t t = 0; t < n_tri_; ++t) {
            sorted[t] = top_.tri[t];
            std::sort(sorted[t].begin(), sorted[t].end());
        }
        std::vector<uint32_t> tord(n_tri_);
        for (size_t t = 0; t < n_tri_; ++t) tord[t] = (uint32_t)t;
        std::sort(tord.begin(), tord.end(), [&](uint32_t a, uint32_t b) {
            return sorted[a] < sorted[b] || (sorted[a] == sorted[b] && a < b);
        });
        for (size_t k = 0; k < n_tri_; ++k) {
            const auto& tv = sorted[tord[k]];
            if (k == 0 || tv != sorted[tord[k - 1]]) rank_tri_verts.push_back(make_uint3(tv[0], tv[1], tv[2]));
            tri_rank[tord[k]] = (uint32_t)rank_tri_verts.size() - 1;
        }
    }
    key_bits_ = 1;
    while ((1ull << key_bits_) < std::max<uint64_t>({(uint64_t)n_all_, rank_edge_verts.size(), rank_tri_verts.size()}))
        ++key_bits_;
    if (key_bits_ > 31) throw Failure{CC_ERR_INVALID_ARGUMENT, "OGC: more than 2^31 vertices, edges or triangles"};
    for (size_t t = 0; t < n_tri_; ++t) {
        const auto& v = top_.tri[t];
        (v[0] < moving || v[1] < moving || v[2] < moving ? tri_moving_h_ : tri_fixed_h_).push_back((uint32_t)t);
    }
    for (size_t e = 0; e < n_edge_; ++e) {
        const auto& v = top_.edges[e];
        (v[0] < moving || v[1] < moving ? edge_moving_h_ : edge_fixed_h_).push_back((uint32_t)e);
    }
    std::vector<uint3> tri_d(n_tri_), te_d(n_tri_);
    for (size_t t = 0; t < n_tri_; ++t) {
        tri_d[t] = make_uint3(top_.tri[t][0], top_.tri[t][1], top_.tri[t][2]);
        te_d[t] = make_uint3(top_.tri_edges[t][0], top_.tri_edges[t][1], top_.tri_edges[t][2]);
    }
    std::vector<uint2> e_d(n_edge_);
    std::vector<int2> o_d(n_edge_);
    for (size_t e = 0; e < n_edge_; ++e) {
        e_d[e] = make_uint2(top_.edges[e][0], top_.edges[e][1]);
        o_d[e] = make_int2(top_.opposites[e][0], top_.opposites[e][1]);
    }
    std::vector<double4> xh(n_all);
    for (size_t i = 0; i < n_all; ++i) xh[i] = make_double4(x_all[3 * i], x_all[3 * i + 1], x_all[3 * i + 2], 0.0);
    tri_.upload(tri_d, stream_);
    tri_edges_.upload(te_d, stream_);
    edges_.upload(e_d, stream_);
    opposites_.upload(o_d, stream_);
    nb_off_.upload(top_.nb_off, stream_);
    nb_.upload(top_.nb, stream_);
    ex_off_.upload(ex_off, stream_);
    ex_.upload(exv, stream_);
    rest_len2_.upload(rl2, stream_);
    edge_rank_.upload(edge_rank, stream_);
    tri_rank_.upload(tri_rank, stream_);
    rank_edge_verts_.upload(rank_edge_verts, stream_);
    rank_edge_id_.upload(rank_edge_id, stream_);
    rank_tri_verts_.upload(rank_tri_verts, stream_);
    x_.upload(xh, stream_);
    fixed_x_.upload(xh.data() + moving, n_all - moving, stream_);
    tri_box_.reserve(n_tri_);
    edge_box_.reserve(n_edge_);
    tri_moving_.upload(tri_moving_h_, stream_);
    tri_fixed_.upload(tri_fixed_h_, stream_);
    edge_moving_.upload(edge_moving_h_, stream_);
    edge_fixed_.upload(edge_fixed_h_, stream_);
    dist_bits_.reserve(n_all);
    radii_.reserve(moving);
    centers_.reserve(moving);
    cache_centers_.reserve(moving);
    inc_count_.reserve(moving + 1);
    inc_off_.reserve(moving + 1);
    inc_cursor_.reserve(moving + 1);
    stats_d_.reserve(1);
    stats_h_.reserve(1);
    std::memset(stats_h_.ptr, 0, sizeof(DetectStats));
    CC_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    CC_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    CC_CUDA(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
    // fixed trees are built once: fixed geometry never moves
    stats_d_.zero(1, stream_);
    refit(false);
    tree_tri_fixed_.build(tri_box_.ptr, tri_fixed_.ptr, (uint32_t)tri_fixed_h_.size(), stream_, &stats_d_.ptr->error);
    tree_edge_fixed_.build(edge_box_.ptr, edge_fixed_.ptr, (uint32_t)edge_fixed_h_.size(), stream_, &stats_d_.ptr->error);
    CC_CUDA(cudaStreamSynchronize(stream_));
}

World::~World() {
    for (cudaEvent_t e : phase_ev_)
        if (e) cudaEventDestroy(e);
    if (fork_) cudaEventDestroy(fork_);
    if (join_) cudaEventDestroy(join_);
    if (side_) cudaStreamDestroy(side_);
}

WorldView World::view() const {
    return {(uint32_t)n_all_,
            (uint32_t)moving_,
            (uint32_t)n_tri_,
            (uint32_t)n_edge_,
            tri_.ptr,
            tri_edges_.ptr,
            edges_.ptr,
            opposites_.ptr,
            nb_off_.ptr,
            nb_.ptr,
            ex_off_.ptr,
            ex_.ptr,
            rest_len2_.ptr,
            x_.ptr,
            tri_box_.ptr,
            edge_box_.ptr};
}

ContactsView World::contacts() const {
    return {(uint32_t)stats_h_.ptr->n_contacts, c_kind_.ptr, c_verts_.ptr, c_eps_.ptr, inc_off_.ptr, inc_.ptr,
            centers_.ptr, radii_.ptr};
}

void World::refit(bool check_fixed) {
    size_t work = std::max(n_all_, std::max(n_tri_, n_edge_));
    k_refit<<<grid_for(work, 256), 256, 0, stream_>>>(view(), fixed_x_.ptr, check_fixed ? 1 : 0, &stats_d_.ptr->error);
    ++launches_;
    CC_CUDA(cudaGetLastError());
}

void World::sync_stats() {
    CC_CUDA(cudaMemcpyAsync(stats_h_.ptr, stats_d_.ptr, sizeof(DetectStats), cudaMemcpyDeviceToHost, stream_));
    CC_CUDA(cudaStreamSynchronize(stream_));
}

static void raise_device_error(unsigned int e) {
    if (e & DERR_NONFINITE_STATE) throw Failure{CC_ERR_INVALID_STATE, "OGC invalid position array"};
    if (e & DERR_FIXED_MOVED) throw Failure{CC_ERR_INVALID_STATE, "OGC fixed geometry changed; rebuild the world"};
    if (e & DERR_DEGENERATE_FACE) throw Failure{CC_ERR_CONTACT, "OGC degenerate face; step rejected"};
    if (e & DERR_STACK_OVERFLOW) throw Failure{CC_ERR_CUDA, "OGC LBVH traversal stack overflow"};
    if (e & DERR_SORT_WAIT) throw Failure{CC_ERR_DEVICE_TIMEOUT, "OGC radix sort look-back wait gave up"};
}

// The moving trees for the current primitive boxes: the triangle tree on the
// side stream, the edge tree on the main one (after fork_, recorded here, the
// side stream waits for the boxes). The caller joins the streams.
int World::update_trees() {
    bool build = !tree_tri_moving_.built || !tree_edge_moving_.built;
    if (!build && tree_period_ > 0 && rebuilds_since_build_ + 1 >= tree_period_) build = true;
    if (build) {
        rebuilds_since_build_ = 0;
        ++tree_builds_;
    } else {
        ++rebuilds_since_build_;
    }
    CC_CUDA(cudaEventRecord(fork_, stream_));
    CC_CUDA(cudaStreamWaitEvent(side_, fork_, 0));
    unsigned int* err = &stats_d_.ptr->error;
    int n = build ? tree_tri_moving_.build(tri_box_.ptr, tri_moving_.ptr, (uint32_t)tri_moving_h_.size(), side_, err)
                  : tree_tri_moving_.refit(tri_box_.ptr, side_);
    n += build ? tree_edge_moving_.build(edge_box_.ptr, edge_moving_.ptr, (uint32_t)edge_moving_h_.size(), stream_, err)
               : tree_edge_moving_.refit(edge_box_.ptr, stream_);
    if (build) n += order_points();
    return n;
}

// A Morton order of all points (the VF queries' order), from the current
// positions; refreshed with the trees' topology.
int World::order_points() {
    const uint32_t n = (uint32_t)n_all_;
    if (n == 0) return 0;
    pt_bounds_.reserve(6);
    pt_code_.reserve(n);
    pt_code_s_.reserve(n);
    pt_ids_.reserve(n);
    point_order_.reserve(n);
    k_bounds_init<<<1, 32, 0, stream_>>>(pt_bounds_.ptr);
    k_point_bounds<<<grid_for(n, 256), 256, 0, stream_>>>(x_.ptr, n, pt_bounds_.ptr);
    k_point_morton<<<grid_for(n, 256), 256, 0, stream_>>>(x_.ptr, n, pt_bounds_.ptr, pt_code_.ptr, pt_ids_.ptr);
    CC_CUDA(cudaGetLastError());
    return 3 + sorter_.sort_pairs(pt_code_.ptr, pt_code_s_.ptr, pt_ids_.ptr, point_order_.ptr, n, 63, stream_,
                                  &stats_d_.ptr->error, DERR_SORT_WAIT);
}

void World::build_candidates(double R, double skin) {
    double search = R + 2.0 * skin + 1e-12;  // candidates.rs:23-28
    double search2 = search * search;
    launches_ += update_trees();
    LbvhView tm = tree_tri_moving_.view(), tf = tree_tri_fixed_.view();
    LbvhView em = tree_edge_moving_.view(), ef = tree_edge_fixed_.view();
    const uint32_t* edges_in_leaf_order = tree_edge_moving_.leaf_prim.ptr;
    if (vf_cap_ == 0) {
        // generous first capacities: the in-plane pairs of a sheet at the
        // candidate radius alone reach ~60 per edge
        vf_cap_ = std::max<size_t>(1024, 48 * n_all_);
        ee_cap_ = std::max<size_t>(1024, 96 * n_edge_);
    }
    for (int attempt = 0; attempt < 8; ++attempt) {
        vf_.reserve(vf_cap_);
        ee_.reserve(ee_cap_);
        // the VF query on the side stream (after its tree), the EE query on
        // the main one: the VF query's one thread per point leaves most of the
        // GPU to the EE query
        // (the side stream also waits for the point order, made on the main
        // stream when the trees are built)
        CC_CUDA(cudaEventRecord(fork_, stream_));
        CC_CUDA(cudaStreamWaitEvent(side_, fork_, 0));
        CC_CUDA(cudaMemsetAsync(&stats_d_.ptr->n_vf, 0, sizeof(unsigned long long), side_));
        CC_CUDA(cudaMemsetAsync(&stats_d_.ptr->n_ee, 0, sizeof(unsigned long long), stream_));
        k_vf_query<<<grid_for(n_all_, 128), 128, 0, side_>>>(view(), point_order_.ptr, tm, tf, search2, vf_.ptr,
                                                              vf_cap_, &stats_d_.ptr->n_vf, &stats_d_.ptr->error);
        k_ee_query<<<grid_for(edge_moving_h_.size(), 128), 128, 0, stream_>>>(
            view(), edges_in_leaf_order, (uint32_t)edge_moving_h_.size(), em, ef, search2, ee_.ptr, ee_cap_,
            &stats_d_.ptr->n_ee, &stats_d_.ptr->error);
        launches_ += 2;
        CC_CUDA(cudaGetLastError());
        CC_CUDA(cudaEventRecord(join_, side_));
        CC_CUDA(cudaStreamWaitEvent(stream_, join_, 0));
        sync_stats();
        raise_device_error(stats_h_.ptr->error);
        bool grow = false;
        if (stats_h_.ptr->n_vf > vf_cap_) {
            vf_cap_ = (size_t)(stats_h_.ptr->n_vf * 1.5) + 1024;
            vf_.release();
            grow = true;
        }
        if (stats_h_.ptr->n_ee > ee_cap_) {
            ee_cap_ = (size_t)(stats_h_.ptr->n_ee * 1.5) + 1024;
            ee_.release();
            grow = true;
        }
        if (!grow) return;
    }
    throw Failure{CC_ERR_CUDA, "OGC candidate buffers could not be sized"};
}

__global__ void k_reset_stats(DetectStats* s, double query_radius) {
    s->n_raw = 0;
    s->n_contacts = 0;
    s->active = 0;
    s->vf_count = 0;
    s->ee_count = 0;
    s->rejections = 0;
    s->min_dist_bits = dbits(query_radius);
    s->n_incident = 0;
    s->max_move_bits = 0;
    s->max_abs_bits = 0;
    s->error = 0;
    s->rebuild = 0;
}

void World::mark(int k) {
    if (!profile_) return;
    if (!phase_ev_[k]) CC_CUDA(cudaEventCreate(&phase_ev_[k]));
    CC_CUDA(cudaEventRecord(phase_ev_[k], stream_));
}

void World::detect(double query_radius, double radius, double relaxation, double stiffness, bool check_fixed,
                   bool prune) {
    (void)stiffness;
    query_radius_ = query_radius;
    DetectStats* sd = stats_d_.ptr;
    mark(0);
    // reset per-detection counters (keep n_vf/n_ee of the cache)
    k_reset_stats<<<1, 1, 0, stream_>>>(sd, query_radius);
    refit(check_fixed);
    k_cover_and_scale<<<grid_for(n_all_, 256), 256, 0, stream_>>>(view(), cache_centers_.ptr, cache_valid_ ? 1 : 0,
                                                                   &sd->max_move_bits, &sd->max_abs_bits);
    launches_ += 2;
    CC_CUDA(cudaGetLastError());
    mark(1);
    sync_stats();
    raise_device_error(stats_h_.ptr->error);
    double max_move;
    {
        unsigned long long b = stats_h_.ptr->max_move_bits;
        std::memcpy(&max_move, &b, 8);
    }
    // Candidates::covers (candidates.rs:15-22)
    bool rebuild = !(cache_valid_ && query_radius <= cache_R_ && max_move <= cache_skin_ * cache_skin_);
    if (rebuild) {
        double R = std::fmax(std::ceil(query_radius / radius) * radius, query_radius);  // world.rs:345
        build_candidates(R, radius);
        cache_valid_ = true;
        cache_R_ = R;
        cache_skin_ = radius;
        CC_CUDA(cudaMemcpyAsync(cache_centers_.ptr, x_.ptr, moving_ * sizeof(double4), cudaMemcpyDeviceToDevice,
                                stream_));
    }
    mark(2);
    unsigned long long n_vf = stats_h_.ptr->n_vf, n_ee = stats_h_.ptr->n_ee;
    // narrow phase
    if (raw_cap_ == 0) raw_cap_ = std::max<size_t>(4096, (size_t)(n_vf + n_ee) / 2 + 4096);
    for (int attempt = 0; attempt < 8; ++attempt) {
        raw_key_.reserve(raw_cap_);
        CC_CUDA(cudaMemsetAsync(&sd->n_raw, 0, sizeof(unsigned long long), stream_));
        CC_CUDA(cudaMemsetAsync(&sd->vf_count, 0, sizeof(unsigned long long) * 3, stream_));
        unsigned long long qbits;
        std::memcpy(&qbits, &query_radius, 8);
        k_fill_u64<<<grid_for(n_all_, 256), 256, 0, stream_>>>(dist_bits_.ptr, n_all_, qbits);
        NarrowOut o{raw_key_.ptr,    raw_cap_,           &sd->n_raw,        dist_bits_.ptr, &sd->vf_count,
                    &sd->ee_count,   &sd->rejections,    edge_rank_.ptr,    tri_rank_.ptr,  key_bits_};
        unsigned long long total = n_vf + n_ee;
        k_narrow<<<grid_for((size_t)total, 128), 128, 0, stream_>>>(view(), vf_.ptr, n_vf, ee_.ptr, n_ee, query_radius,
                                                                    &sd->max_abs_bits, prune ? 1 : 0, o);
        launches_ += 2;
        CC_CUDA(cudaGetLastError());
        mark(3);
        sync_stats();
        if (stats_h_.ptr->n_raw <= raw_cap_) break;
        raw_cap_ = (size_t)(stats_h_.ptr->n_raw * 1.5) + 4096;
        raw_key_.release();
    }
    size_t n_raw = stats_h_.ptr->n_raw;
    if (n_raw > raw_cap_) throw Failure{CC_ERR_CUDA, "OGC contact buffer could not be sized"};
    // canonical order: one keys-only radix sort over the 2W + 2 bits the keys
    // use, then dedup. The unique count stays on the device (sd->n_contacts):
    // the kernels below read it and their grids and buffers are sized for
    // n_raw, so the host learns it only at the detection's final read-back.
    if (n_raw > 0) {
        raw_key_s_.reserve(n_raw);
        uniq_flag_.reserve(n_raw);
        uniq_pos_.reserve(n_raw);
        launches_ += sorter_.sort_keys(raw_key_.ptr, raw_key_s_.ptr, n_raw, (int)(2 * key_bits_ + 2), stream_,
                                       &sd->error, DERR_SORT_WAIT);
        k_unique_flags<<<grid_for(n_raw, 256), 256, 0, stream_>>>(raw_key_s_.ptr, n_raw, uniq_flag_.ptr);
        launches_ += exclusive_sum(uniq_flag_.ptr, uniq_pos_.ptr, n_raw, scan_tmp_, stream_);
        k_unique_count<<<1, 1, 0, stream_>>>(uniq_flag_.ptr, uniq_pos_.ptr, n_raw, &sd->n_contacts);
        c_kind_.reserve(n_raw);
        c_verts_.reserve(n_raw);
        c_eps_.reserve(n_raw);
        RankTables rt{rank_edge_verts_.ptr, rank_edge_id_.ptr, rank_tri_verts_.ptr};
        k_compact<<<grid_for(n_raw, 256), 256, 0, stream_>>>(view(), raw_key_s_.ptr, uniq_flag_.ptr, uniq_pos_.ptr,
                                                             n_raw, rt, key_bits_, c_kind_.ptr, c_verts_.ptr,
                                                             c_eps_.ptr);
        launches_ += 3;
    }
    // incidence (moving vertices), active count, radii
    CC_CUDA(cudaMemsetAsync(inc_count_.ptr, 0, (moving_ + 1) * sizeof(uint32_t), stream_));
    CC_CUDA(cudaMemsetAsync(inc_cursor_.ptr, 0, (moving_ + 1) * sizeof(uint32_t), stream_));
    if (n_raw > 0) {
        k_contact_finalize<<<grid_for(n_raw, 256), 256, 0, stream_>>>(view(), c_kind_.ptr, c_verts_.ptr,
                                                                      &sd->n_contacts, radius, inc_count_.ptr,
                                                                      &sd->active);
        ++launches_;
    }
    launches_ += exclusive_sum(inc_count_.ptr, inc_off_.ptr, moving_ + 1, scan_tmp_, stream_);
    size_t n_inc_bound = 4 * n_raw;  // at most 4 moving vertices per contact
    inc_.reserve(std::max<size_t>(n_inc_bound, 1));
    if (n_raw > 0) {
        k_incidence_scatter<<<grid_for(n_raw, 256), 256, 0, stream_>>>((uint32_t)moving_, c_kind_.ptr, c_verts_.ptr,
                                                                        &sd->n_contacts, inc_off_.ptr, inc_cursor_.ptr,
                                                                        inc_.ptr);
        k_incidence_sort_rows<<<grid_for(moving_, 256), 256, 0, stream_>>>((uint32_t)moving_, inc_off_.ptr, inc_.ptr);
        launches_ += 2;
    }
    if (moving_ > 0)
        k_radii<<<grid_for(moving_, 256), 256, 0, stream_>>>(view(), dist_bits_.ptr, relaxation, query_radius,
                                                             radii_.ptr, centers_.ptr, &sd->min_dist_bits);
    if (moving_ > 0) ++launches_;
    CC_CUDA(cudaMemcpyAsync(&sd->n_incident, inc_off_.ptr + moving_, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            stream_));
    CC_CUDA(cudaGetLastError());
    mark(4);
    sync_stats();
    stats_h_.ptr->n_incident &= 0xffffffffull;
    stats_h_.ptr->rebuild = rebuild ? 1 : 0;
    if (profile_) {
        float t[4];
        for (int k = 0; k < 4; ++k) CC_CUDA(cudaEventElapsedTime(&t[k], phase_ev_[k], phase_ev_[k + 1]));
        phase_ms_.refit = t[0];
        phase_ms_.candidates = t[1];
        phase_ms_.narrow = t[2];
        phase_ms_.canonical = t[3];
    }
    raise_device_error(stats_h_.ptr->error);
}

void World::validate_start() {  // world.rs:242-307
    CC_CUDA(cudaMemsetAsync(&stats_d_.ptr->error, 0, sizeof(unsigned int), stream_));
    unsigned long long none = ~0ull;
    CC_CUDA(cudaMemcpyAsync(&stats_d_.ptr->intersect_key, &none, 8, cudaMemcpyHostToDevice, stream_));
    refit(true);
    launches_ += update_trees();
    CC_CUDA(cudaEventRecord(join_, side_));
    CC_CUDA(cudaStreamWaitEvent(stream_, join_, 0));
    k_intersections<<<grid_for(n_tri_, 128), 128, 0, stream_>>>(view(), tree_tri_moving_.view(),
                                                                tree_tri_fixed_.view(), nullptr,
                                                                &stats_d_.ptr->intersect_key, &stats_d_.ptr->error);
    CC_CUDA(cudaGetLastError());
    sync_stats();
    raise_device_error(stats_h_.ptr->error);
    unsigned long long hit = stats_h_.ptr->intersect_key;
    if (hit != ~0ull) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "OGC initial intersection between faces %llu and %llu; reset/rearrange before simulating",
                      hit >> 32, hit & 0xffffffffull);
        throw Failure{CC_ERR_CONTACT, buf};
    }
    bool was_valid = cache_valid_;
    double R = cache_R_, skin = cache_skin_;
    (void)was_valid;
    (void)R;
    (void)skin;
    detect(1e-5, 1e-5, 0.45, 100000.0, true);
    double md;
    unsigned long long b = stats_h_.ptr->min_dist_bits;
    std::memcpy(&md, &b, 8);
    if (md <= 1e-10)
        throw Failure{CC_ERR_CONTACT, "OGC initial touching/coplanar features: separation must be positive"};
}

void World::fresh_pairs(double search, std::vector<uint32_t>& vf, std::vector<uint32_t>& ee) {
    CC_CUDA(cudaMemsetAsync(&stats_d_.ptr->error, 0, sizeof(unsigned int), stream_));
    refit(true);
    sync_stats();
    raise_device_error(stats_h_.ptr->error);
    // exact search radius: build_candidates adds 2*skin + 1e-12, so pass R
    // such that the sum equals `search`
    double search2 = search * search;
    launches_ += update_trees();
    CC_CUDA(cudaEventRecord(join_, side_));
    CC_CUDA(cudaStreamWaitEvent(stream_, join_, 0));
    LbvhView tm = tree_tri_moving_.view(), tf = tree_tri_fixed_.view();
    LbvhView em = tree_edge_moving_.view(), ef = tree_edge_fixed_.view();
    size_t vcap = std::max<size_t>(1024, 16 * n_all_), ecap = std::max<size_t>(1024, 32 * n_edge_);
    for (int attempt = 0; attempt < 8; ++attempt) {
        DBuf<uint2> a, b;
        a.reserve(vcap);
        b.reserve(ecap);
        // own counters: n_vf / n_ee in the stats belong to the candidate cache
        fresh_counts_.reserve(2);
        CC_CUDA(cudaMemsetAsync(fresh_counts_.ptr, 0, 2 * sizeof(unsigned long long), stream_));
        k_vf_query<<<grid_for(n_all_, 128), 128, 0, stream_>>>(view(), point_order_.ptr, tm, tf, search2, a.ptr,
                                                                vcap, fresh_counts_.ptr, &stats_d_.ptr->error);
        k_ee_query<<<grid_for(edge_moving_h_.size(), 128), 128, 0, stream_>>>(
            view(), tree_edge_moving_.leaf_prim.ptr, (uint32_t)edge_moving_h_.size(), em, ef, search2, b.ptr, ecap,
            fresh_counts_.ptr + 1, &stats_d_.ptr->error);
        CC_CUDA(cudaGetLastError());
        unsigned long long counts[2];
        CC_CUDA(cudaMemcpyAsync(counts, fresh_counts_.ptr, sizeof counts, cudaMemcpyDeviceToHost, stream_));
        sync_stats();
        raise_device_error(stats_h_.ptr->error);
        size_t nv = counts[0], ne = counts[1];
        if (nv > vcap || ne > ecap) {
            vcap = std::max(vcap, nv + 1);
            ecap = std::max(ecap, ne + 1);
            continue;
        }
        std::vector<uint2> hv(nv), he(ne);
        if (nv) CC_CUDA(cudaMemcpy(hv.data(), a.ptr, nv * sizeof(uint2), cudaMemcpyDeviceToHost));
        if (ne) CC_CUDA(cudaMemcpy(he.data(), b.ptr, ne * sizeof(uint2), cudaMemcpyDeviceToHost));
        std::vector<std::array<uint32_t, 2>> sv(nv), se(ne);
        for (size_t i = 0; i < nv; ++i) sv[i] = {hv[i].x, hv[i].y};
        for (size_t i = 0; i < ne; ++i) se[i] = {he[i].x, he[i].y};
        std::sort(sv.begin(), sv.end());
        std::sort(se.begin(), se.end());
        vf.clear();
        ee.clear();
        for (auto& p : sv) vf.insert(vf.end(), p.begin(), p.end());
        for (auto& p : se) ee.insert(ee.end(), p.begin(), p.end());
        return;
    }
    throw Failure{CC_ERR_CUDA, "OGC candidate buffers could not be sized"};
}

void World::download(std::vector<uint32_t>& kind, std::vector<uint32_t>& verts, std::vector<double>& eps,
                     std::vector<uint64_t>& inc_off, std::vector<uint32_t>& inc, std::vector<double>& radii) {
    size_t n = stats_h_.ptr->n_contacts;
    kind.resize(n);
    verts.resize(4 * n);
    eps.resize(n);
    if (n) {
        CC_CUDA(cudaMemcpy(kind.data(), c_kind_.ptr, n * 4, cudaMemcpyDeviceToHost));
        CC_CUDA(cudaMemcpy(verts.data(), c_verts_.ptr, n * 16, cudaMemcpyDeviceToHost));
        CC_CUDA(cudaMemcpy(eps.data(), c_eps_.ptr, n * 8, cudaMemcpyDeviceToHost));
    }
    std::vector<uint32_t> off(moving_ + 1);
    CC_CUDA(cudaMemcpy(off.data(), inc_off_.ptr, (moving_ + 1) * 4, cudaMemcpyDeviceToHost));
    inc_off.assign(off.begin(), off.end());
    inc.resize(off[moving_]);
    if (!inc.empty()) CC_CUDA(cudaMemcpy(inc.data(), inc_.ptr, inc.size() * 4, cudaMemcpyDeviceToHost));
    for (size_t v = 0; v < moving_; ++v) std::sort(inc.begin() + off[v], inc.begin() + off[v + 1]);
    radii.resize(moving_);
    if (moving_) CC_CUDA(cudaMemcpy(radii.data(), radii_.ptr, moving_ * 8, cudaMemcpyDeviceToHost));
}

}  // namespace cc

// ---------------------------------------------------------------------------
// Allocation-free variant of the narrow-phase distance / radius pass.
//
// Some callers cannot call cudaMalloc: an editor's fixed-budget frame worker,
// where an allocation (and the device-wide synchronisation that cudaFree
// implies) would stall the frame, and hosts that reserve all device memory
// up front and hand this library only their own buffers. For them this entry
// point keeps its per-vertex scratch (the running minimum distance of every
// vertex) in the file-scope array below instead of allocating it. The caller
// passes all inputs and outputs as device pointers.
//
// The array holds kNoAllocMaxVertices distance slots plus the global minimum
// and an error word; every GPU that loads the library holds it (2 MiB) until
// the process exits. Every call shares it and it keeps the previous call's
// contents, so each call clears what must start from a known value, and two
// calls whose kernels overlap on the GPU (e.g. on different streams) race.
// Calls made through this entry point from several host threads are
// serialised by a mutex held from the first launch to the read-back, so
// their launches cannot interleave; kernels that another process or another
// copy of the library runs on the same array are outside its reach.
namespace cc {

constexpr uint64_t kNoAllocMaxVertices = 262144;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocMaxVertices + 2];

struct NoAllocArgs {
    const double* x;  // [n_all][3]
    uint32_t n_all, moving, n_tri, n_edge;
    const uint32_t* tri;    // [n_tri][3]
    const uint32_t* edges;  // [n_edge][2]
    const uint32_t* vf;     // [n_vf][2]: point, triangle
    const uint32_t* ee;     // [n_ee][2]: edge, edge (reference operand order)
    unsigned long long n_vf, n_ee;
    double query_radius, relaxation;
    unsigned long long* scratch;  // device address of g_noalloc_scratch
};

__device__ __forceinline__ d3 na_x(const NoAllocArgs& a, uint32_t i) {
    return mk(a.x[3 * (size_t)i], a.x[3 * (size_t)i + 1], a.x[3 * (size_t)i + 2]);
}

__global__ void k_noalloc_clear(NoAllocArgs a) {
    unsigned long long q = dbits(a.query_radius);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_all; i += gridDim.x * blockDim.x)
        a.scratch[i] = q;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.scratch[kNoAllocMaxVertices] = q;
        a.scratch[kNoAllocMaxVertices + 1] = 0ull;
    }
}

// OgcWorld::scan distances (world.rs:461-524): the minimum over pairs with
// d < query_radius, for the point and the triangle's corners (VF) and the
// four edge endpoints (EE). Out-of-range indices set the error word.
__global__ void k_noalloc_pairs(NoAllocArgs a) {
    unsigned long long* dist = a.scratch;
    unsigned long long total = a.n_vf + a.n_ee;
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        if (k < a.n_vf) {
            uint32_t v = a.vf[2 * k], t = a.vf[2 * k + 1];
            if (v >= a.n_all || t >= a.n_tri) {
                atomicOr(&dist[kNoAllocMaxVertices + 1], 1ull);
                continue;
            }
            uint32_t i0 = a.tri[3 * (size_t)t], i1 = a.tri[3 * (size_t)t + 1], i2 = a.tri[3 * (size_t)t + 2];
            if (i0 >= a.n_all || i1 >= a.n_all || i2 >= a.n_all) {
                atomicOr(&dist[kNoAllocMaxVertices + 1], 1ull);
                continue;
            }
            d3 xv = na_x(a, v);
            int kind, which;
            d3 p = closest_on_triangle(xv, na_x(a, i0), na_x(a, i1), na_x(a, i2), kind, which);
            double d = len(xv - p);
            if (d >= a.query_radius) continue;
            unsigned long long db = dbits(d);
            atomicMin(&dist[v], db);
            atomicMin(&dist[i0], db);
            atomicMin(&dist[i1], db);
            atomicMin(&dist[i2], db);
        } else {
            unsigned long long kk = k - a.n_vf;
            uint32_t e = a.ee[2 * kk], f = a.ee[2 * kk + 1];
            if (e >= a.n_edge || f >= a.n_edge) {
                atomicOr(&dist[kNoAllocMaxVertices + 1], 1ull);
                continue;
            }
            uint32_t e0 = a.edges[2 * (size_t)e], e1 = a.edges[2 * (size_t)e + 1];
            uint32_t f0 = a.edges[2 * (size_t)f], f1 = a.edges[2 * (size_t)f + 1];
            if (e0 >= a.n_all || e1 >= a.n_all || f0 >= a.n_all || f1 >= a.n_all) {
                atomicOr(&dist[kNoAllocMaxVertices + 1], 1ull);
                continue;
            }
            d3 pa = na_x(a, e0), pb = na_x(a, e1), pc = na_x(a, f0), pd = na_x(a, f1);
            double s, t;
            closest_segments(pa, pb, pc, pd, s, t);
            d3 p = pa + (pb - pa) * s;
            d3 q = pc + (pd - pc) * t;
            double dist_pq = len(p - q);
            if (dist_pq >= a.query_radius) continue;
            unsigned long long db = dbits(dist_pq);
            atomicMin(&dist[e0], db);
            atomicMin(&dist[e1], db);
            atomicMin(&dist[f0], db);
            atomicMin(&dist[f1], db);
        }
    }
}

// radii = relaxation * d and the minimum over moving vertices (world.rs:394-414)
__global__ void k_noalloc_radii(NoAllocArgs a, double* radii) {
    unsigned long long m = dbits(a.query_radius);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.moving; i += gridDim.x * blockDim.x) {
        unsigned long long b = a.scratch[i];
        m = min(m, b);
        radii[i] = a.relaxation * bitsd(b);
    }
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMin(&a.scratch[kNoAllocMaxVertices], m);
}

__global__ void k_noalloc_store_min(NoAllocArgs a, double* minimum_distance) {
    *minimum_distance = bitsd(a.scratch[kNoAllocMaxVertices]);
}

}  // namespace cc

namespace {
std::mutex g_noalloc_mutex;
unsigned long long* g_noalloc_address[128] = {nullptr};
}  // namespace

extern "C" int32_t cc_ogc_radii_noalloc(const double* x, uint64_t n_all, uint64_t moving, const uint32_t* triangles,
                                        uint64_t n_triangles, const uint32_t* edges, uint64_t n_edges,
                                        const uint32_t* vf_pairs, uint64_t n_vf, const uint32_t* ee_pairs,
                                        uint64_t n_ee, double query_radius, double relaxation, double* radii,
                                        double* minimum_distance, void* stream) {
    using namespace cc;
    if (n_all > kNoAllocMaxVertices) {
        char buf[160];
        std::snprintf(buf, sizeof buf,
                      "cc_ogc_radii_noalloc: %llu vertices exceed the static scratch limit of %llu vertices",
                      (unsigned long long)n_all, (unsigned long long)kNoAllocMaxVertices);
        return record_global_error(CC_ERR_INVALID_ARGUMENT, buf);
    }
    if (!x || !radii || !minimum_distance || moving > n_all || (n_vf && (!vf_pairs || !triangles)) ||
        (n_ee && (!ee_pairs || !edges)) || n_triangles > 0xffffffffull || n_edges > 0xffffffffull ||
        !std::isfinite(query_radius) || !(query_radius > 0.0) || !std::isfinite(relaxation) ||
        !(relaxation > 0.0) || !(relaxation < 0.5))
        return record_global_error(CC_ERR_INVALID_ARGUMENT, "cc_ogc_radii_noalloc: invalid argument");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
        return record_global_error(CC_ERR_CUDA, "cc_ogc_radii_noalloc: no current CUDA device");
    // one call at a time in this process: the launches and the read-back of
    // two host threads must not interleave on the shared scratch array
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    // an earlier, unrelated launch error is not this call's failure
    (void)cudaGetLastError();
    if (!g_noalloc_address[dev]) {
        // once per device, with that device current: the symbol's device address
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
            return record_global_error(CC_ERR_CUDA, "cc_ogc_radii_noalloc: scratch address unavailable");
        g_noalloc_address[dev] = static_cast<unsigned long long*>(p);
    }
    unsigned long long* scratch = g_noalloc_address[dev];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NoAllocArgs a{x, (uint32_t)n_all, (uint32_t)moving, (uint32_t)n_triangles, (uint32_t)n_edges, triangles, edges,
                  vf_pairs, ee_pairs, n_vf, n_ee, query_radius, relaxation, scratch};
    k_noalloc_clear<<<grid_for(n_all + 1, 256), 256, 0, st>>>(a);
    if (n_vf + n_ee) k_noalloc_pairs<<<grid_for((size_t)(n_vf + n_ee), 128), 128, 0, st>>>(a);
    if (moving) k_noalloc_radii<<<grid_for(moving, 256), 256, 0, st>>>(a, radii);
    k_noalloc_store_min<<<1, 1, 0, st>>>(a, minimum_distance);
    if (cudaGetLastError() != cudaSuccess) return record_global_error(CC_ERR_CUDA, "cc_ogc_radii_noalloc: launch failed");
    // read the error word back (into a host variable; nothing is allocated)
    unsigned long long bad = 0;
    if (cudaMemcpyAsync(&bad, scratch + kNoAllocMaxVertices + 1, sizeof bad, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return record_global_error(CC_ERR_CUDA, "cc_ogc_radii_noalloc: device failure");
    if (bad) return record_global_error(CC_ERR_INVALID_ARGUMENT, "cc_ogc_radii_noalloc: index out of range");
    return CC_OK;
}
