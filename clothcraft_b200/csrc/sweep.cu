// VBD colour sweep (replaces the per-colour par_iter of VbdSolver::step,
// src/vbd.rs:337-394, and the `iterate` shader of src/vbd.wgsl:148-182).
//
// One local Newton solve per free vertex of the colour: exact gradient and
// Hessian of every incident term (membrane, bending, stitches, OGC contacts,
// grab) plus inertia, Gershgorin SPD shift, FP64 3x3 solve, then at most ten
// halvings, each clipped to the vertex's OGC ball and accepted on energy
// decrease (src/vbd.rs:353-386). The reference GPU shader uses Gauss-Newton
// Hessians and 8 halvings; this kernel follows the CPU path instead.
//
// A group of G lanes (G in 1..32, chosen per workload) solves one vertex: the
// incident terms are dealt round-robin to the lanes, each lane accumulates a
// partial energy / gradient / Hessian, and a butterfly shuffle reduction gives
// every lane of the group the same bitwise total (each level adds the same two
// partial sums, and addition is commutative), so all lanes take identical
// line-search decisions without a broadcast.
//
// This is the FP64 form (cc_vbd_settings.sweep_precision = CC_SWEEP_FP64):
// every term and the 3x3 solve in FP64, operation for operation as the CPU
// path, so that GPU and CPU iterates agree to the last bits. sweep32.cu holds
// the FP32-assembly form.
#include "sweep_terms.cuh"

namespace cc {

template <int G>
__device__ __forceinline__ void solve_vertex(const SweepView& s, uint32_t v, uint32_t lane, unsigned mask) {
    if (s.pinned[v]) {
        if (lane == 0) s.residual[v] = 0.0;
        return;
    }
    d3 x = ld3(s.x, v);
    d3 y = ld3(s.target, v);
    double m = s.inertia[v];
    d3 g = mk(0, 0, 0);
    Sym H;
    sym_zero(H);
    double e_el = local_part<true, G>(s, v, x, lane, g, H);
    // the OGC ball, loaded here so that its latency hides behind the reductions
    const d3 ctr = ld3(s.contacts.centers, v);
    const double rad = s.contacts.radii[v];
    if (G > 1) {
        e_el = group_sum<G>(e_el, mask);
        g.x = group_sum<G>(g.x, mask);
        g.y = group_sum<G>(g.y, mask);
        g.z = group_sum<G>(g.z, mask);
#pragma unroll
        for (int k = 0; k < 6; ++k) H.a[k] = group_sum<G>(H.a[k], mask);
    }
    d3 xy = x - y;
    g = g + xy * m;
    sym_add_diag(H, m);
    // Gershgorin lower bound and SPD shift (src/vbd.rs:357-370)
    double lower = fmin(fmin(H.a[0] - (fabs(H.a[1]) + fabs(H.a[2])), H.a[3] - (fabs(H.a[1]) + fabs(H.a[4]))),
                        H.a[5] - (fabs(H.a[2]) + fabs(H.a[4])));
    if (lower < 1e-8) sym_add_diag(H, 1e-8 - lower + 0.01 * m);
    // delta = -H^-1 g by adjugate / determinant (glam DMat3::inverse)
    double a00 = H.a[0], a01 = H.a[1], a02 = H.a[2], a11 = H.a[3], a12 = H.a[4], a22 = H.a[5];
    double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
    double det = a00 * c00 + a01 * c01 + a02 * c02;
    double inv = 1.0 / det;
    d3 delta = mk(-(c00 * g.x + c01 * g.y + c02 * g.z) * inv, -(c01 * g.x + c11 * g.y + c12 * g.z) * inv,
                  -(c02 * g.x + c12 * g.y + c22 * g.z) * inv);
    double old = e_el + 0.5 * m * dot(xy, xy);
    d3 accepted = x;
    bool truncated = false;
    double scale = 1.0;
    for (int attempt = 0; attempt < 10; ++attempt) {
        d3 cand = x + delta * scale;
        scale *= 0.5;
        // ContactSet::truncate (src/ogc/world.rs:91-100) with the loaded ball
        bool bound = false;
        {
            d3 d = cand - ctr;
            double l = len(d);
            if (l > rad) {
                bound = true;
                cand = ctr + d * (rad / l);
            }
        }
        truncated = truncated || bound;
        d3 gd;
        Sym Hd;
        double e = local_part<false, G>(s, v, cand, lane, gd, Hd);
        if (G > 1) e = group_sum<G>(e, mask);
        d3 cy = cand - y;
        e += 0.5 * m * dot(cy, cy);
        if (isfin(cand) && isfinite(e) && e <= old + 1e-14) {
            accepted = cand;
            break;
        }
    }
    if (lane == 0) {
        st3(s.x, v, accepted);
        s.residual[v] = dot(g, g);
        s.clipped_flag[v] = truncated ? 1 : 0;
        if (truncated) atomicAdd(s.clipped, 1u);
    }
}

// MINB blocks of BLOCK threads per SM caps the registers (65536 / (MINB*BLOCK)).
// Each group of G lanes solves vertices gi, gi + groups in the grid, ...: one
// vertex per group when the grid covers the colour, several in a persistent grid.
template <int G, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_sweep(SweepView s, const uint32_t* order, uint32_t count) {
    if (s.skip_at && *s.skip_at <= s.iteration) return;  // a refresh detection precedes this iteration
    const uint32_t lane = threadIdx.x & (G - 1);
    const unsigned mask = G >= 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(unsigned)(G - 1)));
    constexpr uint32_t kGroups = BLOCK / G;
    stamp_block_start(s);
    // whole groups step together
    for (uint32_t gi = blockIdx.x * kGroups + threadIdx.x / G; gi < count; gi += gridDim.x * kGroups)
        solve_vertex<G>(s, order[gi], lane, mask);
    stamp_block_end(s);
}

template <int G, int B, int MINB>
static void launch_k(const SweepView& s, const uint32_t* order, uint32_t count, cudaStream_t st, unsigned cap) {
    uint64_t threads = (uint64_t)count * G;
    unsigned grid = (unsigned)((threads + B - 1) / B);
    if (cap && grid > cap) grid = cap;
    k_sweep<G, B, MINB><<<grid, B, 0, st>>>(s, order, count);
}

template <int G, int B, int MINB>
static unsigned resident_k() {
    int dev = 0, sms = 0, per = 0;
    CC_CUDA(cudaGetDevice(&dev));
    CC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweep<G, B, MINB>, B, 0));
    return (unsigned)(sms * (per > 0 ? per : 1));
}

// Dispatch of (lanes, cap, block) to a kernel instance; F(G, B, MINB) is
// called for the instance. Blocks of 64 and 256 threads exist for 4 and 8
// lanes at the register budgets of caps 3-4 (64) and 4, 6, 8 (256).
template <int G, class F>
static auto dispatch_cap(const SweepVariant& v, F&& f) {
    if (v.block == 64) {
        if (v.cap >= 4) return f.template operator()<G, 64, 8>();
        return f.template operator()<G, 64, 6>();
    }
    if (v.block == 256) {
        if (v.cap >= 8) return f.template operator()<G, 256, 4>();
        if (v.cap >= 6) return f.template operator()<G, 256, 3>();
        return f.template operator()<G, 256, 2>();
    }
    if (v.cap >= 8) return f.template operator()<G, 128, 8>();
    if (v.cap >= 6) return f.template operator()<G, 128, 6>();
    if (v.cap == 5) return f.template operator()<G, 128, 5>();
    if (v.cap == 4) return f.template operator()<G, 128, 4>();
    return f.template operator()<G, 128, 3>();
}

template <class F>
static auto dispatch(const SweepVariant& v, F&& f) {
    switch (v.lanes) {
        case 1: return dispatch_cap<1>(SweepVariant{1, v.cap, 128, v.persistent}, f);
        case 2: return dispatch_cap<2>(SweepVariant{2, v.cap, 128, v.persistent}, f);
        case 4: return dispatch_cap<4>(v, f);
        case 16: return dispatch_cap<16>(SweepVariant{16, v.cap, 128, v.persistent}, f);
        case 32: return dispatch_cap<32>(SweepVariant{32, v.cap, 128, v.persistent}, f);
        default: return dispatch_cap<8>(v, f);
    }
}

bool sweep_variant_valid(int variant, bool fp32) {
    if (variant & ~((1 << 19) - 1)) return false;
    SweepVariant v = decode_variant(variant);
    int code = (variant >> 17) & 3;
    if (code == 3) return false;
    bool cap_ok = v.cap == 3 || v.cap == 4 || v.cap == 5 || v.cap == 6 || v.cap == 8;
    bool lanes_ok = fp32 ? (v.lanes == 4 || v.lanes == 8 || v.lanes == 16 || v.lanes == 32)
                         : (v.lanes == 1 || v.lanes == 2 || v.lanes == 4 || v.lanes == 8 || v.lanes == 16 ||
                            v.lanes == 32);
    if (!cap_ok || !lanes_ok) return false;
    if (v.block == 128) return true;
    bool wide = fp32 ? (v.lanes == 8 || v.lanes == 16) : (v.lanes == 4 || v.lanes == 8);
    if (!wide) return false;
    return v.block == 64 ? (v.cap == 3 || v.cap == 4) : (v.cap == 4 || v.cap == 6 || v.cap == 8);
}

namespace {
struct SweepLaunch {
    const SweepView& s;
    const uint32_t* order;
    uint32_t count;
    cudaStream_t st;
    unsigned cap;
    template <int G, int B, int MINB>
    int operator()() const {
        launch_k<G, B, MINB>(s, order, count, st, cap);
        return 0;
    }
};
struct SweepResident {
    template <int G, int B, int MINB>
    unsigned operator()() const {
        return resident_k<G, B, MINB>();
    }
};
}  // namespace

void launch_sweep(const SweepView& s, const uint32_t* order, uint32_t count, int variant, cudaStream_t st,
                  unsigned grid_cap) {
    if (count == 0) return;
    SweepVariant v = decode_variant(variant);
    dispatch(v, SweepLaunch{s, order, count, st, v.persistent ? grid_cap : 0u});
}

unsigned sweep_resident_blocks(int variant) { return dispatch(decode_variant(variant), SweepResident{}); }

// Probe: local e, g, H of every moving vertex at the current positions
// (the f64 gradient check of src/gpu_vbd.rs:305-379, probe of vbd.wgsl:142-147).
__global__ void k_local_blocks(SweepView s, double* energy, double* grad, double* hess) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < s.n; v += gridDim.x * blockDim.x) {
        d3 x = ld3(s.x, v);
        d3 g = mk(0, 0, 0);
        Sym H;
        sym_zero(H);
        double e = local_part<true, 1>(s, v, x, 0, g, H);
        double m = s.inertia ? s.inertia[v] : 0.0;
        d3 y = s.target ? ld3(s.target, v) : x;
        d3 xy = x - y;
        energy[v] = e + 0.5 * m * dot(xy, xy);
        g = g + xy * m;
        grad[3 * v] = g.x;
        grad[3 * v + 1] = g.y;
        grad[3 * v + 2] = g.z;
        double* h = hess + 9 * v;
        h[0] = H.a[0] + m;
        h[1] = H.a[1];
        h[2] = H.a[2];
        h[3] = H.a[1];
        h[4] = H.a[3] + m;
        h[5] = H.a[4];
        h[6] = H.a[2];
        h[7] = H.a[4];
        h[8] = H.a[5] + m;
    }
}

void launch_local_blocks(const SweepView& s, double* energy, double* grad, double* hess, cudaStream_t st) {
    k_local_blocks<<<grid_for(s.n, 128), 128, 0, st>>>(s, energy, grad, hess);
}

// ------------------------------------------ step objective and its gradient
// |dE/dx_v|^2 of every moving vertex at s.x (0 where pinned): the sweep's
// block gradient (inertia + incident terms) without an update. With
// `project`, a vertex on the boundary of its OGC ball (|x - c| >= b) whose
// descent direction -g points out of the ball keeps only the tangential part
// of g: the first-order (KKT) residual of the step's ball-constrained
// problem (ContactSet::truncate, src/ogc/world.rs:91-100). Skipped when
// *skip_at <= iteration (that iteration never ran).
template <int G>
__global__ void __launch_bounds__(128) k_grad_sq(SweepView s, double* out, const unsigned* skip_at, uint32_t iteration,
                                                 int project) {
    if (skip_at && *skip_at <= iteration) return;
    uint32_t t = blockIdx.x * 128 + threadIdx.x;
    uint32_t v = t / G;
    if (v >= s.n) return;  // whole groups leave together
    uint32_t lane = threadIdx.x & (G - 1);
    unsigned mask = G >= 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(unsigned)(G - 1)));
    if (s.pinned[v]) {
        if (lane == 0) out[v] = 0.0;
        return;
    }
    d3 x = ld3(s.x, v);
    d3 g = mk(0, 0, 0);
    Sym H;
    sym_zero(H);
    local_part<true, G, false>(s, v, x, lane, g, H);  // gradient only
    if (G > 1) {
        g.x = group_sum<G>(g.x, mask);
        g.y = group_sum<G>(g.y, mask);
        g.z = group_sum<G>(g.z, mask);
    }
    g = g + (x - ld3(s.target, v)) * s.inertia[v];
    if (project) {
        d3 d = x - ld3(s.contacts.centers, v);
        double l = len(d), b = s.contacts.radii[v];
        double gn = dot(g, d);
        if (l >= b * (1.0 - 1e-9) && l > 0.0 && gn < 0.0) g = g - d * (gn / (l * l));
    }
    if (lane == 0) out[v] = dot(g, g);
}

void launch_grad_sq(const SweepView& s, double* out, const unsigned* skip_at, uint32_t iteration, int variant,
                    bool project, cudaStream_t st) {
    int G = variant & 0xff;
    unsigned grid = (unsigned)(((uint64_t)s.n * (uint64_t)G + 127) / 128);
    if (grid == 0) return;
    int p = project ? 1 : 0;
    switch (G) {
        case 1: k_grad_sq<1><<<grid, 128, 0, st>>>(s, out, skip_at, iteration, p); break;
        case 2: k_grad_sq<2><<<grid, 128, 0, st>>>(s, out, skip_at, iteration, p); break;
        case 4: k_grad_sq<4><<<grid, 128, 0, st>>>(s, out, skip_at, iteration, p); break;
        case 16: k_grad_sq<16><<<grid, 128, 0, st>>>(s, out, skip_at, iteration, p); break;
        case 32: k_grad_sq<32><<<grid, 128, 0, st>>>(s, out, skip_at, iteration, p); break;
        default: k_grad_sq<8><<<grid, 128, 0, st>>>(s, out, skip_at, iteration, p); break;
    }
}

// Energy of every term of the step objective, once each, at s.x:
// [0,n) inertia of free vertices, then triangles, hinges, stitches, contacts
// and the grab (the objective of src/solver.rs:255-296 plus the OGC terms).
__global__ void k_term_energy(SweepView s, ObjectiveCounts c, double* out) {
    uint64_t total = s.n + objective_items(c);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        d3 g = mk(0, 0, 0);
        Sym H;
        double e = 0.0;
        uint64_t k = i;
        if (k < s.n) {
            if (!s.pinned[k]) {
                d3 d = ld3(s.x, (uint32_t)k) - ld3(s.target, (uint32_t)k);
                e = 0.5 * s.inertia[k] * dot(d, d);
            }
        } else if ((k -= s.n) < c.triangles) {
            uint32_t v = (uint32_t)s.tri_v[k].x;
            e = membrane_term<false>(s, (uint32_t)k, 0, ld3(s.x, v), g, H);
        } else if ((k -= c.triangles) < c.hinges) {
            uint32_t v = s.hinge_v[k].x;
            e = bending_term<false>(s, (uint32_t)k, 0, ld3(s.x, v), g, H);
        } else if ((k -= c.hinges) < c.stitches) {
            uint32_t v = s.st_v[s.st_off[k]];
            e = stitch_term<false>(s, (uint32_t)k, v, ld3(s.x, v), g, H);
        } else if ((k -= c.stitches) < c.contacts) {
            uint32_t v = s.contacts.verts[k].x;
            e = contact_term<false>(s, (uint32_t)k, v, ld3(s.x, v), g, H);
        } else if (s.grab.active) {
            uint32_t v = s.grab.v[0];
            e = grab_term<false>(s, v, ld3(s.x, v), g, H);
        }
        out[i] = e;
    }
}

void launch_term_energy(const SweepView& s, const ObjectiveCounts& c, double* out, cudaStream_t st) {
    uint64_t total = s.n + objective_items(c);
    k_term_energy<<<grid_for(total, 256), 256, 0, st>>>(s, c, out);
}

// Deterministic sum, first pass: kSumBlocks fixed-order partial sums.
__global__ void __launch_bounds__(256) k_sum_partial(const double* v, uint64_t n, double* partial,
                                                     const unsigned* skip_at, uint32_t iteration) {
    if (skip_at && *skip_at <= iteration) return;
    __shared__ double sh[256];
    double a = 0.0;
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n; i += (uint64_t)kSumBlocks * 256ull) a += v[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

void launch_sum_partial(const double* v, uint64_t n, double* partial, const unsigned* skip_at, uint32_t iteration,
                        cudaStream_t st) {
    k_sum_partial<<<kSumBlocks, 256, 0, st>>>(v, n, partial, skip_at, iteration);
}


}  // namespace cc
