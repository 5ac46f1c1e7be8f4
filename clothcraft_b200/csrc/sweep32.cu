// VBD colour sweep with FP32 element assembly: the library's fast form of the
// local solve of VbdSolver::step (src/vbd.rs:337-394). sweep.cu holds the FP64
// form, whose arithmetic follows the CPU path operation for operation.
//
// Precision plan (per vertex solve):
//   - positions stay FP64 in HBM; every element's edge vectors are formed as
//     FP64 differences and rounded once to FP32, so they carry FP32 relative
//     precision of the edge (not of the absolute coordinates);
//   - membrane (src/energy.rs:10-29) and bending (src/energy.rs:31-46)
//     energies, gradients and Hessians in FP32 with FP32 accumulation;
//   - OGC contact terms (src/ogc/potential.rs:39-65) in FP64: their
//     closest-feature distances are all within the contact radius, where the
//     barrier needs them exact;
//   - the 3x3 block solve in FP32 unless its condition estimate
//     ||H||inf ||H^-1||inf exceeds 1e6, then in FP64 (adjugate / determinant);
//   - the line search compares energy *differences* e(x + d) - e(x), each
//     element's difference expanded in d (no cancellation of two nearly equal
//     element energies), summed in FP64 with the inertia and contact parts.
//
// The per-element quantities the line search needs (fibre vectors, strains
// and their coefficients in d; hinge normals and their rates) are computed
// once in the derivative pass and staged per lane in shared memory, so the
// up to ten trial evaluations read no global memory for membrane and bending
// terms. A lane's terms beyond the staging slots are recomputed from global
// memory in each trial.
#include <atomic>

#include "sweep_terms.cuh"

namespace cc {

namespace {

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 fmk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float fdot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 fcross(f3 a, f3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ f3 tof(d3 a) { return {(float)a.x, (float)a.y, (float)a.z}; }

struct Sym32 {  // xx xy xz yy yz zz
    float a[6];
};
__device__ __forceinline__ void s32_outer(Sym32& h, f3 u, float s) {
    h.a[0] += s * u.x * u.x;
    h.a[1] += s * u.x * u.y;
    h.a[2] += s * u.x * u.z;
    h.a[3] += s * u.y * u.y;
    h.a[4] += s * u.y * u.z;
    h.a[5] += s * u.z * u.z;
}
__device__ __forceinline__ void s32_outer2(Sym32& h, f3 u, f3 v, float s) {  // h += s (u v^T + v u^T)
    h.a[0] += s * 2.f * u.x * v.x;
    h.a[1] += s * (u.x * v.y + v.x * u.y);
    h.a[2] += s * (u.x * v.z + v.x * u.z);
    h.a[3] += s * 2.f * u.y * v.y;
    h.a[4] += s * (u.y * v.z + v.y * u.z);
    h.a[5] += s * 2.f * u.z * v.z;
}
__device__ __forceinline__ void s32_diag(Sym32& h, float s) {
    h.a[0] += s;
    h.a[3] += s;
    h.a[5] += s;
}

// ------------------------------------------------------------- membrane
// Triangle record in the frame of the solved vertex: fibre vectors w, v of
// F = Ds Dm^-1 (grain-rotated), Green strains ew, ev and shear sh at the
// vertex's current position, and the rates aw, av with which w and v move
// when the vertex moves by d (w(d) = w + aw d, v(d) = v + av d).
struct TriRec {
    f3 w, v;
    float ew, ev, sh, aw, av, area;
    uint32_t mat;
};
constexpr int kTriFields = 13;

__device__ __forceinline__ TriRec tri_rec(const SweepView& s, uint32_t t, uint32_t slot, d3 x) {
    int4 tv = s.tri_v[t];
    double4 cf = s.tri_coef[t];
    d3 x0 = slot == 0 ? x : ld3(s.x, (uint32_t)tv.x);
    d3 x1 = slot == 1 ? x : ld3(s.x, (uint32_t)tv.y);
    d3 x2 = slot == 2 ? x : ld3(s.x, (uint32_t)tv.z);
    // The Green strains are formed in FP64 from the FP64 edge differences and
    // rounded once: 1/2 (w.w - 1) cancels to ~1e-4 of its terms, so an FP32
    // strain would carry ~1e-7 of absolute error, a force noise that left the
    // relative force residual of the 64x64 sheet on a sphere at ~0.19 after
    // 100 steps (FP64: 0.068). Everything after that is FP32.
    const d3 e0 = x1 - x0, e1 = x2 - x0;
    const d3 w64 = e0 * cf.x + e1 * cf.y, v64 = e0 * cf.z + e1 * cf.w;
    float cx = (float)cf.x, cy = (float)cf.y, cz = (float)cf.z, cw = (float)cf.w;
    TriRec r;
    r.w = tof(w64);
    r.v = tof(v64);
    r.ew = (float)((dot(w64, w64) - 1.0) * 0.5);
    r.ev = (float)((dot(v64, v64) - 1.0) * 0.5);
    r.sh = (float)dot(w64, v64);
    r.aw = slot == 0 ? (float)(-(cf.x + cf.y)) : (slot == 1 ? cx : cy);
    r.av = slot == 0 ? (float)(-(cf.z + cf.w)) : (slot == 1 ? cz : cw);
    r.area = (float)s.tri_area[t];
    r.mat = (uint32_t)tv.w;
    return r;
}

// axial (src/energy.rs:10-16) with its first and second derivative, FP32
__device__ __forceinline__ void axial3f(float sv, float k, float c, float delta, float& f1, float& f2) {
    if (c == 1.f) {  // pure quadratic law: the (1 - c) terms are exactly zero
        f1 = k * (c * sv);
        f2 = k * c;
        return;
    }
    float r = sqrtf(sv * sv + delta * delta);
    float ir = 1.f / r;
    float p = (sv + r - delta) * 0.5f;
    float p1 = 0.5f * (1.f + sv * ir);
    float p2 = 0.5f * delta * delta * (ir * ir * ir);
    f1 = k * (c * sv + (1.f - c) * p * p1);
    f2 = k * (c + (1.f - c) * (p1 * p1 + p * p2));
}

__device__ __forceinline__ void tri_derivs(const TriRec& r, const MatParams32& M, f3& g, Sym32& H) {
    float fw1, fw2, fv1, fv2;
    axial3f(r.ew, M.warp, M.c, M.delta, fw1, fw2);
    axial3f(r.ev, M.weft, M.c, M.delta, fv1, fv2);
    f3 q = r.v * r.aw + r.w * r.av;
    g = g + (r.w * (fw1 * r.aw) + r.v * (fv1 * r.av) + q * (M.shear * r.sh)) * r.area;
    s32_outer(H, r.w, r.area * fw2 * r.aw * r.aw);
    s32_outer(H, r.v, r.area * fv2 * r.av * r.av);
    s32_outer(H, q, r.area * M.shear);
    s32_diag(H, r.area * (fw1 * r.aw * r.aw + fv1 * r.av * r.av + 2.f * M.shear * r.sh * r.aw * r.av));
}

// axial(s0 + ds) - axial(s0) without subtracting two energies
__device__ __forceinline__ float daxial(float s0, float ds, float k, float c, float delta) {
    float s1 = s0 + ds;
    float out = c * ds * (s0 + s1);
    if (c != 1.f) {
        float r0 = sqrtf(s0 * s0 + delta * delta), r1 = sqrtf(s1 * s1 + delta * delta);
        float dp = 0.5f * (ds + ds * (s0 + s1) / (r0 + r1));
        float p0 = 0.5f * (s0 + r0 - delta);
        out += (1.f - c) * dp * (2.f * p0 + dp);
    }
    return 0.5f * k * out;
}

// membrane energy change when the solved vertex moves by d
__device__ __forceinline__ float tri_delta(const TriRec& r, const MatParams32& M, f3 d) {
    float wd = fdot(r.w, d), vd = fdot(r.v, d), dd = fdot(d, d);
    float dew = r.aw * wd + 0.5f * r.aw * r.aw * dd;
    float dev = r.av * vd + 0.5f * r.av * r.av * dd;
    float dsh = r.av * wd + r.aw * vd + r.aw * r.av * dd;
    return r.area * (daxial(r.ew, dew, M.warp, M.c, M.delta) + daxial(r.ev, dev, M.weft, M.c, M.delta) +
                     0.5f * M.shear * dsh * (2.f * r.sh + dsh));
}

// -------------------------------------------------------------- bending
// Hinge record: n1 = e x u, n2 = w x e (e = x1 - x0, u = x2 - x0, w = x3 - x0)
// and their rates in the solved vertex, n_k(d) = n_k + a_k x d.
struct HingeRec {
    f3 n1, n2, a1, a2;
    float K;
};
constexpr int kHingeFields = 13;

__device__ __forceinline__ HingeRec hinge_rec(const SweepView& s, uint32_t h, uint32_t slot, d3 x) {
    uint4 hv = s.hinge_v[h];
    d3 x0 = slot == 0 ? x : ld3(s.x, hv.x);
    d3 x1 = slot == 1 ? x : ld3(s.x, hv.y);
    d3 x2 = slot == 2 ? x : ld3(s.x, hv.z);
    d3 x3 = slot == 3 ? x : ld3(s.x, hv.w);
    f3 e = tof(x1 - x0), u = tof(x2 - x0), w = tof(x3 - x0);
    HingeRec r;
    r.n1 = fcross(e, u);
    r.n2 = fcross(w, e);
    const f3 z = fmk(0.f, 0.f, 0.f);
    r.a1 = slot == 0 ? u - e : (slot == 1 ? -u : (slot == 2 ? e : z));
    r.a2 = slot == 0 ? e - w : (slot == 1 ? w : (slot == 3 ? -e : z));
    r.K = (float)s.hinge_k[h];
    return r;
}

// P_k [a]x / l as three columns: P(a x e_j)/l, P y = y - h (h.y)
__device__ __forceinline__ void proj_skew_cols_f(f3 a, f3 h, float inv_l, float sign, f3& c0, f3& c1, f3& c2) {
    f3 e0 = fmk(0.f, a.z, -a.y), e1 = fmk(-a.z, 0.f, a.x), e2 = fmk(a.y, -a.x, 0.f);
    float f = sign * inv_l;
    c0 = c0 + (e0 - h * fdot(h, e0)) * f;
    c1 = c1 + (e1 - h * fdot(h, e1)) * f;
    c2 = c2 + (e2 - h * fdot(h, e2)) * f;
}

// [a]x^T M [a]x for M = -(1/l^2)[d h^T + h d^T + (d.h)(I - 3 h h^T)]
__device__ __forceinline__ void add_curvature_f(Sym32& Hm, f3 a, f3 h, f3 d, float inv_l2, float sign) {
    f3 da = fcross(d, a), ha = fcross(h, a);
    float dh = fdot(d, h);
    float sc = -inv_l2 * sign;
    s32_outer2(Hm, da, ha, sc);
    s32_diag(Hm, sc * dh * fdot(a, a));
    s32_outer(Hm, a, -sc * dh);
    s32_outer(Hm, ha, -3.f * sc * dh);
}

// gradient 2K J^T d and Hessian 2K [J^T J + A1^T M1 A1 - A2^T M2 A2] of
// K |n1/|n1| - n2/|n2||^2 in the solved vertex
__device__ __forceinline__ void hinge_derivs(const HingeRec& r, f3& g, Sym32& H) {
    float il1 = rsqrtf(fdot(r.n1, r.n1));
    float il2 = rsqrtf(fdot(r.n2, r.n2));
    f3 h1 = r.n1 * il1, h2 = r.n2 * il2;
    f3 d = h1 - h2;
    f3 pd1 = d - h1 * fdot(h1, d), pd2 = d - h2 * fdot(h2, d);
    f3 jtd = fcross(pd1, r.a1) * il1 - fcross(pd2, r.a2) * il2;
    g = g + jtd * (2.f * r.K);
    f3 c0 = fmk(0.f, 0.f, 0.f), c1 = c0, c2 = c0;
    proj_skew_cols_f(r.a1, h1, il1, 1.f, c0, c1, c2);
    proj_skew_cols_f(r.a2, h2, il2, -1.f, c0, c1, c2);
    Sym32 Hm;
    Hm.a[0] = fdot(c0, c0);
    Hm.a[1] = fdot(c0, c1);
    Hm.a[2] = fdot(c0, c2);
    Hm.a[3] = fdot(c1, c1);
    Hm.a[4] = fdot(c1, c2);
    Hm.a[5] = fdot(c2, c2);
    add_curvature_f(Hm, r.a1, h1, d, il1 * il1, 1.f);
    add_curvature_f(Hm, r.a2, h2, d, il2 * il2, -1.f);
    float f = 2.f * r.K;
#pragma unroll
    for (int k = 0; k < 6; ++k) H.a[k] += f * Hm.a[k];
}

// unit-normal change n(d)/|n(d)| - n/|n| for n(d) = n + m, expanded so that
// the two nearly equal unit vectors are never subtracted
__device__ __forceinline__ f3 dunit(f3 n, f3 m) {
    float l2 = fdot(n, n);
    float q = 2.f * fdot(n, m) + fdot(m, m);  // |n + m|^2 - |n|^2
    float l = sqrtf(l2), lp = sqrtf(l2 + q);
    return m * (1.f / lp) - n * (q / (l * lp * (l + lp)));
}

// bending energy change when the solved vertex moves by d
__device__ __forceinline__ float hinge_delta(const HingeRec& r, f3 d) {
    f3 dh1 = dunit(r.n1, fcross(r.a1, d));
    f3 dh2 = dunit(r.n2, fcross(r.a2, d));
    f3 d0 = r.n1 * rsqrtf(fdot(r.n1, r.n1)) - r.n2 * rsqrtf(fdot(r.n2, r.n2));
    f3 dd = dh1 - dh2;
    return r.K * fdot(dd, d0 * 2.f + dd);
}

// ------------------------------------------------- shared-memory staging
// A lane's j-th triangle (hinge) record lives in column `tid` of rows
// j, j + JT, ... (one row per field), so the lanes of a warp touch
// consecutive words: no bank conflicts.
template <int G>
struct Stage {
    static constexpr int kTris = 12;    // staged triangles per vertex
    static constexpr int kHinges = 24;  // staged hinges per vertex
    static constexpr int JT = (kTris + G - 1) / G;
    static constexpr int JH = (kHinges + G - 1) / G;
    static constexpr int floats = JT * kTriFields + JH * kHingeFields;  // per thread
};

template <int J, int B>
__device__ __forceinline__ void put_tri(float* base, int j, const TriRec& r) {
    float* p = base + j * B + threadIdx.x;
    const float v[kTriFields] = {r.w.x, r.w.y, r.w.z, r.v.x, r.v.y, r.v.z, r.ew, r.ev, r.sh, r.aw, r.av, r.area,
                                 __uint_as_float(r.mat)};
#pragma unroll
    for (int f = 0; f < kTriFields; ++f) p[f * J * B] = v[f];
}
template <int J, int B>
__device__ __forceinline__ TriRec get_tri(const float* base, int j) {
    const float* p = base + j * B + threadIdx.x;
    TriRec r;
    r.w = fmk(p[0], p[J * B], p[2 * J * B]);
    r.v = fmk(p[3 * J * B], p[4 * J * B], p[5 * J * B]);
    r.ew = p[6 * J * B];
    r.ev = p[7 * J * B];
    r.sh = p[8 * J * B];
    r.aw = p[9 * J * B];
    r.av = p[10 * J * B];
    r.area = p[11 * J * B];
    r.mat = __float_as_uint(p[12 * J * B]);
    return r;
}
template <int J, int B>
__device__ __forceinline__ void put_hinge(float* base, int j, const HingeRec& r) {
    float* p = base + j * B + threadIdx.x;
    const float v[kHingeFields] = {r.n1.x, r.n1.y, r.n1.z, r.n2.x, r.n2.y, r.n2.z, r.a1.x,
                                   r.a1.y, r.a1.z, r.a2.x, r.a2.y, r.a2.z, r.K};
#pragma unroll
    for (int f = 0; f < kHingeFields; ++f) p[f * J * B] = v[f];
}
template <int J, int B>
__device__ __forceinline__ HingeRec get_hinge(const float* base, int j) {
    const float* p = base + j * B + threadIdx.x;
    HingeRec r;
    r.n1 = fmk(p[0], p[J * B], p[2 * J * B]);
    r.n2 = fmk(p[3 * J * B], p[4 * J * B], p[5 * J * B]);
    r.a1 = fmk(p[6 * J * B], p[7 * J * B], p[8 * J * B]);
    r.a2 = fmk(p[9 * J * B], p[10 * J * B], p[11 * J * B]);
    r.K = p[12 * J * B];
    return r;
}

template <int G>
__device__ __forceinline__ float group_sum_f(float x, unsigned mask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(mask, x, o, G);
    return x;
}

// --------------------------------------------------------- vertex solve
template <int G, int B>
__device__ __forceinline__ void solve_vertex32(const SweepView& s, uint32_t v, uint32_t lane, unsigned mask,
                                               float* sm) {
    using St = Stage<G>;
    float* smt = sm;                                 // triangle records
    float* smh = sm + St::JT * kTriFields * B;       // hinge records
    if (s.pinned[v]) {
        if (lane == 0) s.residual[v] = 0.0;
        return;
    }
    const d3 x = ld3(s.x, v);
    const d3 y = ld3(s.target, v);
    const double m = s.inertia[v];
    const uint32_t b0 = s.inc_off[v], b1 = s.inc_off[v + 1];
    const uint2 mid = s.inc_mid[v];
    const uint32_t c0 = s.contacts.inc_off[v], c1 = s.contacts.inc_off[v + 1];
    // ---- derivative pass: FP32 elastic part, FP64 stitch / contact / grab part
    f3 g32 = fmk(0.f, 0.f, 0.f);
    Sym32 H32;
#pragma unroll
    for (int k = 0; k < 6; ++k) H32.a[k] = 0.f;
    {
        int j = 0;
        for (uint32_t k = b0 + lane; k < mid.x; k += G, ++j) {
            uint32_t ent = s.inc[k];
            TriRec r = tri_rec(s, ent & 0x0fffffffu, (ent >> 28) & 3u, x);
            tri_derivs(r, s.mats32[r.mat], g32, H32);
            if (j < St::JT) put_tri<St::JT, B>(smt, j, r);
        }
    }
    {
        int j = 0;
        for (uint32_t k = mid.x + lane; k < mid.y; k += G, ++j) {
            uint32_t ent = s.inc[k];
            HingeRec r = hinge_rec(s, ent & 0x0fffffffu, (ent >> 28) & 3u, x);
            hinge_derivs(r, g32, H32);
            if (j < St::JH) put_hinge<St::JH, B>(smh, j, r);
        }
    }
    d3 g64 = mk(0, 0, 0);
    Sym H64;
    sym_zero(H64);
    double e64 = 0.0;  // this lane's FP64 terms at x
    const bool grab_here = lane == 0 && s.grab.active && (s.grab.v[0] == v || s.grab.v[1] == v || s.grab.v[2] == v);
    const bool lane64 = (mid.y + lane < b1) || (c0 + lane < c1) || grab_here;
    for (uint32_t k = mid.y + lane; k < b1; k += G) e64 += stitch_term<true>(s, s.inc[k] & 0x0fffffffu, v, x, g64, H64);
    for (uint32_t k = c0 + lane; k < c1; k += G) e64 += contact_term<true>(s, s.contacts.inc[k], v, x, g64, H64);
    if (grab_here) e64 += grab_term<true>(s, v, x, g64, H64);
    const bool any64 = G > 1 ? __any_sync(mask, lane64) : lane64;
    if (G > 1) {
        g32.x = group_sum_f<G>(g32.x, mask);
        g32.y = group_sum_f<G>(g32.y, mask);
        g32.z = group_sum_f<G>(g32.z, mask);
#pragma unroll
        for (int k = 0; k < 6; ++k) H32.a[k] = group_sum_f<G>(H32.a[k], mask);
        if (any64) {
            g64.x = group_sum<G>(g64.x, mask);
            g64.y = group_sum<G>(g64.y, mask);
            g64.z = group_sum<G>(g64.z, mask);
#pragma unroll
            for (int k = 0; k < 6; ++k) H64.a[k] = group_sum<G>(H64.a[k], mask);
        }
    }
    const d3 xy = x - y;
    d3 g = mk((double)g32.x, (double)g32.y, (double)g32.z) + g64 + xy * m;
    Sym H;
#pragma unroll
    for (int k = 0; k < 6; ++k) H.a[k] = (double)H32.a[k] + H64.a[k];
    sym_add_diag(H, m);
    // Gershgorin lower bound and SPD shift (src/vbd.rs:357-370)
    double lower = fmin(fmin(H.a[0] - (fabs(H.a[1]) + fabs(H.a[2])), H.a[3] - (fabs(H.a[1]) + fabs(H.a[4]))),
                        H.a[5] - (fabs(H.a[2]) + fabs(H.a[4])));
    if (lower < 1e-8) sym_add_diag(H, 1e-8 - lower + 0.01 * m);
    // delta = -H^-1 g: FP32 adjugate unless the condition estimate exceeds 1e6
    d3 delta;
    {
        float a00 = (float)H.a[0], a01 = (float)H.a[1], a02 = (float)H.a[2], a11 = (float)H.a[3],
              a12 = (float)H.a[4], a22 = (float)H.a[5];
        float k00 = a11 * a22 - a12 * a12, k01 = a02 * a12 - a01 * a22, k02 = a01 * a12 - a02 * a11;
        float k11 = a00 * a22 - a02 * a02, k12 = a01 * a02 - a00 * a12, k22 = a00 * a11 - a01 * a01;
        float det = a00 * k00 + a01 * k01 + a02 * k02;
        float nh = fmaxf(fmaxf(fabsf(a00) + fabsf(a01) + fabsf(a02), fabsf(a01) + fabsf(a11) + fabsf(a12)),
                         fabsf(a02) + fabsf(a12) + fabsf(a22));
        float na = fmaxf(fmaxf(fabsf(k00) + fabsf(k01) + fabsf(k02), fabsf(k01) + fabsf(k11) + fabsf(k12)),
                         fabsf(k02) + fabsf(k12) + fabsf(k22));
        float cond = nh * na / fabsf(det);
        if (cond <= 1e6f) {
            float inv = 1.f / det;
            float gx = (float)g.x, gy = (float)g.y, gz = (float)g.z;
            delta = mk(-(k00 * gx + k01 * gy + k02 * gz) * inv, -(k01 * gx + k11 * gy + k12 * gz) * inv,
                       -(k02 * gx + k12 * gy + k22 * gz) * inv);
        } else {
            double b00 = H.a[0], b01 = H.a[1], b02 = H.a[2], b11 = H.a[3], b12 = H.a[4], b22 = H.a[5];
            double d00 = b11 * b22 - b12 * b12, d01 = b02 * b12 - b01 * b22, d02 = b01 * b12 - b02 * b11;
            double d11 = b00 * b22 - b02 * b02, d12 = b01 * b02 - b00 * b12, d22 = b00 * b11 - b01 * b01;
            double inv = 1.0 / (b00 * d00 + b01 * d01 + b02 * d02);
            delta = mk(-(d00 * g.x + d01 * g.y + d02 * g.z) * inv, -(d01 * g.x + d11 * g.y + d12 * g.z) * inv,
                       -(d02 * g.x + d12 * g.y + d22 * g.z) * inv);
        }
    }
    // ---- line search on energy differences: at most ten halvings, each
    // clipped to the OGC ball, accepted when e(cand) - e(x) <= 1e-14
    d3 accepted = x;
    bool truncated = false;
    double scale = 1.0;
    for (int attempt = 0; attempt < 10; ++attempt) {
        d3 cand = x + delta * scale;
        scale *= 0.5;
        bool bound;
        cand = truncate_ball(s, v, cand, bound);
        truncated = truncated || bound;
        const d3 dd = cand - x;
        const f3 df = tof(dd);
        float de32 = 0.f;
        {
            int j = 0;
            for (uint32_t k = b0 + lane; k < mid.x; k += G, ++j) {
                TriRec r;
                if (j < St::JT) {
                    r = get_tri<St::JT, B>(smt, j);
                } else {
                    uint32_t ent = s.inc[k];
                    r = tri_rec(s, ent & 0x0fffffffu, (ent >> 28) & 3u, x);
                }
                de32 += tri_delta(r, s.mats32[r.mat], df);
            }
        }
        {
            int j = 0;
            for (uint32_t k = mid.x + lane; k < mid.y; k += G, ++j) {
                HingeRec r;
                if (j < St::JH) {
                    r = get_hinge<St::JH, B>(smh, j);
                } else {
                    uint32_t ent = s.inc[k];
                    r = hinge_rec(s, ent & 0x0fffffffu, (ent >> 28) & 3u, x);
                }
                de32 += hinge_delta(r, df);
            }
        }
        double de = (double)de32;
        if (lane64) {
            d3 gd;
            Sym Hd;
            double e1 = 0.0;
            for (uint32_t k = mid.y + lane; k < b1; k += G)
                e1 += stitch_term<false>(s, s.inc[k] & 0x0fffffffu, v, cand, gd, Hd);
            for (uint32_t k = c0 + lane; k < c1; k += G) e1 += contact_term<false>(s, s.contacts.inc[k], v, cand, gd, Hd);
            if (grab_here) e1 += grab_term<false>(s, v, cand, gd, Hd);
            de += e1 - e64;
        }
        if (G > 1) de = group_sum<G>(de, mask);
        de += m * dot(dd, xy) + 0.5 * m * dot(dd, dd);  // inertia
        if (isfin(cand) && isfinite(de) && de <= 1e-14) {
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

template <int G, int B, int MINB>
__global__ void __launch_bounds__(B, MINB) k_sweep32(SweepView s, const uint32_t* order, uint32_t count) {
    extern __shared__ float stage_sm[];
    if (s.skip_at && *s.skip_at <= s.iteration) return;  // a refresh detection precedes this iteration
    const uint32_t lane = threadIdx.x & (G - 1);
    const unsigned mask = G >= 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(unsigned)(G - 1)));
    constexpr uint32_t kGroups = B / G;
    stamp_block_start(s);
    // whole groups step together; a persistent grid loops over the colour
    for (uint32_t gi = blockIdx.x * kGroups + threadIdx.x / G; gi < count; gi += gridDim.x * kGroups)
        solve_vertex32<G, B>(s, order[gi], lane, mask, stage_sm);
    stamp_block_end(s);
}

template <int G, int B>
constexpr size_t stage_bytes() {
    return (size_t)Stage<G>::floats * B * sizeof(float);
}

template <int G, int B, int MINB>
void launch_k32(const SweepView& s, const uint32_t* order, uint32_t count, cudaStream_t st, unsigned cap) {
    constexpr size_t smem = stage_bytes<G, B>();
    static std::atomic<uint64_t> raised{0};  // devices on which the limit is raised
    allow_dynamic_smem_once(k_sweep32<G, B, MINB>, smem, raised);
    uint64_t threads = (uint64_t)count * G;
    unsigned grid = (unsigned)((threads + B - 1) / B);
    if (cap && grid > cap) grid = cap;
    k_sweep32<G, B, MINB><<<grid, B, smem, st>>>(s, order, count);
}

template <int G, int B, int MINB>
unsigned resident_k32() {
    constexpr size_t smem = stage_bytes<G, B>();
    allow_dynamic_smem(k_sweep32<G, B, MINB>, smem);
    int dev = 0, sms = 0, per = 0;
    CC_CUDA(cudaGetDevice(&dev));
    CC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweep32<G, B, MINB>, B, smem));
    return (unsigned)(sms * (per > 0 ? per : 1));
}

// (lanes, cap, block) -> kernel instance; blocks of 64 and 256 threads exist
// for 8 and 16 lanes at the register budgets of caps 3-4 (64) and 4, 6, 8 (256)
template <int G, class F>
auto dispatch_cap32(const SweepVariant& v, F&& f) {
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
auto dispatch32(const SweepVariant& v, F&& f) {
    switch (v.lanes) {
        case 4: return dispatch_cap32<4>(SweepVariant{4, v.cap, 128, v.persistent}, f);
        case 16: return dispatch_cap32<16>(v, f);
        case 32: return dispatch_cap32<32>(SweepVariant{32, v.cap, 128, v.persistent}, f);
        default: return dispatch_cap32<8>(v, f);
    }
}

struct Launch32 {
    const SweepView& s;
    const uint32_t* order;
    uint32_t count;
    cudaStream_t st;
    unsigned cap;
    template <int G, int B, int MINB>
    int operator()() const {
        launch_k32<G, B, MINB>(s, order, count, st, cap);
        return 0;
    }
};
struct Resident32 {
    template <int G, int B, int MINB>
    unsigned operator()() const {
        return resident_k32<G, B, MINB>();
    }
};

}  // namespace

void launch_sweep32(const SweepView& s, const uint32_t* order, uint32_t count, int variant, cudaStream_t st,
                    unsigned grid_cap) {
    if (count == 0) return;
    SweepVariant v = decode_variant(variant);
    dispatch32(v, Launch32{s, order, count, st, v.persistent ? grid_cap : 0u});
}

unsigned sweep32_resident_blocks(int variant) { return dispatch32(decode_variant(variant), Resident32{}); }

}  // namespace cc
