// Device-side terms of the VBD local solve shared by the FP64 sweep
// (sweep.cu) and the FP32-assembly sweep (sweep32.cu): 3x3 symmetric blocks,
// the FP64 membrane and bending terms with exact derivatives, stitches, the
// grab, and the OGC contact energy with its forward-mode (Jet3) derivatives.
#pragma once
#include "sweep.cuh"

namespace cc {

// --------------------------------------------------------------- 3x3 sym
struct Sym {  // xx xy xz yy yz zz
    double a[6];
};
__device__ __forceinline__ void sym_zero(Sym& h) {
#pragma unroll
    for (int i = 0; i < 6; ++i) h.a[i] = 0.0;
}
__device__ __forceinline__ void sym_add_outer(Sym& h, d3 u, double s) {  // h += s u u^T
    h.a[0] += s * u.x * u.x;
    h.a[1] += s * u.x * u.y;
    h.a[2] += s * u.x * u.z;
    h.a[3] += s * u.y * u.y;
    h.a[4] += s * u.y * u.z;
    h.a[5] += s * u.z * u.z;
}
__device__ __forceinline__ void sym_add_outer2(Sym& h, d3 u, d3 v, double s) {  // h += s (u v^T + v u^T)
    h.a[0] += s * 2.0 * u.x * v.x;
    h.a[1] += s * (u.x * v.y + v.x * u.y);
    h.a[2] += s * (u.x * v.z + v.x * u.z);
    h.a[3] += s * 2.0 * u.y * v.y;
    h.a[4] += s * (u.y * v.z + v.y * u.z);
    h.a[5] += s * 2.0 * u.z * v.z;
}
__device__ __forceinline__ void sym_add_diag(Sym& h, double s) {
    h.a[0] += s;
    h.a[3] += s;
    h.a[5] += s;
}

// ----------------------------------------------------------------- terms
// axial (src/energy.rs:10-16) with its first and second derivative. With
// c == 1 (the pure quadratic law, e.g. StVK mapped with compression ratio 1)
// every (1 - c) term is exactly zero, so the square root and the reciprocal
// of the compression branch are skipped; the results are the same bits.
__device__ __forceinline__ void axial3(double s, double k, double c, double delta, double& f, double& f1, double& f2) {
    if (c == 1.0) {
        f = 0.5 * k * (c * s * s);
        f1 = k * (c * s);
        f2 = k * c;
        return;
    }
    double r = sqrt(s * s + delta * delta);
    double ir = 1.0 / r;
    double p = (s + r - delta) * 0.5;
    f = 0.5 * k * (c * s * s + (1.0 - c) * p * p);
    double p1 = 0.5 * (1.0 + s * ir);
    double p2 = 0.5 * delta * delta * (ir * ir * ir);
    f1 = k * (c * s + (1.0 - c) * p * p1);
    f2 = k * (c + (1.0 - c) * (p1 * p1 + p * p2));
}
__device__ __forceinline__ double axial1(double s, double k, double c, double delta) {
    if (c == 1.0) return 0.5 * k * (c * s * s);
    double r = sqrt(s * s + delta * delta);
    double p = (s + r - delta) * 0.5;
    return 0.5 * k * (c * s * s + (1.0 - c) * p * p);
}

__device__ __forceinline__ d3 pos(const SweepView& s, uint32_t i, uint32_t v, d3 p) {
    return i == v ? p : ld3(s.x, i);
}

// membrane (src/energy.rs:17-29) of triangle t with vertex slot `slot` at p.
// D: derivatives; HS: also the Hessian (a gradient-only evaluation skips it)
template <bool D, bool HS = D>
__device__ __forceinline__ double membrane_rec(const SweepView& s, int4 tv, double4 cf, double A, uint32_t slot, d3 p,
                                               d3& g, Sym& H) {
    MatParams M = s.mats[tv.w];
    d3 x0 = slot == 0 ? p : ld3(s.x, (uint32_t)tv.x);
    d3 x1 = slot == 1 ? p : ld3(s.x, (uint32_t)tv.y);
    d3 x2 = slot == 2 ? p : ld3(s.x, (uint32_t)tv.z);
    d3 ds0 = x1 - x0, ds1 = x2 - x0;
    d3 w = ds0 * cf.x + ds1 * cf.y;
    d3 v = ds0 * cf.z + ds1 * cf.w;
    double ew = (dot(w, w) - 1.0) * 0.5;
    double ev = (dot(v, v) - 1.0) * 0.5;
    double sh = dot(w, v);
    if (!D) return A * (axial1(ew, M.warp, M.c, M.delta) + axial1(ev, M.weft, M.c, M.delta) + 0.5 * M.shear * sh * sh);
    double fw, fw1, fw2, fv, fv1, fv2;
    axial3(ew, M.warp, M.c, M.delta, fw, fw1, fw2);
    axial3(ev, M.weft, M.c, M.delta, fv, fv1, fv2);
    double aw = slot == 0 ? -(cf.x + cf.y) : (slot == 1 ? cf.x : cf.y);
    double av = slot == 0 ? -(cf.z + cf.w) : (slot == 1 ? cf.z : cf.w);
    d3 q = v * aw + w * av;
    g = g + (w * (fw1 * aw) + v * (fv1 * av) + q * (M.shear * sh)) * A;
    if (!HS) return A * (fw + fv + 0.5 * M.shear * sh * sh);
    sym_add_outer(H, w, A * fw2 * aw * aw);
    sym_add_outer(H, v, A * fv2 * av * av);
    sym_add_outer(H, q, A * M.shear);
    sym_add_diag(H, A * (fw1 * aw * aw + fv1 * av * av + 2.0 * M.shear * sh * aw * av));
    return A * (fw + fv + 0.5 * M.shear * sh * sh);
}

template <bool D, bool HS = D>
__device__ __forceinline__ double membrane_term(const SweepView& s, uint32_t t, uint32_t slot, d3 p, d3& g, Sym& H) {
    return membrane_rec<D, HS>(s, s.tri_v[t], s.tri_coef[t], s.tri_area[t], slot, p, g, H);
}

// P_k [a]x / l as three columns: P(a x e_j)/l, P y = y - h (h.y)
__device__ __forceinline__ void proj_skew_cols(d3 a, d3 h, double inv_l, double sign, d3& c0, d3& c1, d3& c2) {
    d3 e0 = mk(0.0, a.z, -a.y), e1 = mk(-a.z, 0.0, a.x), e2 = mk(a.y, -a.x, 0.0);
    double f = sign * inv_l;
    c0 = c0 + (e0 - h * dot(h, e0)) * f;
    c1 = c1 + (e1 - h * dot(h, e1)) * f;
    c2 = c2 + (e2 - h * dot(h, e2)) * f;
}

// [a]x^T M [a]x for M = -(1/l^2)[d h^T + h d^T + (d.h)(I - 3 h h^T)]
__device__ __forceinline__ void add_curvature(Sym& Hm, d3 a, d3 h, d3 d, double inv_l2, double sign) {
    d3 da = cross(d, a), ha = cross(h, a);
    double dh = dot(d, h);
    double sc = -inv_l2 * sign;
    sym_add_outer2(Hm, da, ha, sc);
    double aa = dot(a, a);
    sym_add_diag(Hm, sc * dh * aa);
    sym_add_outer(Hm, a, -sc * dh);
    sym_add_outer(Hm, ha, -3.0 * sc * dh);
}

// bending (src/energy.rs:31-46) of hinge h with vertex slot `slot` at p.
// n1 = e x u, n2 = w x e are affine in one vertex: dn_k/dp = [a_k]x.
template <bool D, bool HS = D>
__device__ __forceinline__ double bending_rec(const SweepView& s, uint4 hv, double K, uint32_t slot, d3 p, d3& g,
                                              Sym& H) {
    d3 x0 = slot == 0 ? p : ld3(s.x, hv.x);
    d3 x1 = slot == 1 ? p : ld3(s.x, hv.y);
    d3 x2 = slot == 2 ? p : ld3(s.x, hv.z);
    d3 x3 = slot == 3 ? p : ld3(s.x, hv.w);
    d3 e = x1 - x0, u = x2 - x0, w = x3 - x0;
    d3 n1 = cross(e, u);
    d3 n2 = cross(w, e);
    double il1 = rsqrt(dot(n1, n1));
    double il2 = rsqrt(dot(n2, n2));
    d3 h1 = n1 * il1, h2 = n2 * il2;
    d3 d = h1 - h2;
    double energy = K * dot(d, d);
    if (!D) return energy;
    d3 a1 = slot == 0 ? u - e : (slot == 1 ? -u : (slot == 2 ? e : mk(0, 0, 0)));
    d3 a2 = slot == 0 ? e - w : (slot == 1 ? w : (slot == 3 ? -e : mk(0, 0, 0)));
    // gradient 2K J^T d with J^T d = sum_k s_k ((P_k d) x a_k) / l_k
    d3 pd1 = d - h1 * dot(h1, d), pd2 = d - h2 * dot(h2, d);
    d3 jtd = cross(pd1, a1) * il1 - cross(pd2, a2) * il2;
    g = g + jtd * (2.0 * K);
    if (!HS) return energy;
    // Hessian 2K [J^T J + A1^T M1 A1 - A2^T M2 A2]
    d3 c0 = mk(0, 0, 0), c1 = mk(0, 0, 0), c2 = mk(0, 0, 0);
    proj_skew_cols(a1, h1, il1, 1.0, c0, c1, c2);
    proj_skew_cols(a2, h2, il2, -1.0, c0, c1, c2);
    Sym Hm;
    Hm.a[0] = dot(c0, c0);
    Hm.a[1] = dot(c0, c1);
    Hm.a[2] = dot(c0, c2);
    Hm.a[3] = dot(c1, c1);
    Hm.a[4] = dot(c1, c2);
    Hm.a[5] = dot(c2, c2);
    add_curvature(Hm, a1, h1, d, il1 * il1, 1.0);
    add_curvature(Hm, a2, h2, d, il2 * il2, -1.0);
    double f = 2.0 * K;
#pragma unroll
    for (int k = 0; k < 6; ++k) H.a[k] += f * Hm.a[k];
    return energy;
}

template <bool D, bool HS = D>
__device__ __forceinline__ double bending_term(const SweepView& s, uint32_t hi, uint32_t slot, d3 p, d3& g, Sym& H) {
    return bending_rec<D, HS>(s, s.hinge_v[hi], s.hinge_k[hi], slot, p, g, H);
}

// stitch 0.5 k |sum w_j x_j|^2 (src/vbd.rs:217-227)
template <bool D>
__device__ __forceinline__ double stitch_term(const SweepView& s, uint32_t st, uint32_t v, d3 p, d3& g, Sym& H) {
    d3 d = mk(0, 0, 0);
    double wv = 0.0;
    for (uint32_t k = s.st_off[st]; k < s.st_off[st + 1]; ++k) {
        uint32_t j = s.st_v[k];
        double w = s.st_w[k];
        d = d + pos(s, j, v, p) * w;
        if (j == v) wv += w;
    }
    double K = s.st_k[st];
    if (D) {
        g = g + d * (K * wv);
        sym_add_diag(H, K * wv * wv);
    }
    return 0.5 * K * dot(d, d);
}

// ----------------------------------------------- contact: forward-mode AD
// Jet3 with a symmetric Hessian: the second-order chain rules of
// src/math.rs:46-122, restricted to one vertex's three coordinates.
struct J3 {
    double v;
    double g0, g1, g2;
    double h00, h01, h02, h11, h12, h22;
};
__device__ __forceinline__ J3 jc(double v) { return {v, 0, 0, 0, 0, 0, 0, 0, 0, 0}; }
__device__ __forceinline__ J3 operator+(const J3& a, const J3& b) {
    return {a.v + b.v,     a.g0 + b.g0,   a.g1 + b.g1,   a.g2 + b.g2,   a.h00 + b.h00,
            a.h01 + b.h01, a.h02 + b.h02, a.h11 + b.h11, a.h12 + b.h12, a.h22 + b.h22};
}
__device__ __forceinline__ J3 operator-(const J3& a, const J3& b) {
    return {a.v - b.v,     a.g0 - b.g0,   a.g1 - b.g1,   a.g2 - b.g2,   a.h00 - b.h00,
            a.h01 - b.h01, a.h02 - b.h02, a.h11 - b.h11, a.h12 - b.h12, a.h22 - b.h22};
}
__device__ __forceinline__ J3 operator-(const J3& a) {
    return {-a.v, -a.g0, -a.g1, -a.g2, -a.h00, -a.h01, -a.h02, -a.h11, -a.h12, -a.h22};
}
__device__ __forceinline__ J3 operator*(const J3& a, const J3& b) {
    J3 r;
    r.v = a.v * b.v;
    r.g0 = a.g0 * b.v + a.v * b.g0;
    r.g1 = a.g1 * b.v + a.v * b.g1;
    r.g2 = a.g2 * b.v + a.v * b.g2;
    r.h00 = a.h00 * b.v + a.v * b.h00 + 2.0 * a.g0 * b.g0;
    r.h01 = a.h01 * b.v + a.v * b.h01 + a.g0 * b.g1 + b.g0 * a.g1;
    r.h02 = a.h02 * b.v + a.v * b.h02 + a.g0 * b.g2 + b.g0 * a.g2;
    r.h11 = a.h11 * b.v + a.v * b.h11 + 2.0 * a.g1 * b.g1;
    r.h12 = a.h12 * b.v + a.v * b.h12 + a.g1 * b.g2 + b.g1 * a.g2;
    r.h22 = a.h22 * b.v + a.v * b.h22 + 2.0 * a.g2 * b.g2;
    return r;
}
__device__ __forceinline__ J3 chain(const J3& a, double value, double f1, double f2) {
    J3 r;
    r.v = value;
    r.g0 = f1 * a.g0;
    r.g1 = f1 * a.g1;
    r.g2 = f1 * a.g2;
    r.h00 = f1 * a.h00 + f2 * a.g0 * a.g0;
    r.h01 = f1 * a.h01 + f2 * a.g0 * a.g1;
    r.h02 = f1 * a.h02 + f2 * a.g0 * a.g2;
    r.h11 = f1 * a.h11 + f2 * a.g1 * a.g1;
    r.h12 = f1 * a.h12 + f2 * a.g1 * a.g2;
    r.h22 = f1 * a.h22 + f2 * a.g2 * a.g2;
    return r;
}
__device__ __forceinline__ J3 operator/(const J3& a, const J3& b) {
    return a * chain(b, 1.0 / b.v, -1.0 / (b.v * b.v), 2.0 / (b.v * b.v * b.v));
}
__device__ __forceinline__ J3 ssqrt(const J3& a) {
    double r = sqrt(a.v);
    return chain(a, r, 0.5 / r, -0.25 / (r * r * r));
}
__device__ __forceinline__ J3 sln(const J3& a) { return chain(a, log(a.v), 1.0 / a.v, -1.0 / (a.v * a.v)); }
__device__ __forceinline__ double ssqrt(double x) { return sqrt(x); }
__device__ __forceinline__ double sln(double x) { return log(x); }
__device__ __forceinline__ double sval(double x) { return x; }
__device__ __forceinline__ double sval(const J3& x) { return x.v; }
template <class S>
__device__ __forceinline__ S scst(double v);
template <>
__device__ __forceinline__ double scst<double>(double v) {
    return v;
}
template <>
__device__ __forceinline__ J3 scst<J3>(double v) {
    return jc(v);
}

template <class S>
struct V {
    S x, y, z;
};
template <class S>
__device__ __forceinline__ V<S> vsub(const V<S>& a, const V<S>& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class S>
__device__ __forceinline__ S vdot(const V<S>& a, const V<S>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class S>
__device__ __forceinline__ V<S> vcross(const V<S>& a, const V<S>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// activation (src/ogc/potential.rs:8-22)
template <class S>
__device__ __forceinline__ S activation(const S& d, double r, double k) {
    if (sval(d) >= r) return scst<S>(0.0);
    if (sval(d) <= 0.0) return scst<S>(__longlong_as_double(0x7ff0000000000000ll));
    double tau = 0.5 * r;
    if (sval(d) >= tau) {
        S gg = scst<S>(r) - d;
        return scst<S>(0.5 * k) * gg * gg;
    }
    return scst<S>(0.5 * k * tau * tau) - scst<S>(k * tau * tau) * sln(d / scst<S>(tau));
}

// Contact distance of Contact::energy (src/ogc/potential.rs:39-65) on four
// named points; `degenerate` is set for an EE pair with |n|^2 < 1e-30 (energy 0).
template <class S>
__device__ __forceinline__ S contact_distance(uint32_t kind, const V<S>& p0, const V<S>& p1, const V<S>& p2,
                                              const V<S>& p3, bool& degenerate) {
    degenerate = false;
    if (kind == 0) {
        V<S> v = vsub(p0, p1);
        return ssqrt(vdot(v, v));
    }
    if (kind == 1) {
        V<S> u = vsub(p2, p1);
        V<S> w = vsub(p0, p1);
        S q = vdot(w, u) / vdot(u, u);
        V<S> dd = {w.x - q * u.x, w.y - q * u.y, w.z - q * u.z};
        return ssqrt(vdot(dd, dd));
    }
    if (kind == 2) {
        V<S> n = vcross(vsub(p2, p1), vsub(p3, p1));
        S h = vdot(vsub(p0, p1), n) / ssqrt(vdot(n, n));
        return sval(h) < 0.0 ? -h : h;
    }
    V<S> n = vcross(vsub(p1, p0), vsub(p3, p2));
    if (sval(vdot(n, n)) < 1e-30) {
        degenerate = true;
        return scst<S>(0.0);
    }
    S h = vdot(vsub(p0, p2), n) / ssqrt(vdot(n, n));
    return sval(h) < 0.0 ? -h : h;
}

// Contact::energy (src/ogc/potential.rs:39-65) on four named points.
template <class S>
__device__ __forceinline__ S contact_energy_t(uint32_t kind, double eps, const V<S>& p0, const V<S>& p1,
                                              const V<S>& p2, const V<S>& p3, double r, double k) {
    bool degenerate;
    S d = contact_distance<S>(kind, p0, p1, p2, p3, degenerate);
    if (degenerate) return scst<S>(0.0);
    S e = activation(d, r, k);
    if (kind == 3) {
        V<S> n = vcross(vsub(p1, p0), vsub(p3, p2));
        S q = vdot(n, n) / scst<S>(eps);
        if (sval(q) < 1.0) e = e * q * (scst<S>(2.0) - q);
    }
    return e;
}

// ---- mixed Jet/constant arithmetic: only the moving vertex carries derivatives
__device__ __forceinline__ J3 operator+(const J3& a, double b) {
    J3 r = a;
    r.v += b;
    return r;
}
__device__ __forceinline__ J3 operator+(double a, const J3& b) { return b + a; }
__device__ __forceinline__ J3 operator-(const J3& a, double b) {
    J3 r = a;
    r.v -= b;
    return r;
}
__device__ __forceinline__ J3 operator-(double a, const J3& b) {
    J3 r = -b;
    r.v += a;
    return r;
}
__device__ __forceinline__ J3 operator*(const J3& a, double b) {
    return {a.v * b, a.g0 * b, a.g1 * b, a.g2 * b, a.h00 * b, a.h01 * b, a.h02 * b, a.h11 * b, a.h12 * b, a.h22 * b};
}
__device__ __forceinline__ J3 operator*(double a, const J3& b) { return b * a; }
__device__ __forceinline__ J3 operator/(const J3& a, double b) { return a * (1.0 / b); }
__device__ __forceinline__ J3 operator/(double a, const J3& b) {
    return chain(b, 1.0 / b.v, -1.0 / (b.v * b.v), 2.0 / (b.v * b.v * b.v)) * a;
}
__device__ __forceinline__ J3 to_j3(const J3& a) { return a; }
__device__ __forceinline__ J3 to_j3(double a) { return jc(a); }

template <class A, class B>
struct Pro {
    using T = J3;
};
template <>
struct Pro<double, double> {
    using T = double;
};
template <class A, class B>
__device__ __forceinline__ V<typename Pro<A, B>::T> msub(const V<A>& a, const V<B>& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class A, class B>
__device__ __forceinline__ typename Pro<A, B>::T mdot(const V<A>& a, const V<B>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class A, class B>
__device__ __forceinline__ V<typename Pro<A, B>::T> mcross(const V<A>& a, const V<B>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Contact::energy (src/ogc/potential.rs:39-65) with per-point types.
template <class S0, class S1, class S2, class S3>
__device__ __forceinline__ J3 contact_jet(uint32_t kind, double eps, const V<S0>& p0, const V<S1>& p1,
                                          const V<S2>& p2, const V<S3>& p3, double r, double k) {
    if (kind == 0) {
        auto v = msub(p0, p1);
        return to_j3(activation(ssqrt(mdot(v, v)), r, k));
    }
    if (kind == 1) {
        auto u = msub(p2, p1);
        auto w = msub(p0, p1);
        auto q = mdot(w, u) / mdot(u, u);
        auto dx = w.x - q * u.x;
        auto dy = w.y - q * u.y;
        auto dz = w.z - q * u.z;
        return to_j3(activation(ssqrt(dx * dx + dy * dy + dz * dz), r, k));
    }
    if (kind == 2) {
        auto n = mcross(msub(p2, p1), msub(p3, p1));
        auto h = mdot(msub(p0, p1), n) / ssqrt(mdot(n, n));
        auto d = sval(h) < 0.0 ? -h : h;
        return to_j3(activation(d, r, k));
    }
    auto n = mcross(msub(p1, p0), msub(p3, p2));
    auto nn = mdot(n, n);
    if (sval(nn) < 1e-30) return jc(0.0);
    auto h = mdot(msub(p0, p2), n) / ssqrt(nn);
    auto d = sval(h) < 0.0 ? -h : h;
    J3 e = to_j3(activation(d, r, k));
    J3 q = to_j3(nn / eps);
    if (q.v < 1.0) e = e * q * (2.0 - q);
    return e;
}

__device__ __forceinline__ V<J3> var_point(d3 p) {
    J3 a = jc(p.x), b = jc(p.y), c = jc(p.z);
    a.g0 = 1.0;
    b.g1 = 1.0;
    c.g2 = 1.0;
    return {a, b, c};
}
__device__ __forceinline__ V<double> cst_point(const SweepView& s, uint32_t id) {
    d3 x = ld3(s.x, id);
    return {x.x, x.y, x.z};
}
__device__ __forceinline__ V<double> dpoint(const SweepView& s, uint32_t id, uint32_t v, d3 p) {
    d3 x = pos(s, id, v, p);
    return {x.x, x.y, x.z};
}

template <bool D>
__device__ __forceinline__ double contact_term(const SweepView& s, uint32_t c, uint32_t v, d3 p, d3& g, Sym& H) {
    uint32_t kind = s.contacts.kind[c];
    uint4 cv = s.contacts.verts[c];
    double eps = s.contacts.eps[c];
    if (D) {
        // Inactive term (d >= r): the activation is the constant 0, so the term
        // adds nothing to e, g or H; skip its derivative evaluation.
        bool degenerate;
        double d0 = contact_distance<double>(kind, dpoint(s, cv.x, v, p), dpoint(s, cv.y, v, p),
                                             dpoint(s, cv.z, v, p), dpoint(s, cv.w, v, p), degenerate);
        if (degenerate || d0 >= s.contact_r) return 0.0;
        // the moving vertex's slot among the used ones (unused slots hold 0)
        uint32_t cnt = kind == 0 ? 2u : (kind == 1 ? 3u : 4u);
        int slot = cv.x == v ? 0 : (cv.y == v ? 1 : ((cnt > 2 && cv.z == v) ? 2 : 3));
        double r = s.contact_r, k = s.contact_k;
        J3 e;
        if (slot == 0)
            e = contact_jet(kind, eps, var_point(p), cst_point(s, cv.y), cst_point(s, cv.z), cst_point(s, cv.w), r, k);
        else if (slot == 1)
            e = contact_jet(kind, eps, cst_point(s, cv.x), var_point(p), cst_point(s, cv.z), cst_point(s, cv.w), r, k);
        else if (slot == 2)
            e = contact_jet(kind, eps, cst_point(s, cv.x), cst_point(s, cv.y), var_point(p), cst_point(s, cv.w), r, k);
        else
            e = contact_jet(kind, eps, cst_point(s, cv.x), cst_point(s, cv.y), cst_point(s, cv.z), var_point(p), r, k);
        g = g + mk(e.g0, e.g1, e.g2);
        H.a[0] += e.h00;
        H.a[1] += e.h01;
        H.a[2] += e.h02;
        H.a[3] += e.h11;
        H.a[4] += e.h12;
        H.a[5] += e.h22;
        return e.v;
    }
    return contact_energy_t<double>(kind, eps, dpoint(s, cv.x, v, p), dpoint(s, cv.y, v, p), dpoint(s, cv.z, v, p),
                                    dpoint(s, cv.w, v, p), s.contact_r, s.contact_k);
}

// grab 0.5 k |sum w_j x_j - target|^2 (src/vbd.rs:237-246)
template <bool D>
__device__ __forceinline__ double grab_term(const SweepView& s, uint32_t v, d3 p, d3& g, Sym& H) {
    const GrabDev& G = s.grab;
    d3 d = mk(-G.target[0], -G.target[1], -G.target[2]);
    double wv = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        d = d + pos(s, G.v[j], v, p) * G.w[j];
        if (G.v[j] == v) wv += G.w[j];
    }
    if (D) {
        g = g + d * (G.k * wv);
        sym_add_diag(H, G.k * wv * wv);
    }
    return 0.5 * G.k * dot(d, d);
}

// Partial sum of the incident terms dealt to `lane` of a group of G
// (VbdSolver::local, src/vbd.rs:196-248).
template <bool D, int G, bool HS = D>
__device__ __forceinline__ double local_part(const SweepView& s, uint32_t v, d3 p, uint32_t lane, d3& g, Sym& H) {
    double e = 0.0;
    // entries are grouped by type: one lane-strided loop per type, no per-entry dispatch
    uint32_t b0 = s.inc_off[v], b1 = s.inc_off[v + 1];
    uint2 mid = s.inc_mid[v];
    // each loop loads the next term's record before it evaluates the current one
    {
        uint32_t k = b0 + lane;
        uint32_t ent = k < mid.x ? s.inc[k] : 0u;
        int4 tv = make_int4(0, 0, 0, 0);
        double4 cf = make_double4(0, 0, 0, 0);
        double A = 0.0;
        if (k < mid.x) {
            uint32_t t = ent & 0x0fffffffu;
            tv = s.tri_v[t];
            cf = s.tri_coef[t];
            A = s.tri_area[t];
        }
        for (; k < mid.x; k += G) {
            uint32_t kn = k + G;
            uint32_t en = 0u;
            int4 tvn = tv;
            double4 cfn = cf;
            double An = A;
            if (kn < mid.x) {
                en = s.inc[kn];
                uint32_t t = en & 0x0fffffffu;
                tvn = s.tri_v[t];
                cfn = s.tri_coef[t];
                An = s.tri_area[t];
            }
            e += membrane_rec<D, HS>(s, tv, cf, A, (ent >> 28) & 3u, p, g, H);
            ent = en;
            tv = tvn;
            cf = cfn;
            A = An;
        }
    }
    {
        uint32_t k = mid.x + lane;
        uint32_t ent = k < mid.y ? s.inc[k] : 0u;
        uint4 hv = make_uint4(0, 0, 0, 0);
        double K = 0.0;
        if (k < mid.y) {
            uint32_t h = ent & 0x0fffffffu;
            hv = s.hinge_v[h];
            K = s.hinge_k[h];
        }
        for (; k < mid.y; k += G) {
            uint32_t kn = k + G;
            uint32_t en = 0u;
            uint4 hvn = hv;
            double Kn = K;
            if (kn < mid.y) {
                en = s.inc[kn];
                uint32_t h = en & 0x0fffffffu;
                hvn = s.hinge_v[h];
                Kn = s.hinge_k[h];
            }
            e += bending_rec<D, HS>(s, hv, K, (ent >> 28) & 3u, p, g, H);
            ent = en;
            hv = hvn;
            K = Kn;
        }
    }
    for (uint32_t k = mid.y + lane; k < b1; k += G) e += stitch_term<D>(s, s.inc[k] & 0x0fffffffu, v, p, g, H);
    uint32_t c1 = s.contacts.inc_off[v + 1];
    for (uint32_t k = s.contacts.inc_off[v] + lane; k < c1; k += G) e += contact_term<D>(s, s.contacts.inc[k], v, p, g, H);
    if (lane == 0 && s.grab.active && (s.grab.v[0] == v || s.grab.v[1] == v || s.grab.v[2] == v))
        e += grab_term<D>(s, v, p, g, H);
    return e;
}

template <int G>
__device__ __forceinline__ double group_sum(double x, unsigned mask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(mask, x, o, G);
    return x;
}

__device__ __forceinline__ d3 truncate_ball(const SweepView& s, uint32_t v, d3 proposed, bool& clipped) {  // world.rs:91-100
    d3 c = ld3(s.contacts.centers, v);
    d3 d = proposed - c;
    double l = len(d);
    double b = s.contacts.radii[v];
    if (l > b) {
        clipped = true;
        return c + d * (b / l);
    }
    clipped = false;
    return proposed;
}

}  // namespace cc
