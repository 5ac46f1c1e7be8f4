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
// All arithmetic is FP64: at cloth resolutions the in-plane membrane
// stiffness per vertex (~1e5 N/m) is six to seven orders above the inertia
// term (m/dt^2 ~ 1e-2 N/m), so an FP32 Hessian cannot represent the soft
// (out-of-plane) direction that gravity acts along.
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
__device__ __forceinline__ void sym_add_diag(Sym& h, double s) {
    h.a[0] += s;
    h.a[3] += s;
    h.a[5] += s;
}

struct M33 {
    double m[3][3];  // row-major
};
__device__ __forceinline__ M33 skew(d3 v) {  // [v]x : a -> v x a
    M33 r;
    r.m[0][0] = 0.0;
    r.m[0][1] = -v.z;
    r.m[0][2] = v.y;
    r.m[1][0] = v.z;
    r.m[1][1] = 0.0;
    r.m[1][2] = -v.x;
    r.m[2][0] = -v.y;
    r.m[2][1] = v.x;
    r.m[2][2] = 0.0;
    return r;
}

// ----------------------------------------------------------------- terms
// axial (src/energy.rs:10-16) with its first and second derivative.
__device__ __forceinline__ void axial3(double s, double k, double c, double delta, double& f, double& f1, double& f2) {
    double r = sqrt(s * s + delta * delta);
    double p = (s + r - delta) * 0.5;
    f = 0.5 * k * (c * s * s + (1.0 - c) * p * p);
    double p1 = 0.5 * (1.0 + s / r);
    double p2 = 0.5 * delta * delta / (r * r * r);
    f1 = k * (c * s + (1.0 - c) * p * p1);
    f2 = k * (c + (1.0 - c) * (p1 * p1 + p * p2));
}

__device__ __forceinline__ d3 pos(const SweepView& s, uint32_t i, uint32_t v, d3 p) {
    return i == v ? p : ld3(s.x, i);
}

// membrane (src/energy.rs:17-29) of triangle t with vertex slot `slot` at p.
template <bool D>
__device__ __forceinline__ double membrane_term(const SweepView& s, uint32_t t, uint32_t slot, d3 p, d3& g, Sym& H) {
    int4 tv = s.tri_v[t];
    double4 cf = s.tri_coef[t];
    double A = s.tri_area[t];
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
    double fw, fw1, fw2, fv, fv1, fv2;
    axial3(ew, M.warp, M.c, M.delta, fw, fw1, fw2);
    axial3(ev, M.weft, M.c, M.delta, fv, fv1, fv2);
    double e = A * (fw + fv + 0.5 * M.shear * sh * sh);
    if (D) {
        double aw = slot == 0 ? -(cf.x + cf.y) : (slot == 1 ? cf.x : cf.y);
        double av = slot == 0 ? -(cf.z + cf.w) : (slot == 1 ? cf.z : cf.w);
        d3 q = v * aw + w * av;
        g = g + (w * (fw1 * aw) + v * (fv1 * av) + q * (M.shear * sh)) * A;
        sym_add_outer(H, w, A * fw2 * aw * aw);
        sym_add_outer(H, v, A * fv2 * av * av);
        sym_add_outer(H, q, A * M.shear);
        sym_add_diag(H, A * (fw1 * aw * aw + fv1 * av * av + 2.0 * M.shear * sh * aw * av));
    }
    return e;
}

// bending (src/energy.rs:31-46) of hinge h with vertex slot `slot` at p.
template <bool D>
__device__ __forceinline__ double bending_term(const SweepView& s, uint32_t h, uint32_t slot, d3 p, d3& g, Sym& H) {
    uint4 hv = s.hinge_v[h];
    double K = s.hinge_k[h];
    d3 x0 = slot == 0 ? p : ld3(s.x, hv.x);
    d3 x1 = slot == 1 ? p : ld3(s.x, hv.y);
    d3 x2 = slot == 2 ? p : ld3(s.x, hv.z);
    d3 x3 = slot == 3 ? p : ld3(s.x, hv.w);
    d3 e = x1 - x0, u = x2 - x0, w = x3 - x0;
    d3 n1 = cross(e, u);
    d3 n2 = cross(w, e);
    double l1 = sqrt(dot(n1, n1));
    double l2 = sqrt(dot(n2, n2));
    d3 h1 = n1 / l1, h2 = n2 / l2;
    d3 d = h1 - h2;
    double energy = K * dot(d, d);
    if (D) {
        // dn/dp as cross-product matrices (n1, n2 are affine in one vertex)
        M33 A1, A2;
        bool has1 = slot != 3, has2 = slot != 2;
        if (slot == 0) {
            A1 = skew(u - e);
            A2 = skew(e - w);
        } else if (slot == 1) {
            A1 = skew(-u);
            A2 = skew(w);
        } else if (slot == 2) {
            A1 = skew(e);
        } else {
            A2 = skew(-e);
        }
        // J_k = (I - h h^T) A_k / l_k ; J = J1 - J2
        double J[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) J[i][j] = 0.0;
        double hh1[3] = {h1.x, h1.y, h1.z}, hh2[3] = {h2.x, h2.y, h2.z}, dd[3] = {d.x, d.y, d.z};
        if (has1) {
            for (int j = 0; j < 3; ++j) {
                double hA = hh1[0] * A1.m[0][j] + hh1[1] * A1.m[1][j] + hh1[2] * A1.m[2][j];
                for (int i = 0; i < 3; ++i) J[i][j] += (A1.m[i][j] - hh1[i] * hA) / l1;
            }
        }
        if (has2) {
            for (int j = 0; j < 3; ++j) {
                double hA = hh2[0] * A2.m[0][j] + hh2[1] * A2.m[1][j] + hh2[2] * A2.m[2][j];
                for (int i = 0; i < 3; ++i) J[i][j] -= (A2.m[i][j] - hh2[i] * hA) / l2;
            }
        }
        double gg[3];
        for (int j = 0; j < 3; ++j) gg[j] = 2.0 * K * (J[0][j] * dd[0] + J[1][j] * dd[1] + J[2][j] * dd[2]);
        g = g + mk(gg[0], gg[1], gg[2]);
        double Hm[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Hm[a][b] = J[0][a] * J[0][b] + J[1][a] * J[1][b] + J[2][a] * J[2][b];
        // + A^T M A with M = -(1/l^2)[d h^T + h d^T + (d.h)(I - 3 h h^T)], sign - for n2
        for (int k = 0; k < 2; ++k) {
            if ((k == 0 && !has1) || (k == 1 && !has2)) continue;
            const M33& A = k == 0 ? A1 : A2;
            const double* hk = k == 0 ? hh1 : hh2;
            double l = k == 0 ? l1 : l2;
            double dh = dd[0] * hk[0] + dd[1] * hk[1] + dd[2] * hk[2];
            double M[3][3];
            double sc = -1.0 / (l * l);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    M[i][j] = sc * (dd[i] * hk[j] + hk[i] * dd[j] + dh * ((i == j ? 1.0 : 0.0) - 3.0 * hk[i] * hk[j]));
            double MA[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) MA[i][j] = M[i][0] * A.m[0][j] + M[i][1] * A.m[1][j] + M[i][2] * A.m[2][j];
            double sign = k == 0 ? 1.0 : -1.0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    Hm[a][b] += sign * (A.m[0][a] * MA[0][b] + A.m[1][a] * MA[1][b] + A.m[2][a] * MA[2][b]);
        }
        double f = 2.0 * K;
        H.a[0] += f * Hm[0][0];
        H.a[1] += f * 0.5 * (Hm[0][1] + Hm[1][0]);
        H.a[2] += f * 0.5 * (Hm[0][2] + Hm[2][0]);
        H.a[3] += f * Hm[1][1];
        H.a[4] += f * 0.5 * (Hm[1][2] + Hm[2][1]);
        H.a[5] += f * Hm[2][2];
    }
    return energy;
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
    double e = 0.5 * K * dot(d, d);
    if (D) {
        g = g + d * (K * wv);
        sym_add_diag(H, K * wv * wv);
    }
    return e;
}

// ----------------------------------------------- contact: forward-mode AD
// Jet3 with a symmetric Hessian: the same second-order chain rules as
// src/math.rs:46-122, restricted to one vertex's three coordinates.
struct J3 {
    double v;
    double g[3];
    double h[6];
};
__device__ __forceinline__ J3 jc(double v) {
    J3 r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.g[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.h[i] = 0.0;
    return r;
}
__device__ __forceinline__ J3 jvar(double v, int i) {
    J3 r = jc(v);
    r.g[i] = 1.0;
    return r;
}
__device__ __forceinline__ J3 operator+(const J3& a, const J3& b) {
    J3 r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] + b.g[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) r.h[i] = a.h[i] + b.h[i];
    return r;
}
__device__ __forceinline__ J3 operator-(const J3& a, const J3& b) {
    J3 r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] - b.g[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) r.h[i] = a.h[i] - b.h[i];
    return r;
}
__device__ __forceinline__ J3 operator-(const J3& a) {
    J3 r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.g[i] = -a.g[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) r.h[i] = -a.h[i];
    return r;
}
__device__ __constant__ int kSymI[6] = {0, 0, 0, 1, 1, 2};
__device__ __constant__ int kSymJ[6] = {0, 1, 2, 1, 2, 2};
__device__ __forceinline__ J3 operator*(const J3& a, const J3& b) {
    J3 r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        int i = kSymI[k], j = kSymJ[k];
        r.h[k] = a.h[k] * b.v + a.v * b.h[k] + a.g[i] * b.g[j] + b.g[i] * a.g[j];
    }
    return r;
}
__device__ __forceinline__ J3 chain(const J3& a, double value, double first, double second) {
    J3 r;
    r.v = value;
#pragma unroll
    for (int i = 0; i < 3; ++i) r.g[i] = first * a.g[i];
#pragma unroll
    for (int k = 0; k < 6; ++k) r.h[k] = first * a.h[k] + second * a.g[kSymI[k]] * a.g[kSymJ[k]];
    return r;
}
__device__ __forceinline__ J3 operator/(const J3& a, const J3& b) {
    return a * chain(b, 1.0 / b.v, -1.0 / (b.v * b.v), 2.0 / (b.v * b.v * b.v));
}
__device__ __forceinline__ J3 jsqrt(const J3& a) {
    double r = sqrt(a.v);
    return chain(a, r, 0.5 / r, -0.25 / (r * r * r));
}
__device__ __forceinline__ J3 jln(const J3& a) { return chain(a, log(a.v), 1.0 / a.v, -1.0 / (a.v * a.v)); }
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
__device__ __forceinline__ double ssqrt(double x) { return sqrt(x); }
__device__ __forceinline__ J3 ssqrt(const J3& x) { return jsqrt(x); }
__device__ __forceinline__ double sln(double x) { return log(x); }
__device__ __forceinline__ J3 sln(const J3& x) { return jln(x); }

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

// Contact::energy (src/ogc/potential.rs:39-65)
template <class S>
__device__ __forceinline__ S contact_energy_t(uint32_t kind, double eps, const V<S> p[4], double r, double k) {
    S d;
    if (kind == 0) {
        V<S> v = vsub(p[0], p[1]);
        d = ssqrt(vdot(v, v));
    } else if (kind == 1) {
        V<S> u = vsub(p[2], p[1]);
        V<S> w = vsub(p[0], p[1]);
        S q = vdot(w, u) / vdot(u, u);
        V<S> dd = {w.x - q * u.x, w.y - q * u.y, w.z - q * u.z};
        d = ssqrt(vdot(dd, dd));
    } else if (kind == 2) {
        V<S> n = vcross(vsub(p[2], p[1]), vsub(p[3], p[1]));
        S h = vdot(vsub(p[0], p[1]), n) / ssqrt(vdot(n, n));
        d = sval(h) < 0.0 ? -h : h;
    } else {
        V<S> n = vcross(vsub(p[1], p[0]), vsub(p[3], p[2]));
        if (sval(vdot(n, n)) < 1e-30) return scst<S>(0.0);
        S h = vdot(vsub(p[0], p[2]), n) / ssqrt(vdot(n, n));
        d = sval(h) < 0.0 ? -h : h;
    }
    S e = activation(d, r, k);
    if (kind == 3) {
        V<S> n = vcross(vsub(p[1], p[0]), vsub(p[3], p[2]));
        S q = vdot(n, n) / scst<S>(eps);
        if (sval(q) < 1.0) e = e * q * (scst<S>(2.0) - q);
    }
    return e;
}

template <bool D>
__device__ __forceinline__ double contact_term(const SweepView& s, uint32_t c, uint32_t v, d3 p, d3& g, Sym& H) {
    uint32_t kind = s.contacts.kind[c];
    uint4 cv = s.contacts.verts[c];
    double eps = s.contacts.eps[c];
    uint32_t ids[4] = {cv.x, cv.y, cv.z, cv.w};
    if (D) {
        V<J3> q[4];
        for (int k = 0; k < 4; ++k) {
            if (ids[k] == v) {
                q[k] = {jvar(p.x, 0), jvar(p.y, 1), jvar(p.z, 2)};
            } else {
                d3 x = ld3(s.x, ids[k]);
                q[k] = {jc(x.x), jc(x.y), jc(x.z)};
            }
        }
        J3 e = contact_energy_t<J3>(kind, eps, q, s.contact_r, s.contact_k);
        g = g + mk(e.g[0], e.g[1], e.g[2]);
#pragma unroll
        for (int k = 0; k < 6; ++k) H.a[k] += e.h[k];
        return e.v;
    } else {
        V<double> q[4];
        for (int k = 0; k < 4; ++k) {
            d3 x = pos(s, ids[k], v, p);
            q[k] = {x.x, x.y, x.z};
        }
        return contact_energy_t<double>(kind, eps, q, s.contact_r, s.contact_k);
    }
}

// grab 0.5 k |sum w_j x_j - target|^2 (src/vbd.rs:237-246)
template <bool D>
__device__ __forceinline__ double grab_term(const SweepView& s, uint32_t v, d3 p, d3& g, Sym& H) {
    const GrabDev& G = s.grab;
    d3 d = mk(-G.target[0], -G.target[1], -G.target[2]);
    double wv = 0.0;
    for (int j = 0; j < 3; ++j) {
        d = d + pos(s, G.v[j], v, p) * G.w[j];
        if (G.v[j] == v) wv += G.w[j];
    }
    double e = 0.5 * G.k * dot(d, d);
    if (D) {
        g = g + d * (G.k * wv);
        sym_add_diag(H, G.k * wv * wv);
    }
    return e;
}

// Sum of every incident term (VbdSolver::local, src/vbd.rs:196-248).
template <bool D>
__device__ double local_sum(const SweepView& s, uint32_t v, d3 p, d3& g, Sym& H) {
    double e = 0.0;
    for (uint32_t k = s.inc_off[v]; k < s.inc_off[v + 1]; ++k) {
        uint32_t ent = s.inc[k];
        uint32_t type = ent >> 30, slot = (ent >> 28) & 3u, idx = ent & 0x0fffffffu;
        if (type == TERM_TRI) e += membrane_term<D>(s, idx, slot, p, g, H);
        else if (type == TERM_HINGE) e += bending_term<D>(s, idx, slot, p, g, H);
        else e += stitch_term<D>(s, idx, v, p, g, H);
    }
    for (uint32_t k = s.contacts.inc_off[v]; k < s.contacts.inc_off[v + 1]; ++k)
        e += contact_term<D>(s, s.contacts.inc[k], v, p, g, H);
    if (s.grab.active && (s.grab.v[0] == v || s.grab.v[1] == v || s.grab.v[2] == v)) e += grab_term<D>(s, v, p, g, H);
    return e;
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

__device__ void solve_vertex(const SweepView& s, uint32_t v) {
    if (s.pinned[v]) {
        s.residual[v] = 0.0;
        return;
    }
    d3 x = ld3(s.x, v);
    d3 y = ld3(s.target, v);
    double m = s.inertia[v];
    d3 g = mk(0, 0, 0);
    Sym H;
    sym_zero(H);
    double e_el = local_sum<true>(s, v, x, g, H);
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
        bool bound;
        cand = truncate_ball(s, v, cand, bound);
        truncated = truncated || bound;
        d3 gd;
        Sym Hd;
        double e = local_sum<false>(s, v, cand, gd, Hd);
        d3 cy = cand - y;
        e += 0.5 * m * dot(cy, cy);
        if (isfin(cand) && isfinite(e) && e <= old + 1e-14) {
            accepted = cand;
            break;
        }
    }
    st3(s.x, v, accepted);
    s.residual[v] = dot(g, g);
    s.clipped_flag[v] = truncated ? 1 : 0;
    if (truncated) atomicAdd(s.clipped, 1u);
}

__global__ void __launch_bounds__(128) k_sweep(SweepView s, const uint32_t* order, uint32_t count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) solve_vertex(s, order[i]);
}

void launch_sweep(const SweepView& s, const uint32_t* order, uint32_t count, int lanes, cudaStream_t st) {
    (void)lanes;
    if (count == 0) return;
    k_sweep<<<(count + 127) / 128, 128, 0, st>>>(s, order, count);
}

// Probe: local e, g, H of every moving vertex at the current positions
// (the f64 gradient check of src/gpu_vbd.rs:305-379, probe of vbd.wgsl:142-147).
__global__ void k_local_blocks(SweepView s, double* energy, double* grad, double* hess) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < s.n; v += gridDim.x * blockDim.x) {
        d3 x = ld3(s.x, v);
        d3 g = mk(0, 0, 0);
        Sym H;
        sym_zero(H);
        double e = local_sum<true>(s, v, x, g, H);
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

}  // namespace cc
