// Oracle (test infrastructure only): FP64 restatement of ClothCraft's CPU
// math. Nothing in the product library links this; tests, smoke() and the
// bench's CPU-baseline leg load it as the checker.
//
// Follows, operation for operation where rounding could matter:
//   src/math.rs:4-136     Scalar / Jet<N> second-order forward AD, sub/dot/cross
//   src/energy.rs:10-46   axial, membrane, bending
//   src/ogc/potential.rs  activation, Contact::energy
//   src/ogc/geometry.rs   feasible regions, closest features, distances
// glam 0.34.1 (third-party, Cargo.lock:930-931) supplies DVec3 arithmetic and
// DMat3::inverse; both are restated here (component-wise ops; inverse as
// adjugate / determinant, glam's published cofactor formula).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace oracle {

// ------------------------------------------------------------------ Jet<N>
// src/math.rs:33-122
template <int N>
struct Jet {
    double v;
    double g[N];
    double h[N][N];
};

template <class S>
struct Sc;  // Scalar trait (src/math.rs:4-16)

template <>
struct Sc<double> {
    static double c(double v) { return v; }
    static double value(double x) { return x; }
};

template <int N>
struct Sc<Jet<N>> {
    static Jet<N> c(double v) {
        Jet<N> r;
        r.v = v;
        for (int i = 0; i < N; ++i) {
            r.g[i] = 0.0;
            for (int j = 0; j < N; ++j) r.h[i][j] = 0.0;
        }
        return r;
    }
    static double value(const Jet<N>& x) { return x.v; }
};

template <int N>
inline Jet<N> variable(double v, int i) {  // src/math.rs:41-45
    Jet<N> x = Sc<Jet<N>>::c(v);
    x.g[i] = 1.0;
    return x;
}

template <int N>
inline Jet<N> chain(const Jet<N>& s, double value, double first, double second) {  // src/math.rs:46-54
    Jet<N> r;
    r.v = value;
    for (int i = 0; i < N; ++i) r.g[i] = first * s.g[i];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) r.h[i][j] = first * s.h[i][j] + second * s.g[i] * s.g[j];
    return r;
}

template <int N>
inline Jet<N> operator+(const Jet<N>& a, const Jet<N>& b) {  // src/math.rs:76-85
    Jet<N> r;
    r.v = a.v + b.v;
    for (int i = 0; i < N; ++i) r.g[i] = a.g[i] + b.g[i];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) r.h[i][j] = a.h[i][j] + b.h[i][j];
    return r;
}

template <int N>
inline Jet<N> operator*(const Jet<N>& a, const Jet<N>& b) {  // src/math.rs:100-116
    Jet<N> r;
    r.v = a.v * b.v;
    for (int i = 0; i < N; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            r.h[i][j] = a.h[i][j] * b.v + a.v * b.h[i][j] + a.g[i] * b.g[j] + b.g[i] * a.g[j];
    return r;
}

template <int N>
inline Jet<N> operator-(const Jet<N>& a) {  // src/math.rs:86-91 (self * c(-1))
    return a * Sc<Jet<N>>::c(-1.0);
}

template <int N>
inline Jet<N> operator-(const Jet<N>& a, const Jet<N>& b) {  // src/math.rs:92-97
    return a + (-b);
}

template <int N>
inline Jet<N> operator/(const Jet<N>& a, const Jet<N>& b) {  // src/math.rs:117-122
    return a * chain(b, 1.0 / b.v, -1.0 / (b.v * b.v), 2.0 / (b.v * b.v * b.v));
}

inline double ssqrt(double x) { return std::sqrt(x); }
inline double sln(double x) { return std::log(x); }

template <int N>
inline Jet<N> ssqrt(const Jet<N>& x) {  // src/math.rs:68-71
    double r = std::sqrt(x.v);
    return chain(x, r, 0.5 / r, -0.25 / (r * r * r));
}

template <int N>
inline Jet<N> sln(const Jet<N>& x) {  // src/math.rs:72-74
    return chain(x, std::log(x.v), 1.0 / x.v, -1.0 / (x.v * x.v));
}

template <class S>
inline double val(const S& x) {
    return Sc<S>::value(x);
}
template <class S>
inline S C(double v) {
    return Sc<S>::c(v);
}

template <class S>
struct V3 {
    S a[3];
    S& operator[](int i) { return a[i]; }
    const S& operator[](int i) const { return a[i]; }
};

template <class S>
inline V3<S> vsub(const V3<S>& a, const V3<S>& b) {  // src/math.rs:124-126
    return {{a[0] - b[0], a[1] - b[1], a[2] - b[2]}};
}
template <class S>
inline S vdot(const V3<S>& a, const V3<S>& b) {  // src/math.rs:127-129
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
template <class S>
inline V3<S> vcross(const V3<S>& a, const V3<S>& b) {  // src/math.rs:130-136
    return {{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
}

// ------------------------------------------------------------ plain DVec3
struct D3 {
    double x, y, z;
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline D3 operator-(D3 a) { return {-a.x, -a.y, -a.z}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline double length_squared(D3 a) { return dot(a, a); }
inline double length(D3 a) { return std::sqrt(dot(a, a)); }
inline double distance(D3 a, D3 b) { return length(a - b); }
inline double distance_squared(D3 a, D3 b) { return length_squared(a - b); }
inline bool finite(D3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline bool operator==(D3 a, D3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline D3 vmin(D3 a, D3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline D3 vmax(D3 a, D3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
inline D3 vabs(D3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline double max_element(D3 a) { return std::fmax(std::fmax(a.x, a.y), a.z); }

template <class S>
inline V3<S> lift(D3 p) {
    return {{C<S>(p.x), C<S>(p.y), C<S>(p.z)}};
}

// glam DMat3 restated: columns c0, c1, c2.
struct M3 {
    D3 c[3];
};
inline M3 m3_identity_scaled(double s) { return {{{s, 0, 0}, {0, s, 0}, {0, 0, s}}}; }
inline M3 operator+(const M3& a, const M3& b) {
    return {{a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]}};
}
// DMat3::inverse: adjugate (cross products of columns) over the determinant.
inline M3 inverse(const M3& m) {
    D3 tmp0 = cross(m.c[1], m.c[2]);
    D3 tmp1 = cross(m.c[2], m.c[0]);
    D3 tmp2 = cross(m.c[0], m.c[1]);
    double det = dot(m.c[2], tmp2);
    double inv_det = 1.0 / det;
    // transpose of [tmp0 tmp1 tmp2] scaled
    M3 r;
    r.c[0] = {tmp0.x * inv_det, tmp1.x * inv_det, tmp2.x * inv_det};
    r.c[1] = {tmp0.y * inv_det, tmp1.y * inv_det, tmp2.y * inv_det};
    r.c[2] = {tmp0.z * inv_det, tmp1.z * inv_det, tmp2.z * inv_det};
    return r;
}
inline D3 mul(const M3& m, D3 v) {  // column-major matrix times vector
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}

// ------------------------------------------------------------------ energy
struct Material {  // src/model.rs:7-22
    double warp, weft, shear, compression_ratio, compression_transition;
    double bend_warp, bend_weft, density, thickness, grain_degrees;
};

inline void grain_sin_cos(double degrees, double& s, double& c) {
    double r = degrees * (M_PI / 180.0);  // f64::to_radians
    s = std::sin(r);
    c = std::cos(r);
}

template <class S>
inline S axial(const S& strain, double stiffness, const Material& m) {  // src/energy.rs:10-16
    S delta = C<S>(m.compression_transition);
    S p = (strain + ssqrt(strain * strain + delta * delta) - delta) * C<S>(0.5);
    return C<S>(0.5 * stiffness) *
           (C<S>(m.compression_ratio) * strain * strain + C<S>(1.0 - m.compression_ratio) * p * p);
}

// inv_dm columns: (ix.x, ix.y), (iy.x, iy.y)
template <class S>
inline S membrane(const V3<S> x[3], const double inv_dm[4], double area, const Material& m) {  // src/energy.rs:17-29
    V3<S> ds[2] = {vsub(x[1], x[0]), vsub(x[2], x[0])};
    V3<S> f[2];
    for (int col = 0; col < 2; ++col) {
        double cx = inv_dm[2 * col + 0], cy = inv_dm[2 * col + 1];
        for (int k = 0; k < 3; ++k) f[col][k] = ds[0][k] * C<S>(cx) + ds[1][k] * C<S>(cy);
    }
    double s, c;
    grain_sin_cos(m.grain_degrees, s, c);
    V3<S> w, v;
    for (int i = 0; i < 3; ++i) w[i] = f[0][i] * C<S>(c) + f[1][i] * C<S>(s);
    for (int i = 0; i < 3; ++i) v[i] = f[0][i] * C<S>(-s) + f[1][i] * C<S>(c);
    S ew = (vdot(w, w) - C<S>(1.0)) * C<S>(0.5);
    S ev = (vdot(v, v) - C<S>(1.0)) * C<S>(0.5);
    S shear = vdot(w, v);
    return C<S>(area) * (axial(ew, m.warp, m) + axial(ev, m.weft, m) + C<S>(0.5 * m.shear) * shear * shear);
}

template <class S>
inline S bending(const V3<S> x[4], double weight, const double across[2], const Material& m) {  // src/energy.rs:31-46
    V3<S> edge = vsub(x[1], x[0]);
    V3<S> n1 = vcross(edge, vsub(x[2], x[0]));
    V3<S> n2 = vcross(vsub(x[3], x[0]), edge);
    S length1 = ssqrt(vdot(n1, n1));
    S length2 = ssqrt(vdot(n2, n2));
    V3<S> difference;
    for (int i = 0; i < 3; ++i) difference[i] = n1[i] / length1 - n2[i] / length2;
    double s, c;
    grain_sin_cos(m.grain_degrees, s, c);
    double aw = across[0] * c + across[1] * s;
    double af = -across[0] * s + across[1] * c;
    return C<S>(0.5 * weight * (m.bend_warp * aw * aw + m.bend_weft * af * af)) * vdot(difference, difference);
}

// --------------------------------------------------------------- potential
template <class S>
inline S activation(const S& d, double r, double k) {  // src/ogc/potential.rs:8-22
    if (val(d) >= r) return C<S>(0.0);
    if (val(d) <= 0.0) return C<S>(std::numeric_limits<double>::infinity());
    double tau = 0.5 * r;
    if (val(d) >= tau) {
        S g = C<S>(r) - d;
        return C<S>(0.5 * k) * g * g;
    }
    return C<S>(0.5 * k * tau * tau) - C<S>(k * tau * tau) * sln(d / C<S>(tau));
}

enum Kind : uint8_t { PointPoint = 0, PointEdge = 1, PointFace = 2, EdgeEdge = 3 };  // src/ogc/potential.rs:24-30

struct Contact {  // src/ogc/potential.rs:31-37
    uint8_t kind;
    uint32_t vertices[4];
    uint8_t count;
    double mollifier_epsilon;
};

template <class S>
inline S point_edge_distance(const V3<S>& p, const V3<S>& a, const V3<S>& b) {  // src/ogc/geometry.rs:111-117
    V3<S> u = vsub(b, a);
    V3<S> w = vsub(p, a);
    S q = vdot(w, u) / vdot(u, u);
    V3<S> d;
    for (int k = 0; k < 3; ++k) d[k] = w[k] - q * u[k];
    return ssqrt(vdot(d, d));
}
template <class S>
inline S point_face_distance(const V3<S>& p, const V3<S>& a, const V3<S>& b, const V3<S>& c) {  // geometry.rs:118-122
    V3<S> n = vcross(vsub(b, a), vsub(c, a));
    S h = vdot(vsub(p, a), n) / ssqrt(vdot(n, n));
    if (val(h) < 0.0) return -h;
    return h;
}
template <class S>
inline S edge_edge_distance(const V3<S>& a, const V3<S>& b, const V3<S>& c, const V3<S>& d) {  // geometry.rs:123-127
    V3<S> n = vcross(vsub(b, a), vsub(d, c));
    S h = vdot(vsub(a, c), n) / ssqrt(vdot(n, n));
    if (val(h) < 0.0) return -h;
    return h;
}

template <class S>
inline S contact_energy(const Contact& ct, const V3<S> p[4], double r, double k) {  // potential.rs:39-65
    S d;
    switch (ct.kind) {
        case PointPoint: {
            V3<S> v = vsub(p[0], p[1]);
            d = ssqrt(vdot(v, v));
            break;
        }
        case PointEdge:
            d = point_edge_distance(p[0], p[1], p[2]);
            break;
        case PointFace:
            d = point_face_distance(p[0], p[1], p[2], p[3]);
            break;
        default: {
            V3<S> n = vcross(vsub(p[1], p[0]), vsub(p[3], p[2]));
            if (val(vdot(n, n)) < 1e-30) return C<S>(0.0);
            d = edge_edge_distance(p[0], p[1], p[2], p[3]);
        }
    }
    S e = activation(d, r, k);
    if (ct.kind == EdgeEdge) {
        V3<S> n = vcross(vsub(p[1], p[0]), vsub(p[3], p[2]));
        S q = vdot(n, n) / C<S>(ct.mollifier_epsilon);
        if (val(q) < 1.0) e = e * q * (C<S>(2.0) - q);
    }
    return e;
}

// ---------------------------------------------------------------- geometry
enum FeatureKind { FVertex = 0, FEdge = 1, FFace = 2 };
struct Feature {
    int kind;
    uint32_t id;
};

// closest_segments (src/ogc/geometry.rs:78-107)
inline void closest_segments(D3 a, D3 b, D3 c, D3 d, double& s_out, double& t_out) {
    D3 u = b - a;
    D3 v = d - c;
    D3 w = a - c;
    double aa = length_squared(u);
    double ee = length_squared(v);
    if (aa < 1e-24 || ee < 1e-24) {
        s_out = 0.0;
        t_out = 0.0;
        return;
    }
    double bb = dot(u, v);
    double cc = dot(u, w);
    double ff = dot(v, w);
    double den = aa * ee - bb * bb;
    auto clamp01 = [](double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); };
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

// segment_triangle (src/ogc/geometry.rs:131-147)
inline bool segment_triangle(D3 a, D3 b, D3 p, D3 q, D3 r) {
    D3 e = q - p;
    D3 f = r - p;
    D3 d = b - a;
    D3 h = cross(d, f);
    double det = dot(e, h);
    if (std::fabs(det) < 1e-14) return false;
    D3 s = a - p;
    double u = dot(s, h) / det;
    D3 z = cross(s, e);
    double v = dot(d, z) / det;
    double k = dot(f, z) / det;
    return u >= -1e-10 && v >= -1e-10 && u + v <= 1.0 + 1e-10 && (k >= 1e-10 && k < 1.0 - 1e-10);
}

}  // namespace oracle
