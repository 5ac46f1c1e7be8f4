// Oracle (test infrastructure only): FP64 restatement of the learned-guess
// pieces of the library, for parity tests of its CUDA kernels:
//   - the 24 per-vertex features of a step start (clothcraft_b200/csrc/learned.cu,
//     k_features), computed from this oracle's own prediction
//     (src/vbd/prediction.rs:15-41), inertial target (src/vbd.rs:283-302) and
//     OGC detection (src/ogc/world.rs:308-420);
//   - the 24-64-64-64-3 GELU MLP forward pass and the gradient of the mean
//     squared error (k_mlp_forward_f32, k_mlp_train_tile), in double.
// The reference itself has no learned initial guess; these functions pin the
// library's own extension, not a reference algorithm.
#include <cmath>
#include <cstring>
#include <set>

#include "../include/clothcraft.h"
#include "oracle_vbd.hpp"

using namespace oracle;

struct or_solver;
extern "C" VbdSolver* or_solver_inner(or_solver* s);

namespace {
constexpr int kIn = 24, kH = 64, kOut = 3;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kH, oW4 = oB3 + kH, oB4 = oW4 + kOut * kH, kParams = oB4 + kOut;

double gelu(double z, double* dz) {  // tanh form (Hendrycks & Gimpel 2016)
    const double c0 = 0.7978845608028654, c1 = 0.044715;
    double t = std::tanh(c0 * (z + c1 * z * z * z));
    if (dz) *dz = 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * c0 * (1.0 + 3.0 * c1 * z * z);
    return 0.5 * z * (1.0 + t);
}

struct Net {
    const float* p;
    double W(int off, int o, int i, int in) const { return (double)p[off + o * in + i]; }
};

// forward of one sample keeping pre-activation derivatives for backprop
void forward(const Net& n, const float* f, double a0[kIn], double a1[kH], double g1[kH], double a2[kH], double g2[kH],
             double a3[kH], double g3[kH], double out[kOut]) {
    for (int j = 0; j < kIn; ++j) a0[j] = (double)f[j];
    for (int o = 0; o < kH; ++o) {
        double z = n.p[oB1 + o];
        for (int i = 0; i < kIn; ++i) z += n.W(oW1, o, i, kIn) * a0[i];
        a1[o] = gelu(z, &g1[o]);
    }
    for (int o = 0; o < kH; ++o) {
        double z = n.p[oB2 + o];
        for (int i = 0; i < kH; ++i) z += n.W(oW2, o, i, kH) * a1[i];
        a2[o] = gelu(z, &g2[o]);
    }
    for (int o = 0; o < kH; ++o) {
        double z = n.p[oB3 + o];
        for (int i = 0; i < kH; ++i) z += n.W(oW3, o, i, kH) * a2[i];
        a3[o] = gelu(z, &g3[o]);
    }
    for (int o = 0; o < kOut; ++o) {
        double z = n.p[oB4 + o];
        for (int i = 0; i < kH; ++i) z += n.W(oW4, o, i, kH) * a3[i];
        out[o] = z;
    }
}
}  // namespace

extern "C" {

uint64_t or_mlp_parameter_count(void) { return kParams; }

int32_t or_mlp_forward(const float* params, const float* features, uint64_t n, double* out) {
    Net net{params};
    double a0[kIn], a1[kH], g1[kH], a2[kH], g2[kH], a3[kH], g3[kH];
    for (uint64_t s = 0; s < n; ++s) forward(net, features + s * kIn, a0, a1, g1, a2, g2, a3, g3, out + s * kOut);
    return 0;
}

// L = (1/n) sum_s |MLP(f_s) - t_s|^2 and dL/dparams (double).
int32_t or_mlp_gradients(const float* params, const float* features, const float* targets, uint64_t n, double* grads,
                         double* loss) {
    if (n == 0) return CC_ERR_INVALID_ARGUMENT;
    Net net{params};
    std::memset(grads, 0, kParams * sizeof(double));
    double L = 0.0;
    double a0[kIn], a1[kH], g1[kH], a2[kH], g2[kH], a3[kH], g3[kH], o[kOut];
    double d4[kOut], d3[kH], d2[kH], d1[kH];
    for (uint64_t s = 0; s < n; ++s) {
        forward(net, features + s * kIn, a0, a1, g1, a2, g2, a3, g3, o);
        for (int k = 0; k < kOut; ++k) {
            double r = o[k] - (double)targets[s * kOut + k];
            L += r * r;
            d4[k] = 2.0 * r / (double)n;
        }
        for (int k = 0; k < kOut; ++k) {
            grads[oB4 + k] += d4[k];
            for (int i = 0; i < kH; ++i) grads[oW4 + k * kH + i] += d4[k] * a3[i];
        }
        for (int i = 0; i < kH; ++i) {
            double acc = 0.0;
            for (int k = 0; k < kOut; ++k) acc += net.W(oW4, k, i, kH) * d4[k];
            d3[i] = g3[i] * acc;
        }
        for (int o3 = 0; o3 < kH; ++o3) {
            grads[oB3 + o3] += d3[o3];
            for (int i = 0; i < kH; ++i) grads[oW3 + o3 * kH + i] += d3[o3] * a2[i];
        }
        for (int i = 0; i < kH; ++i) {
            double acc = 0.0;
            for (int k = 0; k < kH; ++k) acc += net.W(oW3, k, i, kH) * d3[k];
            d2[i] = g2[i] * acc;
        }
        for (int o2 = 0; o2 < kH; ++o2) {
            grads[oB2 + o2] += d2[o2];
            for (int i = 0; i < kH; ++i) grads[oW2 + o2 * kH + i] += d2[o2] * a1[i];
        }
        for (int i = 0; i < kH; ++i) {
            double acc = 0.0;
            for (int k = 0; k < kH; ++k) acc += net.W(oW2, k, i, kH) * d2[k];
            d1[i] = g1[i] * acc;
        }
        for (int o1 = 0; o1 < kH; ++o1) {
            grads[oB1 + o1] += d1[o1];
            for (int i = 0; i < kIn; ++i) grads[oW1 + o1 * kIn + i] += d1[o1] * a0[i];
        }
    }
    *loss = L / (double)n;
    return 0;
}

// Features of the step that would start from (x, v, time) with this solver's
// prediction history; out: [free vertices][24] float, in vertex order.
int32_t or_learned_features(or_solver* h, const double* x, const double* v, double time, const cc_vbd_settings* st,
                            float* out) {
    try {
        VbdSolver& s = *or_solver_inner(h);
        const Mesh& mesh = s.mesh;
        size_t n = mesh.n;
        State state;
        state.time = time;
        state.x.resize(n);
        state.v.resize(n);
        for (size_t i = 0; i < n; ++i) {
            state.x[i] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
            state.v[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        }
        VbdSettings vs;
        vs.dt = st->dt;
        vs.iterations = st->iterations;
        vs.damping = st->damping;
        vs.gravity = {st->gravity[0], st->gravity[1], st->gravity[2]};
        vs.contact.radius = st->contact.radius;
        vs.contact.stiffness = st->contact.stiffness;
        vs.contact.relaxation = st->contact.relaxation;
        vs.contact.refresh_fraction = st->contact.refresh_fraction;
        std::vector<D3> guess = s.prediction.guess(state, vs);
        const bool history = s.prediction.valid(state, vs) && s.last_guess.size() == n;
        double damp = 1.0 + vs.damping * vs.dt;
        std::vector<D3> y(n);
        double motion = 0.0;
        for (size_t i = 0; i < n; ++i) {
            y[i] = state.x[i] + (state.v[i] * vs.dt + vs.gravity * (vs.dt * vs.dt)) / damp;
            motion = std::fmax(motion, length(y[i] - state.x[i]));
        }
        double r = vs.contact.radius;
        double rq = std::min(std::max(r + motion, 2.0 * r), 4.0 * r);
        ContactSet cs = s.world.detect(s.world.positions(state.x.data(), n), rq, vs.contact);
        std::vector<std::set<uint32_t>> ring(n);
        std::vector<std::vector<uint32_t>> tris(n);
        for (size_t t = 0; t < mesh.triangles.size(); ++t) {
            const auto& tv = mesh.triangles[t].vertices;
            for (int a = 0; a < 3; ++a) {
                tris[tv[a]].push_back((uint32_t)t);
                for (int b = 0; b < 3; ++b)
                    if (a != b) ring[tv[a]].insert(tv[b]);
            }
        }
        double g = length(vs.gravity);
        double unit = g * vs.dt * vs.dt > 1e-9 ? g * vs.dt * vs.dt : 1e-3;
        size_t row = 0;
        for (size_t vtx = 0; vtx < n; ++vtx) {
            if (mesh.pinned[vtx]) continue;
            const D3 xv = state.x[vtx];
            D3 dy = (y[vtx] - xv) / unit, dg = (guess[vtx] - xv) / unit;
            D3 nb_dg{0, 0, 0}, nb_x{0, 0, 0};
            double elen = 0.0;
            for (uint32_t u : ring[vtx]) {
                nb_x = nb_x + state.x[u];
                elen += length(state.x[u] - xv);
                nb_dg = nb_dg + (guess[u] - state.x[u]) / unit;
            }
            size_t cnt = ring[vtx].size();
            D3 rel{0, 0, 0}, lap{0, 0, 0};
            if (cnt) {
                rel = nb_dg / (double)cnt - dg;
                lap = (nb_x / (double)cnt - xv) / std::fmax(elen / (double)cnt, 1e-12);
            }
            D3 nrm{0, 0, 0};
            double tr = 0.0, shs = 0.0, mx = -1e30;
            for (uint32_t t : tris[vtx]) {
                const Triangle& T = mesh.triangles[t];
                D3 a = state.x[T.vertices[0]], b = state.x[T.vertices[1]], c = state.x[T.vertices[2]];
                D3 ds0 = b - a, ds1 = c - a;
                nrm = nrm + cross(ds0, ds1);
                double sn, cs;
                grain_sin_cos(mesh.materials[T.material].grain_degrees, sn, cs);
                const double* I = T.inv_dm;
                D3 w = ds0 * (I[0] * cs + I[2] * sn) + ds1 * (I[1] * cs + I[3] * sn);
                D3 q = ds0 * (-I[0] * sn + I[2] * cs) + ds1 * (-I[1] * sn + I[3] * cs);
                double ew = 0.5 * (dot(w, w) - 1.0), ef = 0.5 * (dot(q, q) - 1.0);
                tr += ew + ef;
                shs += std::fabs(dot(w, q));
                mx = std::fmax(mx, std::fmax(ew, ef));
            }
            double nl = length(nrm);
            if (nl > 0.0) nrm = nrm / nl;
            if (!tris[vtx].empty()) {
                tr /= (double)tris[vtx].size();
                shs /= (double)tris[vtx].size();
            } else {
                mx = 0.0;
            }
            double dmin = cs.radii[vtx] / vs.contact.relaxation / rq;
            size_t nc = cs.incident[vtx].size();
            D3 pc{0, 0, 0};
            if (history) pc = (xv - s.last_guess[vtx]) / unit;
            double feat[kIn] = {dy.x,
                                dy.y,
                                dy.z,
                                dg.x,
                                dg.y,
                                dg.z,
                                rel.x,
                                rel.y,
                                rel.z,
                                lap.x,
                                lap.y,
                                lap.z,
                                nrm.x,
                                nrm.y,
                                nrm.z,
                                100.0 * tr,
                                100.0 * shs,
                                100.0 * mx,
                                std::fmin(dmin, 1.0),
                                (double)std::min<size_t>(nc, 16) * 0.25,
                                pc.x,
                                pc.y,
                                pc.z,
                                1.0 - (double)cnt / 6.0};
            for (int k = 0; k < kIn; ++k) out[row * kIn + k] = (float)feat[k];
            ++row;
        }
        return 0;
    } catch (const Error& e) {
        return e.code;
    }
}

}  // extern "C"
