// Oracle (test infrastructure only): FP64 Newton reference for the VBD step.
//
// Restates ReferenceSolver::step_problem (src/solver.rs:422-646): implicit
// Euler as minimisation of the incremental potential, element gradients and
// Hessians by forward AD (Jet<9>/Jet<12>, src/energy.rs:68-79), matrix-free
// Jacobi-preconditioned CG with shift escalation (src/solver.rs:150-224,
// 496-545) and an Armijo backtracking line search (src/solver.rs:509-535).
//
// The reference's Newton solver has no OGC term; this oracle adds the step's
// OGC contact set, frozen at one detection, as extra elements with the same
// energy (Contact::energy, src/ogc/potential.rs:39-65). Its inertial term
// m/2|x - x0 - dt v0|^2/dt^2 + m c/(2 dt)|x - x0|^2 - m g.x
// (src/solver.rs:243-254) has the same gradient as VBD's
// m(1+c dt)/dt^2 (x - y) form, so both minimise the same objective.
#include <chrono>
#include <cstring>
#include <numeric>

#include "../include/clothcraft.h"
#include "oracle_vbd.hpp"

namespace oracle {

struct NElement {
    uint32_t verts[4];
    int nv;
    double energy;
    double g[12];
    double h[144];
};

struct NSystem {
    std::vector<NElement> elements;
    std::vector<double> gradient, mass_diag;
    std::vector<char> fixed;
    double energy;
};

struct NewtonInput {
    const VbdSolver* solver;
    const std::vector<D3>* x_old;  // moving
    const std::vector<D3>* v_old;
    const std::vector<D3>* fixed;  // obstacle positions
    const std::vector<Contact>* contacts;
    double dt, damping, r, k;
    D3 gravity;
};

static inline D3 xa(const std::vector<D3>& x, const NewtonInput& in, uint32_t i) {
    size_t n = in.x_old->size();
    return i < n ? x[i] : (*in.fixed)[i - n];
}

template <int N>
static void jet_to_element(const Jet<N>& j, const uint32_t* verts, int nv, NElement& e) {
    e.nv = nv;
    for (int k = 0; k < nv; ++k) e.verts[k] = verts[k];
    e.energy = j.v;
    for (int a = 0; a < N; ++a) e.g[a] = j.g[a];
    for (int a = 0; a < N; ++a)
        for (int b = 0; b < N; ++b) e.h[a * N + b] = j.h[a][b];
}

// geometry_valid (src/solver.rs:235-242) without the sphere collider.
static bool geometry_valid(const Mesh& mesh, const std::vector<D3>& x) {
    for (const auto& p : x)
        if (!finite(p)) return false;
    for (const Triangle& t : mesh.triangles) {
        D3 a = x[t.vertices[0]], b = x[t.vertices[1]], c = x[t.vertices[2]];
        if (!(length(cross(b - a, c - a)) > 2.0 * t.area * 1e-6)) return false;
    }
    return true;
}

// inertial (src/solver.rs:243-254)
static double inertial(const NewtonInput& in, const std::vector<D3>& x) {
    const Mesh& mesh = in.solver->mesh;
    double sum = 0.0;
    for (size_t i = 0; i < x.size(); ++i) {
        D3 y = (*in.x_old)[i] + (*in.v_old)[i] * in.dt;
        sum += mesh.masses[i] * (0.5 * length_squared(x[i] - y) / (in.dt * in.dt) +
                                 0.5 * in.damping / in.dt * length_squared(x[i] - (*in.x_old)[i]) -
                                 dot(in.gravity, x[i]));
    }
    return sum;
}

// objective (src/solver.rs:255-296) + frozen OGC contacts
double newton_objective(const NewtonInput& in, const std::vector<D3>& x) {
    const Mesh& mesh = in.solver->mesh;
    if (!geometry_valid(mesh, x)) return std::numeric_limits<double>::infinity();
    double e = inertial(in, x);
    for (const Triangle& t : mesh.triangles) {
        V3<double> q[3] = {lift<double>(x[t.vertices[0]]), lift<double>(x[t.vertices[1]]), lift<double>(x[t.vertices[2]])};
        e += membrane<double>(q, t.inv_dm, t.area, mesh.materials[t.material]);
    }
    for (const Hinge& h : mesh.hinges) {
        V3<double> q[4] = {lift<double>(x[h.vertices[0]]), lift<double>(x[h.vertices[1]]),
                           lift<double>(x[h.vertices[2]]), lift<double>(x[h.vertices[3]])};
        e += bending<double>(q, h.weight, h.across, mesh.materials[h.material]);
    }
    for (const Stitch& s : mesh.stitches) {
        D3 d{0, 0, 0};
        for (const auto& [j, w] : s.terms) d = d + x[j] * w;
        e += 0.5 * s.stiffness * length_squared(d);
    }
    for (const Contact& c : *in.contacts) {
        V3<double> q[4];
        for (int k = 0; k < 4; ++k) q[k] = lift<double>(xa(x, in, c.vertices[k]));
        e += contact_energy<double>(c, q, in.r, in.k);
    }
    return e;
}

// assemble (src/solver.rs:297-361) + contact elements
static NSystem newton_assemble(const NewtonInput& in, const std::vector<D3>& x, int threads) {
    const Mesh& mesh = in.solver->mesh;
    const size_t n = x.size();
    NSystem sys;
    size_t nt = mesh.triangles.size(), nh = mesh.hinges.size(), nc = in.contacts->size();
    sys.elements.resize(nt + nh + nc);
#pragma omp parallel for num_threads(threads) schedule(static, 256)
    for (size_t t = 0; t < nt; ++t) {
        const Triangle& tr = mesh.triangles[t];
        V3<Jet<9>> p[3];
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) p[i][k] = variable<9>(x[tr.vertices[i]][k], 3 * i + k);
        jet_to_element(membrane<Jet<9>>(p, tr.inv_dm, tr.area, mesh.materials[tr.material]), tr.vertices.data(), 3,
                       sys.elements[t]);
    }
#pragma omp parallel for num_threads(threads) schedule(static, 256)
    for (size_t h = 0; h < nh; ++h) {
        const Hinge& hg = mesh.hinges[h];
        V3<Jet<12>> p[4];
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 3; ++k) p[i][k] = variable<12>(x[hg.vertices[i]][k], 3 * i + k);
        jet_to_element(bending<Jet<12>>(p, hg.weight, hg.across, mesh.materials[hg.material]), hg.vertices.data(), 4,
                       sys.elements[nt + h]);
    }
#pragma omp parallel for num_threads(threads) schedule(static, 64)
    for (size_t c = 0; c < nc; ++c) {
        const Contact& ct = (*in.contacts)[c];
        V3<Jet<12>> p[4];
        for (int i = 0; i < 4; ++i) {
            D3 q = xa(x, in, ct.vertices[i]);
            for (int k = 0; k < 3; ++k) p[i][k] = variable<12>(q[k], 3 * i + k);
        }
        jet_to_element(contact_energy<Jet<12>>(ct, p, in.r, in.k), ct.vertices, 4, sys.elements[nt + nh + c]);
    }
    // stitches (CompiledSeam::elements, src/garment/seam.rs:245-265)
    for (const Stitch& s : mesh.stitches) {
        if (s.terms.size() > 4) continue;  // not produced by the scene generators
        NElement e{};
        e.nv = (int)s.terms.size();
        D3 d{0, 0, 0};
        for (const auto& [j, w] : s.terms) d = d + x[j] * w;
        e.energy = 0.5 * s.stiffness * length_squared(d);
        int m = 3 * e.nv;
        for (int a = 0; a < e.nv; ++a) {
            e.verts[a] = s.terms[a].first;
            for (int k = 0; k < 3; ++k) e.g[3 * a + k] = s.stiffness * s.terms[a].second * d[k];
            for (int b = 0; b < e.nv; ++b)
                for (int k = 0; k < 3; ++k)
                    e.h[(3 * a + k) * m + 3 * b + k] = s.stiffness * s.terms[a].second * s.terms[b].second;
        }
        // repack the (m x m) block into the 12-wide layout used below
        double tmp[144] = {0};
        for (int a = 0; a < m; ++a)
            for (int b = 0; b < m; ++b) tmp[a * 12 + b] = e.h[a * m + b];
        std::memcpy(e.h, tmp, sizeof tmp);
        sys.elements.push_back(e);
    }
    // membrane/bending Jets use N=9 and N=12 strides; normalise to 12-wide
    for (size_t t = 0; t < nt; ++t) {
        double tmp[144] = {0};
        for (int a = 0; a < 9; ++a)
            for (int b = 0; b < 9; ++b) tmp[a * 12 + b] = sys.elements[t].h[a * 9 + b];
        std::memcpy(sys.elements[t].h, tmp, sizeof tmp);
    }
    sys.gradient.assign(3 * n, 0.0);
    sys.mass_diag.assign(3 * n, 0.0);
    sys.fixed.assign(3 * n, 0);
    for (size_t i = 0; i < n; ++i) {
        D3 delta = ((x[i] - (*in.x_old)[i] - (*in.v_old)[i] * in.dt) / (in.dt * in.dt) +
                    (x[i] - (*in.x_old)[i]) * (in.damping / in.dt) - in.gravity) *
                   mesh.masses[i];
        for (int k = 0; k < 3; ++k) {
            sys.gradient[3 * i + k] = delta[k];
            sys.mass_diag[3 * i + k] = mesh.masses[i] * (1.0 / (in.dt * in.dt) + in.damping / in.dt);
            sys.fixed[3 * i + k] = mesh.pinned[i] ? 1 : 0;
        }
    }
    double e_el = 0.0;
    for (const NElement& e : sys.elements) {
        e_el += e.energy;
        for (int a = 0; a < e.nv; ++a) {
            if (e.verts[a] >= n) continue;
            for (int k = 0; k < 3; ++k) sys.gradient[3 * e.verts[a] + k] += e.g[3 * a + k];
        }
    }
    for (size_t i = 0; i < 3 * n; ++i)
        if (sys.fixed[i]) sys.gradient[i] = 0.0;
    sys.energy = inertial(in, x) + e_el;
    return sys;
}

static double vdot_(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// System::diagonal / apply / pcg (src/solver.rs:150-224)
static std::vector<double> sys_diagonal(const NSystem& s, double shift, size_t n) {
    std::vector<double> d(3 * n);
    for (size_t i = 0; i < 3 * n; ++i) d[i] = s.mass_diag[i] + shift;
    for (const NElement& e : s.elements)
        for (int a = 0; a < e.nv; ++a) {
            if (e.verts[a] >= n) continue;
            for (int k = 0; k < 3; ++k) d[3 * e.verts[a] + k] += e.h[(3 * a + k) * 12 + 3 * a + k];
        }
    for (size_t i = 0; i < 3 * n; ++i) d[i] = s.fixed[i] ? 1.0 : std::fmax(d[i], 1e-12);
    return d;
}

// Elements incident to each vertex, in element order (item = element << 2 | slot),
// so that the product can be gathered per row in parallel with the same
// summation order as the element-by-element scatter.
struct VertexElements {
    std::vector<size_t> off;
    std::vector<uint64_t> item;
};
static VertexElements vertex_elements(const NSystem& s, size_t n) {
    VertexElements g;
    g.off.assign(n + 1, 0);
    for (const NElement& e : s.elements)
        for (int a = 0; a < e.nv; ++a)
            if (e.verts[a] < n) ++g.off[e.verts[a] + 1];
    for (size_t i = 0; i < n; ++i) g.off[i + 1] += g.off[i];
    g.item.resize(g.off[n]);
    std::vector<size_t> fill(g.off.begin(), g.off.end() - 1);
    for (size_t k = 0; k < s.elements.size(); ++k) {
        const NElement& e = s.elements[k];
        for (int a = 0; a < e.nv; ++a)
            if (e.verts[a] < n) g.item[fill[e.verts[a]]++] = ((uint64_t)k << 2) | (uint64_t)a;
    }
    return g;
}

static std::vector<double> sys_apply(const NSystem& s, const VertexElements& g, const std::vector<double>& x,
                                     double shift, size_t n, int threads) {
    std::vector<double> out(3 * n);
#pragma omp parallel for num_threads(threads) schedule(static, 256)
    for (size_t v = 0; v < n; ++v) {
        for (int ka = 0; ka < 3; ++ka) {
            size_t gi = 3 * v + ka;
            if (s.fixed[gi]) {
                out[gi] = x[gi];
                continue;
            }
            double o = x[gi] * (s.mass_diag[gi] + shift);
            for (size_t q = g.off[v]; q < g.off[v + 1]; ++q) {
                const NElement& e = s.elements[g.item[q] >> 2];
                int a = (int)(g.item[q] & 3u);
                double acc = 0.0;
                for (int b = 0; b < e.nv; ++b) {
                    if (e.verts[b] >= n) continue;
                    for (int kb = 0; kb < 3; ++kb) {
                        size_t gj = 3 * e.verts[b] + kb;
                        if (!s.fixed[gj]) acc += e.h[(3 * a + ka) * 12 + 3 * b + kb] * x[gj];
                    }
                }
                o += acc;
            }
            out[gi] = o;
        }
    }
    return out;
}

static bool sys_pcg(const NSystem& s, const VertexElements& g, double shift, size_t limit, size_t n,
                    std::vector<double>& x, size_t& its, int threads) {
    std::vector<double> diag = sys_diagonal(s, shift, n);
    x.assign(3 * n, 0.0);
    std::vector<double> r(3 * n), z(3 * n), p(3 * n);
    for (size_t i = 0; i < 3 * n; ++i) r[i] = -s.gradient[i];
    for (size_t i = 0; i < 3 * n; ++i) z[i] = r[i] / diag[i];
    p = z;
    double rz = vdot_(r, z);
    double tol = 1e-5 * std::sqrt(vdot_(r, r));
    for (size_t it = 0; it < limit; ++it) {
        std::vector<double> ap = sys_apply(s, g, p, shift, n, threads);
        double curv = vdot_(p, ap);
        if (!std::isfinite(curv) || curv <= 0.0) {
            its = it + 1;
            return false;
        }
        double alpha = rz / curv;
        for (size_t i = 0; i < 3 * n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * ap[i];
        }
        if (std::sqrt(vdot_(r, r)) <= tol) {
            its = it + 1;
            return true;
        }
        for (size_t i = 0; i < 3 * n; ++i) z[i] = r[i] / diag[i];
        double next = vdot_(r, z);
        double beta = next / rz;
        for (size_t i = 0; i < 3 * n; ++i) p[i] = z[i] + beta * p[i];
        rz = next;
    }
    its = limit;
    return true;
}

static double rms_free(const std::vector<double>& g, const std::vector<char>& fixed) {
    size_t free = 0;
    for (char f : fixed) free += f ? 0 : 1;
    return std::sqrt(vdot_(g, g) / (double)std::max<size_t>(free, 1));
}

struct NewtonResult {
    std::vector<D3> x;
    bool converged = false;
    size_t iterations = 0, pcg_iterations = 0;
    double residual_rms = 0, objective = 0;
};

// step_problem (src/solver.rs:422-646), OGC contacts frozen
NewtonResult newton_step(const NewtonInput& in, int newton_iterations, size_t pcg_iterations, double abs_tol,
                         double rel_tol, int threads) {
    const Mesh& mesh = in.solver->mesh;
    const size_t n = in.x_old->size();
    std::vector<D3> x = *in.x_old;
    for (size_t i = 0; i < n; ++i)
        if (mesh.pinned[i]) x[i] = mesh.pin_positions[i];
    NewtonResult out;
    double tolerance = 0.0;
    for (int iteration = 0; iteration <= newton_iterations; ++iteration) {
        NSystem sys = newton_assemble(in, x, threads);
        double residual = rms_free(sys.gradient, sys.fixed);
        if (!std::isfinite(residual) || !std::isfinite(sys.energy)) throw Error{4, "Non-finite FEM assembly"};
        if (iteration == 0) tolerance = std::fmax(abs_tol, rel_tol * residual);
        out.residual_rms = residual;
        out.objective = sys.energy;
        out.iterations = iteration;
        if (residual <= tolerance) {
            out.converged = true;
            break;
        }
        if (iteration == newton_iterations) break;
        double scale = 1.0;
        for (double d : sys_diagonal(sys, 0.0, n)) scale = std::fmax(scale, d);
        VertexElements elems = vertex_elements(sys, n);
        bool accepted = false;
        std::vector<D3> trial;
        double shift = 0.0;
        for (int attempt = 0; attempt < 12 && !accepted; ++attempt) {
            std::vector<double> dir;
            size_t its = 0;
            bool ok = sys_pcg(sys, elems, shift, pcg_iterations, n, dir, its, threads);
            out.pcg_iterations += its;
            if (ok) {
                double slope = vdot_(sys.gradient, dir);
                if (std::isfinite(slope) && slope < 0.0) {
                    double alpha = 1.0;
                    for (int ls = 0; ls < 24; ++ls) {
                        trial.resize(n);
                        for (size_t i = 0; i < n; ++i)
                            trial[i] = mesh.pinned[i] ? mesh.pin_positions[i]
                                                      : x[i] + D3{dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]} * alpha;
                        double obj = newton_objective(in, trial);
                        if (std::isfinite(obj) && obj <= sys.energy + 1e-4 * alpha * slope) {
                            accepted = true;
                            break;
                        }
                        alpha *= 0.5;
                    }
                }
            }
            if (!accepted) shift = shift == 0.0 ? scale * 1e-6 : shift * 10.0;
        }
        if (!accepted) throw Error{4, "Newton line search failed; state unchanged. Reduce time step."};
        x = trial;
    }
    out.x = x;
    return out;
}

}  // namespace oracle

// ------------------------------------------------------------------ C API
using namespace oracle;

struct or_solver;
extern "C" VbdSolver* or_solver_inner(or_solver* s);

namespace {
std::vector<D3> to_d3n(const double* p, size_t n) {
    std::vector<D3> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    return out;
}
// The step's contact set: detection at the step-start positions with the
// step's query radius (src/vbd.rs:298-307).
std::vector<Contact> step_contacts(VbdSolver& s, const std::vector<D3>& x_old, const std::vector<D3>& v_old,
                                   const cc_vbd_settings* st, double* rq_out) {
    double damp = 1.0 + st->damping * st->dt;
    double motion = 0.0;
    D3 g{st->gravity[0], st->gravity[1], st->gravity[2]};
    for (size_t i = 0; i < x_old.size(); ++i) {
        D3 t = x_old[i] + (v_old[i] * st->dt + g * st->dt * st->dt) / damp;
        motion = std::fmax(motion, distance(t, x_old[i]));
    }
    double r = st->contact.radius;
    double rq = std::min(std::max(r + motion, 2.0 * r), 4.0 * r);
    if (rq_out) *rq_out = rq;
    OgcSettings os;
    os.radius = st->contact.radius;
    os.stiffness = st->contact.stiffness;
    os.relaxation = st->contact.relaxation;
    os.refresh_fraction = st->contact.refresh_fraction;
    ContactSet cs = s.world.detect(s.world.positions(x_old.data(), x_old.size()), rq, os);
    return cs.contacts;
}
}  // namespace

extern "C" {

// FP64 Newton step from (x_old, v_old) with the OGC contacts detected at
// x_old frozen. x_out: [n][3]. Returns 0 or an error code.
int32_t or_newton_step(or_solver* h, const double* x_old, const double* v_old, const cc_vbd_settings* st,
                       int32_t newton_iterations, int32_t pcg_iterations, double abs_tol, double rel_tol,
                       int32_t threads, double* x_out, double* residual_rms, int32_t* converged,
                       int32_t* iterations) {
    try {
        VbdSolver& s = *or_solver_inner(h);
        size_t n = s.mesh.n;
        std::vector<D3> xo = to_d3n(x_old, n), vo = to_d3n(v_old, n);
        std::vector<Contact> contacts = step_contacts(s, xo, vo, st, nullptr);
        std::vector<D3> fixed = s.world.fixed;
        NewtonInput in{&s, &xo, &vo, &fixed, &contacts, st->dt, st->damping, st->contact.radius,
                       st->contact.stiffness, {st->gravity[0], st->gravity[1], st->gravity[2]}};
        NewtonResult r = newton_step(in, newton_iterations, (size_t)pcg_iterations, abs_tol, rel_tol, threads);
        for (size_t i = 0; i < n; ++i) {
            x_out[3 * i] = r.x[i].x;
            x_out[3 * i + 1] = r.x[i].y;
            x_out[3 * i + 2] = r.x[i].z;
        }
        *residual_rms = r.residual_rms;
        *converged = r.converged ? 1 : 0;
        *iterations = (int32_t)r.iterations;
        return 0;
    } catch (const Error& e) {
        return e.code;
    }
}

// Objective value and gradient (free dofs; pinned dofs zero) of the step
// from (x_old, v_old) at x_eval, with the contacts detected at x_old frozen.
int32_t or_step_gradient(or_solver* h, const double* x_old, const double* v_old, const cc_vbd_settings* st,
                         const double* x_eval, int32_t threads, double* energy, double* gradient) {
    try {
        VbdSolver& s = *or_solver_inner(h);
        size_t n = s.mesh.n;
        std::vector<D3> xo = to_d3n(x_old, n), vo = to_d3n(v_old, n), xe = to_d3n(x_eval, n);
        std::vector<Contact> contacts = step_contacts(s, xo, vo, st, nullptr);
        std::vector<D3> fixed = s.world.fixed;
        NewtonInput in{&s, &xo, &vo, &fixed, &contacts, st->dt, st->damping, st->contact.radius,
                       st->contact.stiffness, {st->gravity[0], st->gravity[1], st->gravity[2]}};
        NSystem sys = newton_assemble(in, xe, threads);
        *energy = sys.energy;
        std::memcpy(gradient, sys.gradient.data(), 3 * n * sizeof(double));
        return 0;
    } catch (const Error& e) {
        return e.code;
    }
}

}  // extern "C"
