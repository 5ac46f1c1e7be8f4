// Oracle (test infrastructure only): C entry points of the FP64 restatement.
// They mirror include/clothcraft.h with an `or_` prefix so that parity tests
// call the CUDA library and the oracle the same way. Extra `or_` hooks expose
// the reference's lower-level functions that its own tests exercise.
#include <cstring>
#include <memory>
#include <mutex>

#include "../include/clothcraft.h"
#include "oracle_vbd.hpp"

using namespace oracle;

namespace {
std::mutex g_err_mutex;
std::string g_err;
int g_code = 0;

int set_global(int code, const std::string& m) {
    std::lock_guard<std::mutex> lock(g_err_mutex);
    g_err = m;
    g_code = code;
    return code;
}

int copy_message(const std::string& m, char* buf, uint64_t len) {
    if (buf && len) {
        size_t k = std::min<size_t>(m.size(), len - 1);
        std::memcpy(buf, m.data(), k);
        buf[k] = 0;
    }
    return 0;
}

std::vector<D3> to_d3(const double* p, size_t n) {
    std::vector<D3> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    return out;
}

OgcSettings to_ogc(const cc_ogc_settings* s) {
    OgcSettings o;
    o.radius = s->radius;
    o.stiffness = s->stiffness;
    o.relaxation = s->relaxation;
    o.refresh_fraction = s->refresh_fraction;
    return o;
}

VbdSettings to_vbd(const cc_vbd_settings* s) {
    VbdSettings o;
    o.dt = s->dt;
    o.iterations = s->iterations;
    o.damping = s->damping;
    o.gravity = {s->gravity[0], s->gravity[1], s->gravity[2]};
    o.contact = to_ogc(&s->contact);
    o.residual_tolerance = s->residual_tolerance;
    o.residual_check_every = s->residual_check_every;
    o.stall_refresh = s->stall_refresh;
    o.acceleration = s->acceleration;
    o.init_mode = (int)s->init_mode;
    return o;
}

Grab to_grab(const cc_grab* g) {
    Grab o;
    for (int i = 0; i < 3; ++i) {
        o.vertices[i] = g->vertices[i];
        o.weights[i] = g->weights[i];
    }
    o.target = {g->target[0], g->target[1], g->target[2]};
    o.stiffness = g->stiffness;
    return o;
}

Material to_material(const cc_material& m) {
    return {m.warp,      m.weft,      m.shear,   m.compression_ratio, m.compression_transition,
            m.bend_warp, m.bend_weft, m.density, m.thickness,         m.grain_degrees};
}

Mesh to_mesh(const cc_mesh* m) {
    Mesh out;
    out.n = m->n_vertices;
    for (uint64_t i = 0; i < m->n_materials; ++i) out.materials.push_back(to_material(m->materials[i]));
    for (uint64_t t = 0; t < m->n_triangles; ++t) {
        Triangle tri;
        for (int k = 0; k < 3; ++k) tri.vertices[k] = m->triangles[3 * t + k];
        for (int k = 0; k < 4; ++k) tri.inv_dm[k] = m->inv_dm[4 * t + k];
        tri.area = m->area[t];
        tri.material = m->triangle_material ? m->triangle_material[t] : 0;
        if (tri.material >= out.materials.size()) throw Error{1, "Invalid material binding or mesh topology"};
        for (int k = 0; k < 3; ++k)
            if (tri.vertices[k] >= out.n) throw Error{1, "Invalid material binding or mesh topology"};
        out.triangles.push_back(tri);
    }
    for (uint64_t h = 0; h < m->n_hinges; ++h) {
        Hinge hg;
        for (int k = 0; k < 4; ++k) hg.vertices[k] = m->hinges[4 * h + k];
        hg.weight = m->hinge_weight[h];
        hg.across[0] = m->hinge_across[2 * h];
        hg.across[1] = m->hinge_across[2 * h + 1];
        hg.material = m->hinge_material ? m->hinge_material[h] : 0;
        if (hg.material >= out.materials.size()) throw Error{1, "Invalid material binding or mesh topology"};
        for (int k = 0; k < 4; ++k)
            if (hg.vertices[k] >= out.n) throw Error{1, "Invalid material binding or mesh topology"};
        out.hinges.push_back(hg);
    }
    out.masses.assign(m->masses, m->masses + out.n);
    out.pinned.resize(out.n);
    out.pin_positions.resize(out.n);
    for (uint64_t i = 0; i < out.n; ++i) {
        out.pinned[i] = m->pinned && m->pinned[i];
        if (out.pinned[i])
            out.pin_positions[i] = {m->pin_positions[3 * i], m->pin_positions[3 * i + 1], m->pin_positions[3 * i + 2]};
    }
    for (uint64_t s = 0; s < m->n_stitches; ++s) {
        Stitch st;
        for (uint32_t k = m->stitch_offsets[s]; k < m->stitch_offsets[s + 1]; ++k) {
            if (m->stitch_vertices[k] >= out.n) throw Error{1, "Invalid seam vertex"};
            st.terms.push_back({m->stitch_vertices[k], m->stitch_weights[k]});
        }
        st.stiffness = m->stitch_stiffness[s];
        out.stitches.push_back(st);
    }
    return out;
}

void fill_metrics(const VbdMetrics& m, cc_metrics* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->time_s = m.time_s;
    out->dt_s = m.dt_s;
    out->step_ms = m.step_ms;
    out->detection_ms = m.detection_ms;
    out->solve_ms = m.solve_ms;
    out->refit_ms = m.profile.refit_ms;
    out->candidates_ms = m.profile.candidates_ms;
    out->narrow_ms = m.profile.narrow_ms;
    out->candidate_pairs = m.profile.candidate_pairs;
    out->aabb_rejections = m.profile.aabb_rejections;
    out->iterations = m.iterations;
    out->contacts = m.contacts;
    out->contact_terms = m.contact_terms;
    out->detection_updates = m.detection_updates;
    out->broad_phase_rebuilds = m.broad_phase_rebuilds;
    out->truncated_vertices = m.truncated_vertices;
    out->colors = m.colors;
    out->minimum_distance_m = m.minimum_distance_m;
    out->max_seam_gap_m = m.max_seam_gap_m;
    out->extension_p95_percent = m.extension_p95_percent;
    out->extension_max_percent = m.extension_max_percent;
    out->residual_rms_n = m.residual_rms_n;
    out->has_residual = m.has_residual ? 1 : 0;
    out->has_relative_residual = m.has_relative_residual ? 1 : 0;
    out->relative_residual = m.relative_residual;
    out->initial_relative_residual = m.initial_relative_residual;
    out->relative_force_residual = m.relative_force_residual;
    out->init_used = m.init_used ? 1 : 0;
}

int fill_contacts(const ContactSet& cs, size_t moving, cc_contacts* out) {
    out->n_contacts = cs.contacts.size();
    size_t inc = 0;
    for (const auto& v : cs.incident) inc += v.size();
    out->n_incident = inc;
    out->active_contacts = cs.active_contacts;
    out->vertex_face_candidates = cs.vertex_face_candidates;
    out->edge_edge_candidates = cs.edge_edge_candidates;
    out->candidate_pairs = cs.profile.candidate_pairs;
    out->aabb_rejections = cs.profile.aabb_rejections;
    out->minimum_distance = cs.minimum_distance;
    out->broad_phase_rebuilt = cs.broad_phase_rebuilt ? 1 : 0;
    if (out->contact_capacity < cs.contacts.size() || out->incident_capacity < inc || out->radii_capacity < moving)
        return CC_ERR_CAPACITY;
    for (size_t c = 0; c < cs.contacts.size(); ++c) {
        const Contact& ct = cs.contacts[c];
        if (out->kinds) out->kinds[c] = ct.kind;
        if (out->vertices)
            for (int k = 0; k < 4; ++k) out->vertices[4 * c + k] = ct.vertices[k];
        if (out->counts) out->counts[c] = ct.count;
        if (out->mollifier_epsilon) out->mollifier_epsilon[c] = ct.mollifier_epsilon;
    }
    size_t pos = 0;
    for (size_t v = 0; v < moving; ++v) {
        if (out->incident_offsets) out->incident_offsets[v] = pos;
        for (uint32_t c : cs.incident[v]) {
            if (out->incident) out->incident[pos] = c;
            ++pos;
        }
        if (out->radii) out->radii[v] = cs.radii[v];
    }
    if (out->incident_offsets) out->incident_offsets[moving] = pos;
    return CC_OK;
}
}  // namespace

struct or_world {
    OgcWorld own;
    OgcWorld* w = nullptr;
    std::string err;
    int code = 0;
    int fail(const Error& e) {
        err = e.message;
        code = e.code;
        return e.code;
    }
};

struct or_solver {
    VbdSolver s;
    or_world world_view;
    std::string err;
    int code = 0;
    int fail(const Error& e) {
        err = e.message;
        code = e.code;
        return e.code;
    }
};

extern "C" {

int32_t or_abi_version(void) { return CC_ABI_VERSION; }

int32_t or_global_last_error(char* buf, uint64_t len) {
    std::lock_guard<std::mutex> lock(g_err_mutex);
    copy_message(g_err, buf, len);
    return g_code;
}

int32_t or_last_error(const or_solver* s, char* buf, uint64_t len) {
    copy_message(s->err, buf, len);
    return s->code;
}

int32_t or_world_last_error(const or_world* w, char* buf, uint64_t len) {
    copy_message(w->err, buf, len);
    return w->code;
}

int32_t or_set_threads(or_solver* s, int32_t threads) {
    s->s.threads = threads < 1 ? 1 : threads;
    s->s.world.threads = std::min(2, s->s.threads);  // two narrow-phase lanes (src/ogc/world.rs:332)
    return CC_OK;
}

int32_t or_solver_create(const cc_mesh* mesh, const cc_surface* obstacle, const double* x0, const double* v0,
                         uint64_t n, or_solver** out) {
    try {
        Mesh m = to_mesh(mesh);
        State st;
        st.x = to_d3(x0, n);
        st.v = v0 ? to_d3(v0, n) : std::vector<D3>(n, D3{0, 0, 0});
        std::vector<D3> ox;
        std::vector<std::array<uint32_t, 3>> ot;
        if (obstacle) {
            ox = to_d3(obstacle->vertices, obstacle->n_vertices);
            for (uint64_t t = 0; t < obstacle->n_triangles; ++t)
                ot.push_back({obstacle->triangles[3 * t], obstacle->triangles[3 * t + 1],
                              obstacle->triangles[3 * t + 2]});
        }
        auto h = std::make_unique<or_solver>();
        h->s = VbdSolver::make(m, obstacle ? &ox : nullptr, obstacle ? &ot : nullptr, st);
        h->world_view.w = &h->s.world;
        *out = h.release();
        return CC_OK;
    } catch (const Error& e) {
        return set_global(e.code, e.message);
    }
}

void or_solver_destroy(or_solver* s) { delete s; }

uint64_t or_solver_moving(const or_solver* s) { return s->s.mesh.n; }
uint64_t or_solver_total(const or_solver* s) { return s->s.world.topology.neighbors.size(); }
or_world* or_solver_world(or_solver* s) { return &s->world_view; }

// Correction (rows = free vertices in vertex order, [rows][3] float, the
// layout of the library's network output) for the next learned-init step.
int32_t or_solver_set_learned_correction(or_solver* s, const float* corr, uint64_t rows) {
    size_t n = s->s.mesh.n;
    size_t free_rows = 0;
    for (size_t i = 0; i < n; ++i) free_rows += s->s.mesh.pinned[i] ? 0 : 1;
    if (rows != free_rows) return s->fail(Error{1, "correction rows must equal the free vertices"});
    s->s.learned_correction.assign(n, D3{0, 0, 0});
    size_t r = 0;
    for (size_t i = 0; i < n; ++i) {
        if (s->s.mesh.pinned[i]) continue;
        s->s.learned_correction[i] = D3{(double)corr[3 * r], (double)corr[3 * r + 1], (double)corr[3 * r + 2]};
        ++r;
    }
    return CC_OK;
}

int32_t or_solver_step(or_solver* s, double* x, double* v, double* time, const cc_vbd_settings* settings,
                       const cc_grab* grab, cc_metrics* metrics) {
    try {
        size_t n = s->s.mesh.n;
        State st;
        st.x = to_d3(x, n);
        st.v = to_d3(v, n);
        st.time = *time;
        Grab g;
        if (grab) g = to_grab(grab);
        VbdMetrics m = s->s.step(st, to_vbd(settings), grab ? &g : nullptr);
        for (size_t i = 0; i < n; ++i) {
            x[3 * i] = st.x[i].x;
            x[3 * i + 1] = st.x[i].y;
            x[3 * i + 2] = st.x[i].z;
            v[3 * i] = st.v[i].x;
            v[3 * i + 1] = st.v[i].y;
            v[3 * i + 2] = st.v[i].z;
        }
        *time = st.time;
        fill_metrics(m, metrics);
        return CC_OK;
    } catch (const Error& e) {
        return s->fail(e);
    }
}

int32_t or_solver_colors(or_solver* s, const double* x_all, double query_radius, const cc_ogc_settings* settings,
                         const cc_grab* grab, uint32_t* colors_out, uint32_t* n_colors) {
    try {
        std::vector<D3> x = to_d3(x_all, s->s.world.topology.neighbors.size());
        ContactSet cs = s->s.world.detect(x, query_radius, to_ogc(settings));
        Grab g;
        if (grab) g = to_grab(grab);
        auto colors = s->s.colors(cs, grab ? &g : nullptr);
        for (size_t c = 0; c < colors.size(); ++c)
            for (uint32_t v : colors[c]) colors_out[v] = (uint32_t)c;
        *n_colors = (uint32_t)colors.size();
        return CC_OK;
    } catch (const Error& e) {
        return s->fail(e);
    }
}

int32_t or_solver_local_blocks(or_solver* s, const double* x_all, double query_radius,
                               const cc_vbd_settings* settings, const cc_grab* grab, const double* targets,
                               const double* inertia, double* energy, double* gradient, double* hessian) {
    try {
        VbdSettings vs = to_vbd(settings);
        std::vector<D3> x = to_d3(x_all, s->s.world.topology.neighbors.size());
        ContactSet cs = s->s.world.detect(x, query_radius, vs.contact);
        Grab g;
        if (grab) g = to_grab(grab);
        const size_t n = s->s.mesh.n;
#pragma omp parallel for num_threads(s->s.threads) schedule(dynamic, 64)
        for (size_t v = 0; v < n; ++v) {
            V3<Jet<3>> p;
            for (int k = 0; k < 3; ++k) p[k] = variable<3>(x[v][k], k);
            Jet<3> j = s->s.local<Jet<3>>((uint32_t)v, p, x, cs, vs, grab ? &g : nullptr);
            double m = inertia ? inertia[v] : 0.0;
            D3 t = targets ? D3{targets[3 * v], targets[3 * v + 1], targets[3 * v + 2]} : x[v];
            D3 gr = D3{j.g[0], j.g[1], j.g[2]} + (x[v] - t) * m;
            energy[v] = j.v + 0.5 * m * length_squared(x[v] - t);
            gradient[3 * v] = gr.x;
            gradient[3 * v + 1] = gr.y;
            gradient[3 * v + 2] = gr.z;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) hessian[9 * v + 3 * a + b] = j.h[a][b] + (a == b ? m : 0.0);
        }
        return CC_OK;
    } catch (const Error& e) {
        return s->fail(e);
    }
}

int32_t or_world_create(const double* x, uint64_t n_all, const uint32_t* triangles, uint64_t n_triangles,
                        uint64_t moving, const uint32_t* excluded, uint64_t n_excluded, or_world** out) {
    try {
        std::vector<std::array<uint32_t, 3>> tris(n_triangles);
        for (uint64_t t = 0; t < n_triangles; ++t)
            tris[t] = {triangles[3 * t], triangles[3 * t + 1], triangles[3 * t + 2]};
        std::vector<std::array<uint32_t, 2>> ex(n_excluded);
        for (uint64_t e = 0; e < n_excluded; ++e) ex[e] = {excluded[2 * e], excluded[2 * e + 1]};
        auto h = std::make_unique<or_world>();
        h->own = OgcWorld::make(to_d3(x, n_all), tris, moving, ex);
        h->w = &h->own;
        *out = h.release();
        return CC_OK;
    } catch (const Error& e) {
        return set_global(e.code, e.message);
    }
}

void or_world_destroy(or_world* w) {
    if (w && w->w == &w->own) delete w;
}

int32_t or_world_validate_start(or_world* w, const double* x) {
    try {
        w->w->validate_start(to_d3(x, w->w->topology.neighbors.size()));
        return CC_OK;
    } catch (const Error& e) {
        return w->fail(e);
    }
}

int32_t or_world_detect(or_world* w, const double* x, double query_radius, const cc_ogc_settings* settings,
                        cc_contacts* out) {
    try {
        ContactSet cs = w->w->detect(to_d3(x, w->w->topology.neighbors.size()), query_radius, to_ogc(settings));
        return fill_contacts(cs, w->w->moving, out);
    } catch (const Error& e) {
        return w->fail(e);
    }
}

// Oracle-only: OgcWorld::detect_impl::<false> (no AABB pruning of cached pairs).
int32_t or_world_detect_unpruned(or_world* w, const double* x, double query_radius, const cc_ogc_settings* settings,
                                 cc_contacts* out) {
    try {
        ContactSet cs =
            w->w->detect(to_d3(x, w->w->topology.neighbors.size()), query_radius, to_ogc(settings), false);
        return fill_contacts(cs, w->w->moving, out);
    } catch (const Error& e) {
        return w->fail(e);
    }
}

int32_t or_world_candidates(or_world* w, const double* x, double radius, cc_candidates* out) {
    try {
        w->w->refit(to_d3(x, w->w->topology.neighbors.size()));
        std::vector<std::array<uint32_t, 2>> vf, ee;
        w->w->pairs_at(radius, vf, ee);
        std::sort(vf.begin(), vf.end());
        std::sort(ee.begin(), ee.end());
        out->n_vf = vf.size();
        out->n_ee = ee.size();
        if (out->vf_capacity < vf.size() || out->ee_capacity < ee.size()) return CC_ERR_CAPACITY;
        for (size_t i = 0; i < vf.size(); ++i) {
            out->vf[2 * i] = vf[i][0];
            out->vf[2 * i + 1] = vf[i][1];
        }
        for (size_t i = 0; i < ee.size(); ++i) {
            out->ee[2 * i] = ee[i][0];
            out->ee[2 * i + 1] = ee[i][1];
        }
        return CC_OK;
    } catch (const Error& e) {
        return w->fail(e);
    }
}

uint64_t or_world_edges(const or_world* w, uint32_t* edges_out) {
    const auto& e = w->w->topology.edges;
    if (edges_out)
        for (size_t i = 0; i < e.size(); ++i) {
            edges_out[2 * i] = e[i][0];
            edges_out[2 * i + 1] = e[i][1];
        }
    return e.size();
}

// ------------------------------------------------------------ test hooks
// Jet<1> activation (tests/ogc.rs:17-35).
void or_activation_jet1(double d, double r, double k, double* out3) {
    Jet<1> j = activation(variable<1>(d, 0), r, k);
    out3[0] = j.v;
    out3[1] = j.g[0];
    out3[2] = j.h[0][0];
}
double or_activation(double d, double r, double k) { return activation<double>(d, r, k); }

// Contact::value / Contact::block on four explicit points (potential.rs:66-85).
double or_contact_value(uint8_t kind, uint8_t count, double eps, const double* x12, double r, double k) {
    Contact c{kind, {0, 1, 2, 3}, count, eps};
    std::vector<D3> x = to_d3(x12, 4);
    return contact_value(c, x, r, k);
}
void or_contact_block(uint8_t kind, uint8_t count, double eps, const double* x12, uint32_t vertex, double r, double k,
                      double* e, double* g3, double* h9) {
    Contact c{kind, {0, 1, 2, 3}, count, eps};
    std::vector<D3> x = to_d3(x12, 4);
    V3<Jet<3>> p[4];
    for (int i = 0; i < 4; ++i)
        for (int a = 0; a < 3; ++a) p[i][a] = (uint32_t)i == vertex ? variable<3>(x[i][a], a) : C<Jet<3>>(x[i][a]);
    Jet<3> j = contact_energy<Jet<3>>(c, p, r, k);
    *e = j.v;
    for (int a = 0; a < 3; ++a) g3[a] = j.g[a];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) h9[3 * a + b] = j.h[a][b];
}

// energy::membrane_element / bending_element (src/energy.rs:68-79).
void or_membrane_element(const double* x9, const double* inv_dm4, double area, const cc_material* m, double* e,
                         double* g9, double* h81) {
    V3<Jet<9>> p[3];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) p[i][k] = variable<9>(x9[3 * i + k], 3 * i + k);
    Jet<9> j = membrane<Jet<9>>(p, inv_dm4, area, to_material(*m));
    *e = j.v;
    for (int a = 0; a < 9; ++a) g9[a] = j.g[a];
    for (int a = 0; a < 9; ++a)
        for (int b = 0; b < 9; ++b) h81[9 * a + b] = j.h[a][b];
}
void or_bending_element(const double* x12, double weight, const double* across2, const cc_material* m, double* e,
                        double* g12, double* h144) {
    V3<Jet<12>> p[4];
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 3; ++k) p[i][k] = variable<12>(x12[3 * i + k], 3 * i + k);
    Jet<12> j = bending<Jet<12>>(p, weight, across2, to_material(*m));
    *e = j.v;
    for (int a = 0; a < 12; ++a) g12[a] = j.g[a];
    for (int a = 0; a < 12; ++a)
        for (int b = 0; b < 12; ++b) h144[12 * a + b] = j.h[a][b];
}

// geometry::closest_triangle on one triangle (0,1,2) and query point 3; returns feature kind.
int32_t or_closest_triangle(const double* x12, double* q3) {
    std::vector<D3> x = to_d3(x12, 4);
    Topology top = topology_new(4, {{0, 1, 2}});
    Feature f;
    D3 q = closest_triangle(x[3], 0, x, top, f);
    q3[0] = q.x;
    q3[1] = q.y;
    q3[2] = q.z;
    return f.kind;
}
void or_closest_segments(const double* x12, double* st) {
    std::vector<D3> x = to_d3(x12, 4);
    closest_segments(x[0], x[1], x[2], x[3], st[0], st[1]);
}
int32_t or_segment_triangle(const double* x15) {
    std::vector<D3> x = to_d3(x15, 5);
    return segment_triangle(x[0], x[1], x[2], x[3], x[4]) ? 1 : 0;
}
// geometry::edge_feasible for the edge (a,b) of the given triangle mesh.
int32_t or_edge_feasible(const double* x, uint64_t n, const uint32_t* tris, uint64_t nt, const double* p3, uint32_t a,
                         uint32_t b) {
    std::vector<std::array<uint32_t, 3>> t(nt);
    for (uint64_t i = 0; i < nt; ++i) t[i] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
    Topology top = topology_new(n, t);
    std::vector<D3> xs = to_d3(x, n);
    for (size_t e = 0; e < top.edges.size(); ++e)
        if (top.edges[e][0] == std::min(a, b) && top.edges[e][1] == std::max(a, b))
            return edge_feasible({p3[0], p3[1], p3[2]}, (uint32_t)e, xs, top) ? 1 : 0;
    return -1;
}

// Bvh over explicit boxes (tests/ogc_bvh.rs). boxes: [n][6] = min xyz, max xyz.
struct or_bvh {
    Bvh b;
};
static std::vector<Bounds> to_bounds(const double* boxes, uint64_t n) {
    std::vector<Bounds> out(n);
    for (uint64_t i = 0; i < n; ++i)
        out[i] = {{boxes[6 * i], boxes[6 * i + 1], boxes[6 * i + 2]}, {boxes[6 * i + 3], boxes[6 * i + 4], boxes[6 * i + 5]}};
    return out;
}
or_bvh* or_bvh_create(const double* boxes, const uint8_t* dynamic, uint64_t n) {
    std::vector<bool> d(n);
    for (uint64_t i = 0; i < n; ++i) d[i] = dynamic[i] != 0;
    auto h = new or_bvh;
    h->b = Bvh::make(to_bounds(boxes, n), d);
    return h;
}
void or_bvh_destroy(or_bvh* h) { delete h; }
void or_bvh_refit_dynamic(or_bvh* h, const double* boxes, uint64_t n) {
    std::vector<Bounds> b = to_bounds(boxes, n);
    h->b.refit_dynamic([&](size_t i) { return b[i]; });
}
// Returns the number of pairs (a duplicate visit makes it differ from the set size the caller computes).
uint64_t or_bvh_pairs(const or_bvh* a, const or_bvh* b, double radius, int32_t same, uint32_t* out, uint64_t cap) {
    uint64_t k = 0;
    a->b.pairs(same ? a->b : b->b, radius, same != 0, [&](size_t i, size_t j) {
        if (k < cap) {
            out[2 * k] = (uint32_t)i;
            out[2 * k + 1] = (uint32_t)j;
        }
        ++k;
    });
    return k;
}
uint64_t or_bvh_query(const or_bvh* h, const double* box6, int32_t dynamic_only, uint32_t* out, uint64_t cap) {
    uint64_t k = 0;
    Bounds q{{box6[0], box6[1], box6[2]}, {box6[3], box6[4], box6[5]}};
    h->b.query(q, dynamic_only != 0, [&](size_t i) {
        if (k < cap) out[k] = (uint32_t)i;
        ++k;
    });
    return k;
}
double or_bounds_distance_squared(const double* a6, const double* b6) {
    Bounds a{{a6[0], a6[1], a6[2]}, {a6[3], a6[4], a6[5]}};
    Bounds b{{b6[0], b6[1], b6[2]}, {b6[3], b6[4], b6[5]}};
    return bounds_distance_squared(a, b);
}

// Prediction (src/vbd/prediction.rs) as a standalone object.
struct or_prediction {
    Prediction p;
};
or_prediction* or_prediction_create(void) { return new or_prediction; }
void or_prediction_destroy(or_prediction* p) { delete p; }
void or_prediction_guess(const or_prediction* p, const double* x, const double* v, uint64_t n, double time,
                         const cc_vbd_settings* s, double* out) {
    State st;
    st.x = to_d3(x, n);
    st.v = to_d3(v, n);
    st.time = time;
    auto g = p->p.guess(st, to_vbd(s));
    for (uint64_t i = 0; i < n; ++i) {
        out[3 * i] = g[i].x;
        out[3 * i + 1] = g[i].y;
        out[3 * i + 2] = g[i].z;
    }
}
void or_prediction_record(or_prediction* p, const double* old_v, const double* x, const double* v, uint64_t n,
                          double time, const cc_vbd_settings* s) {
    State st;
    st.x = to_d3(x, n);
    st.v = to_d3(v, n);
    st.time = time;
    p->p.record(to_d3(old_v, n), st, to_vbd(s));
}

// coloring::colors over an explicit graph (CSR) and a contact set in cc_contacts form.
uint32_t or_greedy_colors(uint64_t n, const uint64_t* graph_offsets, const uint32_t* graph_adj,
                          const cc_contacts* contacts, const cc_grab* grab, uint32_t* colors_out) {
    std::vector<std::vector<uint32_t>> graph(n);
    for (uint64_t v = 0; v < n; ++v) graph[v].assign(graph_adj + graph_offsets[v], graph_adj + graph_offsets[v + 1]);
    ContactSet cs;
    cs.contacts.resize(contacts->n_contacts);
    for (uint64_t c = 0; c < contacts->n_contacts; ++c) {
        cs.contacts[c].kind = contacts->kinds[c];
        for (int k = 0; k < 4; ++k) cs.contacts[c].vertices[k] = contacts->vertices[4 * c + k];
        cs.contacts[c].count = contacts->counts[c];
        cs.contacts[c].mollifier_epsilon = contacts->mollifier_epsilon[c];
    }
    cs.incident.assign(n, {});
    for (uint64_t v = 0; v < n; ++v)
        cs.incident[v].assign(contacts->incident + contacts->incident_offsets[v],
                              contacts->incident + contacts->incident_offsets[v + 1]);
    Grab g;
    if (grab) g = to_grab(grab);
    auto colors = greedy_colors(graph, cs, grab ? &g : nullptr);
    for (size_t c = 0; c < colors.size(); ++c)
        for (uint32_t v : colors[c]) colors_out[v] = (uint32_t)c;
    return (uint32_t)colors.size();
}

// diagnostics::extension_percent (src/garment/diagnostics.rs:7-27)
void or_extension_percent(const cc_mesh* mesh, const double* x, double* out2) {
    Mesh m = to_mesh(mesh);
    auto e = extension_percent(m, to_d3(x, m.n));
    out2[0] = e[0];
    out2[1] = e[1];
}

}  // extern "C"

extern "C" VbdSolver* or_solver_inner(or_solver* s) { return &s->s; }
