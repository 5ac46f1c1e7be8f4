// Oracle (test infrastructure only): FP64 restatement of ClothCraft's CPU VBD
// step. Follows src/vbd.rs, src/vbd/prediction.rs, src/vbd/coloring.rs and
// src/garment/diagnostics.rs.
#pragma once
#include <array>
#include <vector>

#include "oracle_ogc.hpp"

namespace oracle {

struct Triangle {  // src/model.rs:91-98
    std::array<uint32_t, 3> vertices;
    double inv_dm[4];  // x_axis.x, x_axis.y, y_axis.x, y_axis.y
    double area;
    uint32_t material;
};
struct Hinge {  // src/model.rs:99-106
    std::array<uint32_t, 4> vertices;
    double weight;
    double across[2];
    uint32_t material;
};
struct Stitch {  // src/vbd.rs:84-88
    std::vector<std::pair<uint32_t, double>> terms;
    double stiffness;
};
struct Mesh {
    size_t n = 0;
    std::vector<Triangle> triangles;
    std::vector<Hinge> hinges;
    std::vector<Material> materials;
    std::vector<double> masses;
    std::vector<bool> pinned;
    std::vector<D3> pin_positions;
    std::vector<Stitch> stitches;
};

struct VbdSettings {  // src/vbd.rs:18-52
    double dt = 1.0 / 240.0;
    size_t iterations = 16;
    double damping = 1.5;
    D3 gravity{0.0, -9.81, 0.0};
    OgcSettings contact;
    // Extension without a reference counterpart (the library's residual
    // target): evaluate ||P grad E(x)|| / ||grad E(y)|| every k iterations and
    // stop at the first evaluation <= tolerance (0 = never stop early).
    double residual_tolerance = 0.0;
    size_t residual_check_every = 0;
    size_t stall_refresh = 0;  // refresh after this many evaluations without a 5 % decrease
    // Extension: Chebyshev semi-iterative acceleration of the sweeps with
    // spectral-radius estimate rho in [0, 1) (0 = off, the reference).
    double acceleration = 0.0;
    // Extension: 1 = start from the library's learned guess (the correction
    // of the adaptive guess is given, see VbdSolver::learned_correction).
    int init_mode = 0;
    bool valid() const;
};

struct Grab {  // src/vbd.rs:54-60
    std::array<uint32_t, 3> vertices;
    std::array<double, 3> weights;
    D3 target;
    double stiffness;
    bool contains(uint32_t v) const { return vertices[0] == v || vertices[1] == v || vertices[2] == v; }
};

struct VbdMetrics {  // src/vbd.rs:61-83
    double time_s = 0, dt_s = 0, step_ms = 0, detection_ms = 0, solve_ms = 0;
    DetectionProfile profile;
    size_t iterations = 0, contacts = 0, contact_terms = 0, detection_updates = 0, broad_phase_rebuilds = 0,
           truncated_vertices = 0, colors = 0;
    double minimum_distance_m = 0, max_seam_gap_m = 0, extension_p95_percent = 0, extension_max_percent = 0;
    bool has_residual = false;
    double residual_rms_n = 0;
    bool has_relative_residual = false;
    double relative_residual = 0, initial_relative_residual = 0;
    double relative_force_residual = 0;  // unprojected, after the last iteration
    bool init_used = false;               // the learned guess replaced the adaptive one
};

struct State {
    std::vector<D3> x, v;
    double time = 0;
};

struct Prediction {  // src/vbd/prediction.rs:6-54
    bool has_last = false;
    State last;
    std::vector<D3> acceleration;
    D3 gravity{0, 0, 0};
    double damping = 0;
    std::vector<D3> guess(const State& state, const VbdSettings& s) const;
    // the history test of guess(): the state is the one last recorded
    bool valid(const State& state, const VbdSettings& s) const;
    void record(const std::vector<D3>& old_velocity, const State& state, const VbdSettings& s);
};

struct VbdSolver {  // src/vbd.rs:89-99
    Prediction prediction;
    std::vector<D3> last_guess;  // adaptive guess of the last step (learned-guess feature)
    // Network output of the next learned-init step: per moving vertex the
    // correction c of the adaptive guess, in units of |g| dt^2 (pinned rows
    // unused). The network itself is checked separately; the step restates
    // what the library does with its output.
    std::vector<D3> learned_correction;
    Mesh mesh;
    OgcWorld world;
    std::vector<std::vector<uint32_t>> triangles, hinges, vertex_stitches, graph;
    int threads = 1;

    static VbdSolver make(const Mesh& mesh, const std::vector<D3>* obstacle_x,
                          const std::vector<std::array<uint32_t, 3>>* obstacle_tris, const State& state);
    std::vector<std::vector<uint32_t>> colors(const ContactSet& contact, const Grab* grab) const;
    template <class S>
    S local(uint32_t v, const V3<S>& p, const std::vector<D3>& x, const ContactSet& contact, const VbdSettings& s,
            const Grab* grab) const;
    VbdMetrics step(State& state, const VbdSettings& settings, const Grab* grab);
    // sum over free vertices of |dE/dx_v|^2 at positions x (all vertices);
    // with `project`, the ball-constraint KKT residual (see grad_sq)
    double grad_sq(const std::vector<D3>& x, const ContactSet& contacts, const std::vector<D3>& target,
                   const std::vector<double>& inertia, const VbdSettings& settings, const Grab* grab,
                   bool project) const;
    // step objective at positions x (all vertices): inertia of the free
    // vertices plus every triangle, hinge, stitch, contact term and the grab
    // once each (the library's k_term_energy items)
    double step_energy(const std::vector<D3>& x, const ContactSet& contacts, const std::vector<D3>& target,
                       const std::vector<double>& inertia, const VbdSettings& settings, const Grab* grab) const;
};

// src/vbd/coloring.rs:5-43
std::vector<std::vector<uint32_t>> greedy_colors(const std::vector<std::vector<uint32_t>>& graph,
                                                 const ContactSet& contact, const Grab* grab);
// src/garment/diagnostics.rs:7-27
std::array<double, 2> extension_percent(const Mesh& mesh, const std::vector<D3>& x);

// src/vbd.rs:196-248
template <class S>
S VbdSolver::local(uint32_t v, const V3<S>& p, const std::vector<D3>& x, const ContactSet& contact,
                   const VbdSettings& settings, const Grab* grab) const {
    auto get = [&](uint32_t i) -> V3<S> { return i == v ? p : lift<S>(x[i]); };
    S value = C<S>(0.0);
    for (uint32_t i : triangles[v]) {
        const Triangle& t = mesh.triangles[i];
        V3<S> q[3] = {get(t.vertices[0]), get(t.vertices[1]), get(t.vertices[2])};
        value = value + membrane<S>(q, t.inv_dm, t.area, mesh.materials[t.material]);
    }
    for (uint32_t i : hinges[v]) {
        const Hinge& h = mesh.hinges[i];
        V3<S> q[4] = {get(h.vertices[0]), get(h.vertices[1]), get(h.vertices[2]), get(h.vertices[3])};
        value = value + bending<S>(q, h.weight, h.across, mesh.materials[h.material]);
    }
    for (uint32_t i : vertex_stitches[v]) {
        const Stitch& st = mesh.stitches[i];
        V3<S> d = {{C<S>(0.0), C<S>(0.0), C<S>(0.0)}};
        for (const auto& [j, w] : st.terms) {
            V3<S> q = get(j);
            for (int k = 0; k < 3; ++k) d[k] = d[k] + C<S>(w) * q[k];
        }
        value = value + C<S>(0.5 * st.stiffness) * vdot(d, d);
    }
    for (uint32_t i : contact.incident[v]) {
        const Contact& c = contact.contacts[i];
        V3<S> q[4] = {get(c.vertices[0]), get(c.vertices[1]), get(c.vertices[2]), get(c.vertices[3])};
        value = value + contact_energy<S>(c, q, settings.contact.radius, settings.contact.stiffness);
    }
    if (grab && grab->contains(v)) {
        V3<S> d = {{C<S>(-grab->target.x), C<S>(-grab->target.y), C<S>(-grab->target.z)}};
        for (int j = 0; j < 3; ++j) {
            V3<S> q = get(grab->vertices[j]);
            for (int k = 0; k < 3; ++k) d[k] = d[k] + C<S>(grab->weights[j]) * q[k];
        }
        value = value + C<S>(0.5 * grab->stiffness) * vdot(d, d);
    }
    return value;
}

}  // namespace oracle
