// Oracle (test infrastructure only): FP64 restatement of ClothCraft's CPU VBD
// step (src/vbd.rs:101-422) and its helpers.
#include "oracle_vbd.hpp"

#include <chrono>
#include <cstdio>

namespace oracle {

static double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

bool VbdSettings::valid() const {  // src/vbd.rs:38-51
    if (!contact.valid()) return false;
    return std::isfinite(dt) && dt >= 1e-6 && dt <= 0.025 && iterations != 0 && iterations <= 200 &&
           std::isfinite(damping) && damping >= 0.0 && finite(gravity) && std::isfinite(acceleration) &&
           acceleration >= 0.0 && acceleration < 1.0;
}

// Chebyshev weight of the k-th iteration since the last (re)start
// (Wang 2015, "A Chebyshev semi-iterative approach for accelerating
// projective and position-based dynamics"): w1 = 1, w2 = 2/(2 - rho^2),
// wk = 4/(4 - rho^2 w(k-1)).
double chebyshev_omega(size_t k, double rho) {
    double r2 = rho * rho, w = 1.0;
    for (size_t j = 2; j <= k; ++j) w = j == 2 ? 2.0 / (2.0 - r2) : 4.0 / (4.0 - r2 * w);
    return w;
}

// src/vbd/prediction.rs:15-41
bool Prediction::valid(const State& state, const VbdSettings& s) const {
    bool ok = false;
    if (has_last) {
        ok = last.time == state.time && last.x.size() == state.x.size() && last.v.size() == state.v.size() &&
             gravity == s.gravity && damping == s.damping;
        for (size_t i = 0; ok && i < state.x.size(); ++i) ok = last.x[i] == state.x[i];
        for (size_t i = 0; ok && i < state.v.size(); ++i) ok = last.v[i] == state.v[i];
    }
    return ok;
}

std::vector<D3> Prediction::guess(const State& state, const VbdSettings& s) const {
    bool valid = this->valid(state, s);
    double g2 = length_squared(s.gravity);
    std::vector<D3> out(state.x.size());
    for (size_t i = 0; i < state.x.size(); ++i) {
        double factor = 1.0;
        if (valid && g2 > 1e-20) {
            double f = dot(acceleration[i], s.gravity) / g2;
            factor = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
        }
        out[i] = state.x[i] + (state.v[i] * s.dt + s.gravity * factor * (s.dt * s.dt)) / (1.0 + s.damping * s.dt);
    }
    return out;
}

// src/vbd/prediction.rs:43-54
void Prediction::record(const std::vector<D3>& old_velocity, const State& state, const VbdSettings& s) {
    acceleration.resize(state.v.size());
    for (size_t i = 0; i < state.v.size(); ++i)
        acceleration[i] = (state.v[i] - old_velocity[i]) / s.dt + state.v[i] * s.damping;
    last = state;
    has_last = true;
    gravity = s.gravity;
    damping = s.damping;
}

// src/vbd/coloring.rs:5-43
std::vector<std::vector<uint32_t>> greedy_colors(const std::vector<std::vector<uint32_t>>& graph,
                                                 const ContactSet& contact, const Grab* grab) {
    const size_t n = graph.size();
    const size_t none = (size_t)-1;
    std::vector<size_t> assigned(n, none);
    std::vector<std::vector<uint32_t>> colors;
    std::vector<size_t> seen(n + 1, none);
    for (size_t v = 0; v < n; ++v) {
        auto mark = [&](size_t i) {
            if (i < n && assigned[i] != none) seen[assigned[i]] = v;
        };
        for (uint32_t i : graph[v]) mark(i);
        for (uint32_t idx : contact.incident[v]) {
            const Contact& c = contact.contacts[idx];
            for (int k = 0; k < c.count; ++k) mark(c.vertices[k]);
        }
        if (grab && grab->contains((uint32_t)v))
            for (uint32_t i : grab->vertices) mark(i);
        size_t c = 0;
        while (seen[c] == v) ++c;
        if (c == colors.size()) colors.emplace_back();
        colors[c].push_back((uint32_t)v);
        assigned[v] = c;
    }
    return colors;
}

// src/garment/diagnostics.rs:7-27 with energy::fiber_frame stretches (src/energy.rs:93-114)
std::array<double, 2> extension_percent(const Mesh& mesh, const std::vector<D3>& x) {
    std::vector<std::pair<double, double>> values;
    values.reserve(mesh.triangles.size());
    for (const Triangle& t : mesh.triangles) {
        const Material& m = mesh.materials[t.material];
        D3 ds0 = x[t.vertices[1]] - x[t.vertices[0]];
        D3 ds1 = x[t.vertices[2]] - x[t.vertices[0]];
        D3 f0 = ds0 * t.inv_dm[0] + ds1 * t.inv_dm[1];
        D3 f1 = ds0 * t.inv_dm[2] + ds1 * t.inv_dm[3];
        double s, c;
        grain_sin_cos(m.grain_degrees, s, c);
        D3 w = f0 * c + f1 * s;
        D3 v = -f0 * s + f1 * c;
        double stretch = std::fmax(length(w), length(v));
        values.push_back({100.0 * std::fmax(stretch - 1.0, 0.0), t.area});
    }
    std::sort(values.begin(), values.end(), [](auto& a, auto& b) { return a.first < b.first; });
    double total = 0.0;
    for (auto& v : values) total += v.second;
    double area = 0.0, p95 = 0.0;
    for (auto& v : values) {
        area += v.second;
        if (area >= 0.95 * total) {
            p95 = v.first;
            break;
        }
    }
    return {p95, values.empty() ? 0.0 : values.back().first};
}

// src/vbd.rs:101-192
VbdSolver VbdSolver::make(const Mesh& mesh, const std::vector<D3>* obstacle_x,
                          const std::vector<std::array<uint32_t, 3>>* obstacle_tris, const State& state) {
    const size_t n = mesh.n;
    if (state.x.size() != n || state.v.size() != n) throw Error{1, "VBD state dimensions do not match garment"};
    for (size_t i = 0; i < n; ++i)
        if (mesh.pinned[i] && distance(state.x[i], mesh.pin_positions[i]) > 1e-10)
            throw Error{1, "VBD pinned positions must match their constraints before initialization"};
    std::vector<D3> x = state.x;
    std::vector<std::array<uint32_t, 3>> faces;
    for (const auto& t : mesh.triangles) faces.push_back(t.vertices);
    if (obstacle_x) {
        if (obstacle_x->empty() || obstacle_tris->empty()) throw Error{1, "Empty/non-finite avatar"};
        for (const auto& p : *obstacle_x)
            if (!finite(p)) throw Error{1, "Empty/non-finite avatar"};
        for (const auto& t : *obstacle_tris) {  // src/avatar.rs:88-97
            if (t[0] >= obstacle_x->size() || t[1] >= obstacle_x->size() || t[2] >= obstacle_x->size())
                throw Error{1, "Invalid avatar index"};
            D3 a = (*obstacle_x)[t[0]], b = (*obstacle_x)[t[1]], c = (*obstacle_x)[t[2]];
            if (length_squared(cross(b - a, c - a)) < 1e-24) throw Error{1, "Degenerate avatar triangle"};
        }
        x.insert(x.end(), obstacle_x->begin(), obstacle_x->end());
        for (const auto& t : *obstacle_tris)
            faces.push_back({t[0] + (uint32_t)n, t[1] + (uint32_t)n, t[2] + (uint32_t)n});
    }
    std::vector<std::array<uint32_t, 2>> excluded;
    for (const Stitch& s : mesh.stitches)
        for (const auto& [a, wa] : s.terms)
            for (const auto& [b, wb] : s.terms)
                if (wa * wb < 0.0) excluded.push_back({std::min(a, b), std::max(a, b)});
    VbdSolver solver;
    solver.mesh = mesh;
    solver.world = OgcWorld::make(x, faces, n, excluded);
    solver.world.validate_start(x);
    solver.triangles.assign(n, {});
    solver.hinges.assign(n, {});
    solver.vertex_stitches.assign(n, {});
    std::vector<std::set<uint32_t>> graph(n);
    auto connect = [&](const uint32_t* ids, size_t count) {
        for (size_t a = 0; a < count; ++a)
            for (size_t b = 0; b < count; ++b)
                if (ids[a] != ids[b]) graph[ids[a]].insert(ids[b]);
    };
    for (size_t i = 0; i < mesh.triangles.size(); ++i) {
        for (uint32_t v : mesh.triangles[i].vertices) solver.triangles[v].push_back((uint32_t)i);
        connect(mesh.triangles[i].vertices.data(), 3);
    }
    for (size_t i = 0; i < mesh.hinges.size(); ++i) {
        for (uint32_t v : mesh.hinges[i].vertices) solver.hinges[v].push_back((uint32_t)i);
        connect(mesh.hinges[i].vertices.data(), 4);
    }
    for (size_t i = 0; i < mesh.stitches.size(); ++i) {
        std::vector<uint32_t> ids;
        for (const auto& t : mesh.stitches[i].terms) ids.push_back(t.first);
        for (uint32_t v : ids) solver.vertex_stitches[v].push_back((uint32_t)i);
        connect(ids.data(), ids.size());
    }
    solver.graph.resize(n);
    for (size_t i = 0; i < n; ++i) solver.graph[i].assign(graph[i].begin(), graph[i].end());
    return solver;
}

std::vector<std::vector<uint32_t>> VbdSolver::colors(const ContactSet& contact, const Grab* grab) const {
    return greedy_colors(graph, contact, grab);
}

namespace {
struct Update {
    uint32_t v;
    D3 p;
    bool truncated;
    double residual;
};
}  // namespace

// src/vbd.rs:250-422
// With `project`, a vertex on the boundary of its OGC ball whose descent
// direction points out of the ball keeps the tangential part of its gradient
// only (first-order residual of the ball-constrained step, ContactSet::truncate).
double VbdSolver::grad_sq(const std::vector<D3>& x, const ContactSet& contacts, const std::vector<D3>& target,
                          const std::vector<double>& inertia, const VbdSettings& settings, const Grab* grab,
                          bool project) const {
    const size_t n = mesh.n;
    std::vector<double> g2(n, 0.0);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 64)
    for (size_t v = 0; v < n; ++v) {
        if (mesh.pinned[v]) continue;
        V3<Jet<3>> p;
        for (int k = 0; k < 3; ++k) p[k] = variable<3>(x[v][k], k);
        Jet<3> jet = local<Jet<3>>((uint32_t)v, p, x, contacts, settings, grab);
        D3 g = D3{jet.g[0], jet.g[1], jet.g[2]} + (x[v] - target[v]) * inertia[v];
        if (project) {
            D3 d = x[v] - contacts.centers[v];
            double l = length(d), b = contacts.radii[v];
            double gn = dot(g, d);
            if (l >= b * (1.0 - 1e-9) && l > 0.0 && gn < 0.0) g = g - d * (gn / (l * l));
        }
        g2[v] = length_squared(g);
    }
    double s = 0.0;
    for (double a : g2) s += a;
    return s;
}

double VbdSolver::step_energy(const std::vector<D3>& x, const ContactSet& contacts, const std::vector<D3>& target,
                              const std::vector<double>& inertia, const VbdSettings& settings,
                              const Grab* grab) const {
    const size_t n = mesh.n;
    double e = 0.0;
    for (size_t v = 0; v < n; ++v)
        if (!mesh.pinned[v]) e += 0.5 * inertia[v] * length_squared(x[v] - target[v]);
    for (const Triangle& t : mesh.triangles) {
        V3<double> q[3] = {lift<double>(x[t.vertices[0]]), lift<double>(x[t.vertices[1]]),
                           lift<double>(x[t.vertices[2]])};
        e += membrane<double>(q, t.inv_dm, t.area, mesh.materials[t.material]);
    }
    for (const Hinge& h : mesh.hinges) {
        V3<double> q[4] = {lift<double>(x[h.vertices[0]]), lift<double>(x[h.vertices[1]]),
                           lift<double>(x[h.vertices[2]]), lift<double>(x[h.vertices[3]])};
        e += bending<double>(q, h.weight, h.across, mesh.materials[h.material]);
    }
    for (const Stitch& st : mesh.stitches) {
        D3 d{0, 0, 0};
        for (const auto& [j, w] : st.terms) d = d + x[j] * w;
        e += 0.5 * st.stiffness * length_squared(d);
    }
    for (const Contact& c : contacts.contacts) {
        V3<double> q[4] = {lift<double>(x[c.vertices[0]]), lift<double>(x[c.vertices[1]]),
                           lift<double>(x[c.vertices[2]]), lift<double>(x[c.vertices[3]])};
        e += contact_energy<double>(c, q, settings.contact.radius, settings.contact.stiffness);
    }
    if (grab) {
        D3 d = grab->target * -1.0;
        for (int j = 0; j < 3; ++j) d = d + x[grab->vertices[j]] * grab->weights[j];
        e += 0.5 * grab->stiffness * length_squared(d);
    }
    return e;
}

VbdMetrics VbdSolver::step(State& state, const VbdSettings& settings, const Grab* grab) {
    if (!settings.valid()) throw Error{1, "Invalid VBD settings"};
    const size_t n = mesh.n;
    bool ok = state.x.size() == n && state.v.size() == n && std::isfinite(state.time);
    for (size_t i = 0; ok && i < n; ++i) ok = finite(state.x[i]) && finite(state.v[i]);
    if (!ok) throw Error{2, "Invalid VBD state"};
    if (grab) {
        double sum = grab->weights[0] + grab->weights[1] + grab->weights[2];
        bool bad = !finite(grab->target) || !std::isfinite(grab->stiffness) || grab->stiffness <= 0.0 ||
                   std::fabs(sum - 1.0) > 1e-8;
        for (int i = 0; i < 3; ++i)
            bad = bad || grab->vertices[i] >= n || !std::isfinite(grab->weights[i]) || grab->weights[i] < 0.0;
        if (bad) throw Error{1, "Invalid mouse attachment"};
    }
    double start = now_ms();
    VbdMetrics metrics;
    metrics.dt_s = settings.dt;
    metrics.iterations = settings.iterations;
    const double dt = settings.dt;
    std::vector<D3> old_velocity = state.v;
    std::vector<D3> guess = prediction.guess(state, settings);
    const double damp = 1.0 + settings.damping * dt;
    std::vector<D3> target(n);
    std::vector<double> inertia(n);
    double predicted_motion = 0.0;
    for (size_t i = 0; i < n; ++i) {
        target[i] = state.x[i] + (state.v[i] * dt + settings.gravity * dt * dt) / damp;
        inertia[i] = mesh.masses[i] * damp / (dt * dt);
        predicted_motion = std::fmax(predicted_motion, distance(target[i], state.x[i]));
    }
    double r = settings.contact.radius;
    double rq = std::min(std::max(r + predicted_motion, 2.0 * r), 4.0 * r);  // f64::clamp
    std::vector<D3> x = world.positions(state.x.data(), n);
    double t_detect = now_ms();
    ContactSet contacts = world.detect(x, rq, settings.contact);
    if (contacts.minimum_distance <= 1e-12)
        throw Error{3, "OGC zero separation; step rejected, reset the arrangement"};
    metrics.detection_ms += now_ms() - t_detect;
    metrics.detection_updates += 1;
    metrics.broad_phase_rebuilds += contacts.broad_phase_rebuilt ? 1 : 0;
    auto add_profile = [&](const DetectionProfile& p) {
        metrics.profile.refit_ms += p.refit_ms;
        metrics.profile.candidates_ms += p.candidates_ms;
        metrics.profile.narrow_ms += p.narrow_ms;
        metrics.profile.candidate_pairs += p.candidate_pairs;
        metrics.profile.aabb_rejections += p.aabb_rejections;
    };
    add_profile(contacts.profile);
    std::vector<std::vector<uint32_t>> colors = this->colors(contacts, grab);
    size_t clipped = 0;
    for (size_t i = 0; i < n; ++i) {
        if (!mesh.pinned[i]) {
            bool b;
            x[i] = contacts.truncate(i, guess[i], b);
            clipped += b ? 1 : 0;
        }
    }
    if (settings.init_mode == 1) {
        // The library's learned guess (clothcraft_b200/csrc/solver.cu,
        // learned_guess): candidates guess + a u c for a = 1, 1/2, 1/4, each
        // clipped to the OGC balls; the lowest step energy replaces the
        // adaptive warm start only if it is strictly lower.
        if (learned_correction.size() != n)
            throw Error{1, "learned initial guess requested but no correction was given"};
        double gl = length(settings.gravity);
        double unit = gl * dt * dt > 1e-9 ? gl * dt * dt : 1e-3;
        double best_e = step_energy(x, contacts, target, inertia, settings, grab);
        std::vector<D3> best;
        size_t clipped_best = clipped;
        for (double a : {1.0, 0.5, 0.25}) {
            std::vector<D3> cand = x;
            size_t cnt = 0;
            for (size_t i = 0; i < n; ++i) {
                if (mesh.pinned[i]) continue;
                D3 p = guess[i] + learned_correction[i] * (unit * a);
                if (!finite(p)) p = guess[i];
                bool b;
                cand[i] = contacts.truncate(i, p, b);
                cnt += b ? 1 : 0;
            }
            double e = step_energy(cand, contacts, target, inertia, settings, grab);
            if (e < best_e) {
                best_e = e;
                best.swap(cand);
                clipped_best = cnt;
                metrics.init_used = true;
            }
        }
        if (metrics.init_used) {
            x.swap(best);
            clipped = clipped_best;
        }
    }
    const bool checks = settings.residual_check_every > 0 || settings.residual_tolerance > 0.0;
    const size_t check_every = settings.residual_check_every > 0 ? settings.residual_check_every : 1;
    double gy2 = 0.0;
    if (checks) {
        std::vector<D3> y_all = world.positions(target.data(), n);
        gy2 = grad_sq(y_all, contacts, target, inertia, settings, grab, false);
        metrics.initial_relative_residual =
            std::sqrt(grad_sq(x, contacts, target, inertia, settings, grab, true) / gy2);
        metrics.has_relative_residual = true;
    }
    std::vector<Update> updates;
    // Chebyshev acceleration: x(k) = w_k (sweep result - x(k-2)) + x(k-2),
    // clipped to the OGC ball, from the second iteration after each
    // (re)start; a refresh detection, and a residual evaluation above the
    // previous one, restart the sequence.
    const bool accelerate = settings.acceleration > 0.0;
    std::vector<D3> acc_prev1, acc_prev2;
    size_t acc_k = 0;
    double acc_g2 = HUGE_VAL;
    if (accelerate) acc_prev1 = x;
    double stall_best = HUGE_VAL;
    size_t stall_count = 0;
    bool stall_pending = false;
    for (size_t it = 0; it < settings.iterations; ++it) {
        if ((clipped > 0 && (double)clipped >= settings.contact.refresh_fraction * (double)n) || stall_pending) {
            stall_pending = false;
            stall_best = HUGE_VAL;
            stall_count = 0;
            double t = now_ms();
            contacts = world.detect(x, rq, settings.contact);
            colors = this->colors(contacts, grab);
            metrics.detection_ms += now_ms() - t;
            metrics.detection_updates += 1;
            metrics.broad_phase_rebuilds += contacts.broad_phase_rebuilt ? 1 : 0;
            add_profile(contacts.profile);
            if (accelerate) {
                acc_k = 0;
                acc_g2 = HUGE_VAL;
                acc_prev1 = x;
            }
        }
        clipped = 0;
        double residual = 0.0;
        for (const auto& color : colors) {
            updates.resize(color.size());
#pragma omp parallel for num_threads(threads) schedule(dynamic, 64)
            for (size_t ci = 0; ci < color.size(); ++ci) {
                uint32_t v = color[ci];
                if (mesh.pinned[v]) {
                    updates[ci] = {v, x[v], false, 0.0};
                    continue;
                }
                V3<Jet<3>> p;
                for (int k = 0; k < 3; ++k) p[k] = variable<3>(x[v][k], k);
                Jet<3> jet = local<Jet<3>>(v, p, x, contacts, settings, grab);
                D3 g = D3{jet.g[0], jet.g[1], jet.g[2]} + (x[v] - target[v]) * inertia[v];
                M3 h;
                for (int col = 0; col < 3; ++col) h.c[col] = {jet.h[0][col], jet.h[1][col], jet.h[2][col]};
                h = h + m3_identity_scaled(inertia[v]);
                double lower = std::numeric_limits<double>::infinity();
                for (int i = 0; i < 3; ++i) {
                    double sum = 0.0;
                    for (int j = 0; j < 3; ++j)
                        if (j != i) sum += std::fabs(h.c[i][j]);
                    lower = std::fmin(lower, h.c[i][i] - sum);
                }
                if (lower < 1e-8) h = h + m3_identity_scaled(1e-8 - lower + 0.01 * inertia[v]);
                D3 delta = -mul(inverse(h), g);
                double old = jet.v + 0.5 * inertia[v] * length_squared(x[v] - target[v]);
                D3 accepted = x[v];
                bool truncated = false;
                double scale = 1.0;
                for (int attempt = 0; attempt < 10; ++attempt) {
                    D3 candidate = x[v] + delta * scale;  // 0.5_f64.powi(attempt) is exact
                    scale *= 0.5;
                    bool bound;
                    candidate = contacts.truncate(v, candidate, bound);
                    truncated = truncated || bound;
                    double e = local<double>(v, lift<double>(candidate), x, contacts, settings, grab) +
                               0.5 * inertia[v] * length_squared(candidate - target[v]);
                    if (finite(candidate) && std::isfinite(e) && e <= old + 1e-14) {
                        accepted = candidate;
                        break;
                    }
                }
                updates[ci] = {v, accepted, truncated, length_squared(g)};
            }
            for (const Update& u : updates) {
                x[u.v] = u.p;
                clipped += u.truncated ? 1 : 0;
                residual += u.residual;
            }
        }
        if (accelerate) {
            double w = chebyshev_omega(++acc_k, settings.acceleration);
            if (acc_k >= 2) {
                for (size_t v = 0; v < n; ++v) {
                    if (mesh.pinned[v]) continue;
                    const D3& p = acc_prev2[v];
                    D3 q{std::fma(w, x[v].x - p.x, p.x), std::fma(w, x[v].y - p.y, p.y),
                         std::fma(w, x[v].z - p.z, p.z)};
                    bool b;
                    x[v] = contacts.truncate(v, q, b);
                }
            }
            acc_prev2.swap(acc_prev1);
            acc_prev1 = x;
        }
        metrics.truncated_vertices += clipped;
        metrics.residual_rms_n = std::sqrt(residual / (double)(3 * n));
        metrics.has_residual = true;
        metrics.colors = colors.size();
        if (checks && ((it + 1) % check_every == 0 || it + 1 == settings.iterations)) {
            double gx2 = grad_sq(x, contacts, target, inertia, settings, grab, true);
            metrics.relative_residual = std::sqrt(gx2 / gy2);
            if (accelerate) {
                if (gx2 > acc_g2) acc_k = 0;
                acc_g2 = gx2;
            }
            if (settings.residual_tolerance > 0.0 &&
                gx2 <= settings.residual_tolerance * settings.residual_tolerance * gy2) {
                metrics.iterations = it + 1;
                break;
            }
            if (settings.residual_tolerance > 0.0 && settings.stall_refresh > 0) {
                if (gx2 < 0.9025 * stall_best) {
                    stall_best = gx2;
                    stall_count = 0;
                } else if (++stall_count >= settings.stall_refresh && clipped > 0 && it + 1 < settings.iterations) {
                    stall_pending = true;
                }
            }
        }
    }
    if (checks)  // the plain force norm of the final iterate, OGC terms in force
        metrics.relative_force_residual =
            std::sqrt(grad_sq(x, contacts, target, inertia, settings, grab, false) / gy2);
    for (const auto& p : x)
        if (!finite(p)) throw Error{4, "Non-finite VBD result; state unchanged"};
    for (size_t i = 0; i < n; ++i)
        if (distance(x[i], contacts.centers[i]) > contacts.radii[i] + 1e-10)
            throw Error{3, "OGC trust-region invariant failed"};
    for (size_t i = 0; i < n; ++i) {
        state.v[i] = (x[i] - state.x[i]) / dt;
        state.x[i] = x[i];
    }
    state.time += dt;
    prediction.record(old_velocity, state, settings);
    last_guess = guess;
    metrics.time_s = state.time;
    metrics.contacts = contacts.active_contacts;
    metrics.contact_terms = contacts.contacts.size();
    metrics.minimum_distance_m = contacts.minimum_distance;
    double gap = 0.0;
    for (const Stitch& s : mesh.stitches) {
        D3 d{0, 0, 0};
        for (const auto& [j, w] : s.terms) d = d + state.x[j] * w;
        gap = std::fmax(gap, length(d));
    }
    metrics.max_seam_gap_m = gap;
    auto ext = extension_percent(mesh, state.x);
    metrics.extension_p95_percent = ext[0];
    metrics.extension_max_percent = ext[1];
    metrics.step_ms = now_ms() - start;
    metrics.solve_ms = metrics.step_ms - metrics.detection_ms;
    return metrics;
}

}  // namespace oracle
