// Oracle (test infrastructure only): FP64 restatement of ClothCraft's OGC
// detection. Each function cites the reference function it follows.
#include <array>
#include <chrono>
#include <cstdio>
#include <numeric>

#include "oracle_ogc.hpp"

namespace oracle {

static double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// src/ogc/topology.rs:13-52
Topology topology_new(size_t n, const std::vector<std::array<uint32_t, 3>>& triangles) {
    Topology top;
    std::map<std::array<uint32_t, 2>, uint32_t> map;
    std::vector<std::set<uint32_t>> neighbors(n);
    for (const auto& t : triangles) {
        if (t[0] >= n || t[1] >= n || t[2] >= n || t[0] == t[1] || t[1] == t[2] || t[0] == t[2])
            throw Error{1, "OGC: invalid triangle indices"};
        std::array<uint32_t, 3> te{};
        for (int k = 0; k < 3; ++k) {
            uint32_t a = t[k], b = t[(k + 1) % 3], c = t[(k + 2) % 3];
            std::array<uint32_t, 2> key{std::min(a, b), std::max(a, b)};
            auto it = map.find(key);
            uint32_t e;
            if (it == map.end()) {
                top.edges.push_back(key);
                top.opposites.emplace_back();
                e = (uint32_t)(top.edges.size() - 1);
                map.emplace(key, e);
            } else {
                e = it->second;
            }
            top.opposites[e].push_back(c);
            neighbors[a].insert(b);
            neighbors[b].insert(a);
            te[k] = e;
        }
        top.triangle_edges.push_back(te);
    }
    for (const auto& o : top.opposites)
        if (o.size() > 2) throw Error{1, "OGC requires manifold triangle edges (at most two incident faces)"};
    top.triangles = triangles;
    top.neighbors.resize(n);
    for (size_t i = 0; i < n; ++i) top.neighbors[i].assign(neighbors[i].begin(), neighbors[i].end());
    return top;
}

// src/ogc/bvh.rs:66-90
Bvh Bvh::make(const std::vector<Bounds>& bounds, const std::vector<bool>& dynamic) {
    Bvh b;
    for (size_t i = 0; i < bounds.size(); ++i)
        if (dynamic[i]) b.order.push_back(i);
    for (size_t i = 0; i < bounds.size(); ++i)
        if (!dynamic[i]) b.order.push_back(i);
    b.primitive_bounds = bounds;
    size_t split = 0;
    for (bool d : dynamic) split += d ? 1 : 0;
    std::pair<size_t, size_t> ranges[2] = {{0, split}, {split, bounds.size()}};
    for (auto [start, end] : ranges) {
        if (start < end) {
            size_t root = b.build(bounds, dynamic, start, end);
            b.roots.push_back(root);
            if (start == 0 && split > 0) b.dynamic_nodes = b.nodes.size();
        }
    }
    return b;
}

// src/ogc/bvh.rs:91-122 (median split on the largest extent, leaf <= 8)
size_t Bvh::build(const std::vector<Bounds>& bounds, const std::vector<bool>& dynamic, size_t start, size_t end) {
    Bounds box = bounds[order[start]];
    for (size_t i = start + 1; i < end; ++i) box = bounds_union(box, bounds[order[i]]);
    size_t id = nodes.size();
    bool dyn = false;
    for (size_t i = start; i < end; ++i) dyn = dyn || dynamic[order[i]];
    nodes.push_back(BvhNode{box, false, {0, 0}, start, end, dyn});
    if (end - start > 8) {
        D3 d = box.max - box.min;
        int axis = (d.x > d.y && d.x > d.z) ? 0 : (d.y > d.z ? 1 : 2);
        std::sort(order.begin() + start, order.begin() + end, [&](size_t a, size_t b) {
            double ka = bounds[a].min[axis] + bounds[a].max[axis];
            double kb = bounds[b].min[axis] + bounds[b].max[axis];
            return ka < kb;
        });
        size_t mid = (start + end) / 2;
        size_t a = build(bounds, dynamic, start, mid);
        size_t c = build(bounds, dynamic, mid, end);
        nodes[id].has_children = true;
        nodes[id].children[0] = a;
        nodes[id].children[1] = c;
    }
    return id;
}

// src/ogc/candidates.rs:15-22
bool Candidates::covers(const D3* moving, size_t n, double r) const {
    if (!(r <= radius) || n != centers.size()) return false;
    for (size_t i = 0; i < n; ++i)
        if (!(distance_squared(moving[i], centers[i]) <= skin * skin)) return false;
    return true;
}

bool OgcSettings::valid() const {  // src/ogc/world.rs:56-70
    return std::isfinite(radius) && radius > 0.0 && std::isfinite(stiffness) && stiffness > 0.0 &&
           std::isfinite(relaxation) && relaxation > 0.0 && relaxation < 0.5 && std::isfinite(refresh_fraction) &&
           refresh_fraction >= 0.0 && refresh_fraction <= 1.0;
}

double contact_value(const Contact& c, const std::vector<D3>& x, double r, double k) {  // potential.rs:66-68
    V3<double> p[4];
    for (int i = 0; i < 4; ++i) p[i] = lift<double>(x[c.vertices[i]]);
    return contact_energy<double>(c, p, r, k);
}

double ContactSet::value(const std::vector<D3>& x, const OgcSettings& s) const {  // world.rs:101-106
    double sum = 0.0;
    for (const auto& c : contacts) sum += contact_value(c, x, s.radius, s.stiffness);
    return sum;
}

// src/ogc/geometry.rs:13-17
bool vertex_feasible(D3 p, uint32_t v, const std::vector<D3>& x, const Topology& top) {
    for (uint32_t j : top.neighbors[v])
        if (!(dot(p - x[v], x[v] - x[j]) >= -1e-14)) return false;
    return true;
}

// src/ogc/geometry.rs:18-29
bool edge_feasible(D3 p, uint32_t e, const std::vector<D3>& x, const Topology& top) {
    D3 a = x[top.edges[e][0]], b = x[top.edges[e][1]];
    D3 u = b - a;
    double t = dot(p - a, u) / length_squared(u);
    if (!(t > 0.0 && t < 1.0)) return false;
    for (uint32_t i : top.opposites[e]) {
        D3 c = x[i];
        D3 q = a + u * (dot(c - a, u) / length_squared(u));
        if (!(dot(p - q, q - c) >= -1e-14)) return false;
    }
    return true;
}

// src/ogc/geometry.rs:31-77 (Ericson region tests)
D3 closest_triangle(D3 p, uint32_t t, const std::vector<D3>& x, const Topology& top, Feature& f) {
    const auto& ids = top.triangles[t];
    D3 a = x[ids[0]], b = x[ids[1]], c = x[ids[2]];
    D3 ab = b - a, ac = c - a, ap = p - a;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) {
        f = {FVertex, ids[0]};
        return a;
    }
    D3 bp = p - b;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) {
        f = {FVertex, ids[1]};
        return b;
    }
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        f = {FEdge, top.triangle_edges[t][0]};
        return a + ab * (d1 / (d1 - d3));
    }
    D3 cp = p - c;
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) {
        f = {FVertex, ids[2]};
        return c;
    }
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        f = {FEdge, top.triangle_edges[t][2]};
        return a + ac * (d2 / (d2 - d6));
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && d4 - d3 >= 0.0 && d5 - d6 >= 0.0) {
        f = {FEdge, top.triangle_edges[t][1]};
        return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    }
    double denom = 1.0 / (va + vb + vc);
    f = {FFace, t};
    return a + ab * (vb * denom) + ac * (vc * denom);
}

// src/ogc/world.rs:126-211
OgcWorld OgcWorld::make(const std::vector<D3>& x, const std::vector<std::array<uint32_t, 3>>& tris, size_t moving,
                        const std::vector<std::array<uint32_t, 2>>& excluded_in) {
    if (moving > x.size()) throw Error{1, "Invalid OGC positions"};
    for (const auto& p : x)
        if (!finite(p)) throw Error{1, "Invalid OGC positions"};
    OgcWorld w;
    w.topology = topology_new(x.size(), tris);
    for (const auto& t : w.topology.triangles) {
        D3 a = x[t[0]], b = x[t[1]], c = x[t[2]];
        if (length_squared(cross(b - a, c - a)) < 1e-24) throw Error{1, "OGC degenerate initial face"};
    }
    const Topology& top = w.topology;
    std::vector<bool> tdyn(top.triangles.size()), edyn(top.edges.size()), pdyn(x.size());
    std::vector<Bounds> tb(top.triangles.size()), eb(top.edges.size()), pb(x.size());
    for (size_t i = 0; i < top.triangles.size(); ++i) {
        const auto& t = top.triangles[i];
        tdyn[i] = t[0] < moving || t[1] < moving || t[2] < moving;
        if (tdyn[i]) w.moving_faces.push_back(i);
        tb[i] = bounds_points({x[t[0]], x[t[1]], x[t[2]]});
    }
    for (size_t i = 0; i < top.edges.size(); ++i) {
        const auto& e = top.edges[i];
        edyn[i] = e[0] < moving || e[1] < moving;
        eb[i] = bounds_points({x[e[0]], x[e[1]]});
    }
    for (size_t i = 0; i < x.size(); ++i) {
        pdyn[i] = i < moving;
        pb[i] = bounds_points({x[i]});
    }
    w.triangles = Bvh::make(tb, tdyn);
    w.edges = Bvh::make(eb, edyn);
    w.rest_edge_length2.resize(top.edges.size());
    for (size_t i = 0; i < top.edges.size(); ++i)
        w.rest_edge_length2[i] = distance_squared(x[top.edges[i][0]], x[top.edges[i][1]]);
    w.points = Bvh::make(pb, pdyn);
    for (auto e : excluded_in) w.excluded.insert({std::min(e[0], e[1]), std::max(e[0], e[1])});
    w.excluded_neighbors.assign(x.size(), {});
    for (const auto& e : w.excluded) {
        if (e[1] >= x.size()) throw Error{1, "OGC invalid excluded vertex"};
        w.excluded_neighbors[e[0]].push_back(e[1]);
        w.excluded_neighbors[e[1]].push_back(e[0]);
    }
    for (auto& v : w.excluded_neighbors) std::sort(v.begin(), v.end());
    w.moving = moving;
    w.fixed.assign(x.begin() + moving, x.end());
    return w;
}

std::vector<D3> OgcWorld::positions(const D3* moving_x, size_t n) const {  // world.rs:212-214
    std::vector<D3> out(moving_x, moving_x + n);
    out.insert(out.end(), fixed.begin(), fixed.end());
    return out;
}

bool OgcWorld::adjacent(uint32_t a, uint32_t b) const {  // world.rs:215-217
    return a == b || std::binary_search(excluded_neighbors[a].begin(), excluded_neighbors[a].end(), b);
}

// src/ogc/world.rs:218-241
void OgcWorld::refit(const std::vector<D3>& x) {
    if (x.size() != topology.neighbors.size()) throw Error{2, "OGC invalid position array"};
    for (const auto& p : x)
        if (!finite(p)) throw Error{2, "OGC invalid position array"};
    for (size_t i = moving; i < x.size(); ++i)
        if (!(x[i] == fixed[i - moving])) throw Error{2, "OGC fixed geometry changed; rebuild the world"};
    for (size_t i : moving_faces) {
        const auto& t = topology.triangles[i];
        D3 a = x[t[0]], b = x[t[1]], c = x[t[2]];
        if (length_squared(cross(b - a, c - a)) < 1e-24) throw Error{3, "OGC degenerate face; step rejected"};
    }
    const Topology& top = topology;
    triangles.refit_dynamic([&](size_t i) {
        const auto& t = top.triangles[i];
        return bounds_points({x[t[0]], x[t[1]], x[t[2]]});
    });
    edges.refit_dynamic([&](size_t i) {
        const auto& e = top.edges[i];
        return bounds_points({x[e[0]], x[e[1]]});
    });
    points.refit_dynamic([&](size_t i) { return bounds_points({x[i]}); });
}

// src/ogc/world.rs:242-307
void OgcWorld::validate_start(const std::vector<D3>& x) {
    refit(x);
    const Topology& top = topology;
    for (size_t i = 0; i < top.triangles.size(); ++i) {
        const auto& t = top.triangles[i];
        bool t_fixed = t[0] >= moving && t[1] >= moving && t[2] >= moving;
        long hit = -1;
        triangles.query(inflate(bounds_points({x[t[0]], x[t[1]], x[t[2]]}), 1e-10), t_fixed, [&](size_t j) {
            const auto& q = top.triangles[j];
            bool q_fixed = q[0] >= moving && q[1] >= moving && q[2] >= moving;
            if (j <= i || (t_fixed && q_fixed)) return;
            for (uint32_t a : t)
                for (uint32_t b : q)
                    if (excluded.count({std::min(a, b), std::max(a, b)})) return;
            auto contains = [](const std::array<uint32_t, 3>& s, uint32_t v) {
                return s[0] == v || s[1] == v || s[2] == v;
            };
            for (int k = 0; k < 3; ++k) {
                bool h1 = !contains(q, t[k]) && !contains(q, t[(k + 1) % 3]) &&
                          segment_triangle(x[t[k]], x[t[(k + 1) % 3]], x[q[0]], x[q[1]], x[q[2]]);
                bool h2 = !contains(t, q[k]) && !contains(t, q[(k + 1) % 3]) &&
                          segment_triangle(x[q[k]], x[q[(k + 1) % 3]], x[t[0]], x[t[1]], x[t[2]]);
                if (h1 || h2) hit = (long)j;
            }
        });
        if (hit >= 0) {
            char buf[256];
            std::snprintf(buf, sizeof buf,
                          "OGC initial intersection between faces %zu and %ld; reset/rearrange before simulating", i,
                          hit);
            throw Error{3, buf};
        }
    }
    OgcSettings s;
    s.radius = 1e-5;
    ContactSet cs = detect(x, 1e-5, s);
    if (cs.minimum_distance <= 1e-10)
        throw Error{3, "OGC initial touching/coplanar features: separation must be positive"};
}

// src/ogc/candidates.rs:23-68 (pair filters) at an explicit search radius
void OgcWorld::pairs_at(double search, std::vector<std::array<uint32_t, 2>>& vf,
                        std::vector<std::array<uint32_t, 2>>& ee) const {
    const Topology& top = topology;
    points.pairs(triangles, search, false, [&](size_t v, size_t t) {
        const auto& ids = top.triangles[t];
        for (uint32_t i : ids)
            if (adjacent((uint32_t)v, i)) return;
        vf.push_back({(uint32_t)v, (uint32_t)t});
    });
    edges.pairs(edges, search, true, [&](size_t e, size_t f) {
        const auto& ids = top.edges[e];
        const auto& js = top.edges[f];
        for (uint32_t i : ids)
            for (uint32_t j : js)
                if (adjacent(i, j)) return;
        // moving edge first for fixed/moving pairs, canonical otherwise
        bool e_fixed = ids[0] >= moving && ids[1] >= moving;
        if (e_fixed)
            ee.push_back({(uint32_t)f, (uint32_t)e});
        else
            ee.push_back({(uint32_t)e, (uint32_t)f});
    });
}

// src/ogc/candidates.rs:23-68
Candidates OgcWorld::build_candidates(const std::vector<D3>& x, double radius, double skin) const {
    Candidates c;
    pairs_at(radius + 2.0 * skin + 1e-12, c.vf, c.ee);
    c.centers.assign(x.begin(), x.begin() + moving);
    c.radius = radius;
    c.skin = skin;
    return c;
}

namespace {
struct Batch {
    std::vector<double> distance;
    std::vector<Contact> found;
    size_t vf = 0, ee = 0, rejected = 0;
};

void add_contact(Batch& out, uint8_t kind, std::array<uint32_t, 4> ids, uint8_t count, double eps) {  // world.rs:435-459
    if (kind == PointPoint && ids[0] > ids[1]) std::swap(ids[0], ids[1]);
    if (kind == PointEdge && ids[1] > ids[2]) std::swap(ids[1], ids[2]);
    if (kind == PointFace) std::sort(ids.begin() + 1, ids.end());
    if (kind == EdgeEdge) {
        std::sort(ids.begin(), ids.begin() + 2);
        std::sort(ids.begin() + 2, ids.end());
        if (ids[0] > ids[2]) {
            std::swap(ids[0], ids[2]);
            std::swap(ids[1], ids[3]);
        }
    }
    Contact c;
    c.kind = kind;
    for (int i = 0; i < 4; ++i) c.vertices[i] = ids[i];
    c.count = count;
    c.mollifier_epsilon = eps;
    out.found.push_back(c);
}
}  // namespace

// src/ogc/world.rs:316-557 (detect_impl + scan)
ContactSet OgcWorld::detect(const std::vector<D3>& x, double query_radius, const OgcSettings& settings, bool prune) {
    if (!settings.valid()) throw Error{1, "Invalid OGC radius, stiffness or trust-region parameters"};
    if (!std::isfinite(query_radius) || query_radius < settings.radius)
        throw Error{1, "OGC query radius must cover the contact radius"};
    double t0 = now_ms();
    refit(x);
    double refit_ms = now_ms() - t0;
    double t1 = now_ms();
    bool rebuilt = !candidates.has_value() || !candidates->covers(x.data(), moving, query_radius);
    if (rebuilt) {
        double R = std::fmax(std::ceil(query_radius / settings.radius) * settings.radius, query_radius);
        candidates = build_candidates(x, R, settings.radius);
    }
    double candidates_ms = now_ms() - t1;
    double t2 = now_ms();
    double scale = query_radius;
    for (const auto& p : x) scale = std::fmax(scale, max_element(vabs(p)));
    double pr = query_radius + 64.0 * std::numeric_limits<double>::epsilon() * scale;
    double padded_radius2 = pr * pr;
    const Topology& top = topology;
    const Candidates& cand = *candidates;
    int lanes = std::max(1, threads);
    std::vector<Batch> batches(lanes);
#pragma omp parallel for num_threads(lanes) schedule(static, 1)
    for (int lane = 0; lane < lanes; ++lane) {
        Batch& B = batches[lane];
        B.distance.assign(x.size(), query_radius);
        for (size_t k = lane; k < cand.vf.size(); k += lanes) {
            uint32_t v = cand.vf[k][0], t = cand.vf[k][1];
            if (prune && bounds_distance_squared(points.primitive_bounds[v], triangles.primitive_bounds[t]) >
                             padded_radius2) {
                B.rejected++;
                continue;
            }
            const auto& ids = top.triangles[t];
            Feature f;
            D3 p = closest_triangle(x[v], t, x, top, f);
            double d = distance(x[v], p);
            if (d >= query_radius) continue;
            B.vf++;
            B.distance[v] = std::fmin(B.distance[v], d);
            for (uint32_t i : ids) B.distance[i] = std::fmin(B.distance[i], d);
            if (f.kind == FVertex) {
                if (vertex_feasible(x[v], f.id, x, top)) add_contact(B, PointPoint, {v, f.id, 0, 0}, 2, 0.0);
            } else if (f.kind == FEdge) {
                if (edge_feasible(x[v], f.id, x, top))
                    add_contact(B, PointEdge, {v, top.edges[f.id][0], top.edges[f.id][1], 0}, 3, 0.0);
            } else {
                add_contact(B, PointFace, {v, ids[0], ids[1], ids[2]}, 4, 0.0);
            }
        }
        for (size_t k = lane; k < cand.ee.size(); k += lanes) {
            uint32_t e = cand.ee[k][0], f = cand.ee[k][1];
            if (prune && bounds_distance_squared(edges.primitive_bounds[e], edges.primitive_bounds[f]) >
                             padded_radius2) {
                B.rejected++;
                continue;
            }
            const auto& ids = top.edges[e];
            const auto& js = top.edges[f];
            D3 a = x[ids[0]], b = x[ids[1]], c = x[js[0]], d = x[js[1]];
            double s, t;
            closest_segments(a, b, c, d, s, t);
            D3 p = a + (b - a) * s;
            D3 q = c + (d - c) * t;
            double dist = distance(p, q);
            if (dist >= query_radius) continue;
            B.ee++;
            for (uint32_t v : {ids[0], ids[1], js[0], js[1]}) B.distance[v] = std::fmin(B.distance[v], dist);
            long end_a = s <= 0.0 ? (long)ids[0] : (s >= 1.0 ? (long)ids[1] : -1);
            long end_b = t <= 0.0 ? (long)js[0] : (t >= 1.0 ? (long)js[1] : -1);
            if ((end_a >= 0 && !vertex_feasible(q, (uint32_t)end_a, x, top)) ||
                (end_b >= 0 && !vertex_feasible(p, (uint32_t)end_b, x, top)))
                continue;
            if (end_a >= 0 && end_b >= 0)
                add_contact(B, PointPoint, {(uint32_t)end_a, (uint32_t)end_b, 0, 0}, 2, 0.0);
            else if (end_a >= 0)
                add_contact(B, PointEdge, {(uint32_t)end_a, js[0], js[1], 0}, 3, 0.0);
            else if (end_b >= 0)
                add_contact(B, PointEdge, {(uint32_t)end_b, ids[0], ids[1], 0}, 3, 0.0);
            else
                add_contact(B, EdgeEdge, {ids[0], ids[1], js[0], js[1]}, 4,
                            1e-3 * rest_edge_length2[e] * rest_edge_length2[f]);
        }
    }
    std::vector<double> dist(x.size(), query_radius);
    std::vector<Contact> found;
    ContactSet out;
    for (auto& B : batches) {
        for (size_t i = 0; i < x.size(); ++i) dist[i] = std::fmin(dist[i], B.distance[i]);
        found.insert(found.end(), B.found.begin(), B.found.end());
        out.vertex_face_candidates += B.vf;
        out.edge_edge_candidates += B.ee;
        out.profile.aabb_rejections += B.rejected;
    }
    auto key_less = [](const Contact& a, const Contact& b) {
        if (a.kind != b.kind) return a.kind < b.kind;
        for (int i = 0; i < 4; ++i)
            if (a.vertices[i] != b.vertices[i]) return a.vertices[i] < b.vertices[i];
        return false;
    };
    auto key_eq = [](const Contact& a, const Contact& b) {
        return a.kind == b.kind && a.vertices[0] == b.vertices[0] && a.vertices[1] == b.vertices[1] &&
               a.vertices[2] == b.vertices[2] && a.vertices[3] == b.vertices[3];
    };
    std::sort(found.begin(), found.end(), key_less);
    found.erase(std::unique(found.begin(), found.end(), key_eq), found.end());
    out.contacts = std::move(found);
    for (const auto& c : out.contacts)
        if (contact_value(c, x, settings.radius, settings.stiffness) > 0.0) out.active_contacts++;
    out.incident.assign(moving, {});
    for (size_t c = 0; c < out.contacts.size(); ++c)
        for (int k = 0; k < out.contacts[c].count; ++k) {
            uint32_t v = out.contacts[c].vertices[k];
            if (v < moving) out.incident[v].push_back((uint32_t)c);
        }
    double md = query_radius;
    for (size_t i = 0; i < moving; ++i) md = std::fmin(md, dist[i]);
    out.minimum_distance = md;
    out.centers.assign(x.begin(), x.begin() + moving);
    out.radii.resize(moving);
    for (size_t i = 0; i < moving; ++i) out.radii[i] = settings.relaxation * dist[i];
    out.broad_phase_rebuilt = rebuilt;
    out.profile.refit_ms = refit_ms;
    out.profile.candidates_ms = candidates_ms;
    out.profile.narrow_ms = now_ms() - t2;
    out.profile.candidate_pairs = cand.vf.size() + cand.ee.size();
    return out;
}

}  // namespace oracle
