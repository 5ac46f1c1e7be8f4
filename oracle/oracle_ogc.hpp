// Oracle (test infrastructure only): FP64 restatement of ClothCraft's OGC
// detection. Follows src/ogc/{topology,bvh,candidates,world,geometry}.rs.
#pragma once
#include <algorithm>
#include <array>
#include <map>
#include <optional>
#include <set>
#include <string>
#include <vector>

#include "oracle_math.hpp"

namespace oracle {

struct Error {
    int code;
    std::string message;
};

// ---------------------------------------------------------------- Topology
struct Topology {  // src/ogc/topology.rs:4-52
    std::vector<std::array<uint32_t, 3>> triangles;
    std::vector<std::array<uint32_t, 2>> edges;
    std::vector<std::array<uint32_t, 3>> triangle_edges;
    std::vector<std::vector<uint32_t>> neighbors;
    std::vector<std::vector<uint32_t>> opposites;
};
Topology topology_new(size_t n, const std::vector<std::array<uint32_t, 3>>& triangles);  // throws Error

// ------------------------------------------------------------------ Bounds
struct Bounds {  // src/ogc/bvh.rs:3-43
    D3 min, max;
};
inline Bounds bounds_empty() {
    double inf = std::numeric_limits<double>::infinity();
    return {{inf, inf, inf}, {-inf, -inf, -inf}};
}
inline Bounds bounds_add(Bounds b, D3 p) { return {vmin(b.min, p), vmax(b.max, p)}; }
inline Bounds bounds_points(std::initializer_list<D3> ps) {
    Bounds b = bounds_empty();
    for (D3 p : ps) b = bounds_add(b, p);
    return b;
}
inline Bounds inflate(Bounds b, double r) { return {b.min - D3{r, r, r}, b.max + D3{r, r, r}}; }
inline bool overlaps(Bounds a, Bounds b) {
    return a.min.x <= b.max.x && a.min.y <= b.max.y && a.min.z <= b.max.z && a.max.x >= b.min.x &&
           a.max.y >= b.min.y && a.max.z >= b.min.z;
}
inline double bounds_distance_squared(Bounds a, Bounds b) {
    D3 d = vmax(vmax(a.min - b.max, b.min - a.max), D3{0, 0, 0});
    return length_squared(d);
}
inline Bounds bounds_union(Bounds a, Bounds b) { return {vmin(a.min, b.min), vmax(a.max, b.max)}; }

// --------------------------------------------------------------------- Bvh
struct BvhNode {
    Bounds bounds;
    bool has_children;
    size_t children[2];
    size_t start, end;
    bool dynamic;
};

struct Bvh {  // src/ogc/bvh.rs:44-243
    std::vector<BvhNode> nodes;
    std::vector<size_t> order;
    std::vector<size_t> roots;
    std::vector<Bounds> primitive_bounds;
    size_t dynamic_nodes = 0;

    static Bvh make(const std::vector<Bounds>& bounds, const std::vector<bool>& dynamic);
    size_t build(const std::vector<Bounds>& bounds, const std::vector<bool>& dynamic, size_t start, size_t end);
    template <class F>
    void refit_dynamic(F bounds_of);
    template <class F>
    void query(Bounds q, bool dynamic_only, F visit) const;
    template <class F>
    void pairs(const Bvh& other, double radius, bool same, F visit) const;
};

template <class F>
void Bvh::refit_dynamic(F bounds_of) {  // bvh.rs:138-154
    for (size_t k = dynamic_nodes; k-- > 0;) {
        BvhNode& n = nodes[k];
        if (n.has_children) {
            n.bounds = bounds_union(nodes[n.children[0]].bounds, nodes[n.children[1]].bounds);
        } else {
            for (size_t i = n.start; i < n.end; ++i) primitive_bounds[order[i]] = bounds_of(order[i]);
            Bounds b = primitive_bounds[order[n.start]];
            for (size_t i = n.start + 1; i < n.end; ++i) b = bounds_union(b, primitive_bounds[order[i]]);
            n.bounds = b;
        }
    }
}

template <class F>
void Bvh::query(Bounds q, bool dynamic_only, F visit) const {  // bvh.rs:155-185
    if (nodes.empty()) return;
    size_t stack[128];
    size_t len = roots.size();
    for (size_t i = 0; i < len; ++i) stack[i] = roots[i];
    while (len > 0) {
        size_t i = stack[--len];
        const BvhNode& n = nodes[i];
        if ((dynamic_only && !n.dynamic) || !overlaps(n.bounds, q)) continue;
        if (n.has_children) {
            stack[len] = n.children[0];
            stack[len + 1] = n.children[1];
            len += 2;
        } else {
            for (size_t k = n.start; k < n.end; ++k) {
                size_t id = order[k];
                if (overlaps(primitive_bounds[id], q)) visit(id);
            }
        }
    }
}

template <class F>
void Bvh::pairs(const Bvh& other, double radius, bool same, F visit) const {  // bvh.rs:198-242
    std::vector<std::pair<size_t, size_t>> stack;
    stack.reserve(128);
    for (size_t i = 0; i < roots.size(); ++i)
        for (size_t j = same ? i : 0; j < other.roots.size(); ++j) stack.push_back({roots[i], other.roots[j]});
    double radius2 = radius * radius;
    while (!stack.empty()) {
        auto [a, b] = stack.back();
        stack.pop_back();
        const BvhNode& na = nodes[a];
        const BvhNode& nb = other.nodes[b];
        if ((!na.dynamic && !nb.dynamic) || bounds_distance_squared(na.bounds, nb.bounds) > radius2) continue;
        if (same && a == b) {
            if (na.has_children) {
                size_t l = na.children[0], r = na.children[1];
                stack.push_back({l, l});
                stack.push_back({l, r});
                stack.push_back({r, r});
                continue;
            }
        } else if (na.has_children && (!nb.has_children || na.end - na.start >= nb.end - nb.start)) {
            stack.push_back({na.children[0], b});
            stack.push_back({na.children[1], b});
            continue;
        } else if (nb.has_children) {
            stack.push_back({a, nb.children[0]});
            stack.push_back({a, nb.children[1]});
            continue;
        }
        for (size_t off = 0; off < na.end - na.start; ++off) {
            size_t i = order[na.start + off];
            size_t start = nb.start + ((same && a == b) ? off + 1 : 0);
            for (size_t k = start; k < nb.end; ++k) {
                size_t j = other.order[k];
                if (bounds_distance_squared(primitive_bounds[i], other.primitive_bounds[j]) <= radius2) {
                    if (same)
                        visit(std::min(i, j), std::max(i, j));
                    else
                        visit(i, j);
                }
            }
        }
    }
}

// -------------------------------------------------------------- Candidates
struct Candidates {  // src/ogc/candidates.rs:5-68
    std::vector<D3> centers;
    double radius, skin;
    std::vector<std::array<uint32_t, 2>> vf, ee;
    bool covers(const D3* moving, size_t n, double r) const;
};

// ------------------------------------------------------------- ContactSet
struct OgcSettings {  // src/ogc/world.rs:33-71
    double radius = 0.003, stiffness = 100000.0, relaxation = 0.45, refresh_fraction = 0.01;
    bool valid() const;
};

struct DetectionProfile {
    double refit_ms = 0, candidates_ms = 0, narrow_ms = 0;
    size_t candidate_pairs = 0, aabb_rejections = 0;
};

struct ContactSet {  // src/ogc/world.rs:73-107
    DetectionProfile profile;
    std::vector<Contact> contacts;
    size_t active_contacts = 0;
    std::vector<std::vector<uint32_t>> incident;
    std::vector<D3> centers;
    std::vector<double> radii;
    double minimum_distance = 0;
    size_t vertex_face_candidates = 0, edge_edge_candidates = 0;
    bool broad_phase_rebuilt = false;

    // Equation 27 clip (world.rs:91-100)
    D3 truncate(size_t v, D3 proposed, bool& clipped) const {
        D3 d = proposed - centers[v];
        double len = length(d);
        double b = radii[v];
        if (len > b) {
            clipped = true;
            return centers[v] + d * (b / len);
        }
        clipped = false;
        return proposed;
    }
    double value(const std::vector<D3>& x, const OgcSettings& s) const;
};

double contact_value(const Contact& c, const std::vector<D3>& x, double r, double k);  // potential.rs:66-68

// ---------------------------------------------------------------- OgcWorld
struct OgcWorld {  // src/ogc/world.rs:111-124
    Topology topology;
    size_t moving = 0;
    std::vector<D3> fixed;
    Bvh triangles, edges, points;
    std::vector<double> rest_edge_length2;
    std::set<std::array<uint32_t, 2>> excluded;
    std::vector<std::vector<uint32_t>> excluded_neighbors;
    std::vector<size_t> moving_faces;
    std::optional<Candidates> candidates;
    int threads = 1;  // narrow-phase lanes (results do not depend on it)

    static OgcWorld make(const std::vector<D3>& x, const std::vector<std::array<uint32_t, 3>>& tris,
                         size_t moving, const std::vector<std::array<uint32_t, 2>>& excluded);  // throws Error
    std::vector<D3> positions(const D3* moving_x, size_t n) const;
    bool adjacent(uint32_t a, uint32_t b) const;
    void refit(const std::vector<D3>& x);
    void validate_start(const std::vector<D3>& x);
    ContactSet detect(const std::vector<D3>& x, double query_radius, const OgcSettings& s, bool prune = true);
    Candidates build_candidates(const std::vector<D3>& x, double radius, double skin) const;
    void pairs_at(double search, std::vector<std::array<uint32_t, 2>>& vf,
                  std::vector<std::array<uint32_t, 2>>& ee) const;
};

// geometry needing topology (src/ogc/geometry.rs:13-77)
bool vertex_feasible(D3 p, uint32_t v, const std::vector<D3>& x, const Topology& top);
bool edge_feasible(D3 p, uint32_t e, const std::vector<D3>& x, const Topology& top);
D3 closest_triangle(D3 p, uint32_t t, const std::vector<D3>& x, const Topology& top, Feature& f);

}  // namespace oracle
