// OGC world on the device: topology, LBVH broad phase, candidate cache, FP64
// narrow phase, canonical contact set. Host class + device views.
#pragma once
#include <array>
#include <vector>

#include "common.cuh"
#include "radix.cuh"

namespace cc {

struct Box {
    double lo[3];
    double hi[3];
};

// One internal LBVH node as a traversal reads it: both children's boxes,
// rounded outward to FP32 (lo down, hi up, so each contains the exact FP64
// box of everything below it), the children's indices and the largest
// primitive id below each child, in one 64-byte record. A visit is one
// record read; only the leaves are tested against their exact FP64 boxes.
//   a = left lo.xyz, left hi.x     b = left hi.yz, right lo.xy
//   c = right lo.z, right hi.xyz   d = left child, right child (bit 31 set:
//   a leaf, by sorted position), largest id below left, below right
struct alignas(16) LNode {
    float4 a, b, c;
    int4 d;
};

// Karras LBVH over a subset of primitives (ids) with boxes in a global array.
struct LbvhView {
    uint32_t m;                 // leaves
    const LNode* node;          // [m-1] internal nodes, root 0
    const uint32_t* leaf_prim;  // [m] primitive id of each sorted leaf
    const Box* leaf_box;        // [m] exact primitive boxes in leaf order
};

// The topology (Morton order, Karras split) comes from build(); refit()
// recomputes the boxes for the current primitive boxes and keeps the
// topology, as the reference's Bvh keeps its tree and refits it
// (src/ogc/bvh.rs). Either way every primitive box is inside its ancestors'
// boxes, so a traversal finds the same pair set.
struct Lbvh {
    uint32_t m = 0;
    bool built = false;
    DBuf<LNode> node;       // [m-1]
    DBuf<int> parent;       // [2m-1]: internal 0..m-2, leaves m-1..2m-2
    DBuf<unsigned> visits;  // [m-1]
    DBuf<uint32_t> leaf_prim, ids_tmp;
    DBuf<Box> leaf_box;     // [m]
    DBuf<unsigned long long> morton, morton_tmp;
    DBuf<unsigned long long> bounds;  // 6 order keys
    RadixSorter sorter;
    // Both return the number of this library's kernels launched.
    int build(const Box* prim_box, const uint32_t* ids, uint32_t m, cudaStream_t s, unsigned int* err);
    int refit(const Box* prim_box, cudaStream_t s);  // after a build over the same primitives
    LbvhView view() const { return {m, node.ptr, leaf_prim.ptr, leaf_box.ptr}; }
};

// Static topology (src/ogc/topology.rs:13-52), built on the host at creation.
struct TopologyHost {
    std::vector<std::array<uint32_t, 3>> tri;
    std::vector<std::array<uint32_t, 3>> tri_edges;
    std::vector<std::array<uint32_t, 2>> edges;
    std::vector<std::array<int32_t, 2>> opposites;
    std::vector<uint32_t> nb_off, nb;  // sorted neighbour CSR
};
TopologyHost build_topology(size_t n, const std::vector<std::array<uint32_t, 3>>& tris);  // throws Failure

// Everything a detection kernel reads.
struct WorldView {
    uint32_t n_all, moving, n_tri, n_edge;
    const uint3* tri;
    const uint3* tri_edges;
    const uint2* edges;
    const int2* opposites;
    const uint32_t* nb_off;
    const uint32_t* nb;
    const uint32_t* ex_off;
    const uint32_t* ex;
    const double* rest_len2;
    const double4* x;     // [n_all]
    Box* tri_box;         // [n_tri]
    Box* edge_box;        // [n_edge]
};

struct DetectStats {  // read back after each detection
    unsigned long long n_vf, n_ee;             // candidate pairs (cache)
    unsigned long long n_raw;                  // raw contacts
    unsigned long long n_contacts;             // unique contacts
    unsigned long long active;
    unsigned long long vf_count, ee_count, rejections;
    unsigned long long min_dist_bits;
    unsigned long long n_incident;
    unsigned long long max_move_bits;          // max |x - cache centre|^2 (moving)
    unsigned long long max_abs_bits;           // max |x| component (all)
    unsigned long long intersect_key;          // validate_start: first (i<<32|j)
    unsigned int error;
    unsigned int rebuild;
};

struct ContactsView {  // canonical contact set for the sweep and colouring
    uint32_t n;
    const uint32_t* kind;   // [n]
    const uint4* verts;     // [n]
    const double* eps;      // [n]
    const uint32_t* inc_off;  // [moving+1]
    const uint32_t* inc;      // contact ids
    const double4* centers;   // [moving]
    const double* radii;      // [moving]
};

class World {
   public:
    World(const double* x_all, size_t n_all, const std::vector<std::array<uint32_t, 3>>& tris, size_t moving,
          const std::vector<std::array<uint32_t, 2>>& excluded, cudaStream_t stream);
    ~World();

    // OgcWorld::detect on the positions currently in x() (n_all entries).
    // check_fixed: verify the fixed block equals the creation positions.
    void detect(double query_radius, double radius, double relaxation, double stiffness, bool check_fixed,
                bool prune = true);
    void validate_start();  // throws Failure
    // Fresh pairs at an exact search radius, sorted, for parity tests.
    void fresh_pairs(double search, std::vector<uint32_t>& vf, std::vector<uint32_t>& ee);

    double4* x() { return x_.ptr; }
    const DetectStats& stats() const { return *stats_h_.ptr; }
    ContactsView contacts() const;
    size_t n_all() const { return n_all_; }
    size_t moving() const { return moving_; }
    size_t n_edges() const { return n_edge_; }
    const TopologyHost& topology() const { return top_; }
    const uint32_t* nb_off() const { return nb_off_.ptr; }
    const uint32_t* nb() const { return nb_.ptr; }
    // download the canonical contact set (for the C ABI / tests)
    void download(std::vector<uint32_t>& kind, std::vector<uint32_t>& verts, std::vector<double>& eps,
                  std::vector<uint64_t>& inc_off, std::vector<uint32_t>& inc, std::vector<double>& radii);
    cudaStream_t stream() const { return stream_; }
    void invalidate_cache() { cache_valid_ = false; }
    uint64_t launches() const { return launches_; }
    // Device time of the last detection's phases (CUDA events; recorded only
    // while profiling is on): refit and cache check, candidate rebuild (0 on a
    // cache hit), narrow phase, canonical set (sort, dedup, incidence, radii).
    struct PhaseMs {
        double refit = 0, candidates = 0, narrow = 0, canonical = 0;
    };
    void set_profiling(bool on) { profile_ = on; }
    const PhaseMs& last_phase_ms() const { return phase_ms_; }
    // LBVH topology policy for the moving trees at a candidate rebuild: 0 =
    // keep the topology of the first build and refit it (the reference's
    // tree), k >= 1 = rebuild it from Morton codes every k-th candidate
    // rebuild and refit in between.
    void set_tree_rebuild_period(uint32_t k) { tree_period_ = k; }
    uint32_t tree_rebuild_period() const { return tree_period_; }
    uint64_t tree_builds() const { return tree_builds_; }

   private:
    WorldView view() const;
    void refit(bool check_fixed);
    void build_candidates(double R, double skin);
    int update_trees();  // moving trees for the current boxes, on two streams
    int order_points();  // point_order_ from the current positions
    void sync_stats();

    cudaStream_t stream_;
    cudaStream_t side_ = nullptr;  // second stream for the triangle side of a rebuild
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    uint32_t tree_period_ = 0;
    uint32_t rebuilds_since_build_ = 0;
    uint64_t tree_builds_ = 0;
    size_t n_all_, moving_, n_tri_, n_edge_;
    TopologyHost top_;
    std::vector<uint32_t> tri_moving_h_, tri_fixed_h_, edge_moving_h_, edge_fixed_h_;

    DBuf<uint3> tri_, tri_edges_;
    DBuf<uint2> edges_;
    DBuf<int2> opposites_;
    DBuf<uint32_t> nb_off_, nb_, ex_off_, ex_;
    DBuf<double> rest_len2_;
    DBuf<double4> x_, fixed_x_;
    DBuf<Box> tri_box_, edge_box_;
    DBuf<uint32_t> tri_moving_, tri_fixed_, edge_moving_, edge_fixed_;
    Lbvh tree_tri_moving_, tree_tri_fixed_, tree_edge_moving_, tree_edge_fixed_;

    // candidate cache (src/ogc/candidates.rs)
    bool cache_valid_ = false;
    double cache_R_ = 0, cache_skin_ = 0;
    DBuf<double4> cache_centers_;
    DBuf<uint2> vf_, ee_;
    size_t vf_cap_ = 0, ee_cap_ = 0;
    DBuf<unsigned long long> fresh_counts_;  // fresh_pairs' own pair counts
    DBuf<uint32_t> point_order_, pt_ids_;     // VF query order (Morton order of all points)
    DBuf<unsigned long long> pt_code_, pt_code_s_, pt_bounds_;

    // narrow phase + canonical set
    DBuf<unsigned long long> raw_key_, raw_key_s_;  // packed contact keys (detect.cu)
    DBuf<uint32_t> uniq_flag_, uniq_pos_;
    DBuf<uint32_t> edge_rank_, tri_rank_, rank_edge_id_;  // contact-key ranks
    DBuf<uint2> rank_edge_verts_;
    DBuf<uint3> rank_tri_verts_;
    uint32_t key_bits_ = 1;
    size_t raw_cap_ = 0;
    DBuf<uint32_t> c_kind_;
    DBuf<uint4> c_verts_;
    DBuf<double> c_eps_;
    DBuf<unsigned long long> dist_bits_;
    DBuf<double> radii_;
    DBuf<double4> centers_;
    DBuf<uint32_t> inc_count_, inc_off_, inc_, inc_cursor_;
    RadixSorter sorter_;
    DBuf<uint32_t> scan_tmp_;
    DBuf<DetectStats> stats_d_;
    Pinned<DetectStats> stats_h_;
    double query_radius_ = 0;
    uint64_t launches_ = 0;
    bool profile_ = false;
    cudaEvent_t phase_ev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    PhaseMs phase_ms_;
    void mark(int k);

    friend struct WorldAccess;
};

}  // namespace cc
