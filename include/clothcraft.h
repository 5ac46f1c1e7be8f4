/*
 * clothcraft.h — C ABI of the B200-native ClothCraft physics step.
 *
 * The library replaces the hybrid wgpu backend of ClothCraft with a CUDA
 * (sm_100a) implementation of the whole step: Vertex Block Descent colour
 * sweeps plus the Offset Geometric Contact (OGC) pipeline, both resident on
 * one GPU. Each entry point names the reference interface it stands in for
 * (paths are inside the ClothCraft source tree).
 *
 * Conventions (mirroring the reference's Rust surface):
 *   - SI units, f64 in and out. Positions and velocities are n x 3 row-major
 *     doubles (the memory image of Vec<DVec3>).
 *   - Every fallible call returns an int32 status (CC_OK on success) and is
 *     transactional: caller arrays are written only on CC_OK
 *     (src/vbd.rs:249,399-405; tests/vbd.rs:88-90).
 *   - The message of the last failure on a handle is read with cc_last_error;
 *     failures without a handle (creation) with cc_global_last_error.
 *   - One handle is driven by one host thread at a time, as GpuVbd is
 *     (RefCell, src/gpu_vbd.rs:15-25). The library owns all device memory.
 *   - Index arrays are uint32. No torch or CUDA types cross this boundary.
 */
#ifndef CLOTHCRAFT_H
#define CLOTHCRAFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CC_ABI_VERSION 3

enum cc_status {
    CC_OK = 0,
    CC_ERR_INVALID_ARGUMENT = 1, /* settings, dimensions, indices          */
    CC_ERR_INVALID_STATE = 2,    /* non-finite state, moved fixed geometry */
    CC_ERR_CONTACT = 3,          /* zero separation, initial intersection, */
                                 /* trust-region invariant                 */
    CC_ERR_NON_FINITE = 4,       /* non-finite result, state unchanged     */
    CC_ERR_CAPACITY = 5,         /* caller buffer too small; sizes written */
    CC_ERR_CUDA = 6,             /* CUDA runtime failure                   */
    CC_ERR_DEVICE_TIMEOUT = 7    /* a bounded device wait gave up          */
};

/* Material (src/model.rs:7-22). grain_degrees rotates the fibre frame. */
typedef struct cc_material {
    double warp, weft, shear;
    double compression_ratio, compression_transition;
    double bend_warp, bend_weft;
    double density, thickness, grain_degrees;
} cc_material;

/* The cloth: Mesh (src/model.rs:91-115) plus the seam stitch terms that
 * VbdSolver::new flattens (src/vbd.rs:128-144, src/garment/seam.rs:215-238).
 * Stitch s covers stitch_vertices/weights[stitch_offsets[s] ..
 * stitch_offsets[s+1]) and has stiffness seam.stiffness * weight_m. */
typedef struct cc_mesh {
    uint64_t n_vertices;
    uint64_t n_triangles;
    const uint32_t* triangles;         /* [n_triangles][3]                     */
    const double* inv_dm;              /* [n_triangles][4]: x_axis.xy, y_axis.xy */
    const double* area;                /* [n_triangles]                        */
    const uint32_t* triangle_material; /* [n_triangles]                        */
    uint64_t n_hinges;
    const uint32_t* hinges;            /* [n_hinges][4]: shared edge a,b; c; d */
    const double* hinge_weight;        /* [n_hinges]                           */
    const double* hinge_across;        /* [n_hinges][2]                        */
    const uint32_t* hinge_material;    /* [n_hinges]                           */
    uint64_t n_materials;
    const cc_material* materials;      /* [n_materials]                        */
    const double* masses;              /* [n_vertices]                         */
    const uint8_t* pinned;             /* [n_vertices], 1 = pinned             */
    const double* pin_positions;       /* [n_vertices][3], read where pinned   */
    uint64_t n_stitches;
    const uint32_t* stitch_offsets;    /* [n_stitches + 1]                     */
    const uint32_t* stitch_vertices;   /* [stitch_offsets[n_stitches]]         */
    const double* stitch_weights;      /* [stitch_offsets[n_stitches]]         */
    const double* stitch_stiffness;    /* [n_stitches]                         */
} cc_mesh;

/* Fixed obstacle: SurfaceMesh (src/avatar.rs:8-11). */
typedef struct cc_surface {
    uint64_t n_vertices;
    const double* vertices;            /* [n_vertices][3] */
    uint64_t n_triangles;
    const uint32_t* triangles;         /* [n_triangles][3] */
} cc_surface;

/* OgcSettings (src/ogc/world.rs:33-71). */
typedef struct cc_ogc_settings {
    double radius;
    double stiffness;
    double relaxation;
    double refresh_fraction;
} cc_ogc_settings;

/* Initial guess of the sweeps. */
enum cc_init_mode {
    CC_INIT_ADAPTIVE = 0, /* Prediction::guess (src/vbd/prediction.rs:15-41) */
    CC_INIT_LEARNED = 1   /* MLP correction of the adaptive guess, kept only */
                          /* when its step energy is lower (cc_mlp_*)        */
};
/* Arithmetic of the colour sweeps (no reference counterpart; the reference's
 * CPU path is FP64, its wgpu shader FP32).
 * CC_SWEEP_FP64: every term and the 3x3 solve in FP64, operation for operation
 *   as the CPU path (the parity form).
 * CC_SWEEP_FP32: membrane and bending energies, gradients and Hessians in FP32
 *   from FP64 edge differences; OGC contact terms in FP64; the 3x3 solve in
 *   FP32 unless its condition estimate exceeds 1e6; the line search compares
 *   energy differences summed in FP64. Detection, the relative residual and
 *   the step energy stay FP64. */
enum cc_sweep_precision {
    CC_SWEEP_FP64 = 0,
    CC_SWEEP_FP32 = 1
};
/* VbdSettings (src/vbd.rs:18-52), plus two extensions without a reference
 * counterpart: the initial-guess mode and a relative-residual target.
 *
 * relative residual = ||P grad E(x)|| / ||grad E(y)|| over free vertices, E
 * the step objective (inertia + membrane + bending + stitches + grab + OGC
 * terms), y the inertial target, P the projection that drops the outward
 * normal part of a vertex's gradient when the vertex sits on the boundary of
 * its OGC ball and its descent direction leaves the ball: the first-order
 * residual of the ball-constrained problem the sweeps solve (without P the
 * norm stalls at the forces the trust region holds back).
 * The OGC terms are those in force when the residual is evaluated (the
 * step's detection, or its latest refresh).
 * residual_check_every = 0: never evaluated (the reference's behaviour).
 * residual_check_every = k > 0: evaluated after every k-th iteration and
 * after the last; with residual_tolerance > 0 the iterations stop at the
 * first evaluation <= residual_tolerance (`iterations` is then the cap).
 * stall_refresh = s > 0 (with a tolerance only): after s evaluations in a
 * row without a 5 % decrease of the residual while vertices are clipped to
 * their OGC balls, the next iteration starts with a refresh detection, as
 * the reference's refresh rule does once refresh_fraction * n vertices clip
 * (src/vbd.rs:326-334); 0 keeps the reference rule alone.
 * acceleration = rho in (0, 1): after every iteration the free vertices move
 * to w_k (x_sweep - x_{k-2}) + x_{k-2}, clipped to their OGC balls, with the
 * Chebyshev weights w_1 = 1, w_2 = 2/(2 - rho^2), w_k = 4/(4 - rho^2 w_{k-1})
 * (Wang 2015). The sequence restarts at the step's start, at every refresh
 * detection and after a residual evaluation that exceeds the previous one,
 * so it is meant for use with residual_check_every > 0. 0 = off: the
 * reference's iteration. */
typedef struct cc_vbd_settings {
    double dt;
    uint32_t iterations;
    uint32_t init_mode;              /* cc_init_mode                        */
    double damping;
    double gravity[3];
    cc_ogc_settings contact;
    double residual_tolerance;       /* 0 = run all `iterations`            */
    uint32_t residual_check_every;   /* 0 = no relative residual            */
    uint32_t stall_refresh;          /* 0 = off                             */
    double acceleration;             /* Chebyshev rho in [0, 1); 0 = off     */
    uint32_t sweep_precision;        /* cc_sweep_precision                  */
    uint32_t reserved1;              /* must be 0                           */
} cc_vbd_settings;

/* Grab (src/vbd.rs:54-60): mouse attachment, weights sum to one. */
typedef struct cc_grab {
    uint32_t vertices[3];
    uint32_t reserved0;
    double weights[3];
    double target[3];
    double stiffness;
} cc_grab;

/* VbdMetrics (src/vbd.rs:61-83) with DetectionProfile (src/ogc/world.rs:14-22). */
typedef struct cc_metrics {
    double time_s, dt_s, step_ms, detection_ms, solve_ms;
    double gpu_compute_ms;          /* device time of the step, CUDA events   */
    double refit_ms, candidates_ms, narrow_ms; /* device time of the detection
                                      phases (profiling on; narrow includes the
                                      canonical sort, incidence and radii)    */
    uint64_t candidate_pairs, aabb_rejections;
    uint64_t iterations, contacts, contact_terms;
    uint64_t detection_updates, broad_phase_rebuilds, truncated_vertices;
    uint64_t colors;                /* colours of the last sweep              */
    double minimum_distance_m, max_seam_gap_m;
    double extension_p95_percent, extension_max_percent;
    double residual_rms_n;
    int32_t has_residual;           /* 1 when residual_rms_n is defined       */
    int32_t reserved0;
    /* device-side accounting of the step (no reference counterpart) */
    double sweep_ms;                /* colour-sweep kernel time (profiling on) */
    uint64_t sweep_launches;        /* colour-sweep kernel launches           */
    uint64_t vertex_solves;         /* local solves: free vertices x sweeps   */
    uint64_t kernel_launches;       /* launches of this library's kernels     */
    uint64_t contact_incidence;     /* entries of the last contact incidence  */
    double color_ms;                /* host time spent colouring              */
    uint64_t color_rounds;          /* greedy-rule rounds of the colourings   */
    /* relative residual (see cc_vbd_settings) after the last iteration and
     * of the initial guess; defined when has_relative_residual = 1 */
    double relative_residual;
    double initial_relative_residual;
    int32_t has_relative_residual;
    int32_t init_used;              /* cc_init_mode the sweeps started from   */
    double init_energy_adaptive;    /* step energy of the adaptive guess and  */
    double init_energy_learned;     /* of the full-scale learned guess        */
                                    /* (learned mode; NaN otherwise)          */
    double init_ms;                 /* device time of the learned guess       */
    /* the plain force norm ||grad E(x)|| / ||grad E(y)|| after the last
     * iteration (no projection P; the same E, y and OGC terms as
     * relative_residual), defined when has_relative_residual = 1 */
    double relative_force_residual;
} cc_metrics;

/* ContactSet (src/ogc/world.rs:73-107) in caller-owned arrays. The contact
 * list is in canonical order: sorted by (kind, vertices), deduplicated. If a
 * capacity is too small the call returns CC_ERR_CAPACITY and fills the
 * n_contacts / n_incident / n_vf_pairs / n_ee_pairs it needs. */
typedef struct cc_contacts {
    /* capacities (in) */
    uint64_t contact_capacity;
    uint64_t incident_capacity;
    uint64_t radii_capacity;          /* >= number of moving vertices */
    /* arrays (out; may be NULL when the matching capacity is 0) */
    uint8_t* kinds;                   /* 0 PointPoint, 1 PointEdge, 2 PointFace, 3 EdgeEdge */
    uint32_t* vertices;               /* [contact][4] */
    uint8_t* counts;
    double* mollifier_epsilon;
    uint64_t* incident_offsets;       /* [moving + 1] */
    uint32_t* incident;               /* contact ids per moving vertex, ascending */
    double* radii;                    /* [moving] */
    /* scalars (out) */
    uint64_t n_contacts;
    uint64_t n_incident;
    uint64_t active_contacts;
    uint64_t vertex_face_candidates;
    uint64_t edge_edge_candidates;
    uint64_t candidate_pairs;
    uint64_t aabb_rejections;
    double minimum_distance;
    int32_t broad_phase_rebuilt;
    int32_t reserved0;
} cc_contacts;

/* Candidate pairs of a fresh broad phase (Candidates::build,
 * src/ogc/candidates.rs:23-68), sorted ascending, for list parity tests. */
typedef struct cc_candidates {
    uint64_t vf_capacity, ee_capacity;
    uint32_t* vf;                     /* [pair][2]: point, triangle */
    uint32_t* ee;                     /* [pair][2]: edge, edge (operand order of the reference) */
    uint64_t n_vf, n_ee;
} cc_candidates;

typedef struct cc_solver cc_solver;
typedef struct cc_world cc_world;

/* ---------------------------------------------------------------- library */
int32_t cc_abi_version(void);
/* Message of the last failure that had no handle (creation). */
int32_t cc_global_last_error(char* buffer, uint64_t length);
/* Message of the last failure on a handle; returns its status. */
int32_t cc_last_error(const cc_solver* solver, char* buffer, uint64_t length);
int32_t cc_world_last_error(const cc_world* world, char* buffer, uint64_t length);
/* Device the library runs on (default 0); call before creating handles. */
int32_t cc_set_device(int32_t device);

/* ----------------------------------------------------------------- solver */
/* VbdSolver::new (src/vbd.rs:101-192): checks dimensions and pins, appends
 * the obstacle, builds stitches and exclusions, OgcWorld::new and
 * validate_start, incidence and the material graph. x0/v0: [n][3]. */
int32_t cc_solver_create(const cc_mesh* mesh, const cc_surface* obstacle,
                         const double* x0, const double* v0, uint64_t n,
                         cc_solver** out);
void cc_solver_destroy(cc_solver* solver);

/* VbdSolver::step (src/vbd.rs:250-422) with GpuVbd::step's slot
 * (src/gpu_vbd.rs:125-131): x, v ([n][3]) and *time are read, and written
 * only on CC_OK. grab may be NULL. metrics may be NULL. */
int32_t cc_solver_step(cc_solver* solver, double* x, double* v, double* time,
                       const cc_vbd_settings* settings, const cc_grab* grab,
                       cc_metrics* metrics);

/* Device-resident stepping: the state stays in HBM between calls.
 * set_state uploads x, v, time; step_resident advances it; get_state reads
 * it back. Same semantics as cc_solver_step otherwise. */
int32_t cc_solver_set_state(cc_solver* solver, const double* x, const double* v, double time);
int32_t cc_solver_get_state(cc_solver* solver, double* x, double* v, double* time);
int32_t cc_solver_step_resident(cc_solver* solver, const cc_vbd_settings* settings,
                                const cc_grab* grab, cc_metrics* metrics);

/* Number of cloth (moving) vertices and of all vertices including the obstacle. */
uint64_t cc_solver_moving(const cc_solver* solver);
uint64_t cc_solver_total(const cc_solver* solver);

/* The CUDA stream (cudaStream_t) every kernel of this solver is launched on,
 * for callers that time the step with CUDA events. No reference counterpart
 * (the wgpu backend times its compute pass with timestamp queries,
 * src/gpu_vbd/cache.rs:16-33). */
void* cc_solver_stream(const cc_solver* solver);
/* When enabled, each chunk of iterations the step enqueues ahead of the
 * device (all iterations without a residual target; max(check_every, 4)
 * with one) is captured into a CUDA graph and launched as one, except the
 * first iteration after each detection, which is launched directly so that
 * the device works while the rest of its chunk is captured. Executable
 * graphs are kept per chunk shape (colour count, placement of the residual
 * checks) and updated in place while the shape recurs.
 * Results are bitwise those of direct launches. On by default (0 launches
 * every kernel directly). Profiling adds no node to the graphs (the sweep
 * kernels stamp their own span). No reference counterpart (the wgpu
 * backend records one dispatch per colour per iteration,
 * src/gpu_vbd.rs:398-404). */
int32_t cc_solver_set_graphs(cc_solver* solver, int32_t enable);
/* When enabled, each iteration's colour sweeps (launched back to back) record
 * their span on the device clock (%globaltimer): the first colour's blocks
 * lower a start stamp to their start times, the last colour's blocks raise an
 * end stamp to their end times, one atomic per block; cc_metrics.sweep_ms
 * reports the summed spans over the iterations the step ran. No event or
 * extra launch is added between the sweeps, so the stepping is timed as it
 * runs unprofiled. Detection phases and the learned guess are timed with
 * CUDA events on the solver stream. */
int32_t cc_solver_set_profiling(cc_solver* solver, int32_t enable);
/* Threads that cooperate on one vertex's local solve (1, 2, 4, 8, 16 or 32),
 * optionally | (cap << 8) with cap = 3, 4, 5, 6 or 8 resident 128-thread
 * blocks per SM (a register budget; default 3; above 3 registers spill to
 * local memory), | (1 << 16) for a persistent grid (at most the resident
 * blocks, each looping over the colour's vertices), | (1 << 17) or (2 << 17)
 * for blocks of 64 or 256 threads (4 or 8 lanes; caps 3-4 or 4, 6, 8) at the
 * same register budget; 0 (the default) lets the solver time the
 * candidates on its first step and keep the fastest. get_lanes returns the
 * same encoding. Two solvers take bitwise-identical steps only with the same
 * setting. No reference counterpart (the wgpu backend always uses a 32-lane
 * workgroup per vertex, src/vbd.wgsl:118-150). */
int32_t cc_solver_set_lanes(cc_solver* solver, int32_t lanes);
int32_t cc_solver_get_lanes(const cc_solver* solver);
/* The same for the CC_SWEEP_FP32 sweep: lanes 4, 8, 16 or 32, optionally
 * | (cap << 8) with cap = 3, 4, 5, 6 or 8, the persistent bit and the block
 * size (64 or 256 threads for 8 or 16 lanes); 0 (the default) autotunes on
 * the first FP32 step. */
int32_t cc_solver_set_lanes32(cc_solver* solver, int32_t lanes);
int32_t cc_solver_get_lanes32(const cc_solver* solver);

/* The solver's OGC world (owned by the solver; do not destroy). */
cc_world* cc_solver_world(cc_solver* solver);

/* Colouring (coloring::colors, src/vbd/coloring.rs:5-43) of the material
 * graph plus a contact set detected at x_all, plus an optional grab.
 * colors_out: [moving] colour per vertex; *n_colors: number of colours. */
int32_t cc_solver_colors(cc_solver* solver, const double* x_all, double query_radius,
                         const cc_ogc_settings* settings, const cc_grab* grab,
                         uint32_t* colors_out, uint32_t* n_colors);

/* Local block of every moving vertex at positions x_all with the contact set
 * detected at x_all (VbdSolver::local with Jet<3>, src/vbd.rs:196-248, plus
 * the inertia of the step, src/vbd.rs:353-356; the GPU probe of
 * src/vbd.wgsl:142-147). targets/inertia: [moving][3] / [moving] or NULL for
 * no inertia. energy [moving], gradient [moving][3], hessian [moving][9]. */
int32_t cc_solver_local_blocks(cc_solver* solver, const double* x_all,
                               double query_radius, const cc_vbd_settings* settings,
                               const cc_grab* grab, const double* targets,
                               const double* inertia, double* energy,
                               double* gradient, double* hessian);

/* FP64 Newton reference step on the GPU, for residual and error references at
 * scale (ReferenceSolver::step_problem, src/solver.rs:422-646: Newton on the
 * implicit-Euler objective, Jacobi-preconditioned CG with shift escalation,
 * Armijo backtracking, stop at RMS gradient <= max(abs_tol, rel_tol r0)).
 * The reference's Newton solver has no OGC term; here the step's contact set,
 * detected at x_old with the step's query radius, enters frozen with
 * Contact::energy (src/ogc/potential.rs:39-65). Hessian-vector products are
 * central differences of the exact FP64 gradient (largest displacement
 * 1e-7 m) instead of assembled element Hessians. x_old, v_old: [n][3] in;
 * x_out: [n][3] out. The solver's own state and history are not changed. */
typedef struct cc_newton_report {
    int32_t converged;
    uint32_t iterations;             /* Newton iterations run                */
    uint64_t pcg_iterations;         /* CG iterations over all solves        */
    double residual_rms_n;           /* RMS gradient over free dofs at x_out */
    double objective_j;              /* step objective at x_out              */
    double relative_force_residual;  /* ||grad E(x_out)|| / ||grad E(y)||   */
    uint64_t contact_terms;          /* frozen OGC contact terms             */
} cc_newton_report;
int32_t cc_solver_newton_step(cc_solver* solver, const double* x_old, const double* v_old,
                              const cc_vbd_settings* settings, uint32_t newton_iterations,
                              uint32_t pcg_iterations, double abs_tol, double rel_tol, double* x_out,
                              cc_newton_report* report);

/* ------------------------------------------------------------------ world */
/* OgcWorld::new (src/ogc/world.rs:126-211). x: [n_all][3]; vertices >= moving
 * are fixed. excluded: [n_excluded][2] vertex pairs never in contact. */
int32_t cc_world_create(const double* x, uint64_t n_all, const uint32_t* triangles,
                        uint64_t n_triangles, uint64_t moving,
                        const uint32_t* excluded, uint64_t n_excluded, cc_world** out);
void cc_world_destroy(cc_world* world);
/* OgcWorld::validate_start (src/ogc/world.rs:242-307). */
int32_t cc_world_validate_start(cc_world* world, const double* x);
/* OgcWorld::detect (src/ogc/world.rs:308-420), candidate cache included. */
int32_t cc_world_detect(cc_world* world, const double* x, double query_radius,
                        const cc_ogc_settings* settings, cc_contacts* out);
/* Fresh broad phase at search radius `radius` (no cache), sorted lists. */
int32_t cc_world_candidates(cc_world* world, const double* x, double radius,
                            cc_candidates* out);
/* Topology sizes: edges of the combined mesh (src/ogc/topology.rs:13-52). */
uint64_t cc_world_edges(const cc_world* world, uint32_t* edges_out);
/* LBVH policy of the moving triangle and edge trees at a candidate rebuild:
 * 0 (the default) builds each tree once, from the Morton codes of the first
 * rebuild's boxes, and refits it at every later rebuild, as the reference
 * keeps its median-split tree and refits it (src/ogc/bvh.rs:66-242);
 * k >= 1 builds the trees again at every k-th rebuild and refits in between.
 * The candidate pair sets do not depend on it (every primitive's box is
 * inside its ancestors' boxes whatever the topology); only the traversal
 * cost does. For a solver, pass cc_solver_world(solver). */
int32_t cc_world_set_tree_rebuild_period(cc_world* world, int32_t period);

/* -------------------------------------------------- batched instances */
/* Many independent cloths stepped as one solver (no reference counterpart;
 * the reference steps one garment per VbdSolver): meshes[k], obstacles[k]
 * (entries with n_vertices = 0 have none; obstacles may be NULL), x0[k], v0[k]
 * ([n_k][3]; v0 or v0[k] may be NULL for rest) are concatenated in order.
 * One colour sweep covers every instance, one detection all of them; the
 * union's colouring equals each instance's own. The step's query radius and
 * refresh rule are taken over the whole batch. Instances must be placed so
 * that none comes within the contact query radius of another. The handle is
 * a cc_solver: step it, read and write its state (vertices in instance
 * order) and destroy it with the cc_solver_* calls. */
int32_t cc_batch_create(const cc_mesh* meshes, const cc_surface* obstacles,
                        const double* const* x0, const double* const* v0, uint64_t count,
                        cc_solver** out);
/* Instance table: first vertex and vertex count of each instance (up to
 * `capacity` entries written); returns the number of instances (0 for a
 * solver made by cc_solver_create). */
uint64_t cc_batch_instances(const cc_solver* solver, uint64_t* first_vertex, uint64_t* vertex_count,
                            uint64_t capacity);
/* ------------------------------------------------------ learned guess */
/* No reference counterpart. A 24-64-64-64-3 GELU MLP predicts, per free
 * vertex, a correction of the adaptive guess from 24 features of the step
 * start (inertial and previous displacement, neighbourhood, local strain,
 * nearest-contact distance). With init_mode = CC_INIT_LEARNED the solver
 * forms guess + a * correction for a = 1, 1/2, 1/4, clips each to the OGC
 * balls (ContactSet::truncate, src/ogc/world.rs:91-100) and starts from the
 * one with the lowest step energy if that is lower than the adaptive guess's
 * energy, else from the adaptive guess; cc_metrics.init_used says which.
 *
 * Arrays marked (device) are device pointers; the calls synchronise their
 * own stream before returning and expect the buffers to be ready. */
typedef struct cc_mlp cc_mlp;
/* New network, Glorot-uniform weights from `seed`, zero biases. */
int32_t cc_mlp_create(uint64_t seed, cc_mlp** out);
void cc_mlp_destroy(cc_mlp* mlp);
int32_t cc_mlp_last_error(const cc_mlp* mlp, char* buffer, uint64_t length);
/* Parameters (float32, host): W1[64][24] b1[64] W2[64][64] b2[64] W3[64][64]
 * b3[64] W4[3][64] b4[3], W[out][in]; count = cc_mlp_parameter_count(). */
uint64_t cc_mlp_parameter_count(void);
int32_t cc_mlp_set_parameters(cc_mlp* mlp, const float* params, uint64_t count);
int32_t cc_mlp_get_parameters(cc_mlp* mlp, float* params, uint64_t count);
/* out (device) [n][3] = MLP(features (device) [n][24]); precision 0 = FP32
 * CUDA cores, 1 = FP16 operands / FP32 accumulation on the tensor cores. */
int32_t cc_mlp_forward(cc_mlp* mlp, const float* features, uint64_t n, float* out, int32_t precision);
/* Gradient (host, [count]) and value (host) of the loss
 * L = (1/n) sum_s |MLP(features_s) - targets_s|^2 (device inputs). */
int32_t cc_mlp_gradients(cc_mlp* mlp, const float* features, const float* targets, uint64_t n,
                         float* grads, float* loss);
/* `steps` Adam steps (beta 0.9/0.999, eps 1e-8) on minibatches of `batch`
 * samples drawn without replacement per epoch (seeded shuffle); losses
 * (host, [steps], may be NULL) receives each minibatch's loss. */
int32_t cc_mlp_train(cc_mlp* mlp, const float* features, const float* targets, uint64_t n,
                     uint32_t batch, uint32_t steps, float learning_rate, uint64_t seed, float* losses);
/* Attach a network to a solver (not owned; NULL detaches). precision as in
 * cc_mlp_forward. */
int32_t cc_solver_set_mlp(cc_solver* solver, cc_mlp* mlp, int32_t precision);
/* Per-iteration record of the last step (no reference counterpart), for
 * convergence studies: relative residual after each iteration (NaN where it
 * was not evaluated) and vertices clipped to their OGC balls in it; entries
 * up to min(capacity, 256). */
int32_t cc_solver_last_step_trace(const cc_solver* solver, double* relative_residual,
                                  uint32_t* clipped, uint32_t capacity);
/* Rows of the training arrays: the solver's free (unpinned) vertices. */
uint64_t cc_solver_free_vertices(const cc_solver* solver);
/* cc_solver_step_resident that also writes one training sample per free
 * vertex, in vertex order: features (device) [rows][24] of the step start and
 * targets (device) [rows][3] = (x_end - adaptive guess) / (|g| dt^2), the
 * correction the network should have predicted for this step's result. */
int32_t cc_solver_step_sample(cc_solver* solver, const cc_vbd_settings* settings,
                              const cc_grab* grab, float* features, float* targets,
                              cc_metrics* metrics);
/* ------------------------------------------------------- allocation-free */
/* No counterpart in the reference. Per-vertex OGC distances and conservative
 * radii for given candidate pairs, without allocating any memory, for callers
 * that cannot call cudaMalloc: a fixed-budget frame worker for which an
 * allocation (and the device-wide synchronisation cudaFree implies) would
 * stall the frame, or a host that reserves all device memory at start-up and
 * passes this library only its own buffers.
 *
 * ALL pointers are device pointers: x [n_all][3]; triangles [n_triangles][3];
 * edges [n_edges][2] (as cc_world_edges returns them); vf_pairs [n_vf][2]
 * (point, triangle) and ee_pairs [n_ee][2] (edge, edge), e.g. the lists of
 * cc_world_candidates at a search radius >= query_radius; outputs radii
 * [moving] and *minimum_distance. Results equal the radii and minimum
 * distance of cc_world_detect for the same positions and query radius.
 *
 * The per-vertex scratch is a static device array of 262,144 vertex slots
 * (2 MiB, held by every GPU that loads the library until exit); larger
 * n_all is rejected with CC_ERR_INVALID_ARGUMENT and a message. Kernels run
 * on `stream` (a cudaStream_t; NULL = legacy default stream) and the call
 * returns after they finish. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture. All calls share the one
 * array, so calls whose kernels overlap on the GPU race. Calls from several
 * host threads of one process are serialised inside the library (a mutex
 * held from the first launch until the call's kernels have finished). */
int32_t cc_ogc_radii_noalloc(const double* x, uint64_t n_all, uint64_t moving, const uint32_t* triangles,
                             uint64_t n_triangles, const uint32_t* edges, uint64_t n_edges,
                             const uint32_t* vf_pairs, uint64_t n_vf, const uint32_t* ee_pairs, uint64_t n_ee,
                             double query_radius, double relaxation, double* radii, double* minimum_distance,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CLOTHCRAFT_H */
