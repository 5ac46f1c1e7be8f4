// VbdSolver on the device and the C ABI of include/clothcraft.h.
//
// The step (VbdSolver::step, src/vbd.rs:250-422) runs entirely on the GPU:
// adaptive initial guess, inertial target, OGC detection, colouring, clipped
// warm start, colour sweeps with refresh detections, final feasibility and
// trust-region checks, commit and history record. The host only sequences
// kernels and reads a few scalars between phases.
#include <chrono>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <set>

#include "color.cuh"
#include "learned.cuh"
#include "sweep.cuh"
#include "newton.cuh"
#include "world.cuh"

using namespace cc;

namespace {
std::mutex g_mutex;
std::string g_error;
int g_code = 0;
int g_device = 0;

int set_global(int code, const std::string& m) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_error = m;
    g_code = code;
    return code;
}
void copy_msg(const std::string& m, char* buf, uint64_t len) {
    if (buf && len) {
        size_t k = std::min<size_t>(m.size(), len - 1);
        std::memcpy(buf, m.data(), k);
        buf[k] = 0;
    }
}
double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}
bool ogc_valid(const cc_ogc_settings& s) {  // src/ogc/world.rs:56-70
    return std::isfinite(s.radius) && s.radius > 0.0 && std::isfinite(s.stiffness) && s.stiffness > 0.0 &&
           std::isfinite(s.relaxation) && s.relaxation > 0.0 && s.relaxation < 0.5 &&
           std::isfinite(s.refresh_fraction) && s.refresh_fraction >= 0.0 && s.refresh_fraction <= 1.0;
}
bool vbd_valid(const cc_vbd_settings& s) {  // src/vbd.rs:38-51
    return ogc_valid(s.contact) && std::isfinite(s.dt) && s.dt >= 1e-6 && s.dt <= 0.025 && s.iterations != 0 &&
           s.iterations <= 200 && std::isfinite(s.damping) && s.damping >= 0.0 && std::isfinite(s.gravity[0]) &&
           std::isfinite(s.gravity[1]) && std::isfinite(s.gravity[2]) && std::isfinite(s.acceleration) &&
           s.acceleration >= 0.0 && s.acceleration < 1.0 &&
           (s.sweep_precision == CC_SWEEP_FP64 || s.sweep_precision == CC_SWEEP_FP32) && s.reserved1 == 0;
}
}  // namespace

// --------------------------------------------------------------- kernels
namespace cc {

int record_global_error(int code, const std::string& message) { return set_global(code, message); }

struct StepScalars {
    unsigned int error;
    unsigned int mismatch;
    unsigned int clipped;
    unsigned int acc_k;         // Chebyshev: iterations since the sequence's (re)start
    double acc_w;               // Chebyshev weight of the current iteration
    double acc_g2;              // Chebyshev: residual of the previous evaluation
    unsigned int refresh_at;    // first iteration whose start needs a refresh detection
    unsigned int converged_at;  // iterations run when the residual target was met
    unsigned int stop_at;       // min(refresh_at, converged_at): later sweeps exit at once
    unsigned int checked_at;    // iterations run at the last residual evaluation
    unsigned int clipped_alt;   // clipped vertices of the learned guess
    unsigned int clipped_iter[256];
    unsigned long long motion_bits;
    unsigned long long seam_gap_bits;
    double residual;
    double ext_total;
    double gy2;        // |grad E(y)|^2, y the inertial target
    double gx2;        // |grad E(x)|^2 at the last evaluation
    double gx2_init;   // |grad E|^2 of the initial guess
    double gx2_plain;  // |grad E(x)|^2 after the last iteration, unprojected
    double e_init[2];  // step energy of the adaptive / full-scale learned guess
    int init_used;
    double gx2_iter[256];   // |P grad E(x)|^2 after iteration it (evaluated ones)
    double stall_best;      // lowest |P grad E|^2 since the last detection (stall refresh)
    unsigned int stall_count;
    double e_cand, best_e;  // learned-guess scale search
    unsigned int clipped_best;
    int take;
    unsigned long long p95_bits, ext_max_bits;  // extension metric keys of the step's end
};

__global__ void k_step_begin(uint32_t n, const double4* x0, const double4* v0, const double4* px, const double4* pv,
                             int has_pred, StepScalars* sc) {
    unsigned int err = 0, mis = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double4 a = x0[i], b = v0[i];
        if (!(isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(b.x) && isfinite(b.y) && isfinite(b.z)))
            err = 1;
        if (has_pred) {
            double4 c = px[i], d = pv[i];
            if (!(a.x == c.x && a.y == c.y && a.z == c.z && b.x == d.x && b.y == d.y && b.z == d.z)) mis = 1;
        }
    }
    if (err) atomicOr(&sc->error, DERR_NONFINITE_STATE);
    if (mis) atomicOr(&sc->mismatch, 1u);
}

// Prediction::guess (src/vbd/prediction.rs:15-41), target and inertia
// (src/vbd.rs:283-302).
__global__ void k_predict(uint32_t n, const double4* x0, const double4* v0, const double4* accel, int history_ok,
                          const StepScalars* sc_in, double dt, double3 g, double damping, const double* masses,
                          double4* guess, double4* target, double* inertia, StepScalars* sc) {
    bool valid = history_ok && sc_in->mismatch == 0;
    double g2 = g.x * g.x + g.y * g.y + g.z * g.z;
    double damp = 1.0 + damping * dt;
    double dt2 = dt * dt;
    double mx = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d3 x = ld3(x0, i), v = ld3(v0, i);
        double factor = 1.0;
        if (valid && g2 > 1e-20) {
            d3 a = ld3(accel, i);
            double f = (a.x * g.x + a.y * g.y + a.z * g.z) / g2;
            factor = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
        }
        d3 gv = mk(g.x, g.y, g.z);
        st3(guess, i, x + (v * dt + gv * factor * dt2) / damp);
        d3 t = x + (v * dt + gv * dt * dt) / damp;
        st3(target, i, t);
        inertia[i] = masses[i] * damp / dt2;
        mx = fmax(mx, len(t - x));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&sc->motion_bits, dbits(mx));
}

__global__ void k_copy_positions(uint32_t n, const double4* src, double4* dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

// Lanes per vertex of the residual evaluation (k_grad_sq, one launch over all
// vertices): 4 is the fastest measured on the fold (36 us per launch against 50
// with 8), whatever the sweep's variant; the residual's value does not depend on it
// beyond the last bits of its sums.
constexpr int kResidualLanes = 4;

// Chebyshev step after iteration `it` (no reference counterpart):
// x = w (x_sweep - x_prev2) + x_prev2 on free vertices, clipped to the OGC
// ball, from the second iteration of a sequence on (acc_k >= 2); `hist`
// holds x_prev2 on entry and the new x on exit (it becomes the previous
// iterate of the next call).
__global__ void k_accelerate(uint32_t n, const uint8_t* pinned, ContactsView c, double4* x, double4* hist,
                             const StepScalars* sc, uint32_t it) {
    if (sc->stop_at <= it) return;  // this iteration was skipped
    const bool extrapolate = sc->acc_k >= 2;
    const double w = sc->acc_w;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d3 p = ld3(x, i);
        if (extrapolate && !pinned[i]) {
            d3 q = ld3(hist, i);
            p = mk(__fma_rn(w, p.x - q.x, q.x), __fma_rn(w, p.y - q.y, q.y), __fma_rn(w, p.z - q.z, q.z));
            d3 ctr = ld3(c.centers, i);
            d3 d = p - ctr;
            double l = len(d);
            double b = c.radii[i];
            if (l > b) p = ctr + d * (b / l);
            st3(x, i, p);
        }
        st3(hist, i, p);
    }
}

// The caller's x and v ([n][3] doubles) are copied as they are, straight from
// or into the caller's memory (DMA when it is pinned), and converted to and
// from the padded device layout on the GPU.
__global__ void k_unpack_state(uint32_t n, const double* io, double4* x, double4* v) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double* a = io + 3 * (size_t)i;
        const double* b = io + 3 * ((size_t)n + i);
        x[i] = make_double4(a[0], a[1], a[2], 0.0);
        v[i] = make_double4(b[0], b[1], b[2], 0.0);
    }
}

__global__ void k_pack_state(uint32_t n, const double4* x, const double4* v, double* io) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double4 a = x[i], b = v[i];
        double* p = io + 3 * (size_t)i;
        double* q = io + 3 * ((size_t)n + i);
        p[0] = a.x;
        p[1] = a.y;
        p[2] = a.z;
        q[0] = b.x;
        q[1] = b.y;
        q[2] = b.z;
    }
}

void launch_unpack_state(size_t n, const double* io, double4* x, double4* v, cudaStream_t st) {
    k_unpack_state<<<grid_for(n, 256), 256, 0, st>>>((uint32_t)n, io, x, v);
    CC_CUDA(cudaGetLastError());
}

void launch_pack_state(size_t n, const double4* x, const double4* v, double* io, cudaStream_t st) {
    k_pack_state<<<grid_for(n, 256), 256, 0, st>>>((uint32_t)n, x, v, io);
    CC_CUDA(cudaGetLastError());
}

// Conservative warm start (src/vbd.rs:316-324)
__global__ void k_warm_start(uint32_t n, const uint8_t* pinned, const double4* guess, ContactsView c, double4* x,
                             unsigned int* clipped) {
    unsigned int cnt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (pinned[i]) continue;
        d3 p = ld3(guess, i);
        d3 ctr = ld3(c.centers, i);
        d3 d = p - ctr;
        double l = len(d);
        double b = c.radii[i];
        if (l > b) {
            p = ctr + d * (b / l);
            ++cnt;
        }
        st3(x, i, p);
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(clipped, cnt);
}

// Refresh rule after iteration `it` (src/vbd.rs:326): the next iteration
// starts with a new detection when at least refresh_fraction * n vertices
// were clipped. Later sweeps already enqueued see refresh_at and skip.
// With acceleration (rho2 = rho^2 > 0) it also advances the Chebyshev
// sequence (Wang 2015, "A Chebyshev semi-iterative approach for accelerating
// projective and position-based dynamics"): w1 = 1, w2 = 2/(2 - rho^2),
// wk = 4/(4 - rho^2 w(k-1)), rounded operation by operation as on the CPU.
__global__ void k_refresh_rule(StepScalars* sc, uint32_t it, uint32_t iterations, double threshold, double rho2) {
    if (sc->stop_at <= it) return;  // this iteration was skipped
    if (rho2 > 0.0) {
        unsigned int k = ++sc->acc_k;
        double w = 1.0;
        if (k == 2) w = __ddiv_rn(2.0, __dsub_rn(2.0, rho2));
        else if (k > 2) w = __ddiv_rn(4.0, __dsub_rn(4.0, __dmul_rn(rho2, sc->acc_w)));
        sc->acc_w = w;
    }
    unsigned int c = sc->clipped_iter[it];
    if (c > 0 && (double)c >= threshold && it + 1 < iterations) {
        sc->refresh_at = it + 1;
        sc->stop_at = min(sc->stop_at, it + 1);
    }
}

// Relative-residual rule after iteration `it`: |grad E(x)|^2 from the
// partial sums; with a target, iterations stop at the first evaluation with
// |grad E(x)| <= tol |grad E(y)|. No reference counterpart (the reference
// always runs `iterations` sweeps).
// With `stall` = k > 0, k evaluations in a row without a 5 % decrease of the
// residual, while vertices are being clipped, request a refresh detection
// before the next iteration (new OGC balls around the current positions).
// With acceleration, an evaluation above the previous one restarts the
// Chebyshev sequence (the next iteration is a plain sweep again).
__global__ void __launch_bounds__(256) k_residual_rule(StepScalars* sc, const double* partial, uint32_t it,
                                                       uint32_t iterations, double tol2, int stop, uint32_t stall,
                                                       int accelerate) {
    if (sc->stop_at <= it) return;  // uniform: every thread reads it before thread 0 writes
    double g2 = block_sum_partials(partial);
    if (threadIdx.x == 0) {
        sc->gx2 = g2;
        sc->gx2_iter[it] = g2;
        sc->checked_at = it + 1;
        if (accelerate) {
            if (g2 > sc->acc_g2) sc->acc_k = 0;
            sc->acc_g2 = g2;
        }
        if (stop && g2 <= tol2 * sc->gy2 && sc->converged_at > it + 1) {
            sc->converged_at = it + 1;
            if (it + 1 < iterations) sc->stop_at = min(sc->stop_at, it + 1);
        } else if (stop && stall) {
            if (g2 < 0.9025 * sc->stall_best) {
                sc->stall_best = g2;
                sc->stall_count = 0;
            } else if (++sc->stall_count >= stall && sc->clipped_iter[it] > 0 && it + 1 < iterations) {
                sc->refresh_at = min(sc->refresh_at, it + 1);
                sc->stop_at = min(sc->stop_at, it + 1);
            }
        }
    }
}

// Sum of the partials into *out (one block of 256 threads).
__global__ void __launch_bounds__(256) k_store_sum(const double* partial, double* out) {
    double v = block_sum_partials(partial);
    if (threadIdx.x == 0) *out = v;
}

// Scale search of the learned guess: keep the candidate if its energy is
// lower than the best so far (the adaptive guess's to begin with).
__global__ void k_decide_guess(StepScalars* sc) {
    sc->take = sc->e_cand < sc->best_e ? 1 : 0;
    if (sc->take) {
        sc->best_e = sc->e_cand;
        sc->clipped_best = sc->clipped_alt;
        sc->init_used = 1;
    }
}
__global__ void k_take_guess(uint32_t n, const double4* alt, double4* best, const StepScalars* sc) {
    if (!sc->take) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) best[i] = alt[i];
}
__global__ void k_commit_guess(uint32_t n, const double4* best, double4* x, StepScalars* sc) {
    if (!sc->init_used) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = best[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->clipped = sc->clipped_best;
}

// finite result and trust-region invariant (src/vbd.rs:399-405), residual sum
__global__ void k_step_finish(uint32_t n, const double4* x, ContactsView c, const double* residual, StepScalars* sc) {
    unsigned int err = 0;
    double r = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d3 p = ld3(x, i);
        if (!isfin(p)) err |= DERR_NONFINITE_RESULT;
        else if (len(p - ld3(c.centers, i)) > c.radii[i] + 1e-10) err |= DERR_TRUST_REGION;
        r += residual[i];
    }
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sc->residual, r);
    if (err) atomicOr(&sc->error, err);
}

// commit + Prediction::record (src/vbd.rs:406-411, prediction.rs:43-54)
__global__ void k_commit(uint32_t n, const double4* x, double4* x0, double4* v0, double4* px, double4* pv,
                         double4* accel, double dt, double damping, const double4* guess, double4* prev_corr) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d3 p = ld3(x, i), xo = ld3(x0, i), vo = ld3(v0, i);
        st3(prev_corr, i, p - ld3(guess, i));  // learned-guess feature of the next step
        d3 v = (p - xo) / dt;
        st3(x0, i, p);
        st3(v0, i, v);
        st3(px, i, p);
        st3(pv, i, v);
        st3(accel, i, (v - vo) / dt + v * damping);
    }
}

// extension_percent inputs (src/garment/diagnostics.rs:7-27) and seam gap
__global__ void k_stretch(uint32_t nt, const int4* tv, const double4* coef, const double* area, const double4* x,
                          unsigned long long* key, double* w) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        int4 v = tv[t];
        double4 cf = coef[t];
        d3 x0 = ld3(x, v.x), ds0 = ld3(x, v.y) - x0, ds1 = ld3(x, v.z) - x0;
        d3 ww = ds0 * cf.x + ds1 * cf.y;
        d3 vv = ds0 * cf.z + ds1 * cf.w;
        double st = fmax(len(ww), len(vv));
        double e = 100.0 * fmax(st - 1.0, 0.0);
        key[t] = order_key(e);
        w[t] = area[t];
    }
}

// extension P95 (the first sorted key whose cumulative area reaches 95 % of the
// total) and maximum, into the step scalars (read with the step's last sync)
__global__ void k_p95(uint32_t nt, const unsigned long long* key_sorted, const double* cum, StepScalars* sc) {
    const double total = cum[nt - 1];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        bool hit = cum[t] >= 0.95 * total && (t == 0 || !(cum[t - 1] >= 0.95 * total));
        if (hit) sc->p95_bits = key_sorted[t];
        if (t == nt - 1) sc->ext_max_bits = key_sorted[t];
    }
}

__global__ void k_seam_gap(uint32_t ns, const uint32_t* off, const uint32_t* sv, const double* sw, const double4* x,
                           StepScalars* sc) {
    double m = 0.0;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
        d3 d = mk(0, 0, 0);
        for (uint32_t k = off[s]; k < off[s + 1]; ++k) d = d + ld3(x, sv[k]) * sw[k];
        m = fmax(m, len(d));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&sc->seam_gap_bits, dbits(m));
}

}  // namespace cc

// ---------------------------------------------------------------- handles
struct cc_world {
    std::unique_ptr<World> own;
    World* w = nullptr;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    std::string err;
    int code = 0;
    int fail(const Failure& f) {
        err = f.message;
        code = f.code;
        return f.code;
    }
    ~cc_world() {
        own.reset();
        if (owns_stream && stream) cudaStreamDestroy(stream);
    }
};

struct cc_mlp {
    std::unique_ptr<Mlp> net;
    cudaStream_t stream = nullptr;
    DBuf<uint32_t> perm;
    DBuf<float> losses;
    std::string err;
    int code = 0;
    int fail(const Failure& f) {
        err = f.message;
        code = f.code;
        return f.code;
    }
    ~cc_mlp() {
        net.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

struct cc_solver {
    cudaStream_t stream = nullptr;
    uint32_t n = 0, n_all = 0, n_tri = 0, n_stitch = 0;
    std::unique_ptr<World> world;
    cc_world world_view;
    Coloring coloring;
    // static sweep data
    DBuf<int4> tri_v;
    DBuf<double4> tri_coef;
    DBuf<double> tri_area;
    DBuf<MatParams> mats;
    DBuf<MatParams32> mats32;
    DBuf<uint4> hinge_v;
    DBuf<double> hinge_k;
    DBuf<uint32_t> st_off, st_v;
    DBuf<double> st_w, st_k;
    DBuf<uint32_t> inc_off, inc, lo_off, lo;
    DBuf<uint2> inc_mid;  // per vertex: first hinge entry, first stitch entry
    DBuf<uint8_t> pinned;
    DBuf<double> masses;
    // state and per-step buffers
    DBuf<double4> x0, v0, guess, target, pred_x, pred_v, accel;
    DBuf<double> inertia, residual;
    DBuf<unsigned char> clipped_flag;
    DBuf<StepScalars> sc;
    Pinned<StepScalars> sc_h;
    Pinned<double4> stage;
    DBuf<double> io;  // [2][n][3] device copy of a caller's x and v (host layout)
    double time = 0.0;
    bool has_pred = false;
    double pred_time = 0.0, pred_damping = 0.0;
    double pred_g[3] = {0, 0, 0};
    // metrics scratch
    DBuf<unsigned long long> ext_key, ext_key_s;
    DBuf<double> ext_w, ext_w_s, ext_cum;
    RadixSorter ext_sorter;
    DBuf<double> ext_scan;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, tune0 = nullptr, tune1 = nullptr;
    bool profiling = false;
    // profiling: per-iteration sweep-span stamps (ns, %globaltimer) written by the
    // first and last colour's blocks; no event is recorded between the sweeps
    DBuf<unsigned long long> stamp_s, stamp_e;
    Pinned<unsigned long long> stamp_h;
    uint64_t own_launches = 0;
    uint32_t n_free = 0;
    int lanes = 0;          // vertices are solved by groups of `lanes` threads; 0 = autotune on next step
    int lanes32 = 0;        // the same for the FP32-assembly sweep
    DBuf<double4> x_backup;
    std::vector<double> tune_ms;
    // objective and relative residual
    uint32_t n_hinge = 0;
    DBuf<double4> alt;  // [n_all] second position array (fixed part = obstacle)
    DBuf<double> gsq, term_e, partial;
    Pinned<unsigned int> stop_h;  // two slots, one per chunk in flight
    cudaEvent_t chunk_ev[2] = {nullptr, nullptr};
    // learned initial guess
    cc_mlp* mlp = nullptr;  // attached, not owned
    int mlp_precision = 1;
    DBuf<uint32_t> ring_off, ring, row;
    double mean_mass = 1.0;
    DBuf<float> feat, corr;
    DBuf<double4> best, prev_corr;
    DBuf<double4> acc_a, acc_b;  // Chebyshev history: the last two iterates
    bool step_history = false;  // the adaptive-guess history test of the current step (host part)
    float* sample_features = nullptr;  // caller device buffers of cc_solver_step_sample
    float* sample_targets = nullptr;
    cudaEvent_t learn0 = nullptr, learn1 = nullptr;
    bool learn_timed = false;
    // Newton reference step (cc_solver_newton_step)
    DBuf<double4> nt_x0, nt_v0, nt_guess, nt_target, nt_y, nt_out;
    DBuf<double> nt_inertia;
    // batched instances (cc_batch_create): first vertex and count of each
    std::vector<uint64_t> inst_first, inst_count;
    std::string err;
    int code = 0;
    int fail(const Failure& f) {
        err = f.message;
        code = f.code;
        return f.code;
    }
    ~cc_solver() {
        world.reset();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (tune0) cudaEventDestroy(tune0);
        if (tune1) cudaEventDestroy(tune1);
        for (auto e : chunk_ev)
            if (e) cudaEventDestroy(e);
        if (learn0) cudaEventDestroy(learn0);
        if (learn1) cudaEventDestroy(learn1);
        for (auto& e : graph_cache)
            if (e.second) cudaGraphExecDestroy(e.second);
        if (stream) cudaStreamDestroy(stream);
    }

    SweepView sweep_view(const ContactsView& cv, const cc_vbd_settings& s, const cc_grab* grab) {
        SweepView v{};
        v.n = n;
        v.x = world->x();
        v.target = target.ptr;
        v.inertia = inertia.ptr;
        v.pinned = pinned.ptr;
        v.inc_off = inc_off.ptr;
        v.inc_mid = inc_mid.ptr;
        v.inc = inc.ptr;
        v.tri_v = tri_v.ptr;
        v.tri_coef = tri_coef.ptr;
        v.tri_area = tri_area.ptr;
        v.mats = mats.ptr;
        v.mats32 = mats32.ptr;
        v.hinge_v = hinge_v.ptr;
        v.hinge_k = hinge_k.ptr;
        v.st_off = st_off.ptr;
        v.st_v = st_v.ptr;
        v.st_w = st_w.ptr;
        v.st_k = st_k.ptr;
        v.contacts = cv;
        v.contact_r = s.contact.radius;
        v.contact_k = s.contact.stiffness;
        v.grab.active = grab ? 1 : 0;
        if (grab)
            for (int k = 0; k < 3; ++k) {
                v.grab.v[k] = grab->vertices[k];
                v.grab.w[k] = grab->weights[k];
                v.grab.target[k] = grab->target[k];
            }
        v.grab.k = grab ? grab->stiffness : 0.0;
        v.residual = residual.ptr;
        v.clipped = &sc.ptr->clipped;
        v.clipped_flag = clipped_flag.ptr;
        return v;
    }

    ColorView color_view(const ContactsView& cv, const cc_grab* grab) {
        ColorView c{};
        c.n = n;
        c.lo_off = lo_off.ptr;
        c.lo = lo.ptr;
        c.contacts = cv;
        c.grab_active = grab ? 1 : 0;
        if (grab)
            for (int k = 0; k < 3; ++k) c.grab_v[k] = grab->vertices[k];
        return c;
    }

    void read_scalars() {
        CC_CUDA(cudaMemcpyAsync(sc_h.ptr, sc.ptr, sizeof(StepScalars), cudaMemcpyDeviceToHost, stream));
        CC_CUDA(cudaStreamSynchronize(stream));
    }

    void detect(double rq, const cc_ogc_settings& s, cc_metrics* m, double& det_ms) {
        double t = now_ms();
        world->set_profiling(profiling);
        world->detect(rq, s.radius, s.relaxation, s.stiffness, false);
        det_ms += now_ms() - t;
        if (m && profiling) {
            const World::PhaseMs& p = world->last_phase_ms();
            m->refit_ms += p.refit;
            m->candidates_ms += p.candidates;
            m->narrow_ms += p.narrow + p.canonical;
        }
        if (m) {
            m->detection_updates += 1;
            m->broad_phase_rebuilds += world->stats().rebuild;
            m->candidate_pairs += world->stats().n_vf + world->stats().n_ee;
            m->aabb_rejections += world->stats().rejections;
        }
    }

    // CUDA-graph launch of the iteration chunks (cc_solver_set_graphs)
    bool graphs = true;
    // executable graphs by shape (node count): a batch's lead chunk and the
    // full chunks after it have different shapes, and each keeps its own
    // executable, updated in place while its shape holds
    std::vector<std::pair<size_t, cudaGraphExec_t>> graph_cache;
    static constexpr size_t kGraphCacheSize = 6;
    uint64_t graph_instantiations = 0, graph_updates = 0;
    void launch_captured_chunk() {
        cudaGraph_t g = nullptr;
        CC_CUDA(cudaStreamEndCapture(stream, &g));
        size_t nodes = 0;
        cudaError_t ce = cudaGraphGetNodes(g, nullptr, &nodes);
        if (ce != cudaSuccess) {
            cudaGraphDestroy(g);
            cuda_check(ce, "cudaGraphGetNodes");
        }
        cudaGraphExec_t* slot = nullptr;
        for (auto& e : graph_cache)
            if (e.first == nodes) slot = &e.second;
        bool updated = false;
        if (slot && *slot) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(*slot, g, &info) == cudaSuccess) {
                ++graph_updates;
                updated = true;
            } else {
                (void)cudaGetLastError();  // another topology with the same node count: not an error
                cudaGraphExecDestroy(*slot);
                *slot = nullptr;
            }
        }
        if (!updated) {
            if (!slot) {
                if (graph_cache.size() >= kGraphCacheSize) {  // drop the oldest shape
                    if (graph_cache.front().second) cudaGraphExecDestroy(graph_cache.front().second);
                    graph_cache.erase(graph_cache.begin());
                }
                graph_cache.push_back({nodes, nullptr});
                slot = &graph_cache.back().second;
            }
            cudaError_t e = cudaGraphInstantiate(slot, g, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                *slot = nullptr;
                cuda_check(e, "cudaGraphInstantiate");
            }
            ++graph_instantiations;
        }
        CC_CUDA(cudaGraphDestroy(g));
        CC_CUDA(cudaGraphLaunch(*slot, stream));
    }
    void step(const cc_vbd_settings& s, const cc_grab* grab, cc_metrics* out);
    void autotune(const SweepView& sv, bool fp32);
    std::map<int, unsigned> resident_;  // resident blocks of each variant's kernel (fp32 variants | 1 << 30)
    unsigned grid_cap(int variant, bool fp32) {
        if (!(variant & kVariantPersistent)) return 0;
        int key = variant | (fp32 ? 1 << 30 : 0);
        auto it = resident_.find(key);
        if (it != resident_.end()) return it->second;
        unsigned r = fp32 ? sweep32_resident_blocks(variant) : sweep_resident_blocks(variant);
        resident_[key] = r;
        return r;
    }
    void launch_variant(const SweepView& sv, const uint32_t* order, uint32_t count, int variant, bool fp32) {
        if (fp32) launch_sweep32(sv, order, count, variant, stream, grid_cap(variant, true));
        else launch_sweep(sv, order, count, variant, stream, grid_cap(variant, false));
    }
    void sweep(const SweepView& sv, const uint32_t* order, uint32_t count, bool fp32) {
        launch_variant(sv, order, count, fp32 ? lanes32 : lanes, fp32);
    }
    ObjectiveCounts counts() const {
        return ObjectiveCounts{n_tri, n_hinge, n_stitch, world->stats().n_contacts};
    }
    FeatureView feature_view(const ContactsView& cv, const cc_vbd_settings& s, double rq) {
        FeatureView f{};
        f.n = n;
        f.x0 = x0.ptr;
        f.v0 = v0.ptr;
        f.guess = guess.ptr;
        f.target = target.ptr;
        f.pinned = pinned.ptr;
        f.masses = masses.ptr;
        f.mean_mass = mean_mass;
        f.ring_off = ring_off.ptr;
        f.ring = ring.ptr;
        f.inc_off = inc_off.ptr;
        f.inc = inc.ptr;
        f.tri_v = tri_v.ptr;
        f.tri_coef = tri_coef.ptr;
        f.contacts = cv;
        f.query_radius = rq;
        f.relaxation = s.contact.relaxation;
        f.dt = s.dt;
        double g = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]);
        f.unit = g * s.dt * s.dt > 1e-9 ? g * s.dt * s.dt : 1e-3;
        f.row = row.ptr;
        f.prev_corr = prev_corr.ptr;
        f.history = step_history ? 1 : 0;
        f.mismatch = &sc.ptr->mismatch;
        return f;
    }
    void learned_guess(const cc_vbd_settings& s, const cc_grab* grab, const ContactsView& cv, double rq,
                       const float* features);
    // |grad E|^2 over moving vertices at view.x into `dst` (device).
    void grad_sq_into(const SweepView& view, double* dst, bool project) {
        launch_grad_sq(view, gsq.ptr, nullptr, 0, kResidualLanes, project, stream);
        launch_sum_partial(gsq.ptr, n, partial.ptr, nullptr, 0, stream);
        k_store_sum<<<1, 256, 0, stream>>>(partial.ptr, dst);
        own_launches += 3;
    }
    // step energy at view.x into `dst` (device).
    void energy_into(const SweepView& view, double* dst) {
        ObjectiveCounts c = counts();
        uint64_t items = n + objective_items(c);
        term_e.reserve(items);
        launch_term_energy(view, c, term_e.ptr, stream);
        launch_sum_partial(term_e.ptr, items, partial.ptr, nullptr, 0, stream);
        k_store_sum<<<1, 256, 0, stream>>>(partial.ptr, dst);
        own_launches += 3;
    }
    void color(const ContactsView& cv, const cc_grab* grab, cc_metrics& m) {
        double t = now_ms();
        coloring.set_error_word(&sc.ptr->error);
        coloring.compute(color_view(cv, grab), stream);
        m.color_ms += now_ms() - t;
        m.color_rounds += coloring.last_iterations();
    }
};

// Project autotuner: time one full colour sweep per candidate group width on
// a backup of the positions (restored after each trial) and keep the fastest.
void cc_solver::autotune(const SweepView& sv_in, bool fp32) {
    // lanes per vertex | register cap (resident 128-thread blocks per SM: 3, 4, 5,
    // 6 or 8; above 3 the compiler spills to local memory) << 8
    // | kVariantPersistent: a grid of the resident blocks looping over the colour;
    // | 1 << 17 or 2 << 17: blocks of 64 or 256 threads at the same register budget
    constexpr int P = kVariantPersistent, B64 = 1 << 17, B256 = 2 << 17;
    static const int kCandidates64[] = {1 | 3 << 8,      2 | 3 << 8,       4 | 3 << 8,      4 | 4 << 8,
                                        4 | 5 << 8,      4 | 6 << 8,       8 | 3 << 8,      8 | 4 << 8,
                                        8 | 5 << 8,      8 | 6 << 8,       8 | 8 << 8,      16 | 3 << 8,
                                        16 | 4 << 8,     16 | 6 << 8,      16 | 8 << 8,     32 | 3 << 8,
                                        4 | 4 << 8 | P,  8 | 4 << 8 | P,   8 | 3 << 8 | P,  4 | 4 << 8 | B64,
                                        8 | 4 << 8 | B64, 8 | 4 << 8 | B256, 4 | 4 << 8 | B256, 8 | 4 << 8 | B64 | P};
    static const int kCandidates32[] = {4 | 3 << 8,       4 | 4 << 8,        8 | 3 << 8,      8 | 4 << 8,
                                        8 | 5 << 8,       8 | 6 << 8,        8 | 8 << 8,      16 | 3 << 8,
                                        16 | 4 << 8,      16 | 6 << 8,       16 | 8 << 8,     32 | 3 << 8,
                                        32 | 4 << 8,      8 | 4 << 8 | P,    16 | 4 << 8 | P, 8 | 4 << 8 | B64,
                                        16 | 4 << 8 | B64, 8 | 4 << 8 | B256, 16 | 4 << 8 | B256};
    const int* cands = fp32 ? kCandidates32 : kCandidates64;
    const size_t n_cands = fp32 ? sizeof(kCandidates32) / sizeof(int) : sizeof(kCandidates64) / sizeof(int);
    SweepView sv = sv_in;  // trial sweeps never skip and count into a scratch counter
    sv.skip_at = nullptr;
    sv.clipped = &sc.ptr->clipped;
    x_backup.reserve(n);
    CC_CUDA(cudaMemcpyAsync(x_backup.ptr, world->x(), n * sizeof(double4), cudaMemcpyDeviceToDevice, stream));
    const auto& off = coloring.offsets();
    tune_ms.clear();
    float best = 1e30f;
    int best_g = fp32 ? (8 | 4 << 8) : (8 | 3 << 8);
    for (size_t ci = 0; ci < n_cands; ++ci) {
        const int g = cands[ci];
        float total = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {  // first repetition warms caches; keep the fastest of the rest
            CC_CUDA(cudaEventRecord(tune0, stream));
            for (int sweep = 0; sweep < 2; ++sweep)  // two consecutive sweeps, as the iterations run
                for (uint32_t c = 0; c < coloring.n_colors(); ++c)
                    launch_variant(sv, coloring.order() + off[c], off[c + 1] - off[c], g, fp32);
            CC_CUDA(cudaEventRecord(tune1, stream));
            CC_CUDA(cudaMemcpyAsync(world->x(), x_backup.ptr, n * sizeof(double4), cudaMemcpyDeviceToDevice, stream));
            CC_CUDA(cudaEventSynchronize(tune1));
            CC_CUDA(cudaGetLastError());
            float t = 0.f;
            CC_CUDA(cudaEventElapsedTime(&t, tune0, tune1));
            if (rep > 0) total = std::min(total, t);
            own_launches += 2 * coloring.n_colors();
        }
        tune_ms.push_back(total);
        if (total < best) {
            best = total;
            best_g = g;
        }
    }
    CC_CUDA(cudaMemsetAsync(&sc.ptr->clipped, 0, sizeof(unsigned int), stream));
    if (fp32) lanes32 = best_g;
    else lanes = best_g;
}

// MLP correction of the adaptive guess at three scales, clipped to the OGC
// balls; the lowest-energy candidate replaces the adaptive warm start (already
// in world->x()) only when its step energy is lower.
void cc_solver::learned_guess(const cc_vbd_settings& s, const cc_grab* grab, const ContactsView& cv, double rq,
                              const float* features) {
    if (!mlp) throw Failure{CC_ERR_INVALID_ARGUMENT, "learned initial guess requested but no MLP is attached"};
    FeatureView f = feature_view(cv, s, rq);
    corr.reserve((size_t)n_free * kMlpOut);
    mlp->net->forward(features, n_free, corr.ptr, mlp_precision, stream);
    // Candidates guess + a u c for a in {1, 1/2, 1/4}, each clipped to the OGC
    // balls; the one with the lowest step energy is kept if it is lower than
    // the adaptive guess's energy, which is kept otherwise.
    SweepView sa = sweep_view(cv, s, grab);
    best.reserve(n);
    energy_into(sa, &sc.ptr->e_init[0]);
    CC_CUDA(cudaMemcpyAsync(&sc.ptr->best_e, &sc.ptr->e_init[0], 8, cudaMemcpyDeviceToDevice, stream));
    for (double a : {1.0, 0.5, 0.25}) {
        CC_CUDA(cudaMemsetAsync(&sc.ptr->clipped_alt, 0, sizeof(unsigned int), stream));
        launch_learned_warm_start(f, corr.ptr, a, alt.ptr, &sc.ptr->clipped_alt, stream);
        SweepView sl = sa;
        sl.x = alt.ptr;
        energy_into(sl, &sc.ptr->e_cand);
        if (a == 1.0) CC_CUDA(cudaMemcpyAsync(&sc.ptr->e_init[1], &sc.ptr->e_cand, 8, cudaMemcpyDeviceToDevice, stream));
        k_decide_guess<<<1, 1, 0, stream>>>(sc.ptr);
        k_take_guess<<<grid_for(n, 256), 256, 0, stream>>>(n, alt.ptr, best.ptr, sc.ptr);
        own_launches += 3;
    }
    k_commit_guess<<<grid_for(n, 256), 256, 0, stream>>>(n, best.ptr, world->x(), sc.ptr);
    ++own_launches;
    CC_CUDA(cudaGetLastError());
}

void cc_solver::step(const cc_vbd_settings& s, const cc_grab* grab, cc_metrics* out) {
    if (!vbd_valid(s)) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid VBD settings"};
    if (!std::isfinite(time)) throw Failure{CC_ERR_INVALID_STATE, "Invalid VBD state"};
    if (grab) {
        double sum = grab->weights[0] + grab->weights[1] + grab->weights[2];
        bool bad = !std::isfinite(grab->target[0]) || !std::isfinite(grab->target[1]) ||
                   !std::isfinite(grab->target[2]) || !std::isfinite(grab->stiffness) || grab->stiffness <= 0.0 ||
                   std::fabs(sum - 1.0) > 1e-8;
        for (int i = 0; i < 3; ++i)
            bad = bad || grab->vertices[i] >= n || !std::isfinite(grab->weights[i]) || grab->weights[i] < 0.0;
        if (bad) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid mouse attachment"};
    }
    double t_start = now_ms();
    cc_metrics m;
    std::memset(&m, 0, sizeof m);
    uint64_t launches0 = own_launches + world->launches() + coloring.launches();
    m.dt_s = s.dt;
    m.iterations = s.iterations;
    CC_CUDA(cudaEventRecord(ev0, stream));
    CC_CUDA(cudaMemsetAsync(sc.ptr, 0, sizeof(StepScalars), stream));
    int gb = grid_for(n, 256);
    k_step_begin<<<gb, 256, 0, stream>>>(n, x0.ptr, v0.ptr, pred_x.ptr, pred_v.ptr, has_pred ? 1 : 0, sc.ptr);
    bool history = has_pred && pred_time == time && pred_g[0] == s.gravity[0] && pred_g[1] == s.gravity[1] &&
                   pred_g[2] == s.gravity[2] && pred_damping == s.damping;
    step_history = history;
    double3 g3 = make_double3(s.gravity[0], s.gravity[1], s.gravity[2]);
    k_predict<<<gb, 256, 0, stream>>>(n, x0.ptr, v0.ptr, accel.ptr, history ? 1 : 0, sc.ptr, s.dt, g3, s.damping,
                                      masses.ptr, guess.ptr, target.ptr, inertia.ptr, sc.ptr);
    own_launches += 2;
    CC_CUDA(cudaGetLastError());
    read_scalars();
    if (sc_h.ptr->error & DERR_NONFINITE_STATE) throw Failure{CC_ERR_INVALID_STATE, "Invalid VBD state"};
    double motion;
    std::memcpy(&motion, &sc_h.ptr->motion_bits, 8);
    double r = s.contact.radius;
    double rq = std::min(std::max(r + motion, 2.0 * r), 4.0 * r);
    k_copy_positions<<<gb, 256, 0, stream>>>(n, x0.ptr, world->x());
    ++own_launches;
    double det_ms = 0.0;
    detect(rq, s.contact, &m, det_ms);
    double md;
    {
        unsigned long long b = world->stats().min_dist_bits;
        std::memcpy(&md, &b, 8);
    }
    if (md <= 1e-12) throw Failure{CC_ERR_CONTACT, "OGC zero separation; step rejected, reset the arrangement"};
    ContactsView cv = world->contacts();
    color(cv, grab, m);
    CC_CUDA(cudaMemsetAsync(&sc.ptr->clipped, 0, sizeof(unsigned int), stream));
    k_warm_start<<<gb, 256, 0, stream>>>(n, pinned.ptr, guess.ptr, cv, world->x(), &sc.ptr->clipped);
    ++own_launches;
    const bool checks = s.residual_check_every > 0 || s.residual_tolerance > 0.0;
    const uint32_t check_every = s.residual_check_every > 0 ? s.residual_check_every : 1;
    learn_timed = false;
    if (s.init_mode == CC_INIT_LEARNED || sample_features) {
        // features of the step start (the learned guess's input; training samples)
        CC_CUDA(cudaEventRecord(learn0, stream));
        learn_timed = true;
        FeatureView f = feature_view(cv, s, rq);
        float* fout = sample_features;
        if (!fout) {
            feat.reserve((size_t)n_free * kMlpIn);
            fout = feat.ptr;
        }
        launch_features(f, fout, stream);
        ++own_launches;
        if (s.init_mode == CC_INIT_LEARNED) learned_guess(s, grab, cv, rq, fout);
        CC_CUDA(cudaEventRecord(learn1, stream));
    }
    if (checks) {
        // denominator |grad E(y)|^2 (alt holds y), then the initial guess's residual
        SweepView sy = sweep_view(cv, s, grab);
        sy.x = alt.ptr;
        k_copy_positions<<<gb, 256, 0, stream>>>(n, target.ptr, alt.ptr);
        ++own_launches;
        grad_sq_into(sy, &sc.ptr->gy2, false);
        grad_sq_into(sweep_view(cv, s, grab), &sc.ptr->gx2_init, true);
    }
    CC_CUDA(cudaGetLastError());
    read_scalars();
    size_t clipped = sc_h.ptr->clipped;
    // Iterations are enqueued ahead of the device: k_refresh_rule (and, with a
    // residual target, k_residual_rule) decide on the device and later sweeps
    // exit at once. Without a target all iterations go in one batch and the
    // host syncs once; with one, they go in chunks and the host reads the
    // previous chunk's stop flag while the next chunk runs. After a refresh
    // the host redoes detection and colouring and resumes at that iteration.
    const double threshold = s.contact.refresh_fraction * (double)n;
    const double tol2 = s.residual_tolerance * s.residual_tolerance;
    const bool target_on = s.residual_tolerance > 0.0;
    const bool accelerate = s.acceleration > 0.0;
    const double rho2 = accelerate ? s.acceleration * s.acceleration : 0.0;
    if (accelerate) {
        acc_a.reserve(n);
        acc_b.reserve(n);
    }
    bool need_refresh = clipped > 0 && (double)clipped >= threshold;
    if (profiling) {
        stamp_s.reserve(s.iterations);
        stamp_e.reserve(s.iterations);
        stamp_h.reserve(2 * (size_t)s.iterations);
    }
    uint32_t it0 = 0, executed = s.iterations;
    CC_CUDA(cudaMemsetAsync(&sc.ptr->converged_at, 0xff, sizeof(unsigned int), stream));
    if (checks) CC_CUDA(cudaMemsetAsync(sc.ptr->gx2_iter, 0xff, sizeof(sc.ptr->gx2_iter), stream));  // NaN: not evaluated
    while (it0 < s.iterations) {
        if (need_refresh) {
            detect(rq, s.contact, &m, det_ms);
            cv = world->contacts();
            color(cv, grab, m);
        }
        SweepView sv = sweep_view(cv, s, grab);
        sv.skip_at = &sc.ptr->stop_at;
        const bool fp32 = s.sweep_precision == CC_SWEEP_FP32;
        if ((fp32 ? lanes32 : lanes) == 0) autotune(sv, fp32);
        // the Chebyshev sequence restarts with every batch (the step's start or a refresh)
        double4* acc_prev1 = acc_a.ptr;
        double4* acc_prev2 = acc_b.ptr;
        if (accelerate) {
            CC_CUDA(cudaMemcpyAsync(acc_prev1, world->x(), n * sizeof(double4), cudaMemcpyDeviceToDevice, stream));
            CC_CUDA(cudaMemsetAsync(&sc.ptr->acc_k, 0, sizeof(unsigned int), stream));
            CC_CUDA(cudaMemsetAsync(&sc.ptr->acc_g2, 0x7f, sizeof(double), stream));  // ~1.4e306
        }
        CC_CUDA(cudaMemsetAsync(&sc.ptr->refresh_at, 0xff, 2 * sizeof(unsigned int), stream));  // + converged_at
        CC_CUDA(cudaMemsetAsync(&sc.ptr->stall_best, 0x7f, sizeof(double), stream));  // ~1.4e306
        CC_CUDA(cudaMemsetAsync(&sc.ptr->stall_count, 0, sizeof(unsigned int), stream));
        CC_CUDA(cudaMemsetAsync(&sc.ptr->stop_at, 0xff, sizeof(unsigned int), stream));
        CC_CUDA(cudaMemsetAsync(&sc.ptr->clipped_iter[it0], 0, (s.iterations - it0) * sizeof(unsigned int), stream));
        const auto& off = coloring.offsets();
        if (profiling) {  // this batch's iterations are (re)timed from scratch
            CC_CUDA(cudaMemsetAsync(stamp_s.ptr + it0, 0xff, (s.iterations - it0) * sizeof(unsigned long long), stream));
            CC_CUDA(cudaMemsetAsync(stamp_e.ptr + it0, 0, (s.iterations - it0) * sizeof(unsigned long long), stream));
        }
        uint32_t first_color = 0, last_color = 0;
        {
            bool any = false;
            for (uint32_t c = 0; c < coloring.n_colors(); ++c)
                if (off[c + 1] > off[c]) {
                    if (!any) first_color = c;
                    last_color = c;
                    any = true;
                }
        }
        const uint32_t chunk = target_on ? std::max<uint32_t>(check_every, 4) : s.iterations;
        uint32_t chunks = 0;
        // graph mode: each chunk's launches (after a batch's first iteration)
        // are captured into a CUDA graph; the executable graph of the chunk's
        // shape is updated in place, and a new shape (another colour count or
        // placement of the residual checks) is instantiated once and kept
        const bool capture = graphs;
        for (uint32_t c0 = it0; c0 < s.iterations; c0 += chunk) {
            uint32_t c1 = std::min(s.iterations, c0 + chunk);
            // the batch's first iteration goes out as direct launches: the GPU
            // starts on it while the host captures the rest of the lead chunk
            // (the capture and the executable-graph update of the first chunk
            // after a detection would otherwise leave the GPU idle)
            const uint32_t cap_from = (capture && c0 == it0) ? c0 + 1 : c0;
            bool capturing = false;
            try {
            for (uint32_t it = c0; it < c1; ++it) {
                if (capture && it == cap_from) {
                    CC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
                    capturing = true;
                }
                sv.iteration = it;
                sv.clipped = &sc.ptr->clipped_iter[it];
                // profiling: the iteration's back-to-back colour sweeps stamp
                // their span (first colour's earliest block start, last
                // colour's latest block end)
                sv.stamp_start = profiling ? stamp_s.ptr + it : nullptr;
                sv.stamp_end = profiling ? stamp_e.ptr + it : nullptr;
                for (uint32_t c = 0; c < coloring.n_colors(); ++c) {
                    uint32_t cnt = off[c + 1] - off[c];
                    if (cnt == 0) continue;
                    sv.stamp_first = c == first_color ? 1u : 0u;
                    sv.stamp_last = c == last_color ? 1u : 0u;
                    sweep(sv, coloring.order() + off[c], cnt, fp32);
                    ++own_launches;
                }
                k_refresh_rule<<<1, 1, 0, stream>>>(sc.ptr, it, s.iterations, threshold, rho2);
                if (accelerate) {
                    k_accelerate<<<gb, 256, 0, stream>>>(n, pinned.ptr, cv, world->x(), acc_prev2, sc.ptr, it);
                    std::swap(acc_prev1, acc_prev2);
                    ++own_launches;
                }
                ++own_launches;
                if (checks && ((it + 1) % check_every == 0 || it + 1 == s.iterations)) {
                    launch_grad_sq(sv, gsq.ptr, &sc.ptr->stop_at, it, kResidualLanes, true, stream);
                    launch_sum_partial(gsq.ptr, n, partial.ptr, &sc.ptr->stop_at, it, stream);
                    k_residual_rule<<<1, 256, 0, stream>>>(sc.ptr, partial.ptr, it, s.iterations, tol2,
                                                           target_on ? 1 : 0, s.stall_refresh, accelerate ? 1 : 0);
                    own_launches += 3;
                }
            }
            } catch (...) {
                if (capturing) {  // leave the stream out of capture mode before the failure propagates
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(stream, &g);
                    if (g) cudaGraphDestroy(g);
                }
                throw;
            }
            if (capturing) launch_captured_chunk();
            CC_CUDA(cudaGetLastError());
            if (c1 >= s.iterations || !target_on) break;
            // look ahead: enqueue the next chunk before waiting on this one's stop flag
            unsigned int slot = chunks & 1u;
            CC_CUDA(cudaMemcpyAsync(stop_h.ptr + slot, &sc.ptr->stop_at, sizeof(unsigned int),
                                    cudaMemcpyDeviceToHost, stream));
            CC_CUDA(cudaEventRecord(chunk_ev[slot], stream));
            if (chunks > 0) {
                CC_CUDA(cudaEventSynchronize(chunk_ev[slot ^ 1u]));
                if (stop_h.ptr[slot ^ 1u] != 0xffffffffu) break;
            }
            ++chunks;
        }
        read_scalars();
        uint32_t ra = sc_h.ptr->refresh_at, ca = sc_h.ptr->converged_at;
        uint32_t done_to = std::min(std::min(ra, ca), s.iterations);
        m.sweep_launches += (uint64_t)(done_to - it0) * coloring.n_colors();
        if (ca <= s.iterations && ca <= ra) {
            executed = ca;
            break;
        }
        if (ra < s.iterations) {
            it0 = ra;
            need_refresh = true;
        } else {
            it0 = s.iterations;
        }
    }
    if (checks) {
        // the plain force norm of the final iterate with the OGC terms in force
        grad_sq_into(sweep_view(cv, s, grab), &sc.ptr->gx2_plain, false);
        CC_CUDA(cudaGetLastError());
    }
    for (uint32_t it = 0; it < executed; ++it) m.truncated_vertices += sc_h.ptr->clipped_iter[it];
    m.iterations = executed;
    m.vertex_solves = (uint64_t)n_free * executed;
    if (checks) {
        double gy = std::sqrt(sc_h.ptr->gy2);
        m.has_relative_residual = 1;
        m.relative_residual = std::sqrt(sc_h.ptr->gx2) / gy;
        m.initial_relative_residual = std::sqrt(sc_h.ptr->gx2_init) / gy;
    }
    m.init_used = sc_h.ptr->init_used;
    m.init_energy_adaptive = m.init_energy_learned = std::nan("");
    if (s.init_mode == CC_INIT_LEARNED) {
        m.init_energy_adaptive = sc_h.ptr->e_init[0];
        m.init_energy_learned = sc_h.ptr->e_init[1];
    }
    if (sample_targets) {
        launch_targets(feature_view(cv, s, rq), world->x(), sample_targets, stream);
        ++own_launches;
    }
    m.colors = coloring.n_colors();
    CC_CUDA(cudaMemsetAsync(&sc.ptr->residual, 0, sizeof(double), stream));
    k_step_finish<<<gb, 256, 0, stream>>>(n, world->x(), cv, residual.ptr, sc.ptr);
    ++own_launches;
    CC_CUDA(cudaGetLastError());
    read_scalars();
    if (sc_h.ptr->error & DERR_SORT_WAIT)
        throw Failure{CC_ERR_DEVICE_TIMEOUT, "colour sort look-back wait gave up; state unchanged"};
    if (sc_h.ptr->error & DERR_NONFINITE_RESULT) throw Failure{CC_ERR_NON_FINITE, "Non-finite VBD result; state unchanged"};
    if (checks) m.relative_force_residual = std::sqrt(sc_h.ptr->gx2_plain / sc_h.ptr->gy2);
    if (sc_h.ptr->error & DERR_TRUST_REGION) throw Failure{CC_ERR_CONTACT, "OGC trust-region invariant failed"};
    m.residual_rms_n = std::sqrt(sc_h.ptr->residual / (double)(3 * (size_t)n));
    m.has_residual = 1;
    k_commit<<<gb, 256, 0, stream>>>(n, world->x(), x0.ptr, v0.ptr, pred_x.ptr, pred_v.ptr, accel.ptr, s.dt,
                                     s.damping, guess.ptr, prev_corr.ptr);
    ++own_launches;
    time += s.dt;
    has_pred = true;
    pred_time = time;
    pred_damping = s.damping;
    for (int k = 0; k < 3; ++k) pred_g[k] = s.gravity[k];
    // metrics: seam gap, extension P95/max
    if (n_stitch) k_seam_gap<<<grid_for(n_stitch, 256), 256, 0, stream>>>(n_stitch, st_off.ptr, st_v.ptr, st_w.ptr,
                                                                            x0.ptr, sc.ptr);
    if (n_stitch) ++own_launches;
    double p95 = 0.0, emax = 0.0;
    if (n_tri) {
        k_stretch<<<grid_for(n_tri, 256), 256, 0, stream>>>(n_tri, tri_v.ptr, tri_coef.ptr, tri_area.ptr, x0.ptr,
                                                            ext_key.ptr, ext_w.ptr);
        own_launches += 2;  // k_stretch and k_p95
        own_launches += ext_sorter.sort_pairs(ext_key.ptr, ext_key_s.ptr, ext_w.ptr, ext_w_s.ptr, n_tri, 64, stream,
                                              &sc.ptr->error, DERR_SORT_WAIT);
        own_launches += inclusive_sum(ext_w_s.ptr, ext_cum.ptr, n_tri, ext_scan, stream);
        k_p95<<<grid_for(n_tri, 256), 256, 0, stream>>>(n_tri, ext_key_s.ptr, ext_cum.ptr, sc.ptr);
    }
    CC_CUDA(cudaEventRecord(ev1, stream));
    read_scalars();
    if (n_tri) {
        p95 = from_order_key(sc_h.ptr->p95_bits);
        emax = from_order_key(sc_h.ptr->ext_max_bits);
    }
    const bool metric_sort_failed = (sc_h.ptr->error & DERR_SORT_WAIT) != 0;  // the step is committed already
    float gms = 0.f;
    CC_CUDA(cudaEventElapsedTime(&gms, ev0, ev1));
    double gap;
    std::memcpy(&gap, &sc_h.ptr->seam_gap_bits, 8);
    m.time_s = time;
    m.contacts = world->stats().active;
    m.contact_terms = world->stats().n_contacts;
    m.minimum_distance_m = md;
    {
        unsigned long long b = world->stats().min_dist_bits;
        std::memcpy(&m.minimum_distance_m, &b, 8);
    }
    m.max_seam_gap_m = n_stitch ? gap : 0.0;
    m.extension_p95_percent = metric_sort_failed ? std::nan("") : p95;
    m.extension_max_percent = metric_sort_failed ? std::nan("") : emax;
    m.detection_ms = det_ms;
    m.gpu_compute_ms = gms;
    if (profiling && executed > 0) {
        // iterations skipped after a refresh or a stop never stamp: their
        // slots keep the empty values and are left out
        CC_CUDA(cudaMemcpyAsync(stamp_h.ptr, stamp_s.ptr, executed * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, stream));
        CC_CUDA(cudaMemcpyAsync(stamp_h.ptr + executed, stamp_e.ptr, executed * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, stream));
        CC_CUDA(cudaStreamSynchronize(stream));
        double sw = 0.0;
        for (uint32_t it = 0; it < executed; ++it) {
            unsigned long long a = stamp_h.ptr[it], b = stamp_h.ptr[executed + it];
            if (a != ~0ull && b >= a) sw += (double)(b - a) * 1e-6;
        }
        m.sweep_ms = sw;
    }
    if (learn_timed) {
        float lt = 0.f;
        CC_CUDA(cudaEventElapsedTime(&lt, learn0, learn1));
        m.init_ms = lt;
    }
    m.kernel_launches = own_launches + world->launches() + coloring.launches() - launches0;
    m.contact_incidence = world->stats().n_incident;
    m.step_ms = now_ms() - t_start;
    m.solve_ms = m.step_ms - det_ms;
    if (out) *out = m;
}

// ----------------------------------------------------------- C entry points
extern "C" {

int32_t cc_abi_version(void) { return CC_ABI_VERSION; }

int32_t cc_global_last_error(char* buffer, uint64_t length) {
    std::lock_guard<std::mutex> lock(g_mutex);
    copy_msg(g_error, buffer, length);
    return g_code;
}

int32_t cc_last_error(const cc_solver* s, char* buffer, uint64_t length) {
    copy_msg(s->err, buffer, length);
    return s->code;
}

int32_t cc_world_last_error(const cc_world* w, char* buffer, uint64_t length) {
    copy_msg(w->err, buffer, length);
    return w->code;
}

int32_t cc_set_device(int32_t device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return set_global(CC_ERR_CUDA, "cc_set_device: no such CUDA device");
    g_device = device;
    return CC_OK;
}

int32_t cc_solver_create(const cc_mesh* mesh, const cc_surface* obstacle, const double* x0, const double* v0,
                         uint64_t n, cc_solver** out) {
    try {
        if (!mesh || !x0 || !out) throw Failure{CC_ERR_INVALID_ARGUMENT, "null argument"};
        if (mesh->n_vertices != n) throw Failure{CC_ERR_INVALID_ARGUMENT, "VBD state dimensions do not match garment"};
        CC_CUDA(cudaSetDevice(g_device));
        auto h = std::make_unique<cc_solver>();
        CC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        CC_CUDA(cudaEventCreate(&h->ev0));
        CC_CUDA(cudaEventCreate(&h->ev1));
        CC_CUDA(cudaEventCreate(&h->tune0));
        CC_CUDA(cudaEventCreate(&h->tune1));
        cudaStream_t st = h->stream;
        h->n = (uint32_t)n;
        // pins must match their constraints (src/vbd.rs:110-120)
        for (uint64_t i = 0; i < n; ++i) {
            if (mesh->pinned && mesh->pinned[i]) {
                double dx = x0[3 * i] - mesh->pin_positions[3 * i], dy = x0[3 * i + 1] - mesh->pin_positions[3 * i + 1],
                       dz = x0[3 * i + 2] - mesh->pin_positions[3 * i + 2];
                if (std::sqrt(dx * dx + dy * dy + dz * dz) > 1e-10)
                    throw Failure{CC_ERR_INVALID_ARGUMENT,
                                  "VBD pinned positions must match their constraints before initialization"};
            }
        }
        for (uint64_t i = 0; i < 3 * n; ++i)
            if (!std::isfinite(x0[i]) || (v0 && !std::isfinite(v0[i])))
                throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid OGC positions"};
        // combined positions and faces (src/vbd.rs:121-127)
        std::vector<double> xall(x0, x0 + 3 * n);
        std::vector<std::array<uint32_t, 3>> faces;
        for (uint64_t t = 0; t < mesh->n_triangles; ++t) {
            std::array<uint32_t, 3> f{mesh->triangles[3 * t], mesh->triangles[3 * t + 1], mesh->triangles[3 * t + 2]};
            for (uint32_t v : f)
                if (v >= n) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid material binding or mesh topology"};
            faces.push_back(f);
        }
        if (obstacle) {  // SurfaceMesh::validate (src/avatar.rs:83-98)
            if (obstacle->n_vertices == 0 || obstacle->n_triangles == 0)
                throw Failure{CC_ERR_INVALID_ARGUMENT, "Empty/non-finite avatar"};
            for (uint64_t i = 0; i < 3 * obstacle->n_vertices; ++i)
                if (!std::isfinite(obstacle->vertices[i])) throw Failure{CC_ERR_INVALID_ARGUMENT, "Empty/non-finite avatar"};
            for (uint64_t t = 0; t < obstacle->n_triangles; ++t) {
                uint32_t a = obstacle->triangles[3 * t], b = obstacle->triangles[3 * t + 1],
                         c = obstacle->triangles[3 * t + 2];
                if (a >= obstacle->n_vertices || b >= obstacle->n_vertices || c >= obstacle->n_vertices)
                    throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid avatar index"};
                auto P = [&](uint32_t i) {
                    return mk(obstacle->vertices[3 * i], obstacle->vertices[3 * i + 1], obstacle->vertices[3 * i + 2]);
                };
                if (len2(cross(P(b) - P(a), P(c) - P(a))) < 1e-24)
                    throw Failure{CC_ERR_INVALID_ARGUMENT, "Degenerate avatar triangle"};
                faces.push_back({a + (uint32_t)n, b + (uint32_t)n, c + (uint32_t)n});
            }
            xall.insert(xall.end(), obstacle->vertices, obstacle->vertices + 3 * obstacle->n_vertices);
        }
        size_t n_all = xall.size() / 3;
        h->n_all = (uint32_t)n_all;
        // stitches and their contact exclusions (src/vbd.rs:128-144)
        std::vector<std::array<uint32_t, 2>> excluded;
        uint64_t S = mesh->n_stitches;
        for (uint64_t s = 0; s < S; ++s) {
            for (uint32_t a = mesh->stitch_offsets[s]; a < mesh->stitch_offsets[s + 1]; ++a) {
                if (mesh->stitch_vertices[a] >= n) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid seam vertex"};
                for (uint32_t b = mesh->stitch_offsets[s]; b < mesh->stitch_offsets[s + 1]; ++b)
                    if (mesh->stitch_weights[a] * mesh->stitch_weights[b] < 0.0)
                        excluded.push_back({std::min(mesh->stitch_vertices[a], mesh->stitch_vertices[b]),
                                            std::max(mesh->stitch_vertices[a], mesh->stitch_vertices[b])});
            }
        }
        h->world = std::make_unique<World>(xall.data(), n_all, faces, n, excluded, st);
        h->world->validate_start();
        h->world_view.w = h->world.get();
        h->world_view.stream = st;
        // materials
        std::vector<MatParams> mats;
        for (uint64_t k = 0; k < mesh->n_materials; ++k) {
            const cc_material& M = mesh->materials[k];
            mats.push_back({M.warp, M.weft, M.shear, M.compression_ratio, M.compression_transition});
        }
        if (mats.empty()) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid material binding or mesh topology"};
        auto grain = [&](uint32_t mat, double& sn, double& cs) {
            double r = mesh->materials[mat].grain_degrees * (M_PI / 180.0);
            sn = std::sin(r);
            cs = std::cos(r);
        };
        // triangles: grain-rotated inverse rest matrix columns
        uint64_t T = mesh->n_triangles;
        h->n_tri = (uint32_t)T;
        std::vector<int4> tv(T);
        std::vector<double4> tc(T);
        std::vector<double> ta(T);
        std::vector<std::vector<uint32_t>> inc(n);
        std::vector<std::set<uint32_t>> graph(n), ring1(n);
        auto connect = [&](const uint32_t* ids, size_t k) {
            for (size_t a = 0; a < k; ++a)
                for (size_t b = 0; b < k; ++b)
                    if (ids[a] != ids[b]) graph[ids[a]].insert(ids[b]);
        };
        for (uint64_t t = 0; t < T; ++t) {
            uint32_t mat = mesh->triangle_material ? mesh->triangle_material[t] : 0;
            if (mat >= mats.size()) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid material binding or mesh topology"};
            const double* I = mesh->inv_dm + 4 * t;
            double sn, cs;
            grain(mat, sn, cs);
            tv[t] = make_int4((int)mesh->triangles[3 * t], (int)mesh->triangles[3 * t + 1],
                              (int)mesh->triangles[3 * t + 2], (int)mat);
            tc[t] = make_double4(I[0] * cs + I[2] * sn, I[1] * cs + I[3] * sn, -I[0] * sn + I[2] * cs,
                                 -I[1] * sn + I[3] * cs);
            ta[t] = mesh->area[t];
            for (uint32_t k = 0; k < 3; ++k) inc[mesh->triangles[3 * t + k]].push_back(pack_term(TERM_TRI, k, (uint32_t)t));
            connect(mesh->triangles + 3 * t, 3);
            for (uint32_t a = 0; a < 3; ++a)
                for (uint32_t b = 0; b < 3; ++b)
                    if (a != b) ring1[mesh->triangles[3 * t + a]].insert(mesh->triangles[3 * t + b]);
        }
        uint64_t Hn = mesh->n_hinges;
        std::vector<uint4> hv(Hn);
        std::vector<double> hk(Hn);
        for (uint64_t i = 0; i < Hn; ++i) {
            const uint32_t* v = mesh->hinges + 4 * i;
            for (int k = 0; k < 4; ++k)
                if (v[k] >= n) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid material binding or mesh topology"};
            uint32_t mat = mesh->hinge_material ? mesh->hinge_material[i] : 0;
            if (mat >= mats.size()) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid material binding or mesh topology"};
            double sn, cs;
            grain(mat, sn, cs);
            double ax = mesh->hinge_across[2 * i], ay = mesh->hinge_across[2 * i + 1];
            double aw = ax * cs + ay * sn, af = -ax * sn + ay * cs;
            const cc_material& M = mesh->materials[mat];
            hv[i] = make_uint4(v[0], v[1], v[2], v[3]);
            hk[i] = 0.5 * mesh->hinge_weight[i] * (M.bend_warp * aw * aw + M.bend_weft * af * af);
            for (uint32_t k = 0; k < 4; ++k) inc[v[k]].push_back(pack_term(TERM_HINGE, k, (uint32_t)i));
            connect(v, 4);
        }
        h->n_stitch = (uint32_t)S;
        std::vector<uint32_t> so(S + 1, 0), sv;
        std::vector<double> sw, sk(S);
        for (uint64_t s = 0; s < S; ++s) {
            std::vector<uint32_t> ids;
            for (uint32_t k = mesh->stitch_offsets[s]; k < mesh->stitch_offsets[s + 1]; ++k) {
                sv.push_back(mesh->stitch_vertices[k]);
                sw.push_back(mesh->stitch_weights[k]);
                ids.push_back(mesh->stitch_vertices[k]);
            }
            so[s + 1] = (uint32_t)sv.size();
            sk[s] = mesh->stitch_stiffness[s];
            for (uint32_t v : ids) inc[v].push_back(pack_term(TERM_STITCH, 0, (uint32_t)s));
            connect(ids.data(), ids.size());
        }
        std::vector<uint32_t> io(n + 1, 0), iv, lo_o(n + 1, 0), lo_v;
        std::vector<uint2> mid(n);
        for (uint64_t v = 0; v < n; ++v) {
            io[v + 1] = io[v] + (uint32_t)inc[v].size();
            // entries are grouped by type (triangles, hinges, stitches): record the boundaries
            uint32_t hb = io[v], sb = io[v];
            for (uint32_t e : inc[v]) {
                uint32_t type = e >> 30;
                if (type == TERM_TRI) ++hb, ++sb;
                else if (type == TERM_HINGE) ++sb;
            }
            mid[v] = make_uint2(hb, sb);
            iv.insert(iv.end(), inc[v].begin(), inc[v].end());
            for (uint32_t u : graph[v])
                if (u < v) lo_v.push_back(u);
            lo_o[v + 1] = (uint32_t)lo_v.size();
        }
        std::vector<uint8_t> pin(n, 0);
        if (mesh->pinned)
            for (uint64_t i = 0; i < n; ++i) pin[i] = mesh->pinned[i] ? 1 : 0;
        h->n_free = 0;
        std::vector<uint32_t> rows(n, 0), rg_o(n + 1, 0), rg_v;
        double msum = 0.0;
        for (uint64_t i = 0; i < n; ++i) {
            rows[i] = h->n_free;
            h->n_free += pin[i] ? 0 : 1;
            msum += mesh->masses[i];
            rg_v.insert(rg_v.end(), ring1[i].begin(), ring1[i].end());
            rg_o[i + 1] = (uint32_t)rg_v.size();
        }
        h->mean_mass = n ? msum / (double)n : 1.0;
        h->n_hinge = (uint32_t)Hn;
        for (uint64_t i = 0; i < n; ++i)
            if (!(mesh->masses[i] > 0.0) || !std::isfinite(mesh->masses[i]))
                throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid material binding or mesh topology"};
        h->mats.upload(mats, st);
        {
            std::vector<MatParams32> m32;
            for (const MatParams& M : mats)
                m32.push_back({(float)M.warp, (float)M.weft, (float)M.shear, (float)M.c, (float)M.delta});
            h->mats32.upload(m32, st);
        }
        h->tri_v.upload(tv, st);
        h->tri_coef.upload(tc, st);
        h->tri_area.upload(ta, st);
        h->hinge_v.upload(hv, st);
        h->hinge_k.upload(hk, st);
        h->st_off.upload(so, st);
        h->st_v.upload(sv, st);
        h->st_w.upload(sw, st);
        h->st_k.upload(sk, st);
        h->inc_off.upload(io, st);
        h->inc_mid.upload(mid, st);
        h->inc.upload(iv, st);
        h->lo_off.upload(lo_o, st);
        h->lo.upload(lo_v, st);
        h->pinned.upload(pin, st);
        h->row.upload(rows, st);
        h->ring_off.upload(rg_o, st);
        h->ring.upload(rg_v, st);
        h->alt.reserve(n_all);
        CC_CUDA(cudaMemcpyAsync(h->alt.ptr, h->world->x(), n_all * sizeof(double4), cudaMemcpyDeviceToDevice, st));
        h->gsq.reserve(n);
        h->partial.reserve(kSumBlocks);
        h->stop_h.reserve(2);
        CC_CUDA(cudaEventCreateWithFlags(&h->chunk_ev[0], cudaEventDisableTiming));
        CC_CUDA(cudaEventCreateWithFlags(&h->chunk_ev[1], cudaEventDisableTiming));
        CC_CUDA(cudaEventCreate(&h->learn0));
        CC_CUDA(cudaEventCreate(&h->learn1));
        h->masses.upload(mesh->masses, n, st);
        for (auto* b : {&h->x0, &h->v0, &h->guess, &h->target, &h->pred_x, &h->pred_v, &h->accel, &h->prev_corr})
            b->reserve(n);
        h->inertia.reserve(n);
        h->residual.reserve(n);
        h->clipped_flag.reserve(n);
        h->sc.reserve(1);
        h->sc_h.reserve(1);
        h->stage.reserve(2 * n);
        h->io.reserve(6 * n);
        h->ext_key.reserve(T);
        h->ext_key_s.reserve(T);
        h->ext_w.reserve(T);
        h->ext_w_s.reserve(T);
        h->ext_cum.reserve(T);
        h->residual.zero(n, st);
        h->coloring.init((uint32_t)n, st);
        // initial state
        for (uint64_t i = 0; i < n; ++i) {
            h->stage.ptr[i] = make_double4(x0[3 * i], x0[3 * i + 1], x0[3 * i + 2], 0.0);
            h->stage.ptr[n + i] = v0 ? make_double4(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2], 0.0) : make_double4(0, 0, 0, 0);
        }
        CC_CUDA(cudaMemcpyAsync(h->x0.ptr, h->stage.ptr, n * sizeof(double4), cudaMemcpyHostToDevice, st));
        CC_CUDA(cudaMemcpyAsync(h->v0.ptr, h->stage.ptr + n, n * sizeof(double4), cudaMemcpyHostToDevice, st));
        CC_CUDA(cudaStreamSynchronize(st));
        *out = h.release();
        return CC_OK;
    } catch (const Failure& f) {
        return set_global(f.code, f.message);
    } catch (const std::exception& e) {
        return set_global(CC_ERR_CUDA, e.what());
    }
}

void cc_solver_destroy(cc_solver* s) { delete s; }
uint64_t cc_solver_moving(const cc_solver* s) { return s->n; }
uint64_t cc_solver_total(const cc_solver* s) { return s->n_all; }
void* cc_solver_stream(const cc_solver* s) { return (void*)s->stream; }
int32_t cc_solver_set_graphs(cc_solver* s, int32_t enable) {
    s->graphs = enable != 0;
    return CC_OK;
}
int32_t cc_solver_set_profiling(cc_solver* s, int32_t enable) {
    s->profiling = enable != 0;
    return CC_OK;
}
// 0, or a sweep variant with the cap defaulting to 3
static int normalize_variant(int32_t v) {
    if (v == 0) return 0;
    if (((v >> 8) & 0xff) == 0) v |= 3 << 8;
    return v;
}

int32_t cc_solver_set_lanes(cc_solver* s, int32_t lanes) {
    int v = normalize_variant(lanes);
    if (v != 0 && !sweep_variant_valid(v, false))
        return s->fail(Failure{CC_ERR_INVALID_ARGUMENT,
                               "lanes must be 0 (autotune) or a power of two up to 32, optionally | cap << 8 with "
                               "cap 3, 4, 5, 6 or 8, | 1 << 16 (persistent grid), | 1 << 17 or 2 << 17 (64- or "
                               "256-thread blocks, 4 or 8 lanes)"});
    s->lanes = v;
    return CC_OK;
}
int32_t cc_solver_get_lanes(const cc_solver* s) { return s->lanes; }
int32_t cc_solver_set_lanes32(cc_solver* s, int32_t lanes) {
    int v = normalize_variant(lanes);
    if (v != 0 && !sweep_variant_valid(v, true))
        return s->fail(Failure{CC_ERR_INVALID_ARGUMENT,
                               "FP32 sweep lanes must be 0 (autotune), 4, 8, 16 or 32, optionally | cap << 8 "
                               "with cap 3, 4, 5, 6 or 8, | 1 << 16 (persistent grid), | 1 << 17 or 2 << 17 "
                               "(64- or 256-thread blocks, 8 or 16 lanes)"});
    s->lanes32 = v;
    return CC_OK;
}
int32_t cc_solver_get_lanes32(const cc_solver* s) { return s->lanes32; }
cc_world* cc_solver_world(cc_solver* s) { return &s->world_view; }

static void upload_state(cc_solver* s, const double* x, const double* v) {
    size_t n = s->n;
    if (n == 0) return;
    CC_CUDA(cudaMemcpyAsync(s->io.ptr, x, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CC_CUDA(cudaMemcpyAsync(s->io.ptr + 3 * n, v, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    launch_unpack_state(n, s->io.ptr, s->x0.ptr, s->v0.ptr, s->stream);
}

static void download_state(cc_solver* s, double* x, double* v) {
    size_t n = s->n;
    if (n == 0) return;
    launch_pack_state(n, s->x0.ptr, s->v0.ptr, s->io.ptr, s->stream);
    CC_CUDA(cudaMemcpyAsync(x, s->io.ptr, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CC_CUDA(cudaMemcpyAsync(v, s->io.ptr + 3 * n, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CC_CUDA(cudaStreamSynchronize(s->stream));
}

int32_t cc_solver_set_state(cc_solver* s, const double* x, const double* v, double time) {
    try {
        upload_state(s, x, v);
        s->time = time;
        CC_CUDA(cudaStreamSynchronize(s->stream));
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

int32_t cc_solver_get_state(cc_solver* s, double* x, double* v, double* time) {
    try {
        download_state(s, x, v);
        if (time) *time = s->time;
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

int32_t cc_solver_step_resident(cc_solver* s, const cc_vbd_settings* settings, const cc_grab* grab,
                                cc_metrics* metrics) {
    // The resident state is the last committed one; a failed step leaves it
    // (and the prediction history) untouched.
    double t0 = s->time;
    try {
        s->step(*settings, grab, metrics);
        return CC_OK;
    } catch (const Failure& f) {
        s->time = t0;
        return s->fail(f);
    }
}

int32_t cc_solver_newton_step(cc_solver* s, const double* x_old, const double* v_old,
                              const cc_vbd_settings* settings, uint32_t newton_iterations, uint32_t pcg_iterations,
                              double abs_tol, double rel_tol, double* x_out, cc_newton_report* report) {
    try {
        if (!settings || !vbd_valid(*settings) || !x_old || !v_old || !x_out || newton_iterations > 1000 ||
            pcg_iterations == 0 || !(abs_tol >= 0.0) || !(rel_tol >= 0.0))
            throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid Newton settings"};
        const cc_vbd_settings& st = *settings;
        const uint32_t n = s->n, n_all = s->n_all;
        cudaStream_t stream = s->stream;
        for (DBuf<double4>* b : {&s->nt_x0, &s->nt_v0, &s->nt_guess, &s->nt_target}) b->reserve(n);
        s->nt_y.reserve(n_all);
        s->nt_out.reserve(n_all);
        s->nt_inertia.reserve(n);
        // the caller's state in the device layout (the solver's own state is untouched)
        s->io.reserve(6 * (size_t)n);
        CC_CUDA(cudaMemcpyAsync(s->io.ptr, x_old, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, stream));
        CC_CUDA(cudaMemcpyAsync(s->io.ptr + 3 * (size_t)n, v_old, 3 * (size_t)n * sizeof(double),
                                cudaMemcpyHostToDevice, stream));
        launch_unpack_state(n, s->io.ptr, s->nt_x0.ptr, s->nt_v0.ptr, stream);
        // inertial target, inertia and the step's query radius (src/vbd.rs:283-307)
        CC_CUDA(cudaMemsetAsync(s->sc.ptr, 0, sizeof(StepScalars), stream));
        int gb = grid_for(n, 256);
        double3 g3 = make_double3(st.gravity[0], st.gravity[1], st.gravity[2]);
        k_predict<<<gb, 256, 0, stream>>>(n, s->nt_x0.ptr, s->nt_v0.ptr, s->accel.ptr, 0, s->sc.ptr, st.dt, g3,
                                          st.damping, s->masses.ptr, s->nt_guess.ptr, s->nt_target.ptr,
                                          s->nt_inertia.ptr, s->sc.ptr);
        CC_CUDA(cudaGetLastError());
        s->read_scalars();
        double motion;
        std::memcpy(&motion, &s->sc_h.ptr->motion_bits, 8);
        double r = st.contact.radius;
        double rq = std::min(std::max(r + motion, 2.0 * r), 4.0 * r);
        // the step's OGC contact set at x_old, frozen for the whole solve
        k_copy_positions<<<gb, 256, 0, stream>>>(n, s->nt_x0.ptr, s->world->x());
        s->world->detect(rq, r, st.contact.relaxation, st.contact.stiffness, false);
        ContactsView cv = s->world->contacts();
        NewtonProblem pb;
        pb.view = s->sweep_view(cv, st, nullptr);
        pb.view.target = s->nt_target.ptr;
        pb.view.inertia = s->nt_inertia.ptr;
        pb.n_all = n_all;
        pb.n_free = s->n_free;
        pb.n_tri = s->n_tri;
        pb.counts = s->counts();
        CC_CUDA(cudaMemcpyAsync(s->nt_y.ptr, s->world->x(), n_all * sizeof(double4), cudaMemcpyDeviceToDevice, stream));
        k_copy_positions<<<gb, 256, 0, stream>>>(n, s->nt_target.ptr, s->nt_y.ptr);
        pb.y_all = s->nt_y.ptr;
        double gy2 = 0.0;
        NewtonResult res = newton_solve(pb, s->world->x(), newton_iterations, pcg_iterations, abs_tol, rel_tol,
                                        s->nt_out.ptr, &gy2, stream);
        launch_pack_state(n, s->nt_out.ptr, s->nt_v0.ptr, s->io.ptr, stream);
        CC_CUDA(cudaMemcpyAsync(x_out, s->io.ptr, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CC_CUDA(cudaStreamSynchronize(stream));
        if (report) {
            report->converged = res.converged ? 1 : 0;
            report->iterations = res.iterations;
            report->pcg_iterations = res.pcg_iterations;
            report->residual_rms_n = res.residual_rms;
            report->objective_j = res.objective;
            report->relative_force_residual = gy2 > 0.0 ? std::sqrt(res.gradient_sq / gy2) : 0.0;
            report->contact_terms = s->world->stats().n_contacts;
        }
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

int32_t cc_solver_step(cc_solver* s, double* x, double* v, double* time, const cc_vbd_settings* settings,
                       const cc_grab* grab, cc_metrics* metrics) {
    try {
        upload_state(s, x, v);
        s->time = *time;
        s->step(*settings, grab, metrics);
        download_state(s, x, v);
        *time = s->time;
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

static void upload_all(World* w, const double* x_all, cudaStream_t st, Pinned<double4>& stage) {
    size_t N = w->n_all();
    stage.reserve(N);
    for (size_t i = 0; i < N; ++i) stage.ptr[i] = make_double4(x_all[3 * i], x_all[3 * i + 1], x_all[3 * i + 2], 0.0);
    CC_CUDA(cudaMemcpyAsync(w->x(), stage.ptr, N * sizeof(double4), cudaMemcpyHostToDevice, st));
    CC_CUDA(cudaStreamSynchronize(st));
}

int32_t cc_solver_colors(cc_solver* s, const double* x_all, double query_radius, const cc_ogc_settings* settings,
                         const cc_grab* grab, uint32_t* colors_out, uint32_t* n_colors) {
    try {
        if (!ogc_valid(*settings)) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid OGC radius, stiffness or trust-region parameters"};
        Pinned<double4> stage;
        upload_all(s->world.get(), x_all, s->stream, stage);
        s->world->detect(query_radius, settings->radius, settings->relaxation, settings->stiffness, true);
        s->coloring.compute(s->color_view(s->world->contacts(), grab), s->stream);
        std::vector<uint32_t> c;
        s->coloring.download(c);
        std::copy(c.begin(), c.end(), colors_out);
        *n_colors = s->coloring.n_colors();
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

int32_t cc_solver_local_blocks(cc_solver* s, const double* x_all, double query_radius,
                               const cc_vbd_settings* settings, const cc_grab* grab, const double* targets,
                               const double* inertia, double* energy, double* gradient, double* hessian) {
    try {
        if (!ogc_valid(settings->contact))
            throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid OGC radius, stiffness or trust-region parameters"};
        Pinned<double4> stage;
        upload_all(s->world.get(), x_all, s->stream, stage);
        size_t n = s->n;
        if (targets) {
            std::vector<double4> t(n);
            for (size_t i = 0; i < n; ++i) t[i] = make_double4(targets[3 * i], targets[3 * i + 1], targets[3 * i + 2], 0);
            s->target.upload(t, s->stream);
        }
        if (inertia) s->inertia.upload(inertia, n, s->stream);
        s->world->detect(query_radius, settings->contact.radius, settings->contact.relaxation,
                         settings->contact.stiffness, true);
        SweepView sv = s->sweep_view(s->world->contacts(), *settings, grab);
        if (!targets) sv.target = nullptr;
        if (!inertia) sv.inertia = nullptr;
        DBuf<double> e, g, h;
        e.reserve(n);
        g.reserve(3 * n);
        h.reserve(9 * n);
        launch_local_blocks(sv, e.ptr, g.ptr, h.ptr, s->stream);
        CC_CUDA(cudaGetLastError());
        CC_CUDA(cudaMemcpyAsync(energy, e.ptr, n * 8, cudaMemcpyDeviceToHost, s->stream));
        CC_CUDA(cudaMemcpyAsync(gradient, g.ptr, 3 * n * 8, cudaMemcpyDeviceToHost, s->stream));
        CC_CUDA(cudaMemcpyAsync(hessian, h.ptr, 9 * n * 8, cudaMemcpyDeviceToHost, s->stream));
        CC_CUDA(cudaStreamSynchronize(s->stream));
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

int32_t cc_world_create(const double* x, uint64_t n_all, const uint32_t* triangles, uint64_t n_triangles,
                        uint64_t moving, const uint32_t* excluded, uint64_t n_excluded, cc_world** out) {
    try {
        CC_CUDA(cudaSetDevice(g_device));
        auto h = std::make_unique<cc_world>();
        CC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->owns_stream = true;
        std::vector<std::array<uint32_t, 3>> tris(n_triangles);
        for (uint64_t t = 0; t < n_triangles; ++t) tris[t] = {triangles[3 * t], triangles[3 * t + 1], triangles[3 * t + 2]};
        std::vector<std::array<uint32_t, 2>> ex(n_excluded);
        for (uint64_t e = 0; e < n_excluded; ++e) ex[e] = {excluded[2 * e], excluded[2 * e + 1]};
        h->own = std::make_unique<World>(x, n_all, tris, moving, ex, h->stream);
        h->w = h->own.get();
        *out = h.release();
        return CC_OK;
    } catch (const Failure& f) {
        return set_global(f.code, f.message);
    }
}

void cc_world_destroy(cc_world* w) {
    if (w && w->own) delete w;
}

int32_t cc_world_set_tree_rebuild_period(cc_world* w, int32_t period) {
    if (!w) return CC_ERR_INVALID_ARGUMENT;
    if (period < 0) return w->fail(Failure{CC_ERR_INVALID_ARGUMENT, "tree rebuild period must be >= 0"});
    w->w->set_tree_rebuild_period((uint32_t)period);
    return CC_OK;
}

int32_t cc_world_validate_start(cc_world* w, const double* x) {
    try {
        Pinned<double4> stage;
        upload_all(w->w, x, w->w->stream(), stage);
        w->w->validate_start();
        return CC_OK;
    } catch (const Failure& f) {
        return w->fail(f);
    }
}

int32_t cc_world_detect(cc_world* w, const double* x, double query_radius, const cc_ogc_settings* settings,
                        cc_contacts* out) {
    try {
        if (!ogc_valid(*settings))
            throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid OGC radius, stiffness or trust-region parameters"};
        if (!std::isfinite(query_radius) || query_radius < settings->radius)
            throw Failure{CC_ERR_INVALID_ARGUMENT, "OGC query radius must cover the contact radius"};
        Pinned<double4> stage;
        upload_all(w->w, x, w->w->stream(), stage);
        w->w->detect(query_radius, settings->radius, settings->relaxation, settings->stiffness, true);
        const DetectStats& st = w->w->stats();
        std::vector<uint32_t> kind, verts, inc;
        std::vector<double> eps, radii;
        std::vector<uint64_t> inc_off;
        w->w->download(kind, verts, eps, inc_off, inc, radii);
        size_t moving = w->w->moving();
        out->n_contacts = kind.size();
        out->n_incident = inc.size();
        out->active_contacts = st.active;
        out->vertex_face_candidates = st.vf_count;
        out->edge_edge_candidates = st.ee_count;
        out->candidate_pairs = st.n_vf + st.n_ee;
        out->aabb_rejections = st.rejections;
        std::memcpy(&out->minimum_distance, &st.min_dist_bits, 8);
        out->broad_phase_rebuilt = st.rebuild ? 1 : 0;
        if (out->contact_capacity < kind.size() || out->incident_capacity < inc.size() || out->radii_capacity < moving)
            return CC_ERR_CAPACITY;
        for (size_t c = 0; c < kind.size(); ++c) {
            if (out->kinds) out->kinds[c] = (uint8_t)kind[c];
            if (out->vertices)
                for (int k = 0; k < 4; ++k) out->vertices[4 * c + k] = verts[4 * c + k];
            if (out->counts) out->counts[c] = (uint8_t)(kind[c] == 0 ? 2 : (kind[c] == 1 ? 3 : 4));
            if (out->mollifier_epsilon) out->mollifier_epsilon[c] = eps[c];
        }
        if (out->incident_offsets) std::copy(inc_off.begin(), inc_off.end(), out->incident_offsets);
        if (out->incident) std::copy(inc.begin(), inc.end(), out->incident);
        if (out->radii) std::copy(radii.begin(), radii.end(), out->radii);
        return CC_OK;
    } catch (const Failure& f) {
        return w->fail(f);
    }
}

int32_t cc_world_candidates(cc_world* w, const double* x, double radius, cc_candidates* out) {
    try {
        Pinned<double4> stage;
        upload_all(w->w, x, w->w->stream(), stage);
        std::vector<uint32_t> vf, ee;
        w->w->fresh_pairs(radius, vf, ee);
        out->n_vf = vf.size() / 2;
        out->n_ee = ee.size() / 2;
        if (out->vf_capacity < out->n_vf || out->ee_capacity < out->n_ee) return CC_ERR_CAPACITY;
        std::copy(vf.begin(), vf.end(), out->vf);
        std::copy(ee.begin(), ee.end(), out->ee);
        return CC_OK;
    } catch (const Failure& f) {
        return w->fail(f);
    }
}

uint64_t cc_world_edges(const cc_world* w, uint32_t* edges_out) {
    const auto& e = w->w->topology().edges;
    if (edges_out)
        for (size_t i = 0; i < e.size(); ++i) {
            edges_out[2 * i] = e[i][0];
            edges_out[2 * i + 1] = e[i][1];
        }
    return e.size();
}

// ------------------------------------------------------- learned guess
namespace {
uint64_t mix64(uint64_t& st) {
    uint64_t z = (st += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
}  // namespace

int32_t cc_mlp_create(uint64_t seed, cc_mlp** out) {
    try {
        if (!out) throw Failure{CC_ERR_INVALID_ARGUMENT, "null argument"};
        CC_CUDA(cudaSetDevice(g_device));
        auto h = std::make_unique<cc_mlp>();
        CC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->net = std::make_unique<Mlp>(seed);
        *out = h.release();
        return CC_OK;
    } catch (const Failure& f) {
        return set_global(f.code, f.message);
    }
}

void cc_mlp_destroy(cc_mlp* m) { delete m; }
uint64_t cc_mlp_parameter_count(void) { return (uint64_t)kMlpParams; }

int32_t cc_mlp_last_error(const cc_mlp* m, char* buffer, uint64_t length) {
    copy_msg(m->err, buffer, length);
    return m->code;
}

int32_t cc_mlp_set_parameters(cc_mlp* m, const float* params, uint64_t count) {
    try {
        if (!params || count != (uint64_t)kMlpParams)
            throw Failure{CC_ERR_INVALID_ARGUMENT, "MLP parameter count must be cc_mlp_parameter_count()"};
        for (uint64_t i = 0; i < count; ++i)
            if (!std::isfinite(params[i])) throw Failure{CC_ERR_INVALID_ARGUMENT, "non-finite MLP parameter"};
        m->net->set_params(params, m->stream);
        return CC_OK;
    } catch (const Failure& f) {
        return m->fail(f);
    }
}

int32_t cc_mlp_get_parameters(cc_mlp* m, float* params, uint64_t count) {
    try {
        if (!params || count != (uint64_t)kMlpParams)
            throw Failure{CC_ERR_INVALID_ARGUMENT, "MLP parameter count must be cc_mlp_parameter_count()"};
        m->net->get_params(params, m->stream);
        return CC_OK;
    } catch (const Failure& f) {
        return m->fail(f);
    }
}

int32_t cc_mlp_forward(cc_mlp* m, const float* features, uint64_t n, float* out, int32_t precision) {
    try {
        if ((n && (!features || !out)) || (precision != 0 && precision != 1))
            throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_mlp_forward: bad arguments"};
        m->net->forward(features, n, out, precision, m->stream);
        CC_CUDA(cudaStreamSynchronize(m->stream));
        if (precision == 1 && m->net->read_error(m->stream))
            throw Failure{CC_ERR_DEVICE_TIMEOUT, "tensor-core MLP: a bounded wait gave up"};
        return CC_OK;
    } catch (const Failure& f) {
        return m->fail(f);
    }
}

int32_t cc_mlp_gradients(cc_mlp* m, const float* features, const float* targets, uint64_t n, float* grads,
                         float* loss) {
    try {
        if (!features || !targets || !grads || !loss || n == 0)
            throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_mlp_gradients: bad arguments"};
        m->net->gradients(features, targets, nullptr, n, m->net->grad_buffer(), m->net->loss_buffer(), m->stream);
        CC_CUDA(cudaMemcpyAsync(grads, m->net->grad_buffer(), kMlpParams * sizeof(float), cudaMemcpyDeviceToHost,
                                m->stream));
        CC_CUDA(cudaMemcpyAsync(loss, m->net->loss_buffer(), sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        CC_CUDA(cudaStreamSynchronize(m->stream));
        return CC_OK;
    } catch (const Failure& f) {
        return m->fail(f);
    }
}

int32_t cc_mlp_train(cc_mlp* m, const float* features, const float* targets, uint64_t n, uint32_t batch,
                     uint32_t steps, float learning_rate, uint64_t seed, float* losses) {
    try {
        if (!features || !targets || n == 0 || batch == 0 || steps == 0 || !(learning_rate > 0.0f))
            throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_mlp_train: bad arguments"};
        if (n > 0xffffffffull) throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_mlp_train: at most 2^32-1 samples"};
        uint64_t b = std::min<uint64_t>(batch, n);
        m->perm.reserve(n);
        m->losses.reserve(steps);
        std::vector<uint32_t> perm(n);
        for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
        uint64_t rng = seed, pos = n;  // pos = n forces a shuffle first
        for (uint32_t t = 0; t < steps; ++t) {
            if (pos + b > n) {  // new epoch: Fisher-Yates shuffle, upload
                CC_CUDA(cudaStreamSynchronize(m->stream));
                for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[mix64(rng) % (i + 1)]);
                CC_CUDA(cudaMemcpyAsync(m->perm.ptr, perm.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                        m->stream));
                pos = 0;
            }
            m->net->gradients(features, targets, m->perm.ptr + pos, b, m->net->grad_buffer(), m->losses.ptr + t,
                              m->stream);
            m->net->adam(m->net->grad_buffer(), learning_rate, 0.9f, 0.999f, 1e-8f, m->stream);
            pos += b;
        }
        if (losses)
            CC_CUDA(cudaMemcpyAsync(losses, m->losses.ptr, steps * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        CC_CUDA(cudaStreamSynchronize(m->stream));
        return CC_OK;
    } catch (const Failure& f) {
        return m->fail(f);
    }
}

int32_t cc_solver_set_mlp(cc_solver* s, cc_mlp* m, int32_t precision) {
    if (precision != 0 && precision != 1)
        return s->fail(Failure{CC_ERR_INVALID_ARGUMENT, "MLP precision must be 0 (FP32) or 1 (FP16 tensor cores)"});
    s->mlp = m;
    s->mlp_precision = precision;
    return CC_OK;
}

uint64_t cc_solver_free_vertices(const cc_solver* s) { return s->n_free; }

int32_t cc_solver_last_step_trace(const cc_solver* s, double* relative_residual, uint32_t* clipped,
                                  uint32_t capacity) {
    uint32_t k = std::min<uint32_t>(capacity, 256u);
    double gy2 = s->sc_h.ptr->gy2;
    for (uint32_t i = 0; i < k; ++i) {
        double g = s->sc_h.ptr->gx2_iter[i];
        if (relative_residual) relative_residual[i] = std::isnan(g) ? g : std::sqrt(g / gy2);
        if (clipped) clipped[i] = s->sc_h.ptr->clipped_iter[i];
    }
    return CC_OK;
}

int32_t cc_solver_step_sample(cc_solver* s, const cc_vbd_settings* settings, const cc_grab* grab, float* features,
                              float* targets, cc_metrics* metrics) {
    try {
        if (!settings || !features || !targets) throw Failure{CC_ERR_INVALID_ARGUMENT, "null argument"};
        s->sample_features = features;
        s->sample_targets = targets;
        try {
            s->step(*settings, grab, metrics);
        } catch (...) {
            s->sample_features = s->sample_targets = nullptr;
            throw;
        }
        s->sample_features = s->sample_targets = nullptr;
        return CC_OK;
    } catch (const Failure& f) {
        return s->fail(f);
    }
}

// ------------------------------------------------------ batched instances
// Many independent cloths as one solver: meshes concatenated (vertex, triangle,
// hinge, stitch and material indices offset), obstacles concatenated. Each
// colour sweep then covers every instance in one launch, detection builds
// one hierarchy for all of them, and the colouring of the union equals each
// instance's own greedy colouring (instances share no edges). Contact between
// instances is the caller's to avoid by placement: detection finds any pair
// within the query radius, whichever instances it joins.
int32_t cc_batch_create(const cc_mesh* meshes, const cc_surface* obstacles, const double* const* x0,
                        const double* const* v0, uint64_t count, cc_solver** out) {
    try {
        if (!meshes || !x0 || !out || count == 0) throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_batch_create: bad arguments"};
        std::vector<uint32_t> tri, tmat, hin, hmat, soff{0}, sv;
        std::vector<double> inv, area, hw, hac, masses, ppos, sw, sk, xs, vs;
        std::vector<uint8_t> pin;
        std::vector<cc_material> mats;
        std::vector<double> ov;
        std::vector<uint32_t> ot;
        std::vector<uint64_t> first, cnt;
        uint64_t nv = 0, obase = 0;
        for (uint64_t k = 0; k < count; ++k) {
            const cc_mesh& m = meshes[k];
            if (!x0[k]) throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_batch_create: missing positions"};
            uint32_t mbase = (uint32_t)mats.size(), vb = (uint32_t)nv;
            first.push_back(nv);
            cnt.push_back(m.n_vertices);
            for (uint64_t i = 0; i < m.n_materials; ++i) mats.push_back(m.materials[i]);
            for (uint64_t t = 0; t < m.n_triangles; ++t) {
                for (int c = 0; c < 3; ++c) tri.push_back(m.triangles[3 * t + c] + vb);
                for (int c = 0; c < 4; ++c) inv.push_back(m.inv_dm[4 * t + c]);
                area.push_back(m.area[t]);
                tmat.push_back((m.triangle_material ? m.triangle_material[t] : 0) + mbase);
            }
            for (uint64_t h = 0; h < m.n_hinges; ++h) {
                for (int c = 0; c < 4; ++c) hin.push_back(m.hinges[4 * h + c] + vb);
                hw.push_back(m.hinge_weight[h]);
                hac.push_back(m.hinge_across[2 * h]);
                hac.push_back(m.hinge_across[2 * h + 1]);
                hmat.push_back((m.hinge_material ? m.hinge_material[h] : 0) + mbase);
            }
            for (uint64_t i = 0; i < m.n_vertices; ++i) {
                masses.push_back(m.masses[i]);
                pin.push_back(m.pinned ? m.pinned[i] : 0);
                for (int c = 0; c < 3; ++c) {
                    ppos.push_back(m.pin_positions ? m.pin_positions[3 * i + c] : 0.0);
                    xs.push_back(x0[k][3 * i + c]);
                    vs.push_back(v0 && v0[k] ? v0[k][3 * i + c] : 0.0);
                }
            }
            for (uint64_t st = 0; st < m.n_stitches; ++st) {
                for (uint32_t a = m.stitch_offsets[st]; a < m.stitch_offsets[st + 1]; ++a) {
                    sv.push_back(m.stitch_vertices[a] + vb);
                    sw.push_back(m.stitch_weights[a]);
                }
                soff.push_back((uint32_t)sv.size());
                sk.push_back(m.stitch_stiffness[st]);
            }
            if (obstacles && obstacles[k].n_vertices) {
                const cc_surface& o = obstacles[k];
                for (uint64_t i = 0; i < 3 * o.n_vertices; ++i) ov.push_back(o.vertices[i]);
                for (uint64_t t = 0; t < 3 * o.n_triangles; ++t) {
                    if (o.triangles[t] >= o.n_vertices) throw Failure{CC_ERR_INVALID_ARGUMENT, "Invalid avatar index"};
                    ot.push_back(o.triangles[t] + (uint32_t)obase);
                }
                obase += o.n_vertices;
            }
            nv += m.n_vertices;
        }
        if (nv > 0x0fffffffull) throw Failure{CC_ERR_INVALID_ARGUMENT, "cc_batch_create: too many vertices"};
        cc_mesh u{};
        u.n_vertices = nv;
        u.n_triangles = area.size();
        u.triangles = tri.data();
        u.inv_dm = inv.data();
        u.area = area.data();
        u.triangle_material = tmat.data();
        u.n_hinges = hw.size();
        u.hinges = hin.data();
        u.hinge_weight = hw.data();
        u.hinge_across = hac.data();
        u.hinge_material = hmat.data();
        u.n_materials = mats.size();
        u.materials = mats.data();
        u.masses = masses.data();
        u.pinned = pin.data();
        u.pin_positions = ppos.data();
        u.n_stitches = sk.size();
        u.stitch_offsets = soff.data();
        u.stitch_vertices = sv.data();
        u.stitch_weights = sw.data();
        u.stitch_stiffness = sk.data();
        cc_surface os{obase, ov.data(), ot.size() / 3, ot.data()};
        int32_t rc = cc_solver_create(&u, obase ? &os : nullptr, xs.data(), vs.data(), nv, out);
        if (rc != CC_OK) return rc;
        (*out)->inst_first = first;
        (*out)->inst_count = cnt;
        return CC_OK;
    } catch (const Failure& f) {
        return set_global(f.code, f.message);
    }
}

uint64_t cc_batch_instances(const cc_solver* s, uint64_t* first_vertex, uint64_t* vertex_count, uint64_t capacity) {
    uint64_t k = s->inst_first.size();
    for (uint64_t i = 0; i < k && i < capacity; ++i) {
        if (first_vertex) first_vertex[i] = s->inst_first[i];
        if (vertex_count) vertex_count[i] = s->inst_count[i];
    }
    return k;
}

}  // extern "C"
