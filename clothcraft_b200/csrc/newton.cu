// FP64 Newton reference step on the GPU: ReferenceSolver::step_problem
// (src/solver.rs:422-646) for the VBD step's objective, with the step's OGC
// contact set frozen at one detection (the reference's Newton solver has no
// OGC term; the contacts enter with Contact::energy, src/ogc/potential.rs:39-65).
//
// Algorithm, as the reference: Newton iterations on the implicit-Euler
// objective; per iteration a Jacobi-preconditioned CG solve (tolerance 1e-5
// of the initial residual, at most pcg_iterations) with shift escalation
// 0, 1e-6 scale, x10 ... on a failed solve or line search (12 attempts), and
// an Armijo backtracking line search (c = 1e-4, 24 halvings), stopping at an
// RMS gradient over the free degrees of freedom <= max(abs_tol, rel_tol r0).
//
// One difference in form: the reference multiplies by assembled element
// Hessians; here the Hessian-vector product is the central difference of the
// exact FP64 gradient, H p = (g(x + h p) - g(x - h p)) / 2h with the largest
// displacement |h p| = 1e-7 m, so no 12x12 element matrices are stored. The
// Jacobi diagonal is exact (the diagonal of each vertex's 3x3 block).
#include <cmath>
#include <limits>
#include <vector>

#include "newton.cuh"
#include "sweep_terms.cuh"

namespace cc {

namespace {

constexpr int kLanes = 4;       // lanes per vertex of the gradient evaluations
constexpr int kBlocks = kSumBlocks;

// g_out[3v..3v+2] = dE/dx_v at s.x for moving vertex v (0 where pinned)
template <int G>
__global__ void __launch_bounds__(128) k_nt_gradient(SweepView s, double* g_out) {
    uint32_t t = blockIdx.x * 128 + threadIdx.x;
    uint32_t v = t / G;
    if (v >= s.n) return;
    uint32_t lane = threadIdx.x & (G - 1);
    unsigned mask = G >= 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(unsigned)(G - 1)));
    if (s.pinned[v]) {
        if (lane == 0) g_out[3 * v] = g_out[3 * v + 1] = g_out[3 * v + 2] = 0.0;
        return;
    }
    d3 x = ld3(s.x, v);
    d3 g = mk(0, 0, 0);
    Sym H;
    sym_zero(H);
    local_part<true, G, false>(s, v, x, lane, g, H);
    if (G > 1) {
        g.x = group_sum<G>(g.x, mask);
        g.y = group_sum<G>(g.y, mask);
        g.z = group_sum<G>(g.z, mask);
    }
    g = g + (x - ld3(s.target, v)) * s.inertia[v];
    if (lane == 0) {
        g_out[3 * v] = g.x;
        g_out[3 * v + 1] = g.y;
        g_out[3 * v + 2] = g.z;
    }
}

// Jacobi diagonal of System::diagonal (src/solver.rs:150-161): inertia +
// shift + the diagonal of every incident term's Hessian; 1 on fixed dofs.
__global__ void k_nt_diagonal(SweepView s, double shift, double* diag) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < s.n; v += gridDim.x * blockDim.x) {
        if (s.pinned[v]) {
            diag[3 * v] = diag[3 * v + 1] = diag[3 * v + 2] = 1.0;
            continue;
        }
        d3 x = ld3(s.x, v);
        d3 g = mk(0, 0, 0);
        Sym H;
        sym_zero(H);
        local_part<true, 1>(s, v, x, 0, g, H);
        double m = s.inertia[v];
        diag[3 * v] = fmax(H.a[0] + m + shift, 1e-12);
        diag[3 * v + 1] = fmax(H.a[3] + m + shift, 1e-12);
        diag[3 * v + 2] = fmax(H.a[5] + m + shift, 1e-12);
    }
}

// out = x + a d on free vertices (pinned keep x); fixed obstacle untouched
__global__ void k_nt_move(uint32_t n, const uint8_t* pinned, const double4* x, const double* d, double a,
                          double4* out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        d3 p = ld3(x, v);
        if (!pinned[v]) p = p + mk(d[3 * v], d[3 * v + 1], d[3 * v + 2]) * a;
        st3(out, v, p);
    }
}

// ap = (gp - gm) * inv2h + shift p
__global__ void k_nt_fd(size_t m, const double* gp, const double* gm, double inv2h, const double* p, double shift,
                        double* ap) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        ap[i] = (gp[i] - gm[i]) * inv2h + shift * p[i];
}

// Deterministic dot product: kBlocks fixed-order partials of a[i] b[i]
__global__ void __launch_bounds__(256) k_nt_dot_partial(const double* a, const double* b, size_t m,
                                                        double* partial) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (size_t i = blockIdx.x * 256ull + threadIdx.x; i < m; i += (size_t)kBlocks * 256ull) acc += a[i] * b[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}
__global__ void __launch_bounds__(256) k_nt_store(const double* partial, double* out) {
    double v = block_sum_partials(partial);
    if (threadIdx.x == 0) *out = v;
}
// max |a_i| (non-negative doubles order as their bits)
__global__ void k_nt_absmax(const double* a, size_t m, unsigned long long* out) {
    unsigned long long b = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        b = max(b, dbits(fabs(a[i])));
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, b);
}

// CG updates (src/solver.rs:205-220)
__global__ void k_nt_cg_step(size_t m, double alpha, const double* p, const double* ap, double* x, double* r) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        r[i] -= alpha * ap[i];
    }
}
__global__ void k_nt_precond(size_t m, const double* r, const double* diag, double* z) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        z[i] = r[i] / diag[i];
}
__global__ void k_nt_direction(size_t m, const double* z, double beta, double* p) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}
__global__ void k_nt_negate(size_t m, const double* g, double* r) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        r[i] = -g[i];
}

// geometry_valid (src/solver.rs:235-242): finite positions and no collapsed
// triangle (|cross| > 2 area 1e-6); sets *bad otherwise
__global__ void k_nt_geometry(uint32_t n, uint32_t nt, const int4* tri_v, const double* area, const double4* x,
                              unsigned int* bad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n + nt; i += gridDim.x * blockDim.x) {
        if (i < n) {
            if (!isfin(ld3(x, i))) atomicOr(bad, 1u);
        } else {
            int4 t = tri_v[i - n];
            d3 a = ld3(x, (uint32_t)t.x), b = ld3(x, (uint32_t)t.y), c = ld3(x, (uint32_t)t.z);
            if (!(len(cross(b - a, c - a)) > 2.0 * area[i - n] * 1e-6)) atomicOr(bad, 1u);
        }
    }
}

struct NewtonScratch {
    DBuf<double> g, gp, gm, diag, d, r, z, p, ap, partial, scalars, term_e;
    DBuf<double4> x, trial, probe;
    DBuf<unsigned long long> maxbits;
    DBuf<unsigned int> bad;
    Pinned<double> h_scalar;
    Pinned<unsigned long long> h_bits;
    Pinned<unsigned int> h_bad;
};

class Newton {
   public:
    Newton(const NewtonProblem& pb, cudaStream_t st) : pb_(pb), st_(st) {
        const size_t m = 3 * (size_t)pb.view.n;
        for (DBuf<double>* b : {&w_.g, &w_.gp, &w_.gm, &w_.diag, &w_.d, &w_.r, &w_.z, &w_.p, &w_.ap}) b->reserve(m);
        w_.partial.reserve(kBlocks);
        w_.scalars.reserve(1);
        w_.x.reserve(pb.n_all);
        w_.trial.reserve(pb.n_all);
        w_.probe.reserve(pb.n_all);
        w_.maxbits.reserve(1);
        w_.bad.reserve(1);
        w_.h_scalar.reserve(1);
        w_.h_bits.reserve(1);
        w_.h_bad.reserve(1);
        m_ = m;
    }

    NewtonResult run(const double4* x_start, uint32_t newton_iterations, uint32_t pcg_iterations, double abs_tol,
                     double rel_tol) {
        NewtonResult out;
        // all three position buffers carry the fixed obstacle after the cloth
        for (DBuf<double4>* b : {&w_.x, &w_.trial, &w_.probe})
            CC_CUDA(cudaMemcpyAsync(b->ptr, x_start, pb_.n_all * sizeof(double4), cudaMemcpyDeviceToDevice, st_));
        double tolerance = 0.0;
        size_t free_dofs = 3 * (size_t)pb_.n_free;
        for (uint32_t iteration = 0; iteration <= newton_iterations; ++iteration) {
            gradient(w_.x.ptr, w_.g.ptr);
            double gg = dot(w_.g.ptr, w_.g.ptr);
            double energy = objective(w_.x.ptr);
            double residual = std::sqrt(gg / (double)std::max<size_t>(free_dofs, 1));
            if (!std::isfinite(residual) || !std::isfinite(energy))
                throw Failure{CC_ERR_NON_FINITE, "Non-finite FEM assembly; step rolled back"};
            if (iteration == 0) tolerance = std::fmax(abs_tol, rel_tol * residual);
            out.residual_rms = residual;
            out.objective = energy;
            out.gradient_sq = gg;
            out.iterations = iteration;
            if (residual <= tolerance) {
                out.converged = true;
                break;
            }
            if (iteration == newton_iterations) break;
            diagonal(0.0);
            double scale = std::fmax(1.0, absmax(w_.diag.ptr));
            bool accepted = false;
            double shift = 0.0;
            for (int attempt = 0; attempt < 12 && !accepted; ++attempt) {
                uint64_t its = 0;
                bool ok = pcg(shift, pcg_iterations, its);
                out.pcg_iterations += its;
                if (ok) {
                    double slope = dot(w_.g.ptr, w_.d.ptr);
                    if (std::isfinite(slope) && slope < 0.0) {
                        double alpha = 1.0;
                        for (int ls = 0; ls < 24; ++ls) {
                            move(w_.x.ptr, w_.d.ptr, alpha, w_.trial.ptr);
                            double obj = objective(w_.trial.ptr);
                            if (std::isfinite(obj) && obj <= energy + 1e-4 * alpha * slope) {
                                accepted = true;
                                break;
                            }
                            alpha *= 0.5;
                        }
                    }
                }
                if (!accepted) shift = shift == 0.0 ? scale * 1e-6 : shift * 10.0;
            }
            if (!accepted) throw Failure{CC_ERR_NON_FINITE, "Newton line search failed; state unchanged. Reduce time step."};
            std::swap(w_.x.ptr, w_.trial.ptr);
        }
        out.x = w_.x.ptr;
        return out;
    }

    // |grad E|^2 over free vertices at positions x (device, [n_all])
    double gradient_sq_at(const double4* x) {
        gradient(x, w_.gp.ptr);
        return dot(w_.gp.ptr, w_.gp.ptr);
    }

   private:
    void gradient(const double4* x, double* out) {
        SweepView s = pb_.view;
        s.x = const_cast<double4*>(x);
        unsigned grid = (unsigned)(((uint64_t)s.n * kLanes + 127) / 128);
        if (grid) k_nt_gradient<kLanes><<<grid, 128, 0, st_>>>(s, out);
        CC_CUDA(cudaGetLastError());
    }
    void diagonal(double shift) {
        SweepView s = pb_.view;
        s.x = w_.x.ptr;
        k_nt_diagonal<<<grid_for(s.n, 128), 128, 0, st_>>>(s, shift, w_.diag.ptr);
    }
    double read_scalar() {
        CC_CUDA(cudaMemcpyAsync(w_.h_scalar.ptr, w_.scalars.ptr, sizeof(double), cudaMemcpyDeviceToHost, st_));
        CC_CUDA(cudaStreamSynchronize(st_));
        return *w_.h_scalar.ptr;
    }
    double dot(const double* a, const double* b) {
        k_nt_dot_partial<<<kBlocks, 256, 0, st_>>>(a, b, m_, w_.partial.ptr);
        k_nt_store<<<1, 256, 0, st_>>>(w_.partial.ptr, w_.scalars.ptr);
        return read_scalar();
    }
    double absmax(const double* a) {
        CC_CUDA(cudaMemsetAsync(w_.maxbits.ptr, 0, sizeof(unsigned long long), st_));
        k_nt_absmax<<<grid_for(m_, 256), 256, 0, st_>>>(a, m_, w_.maxbits.ptr);
        CC_CUDA(cudaMemcpyAsync(w_.h_bits.ptr, w_.maxbits.ptr, 8, cudaMemcpyDeviceToHost, st_));
        CC_CUDA(cudaStreamSynchronize(st_));
        double v;
        std::memcpy(&v, w_.h_bits.ptr, 8);
        return v;
    }
    void move(const double4* x, const double* d, double a, double4* out) {
        k_nt_move<<<grid_for(pb_.view.n, 256), 256, 0, st_>>>(pb_.view.n, pb_.view.pinned, x, d, a, out);
    }
    // step objective (VBD inertia form; the reference's form differs by a
    // constant) or +inf for invalid geometry
    double objective(const double4* x) {
        CC_CUDA(cudaMemsetAsync(w_.bad.ptr, 0, sizeof(unsigned int), st_));
        k_nt_geometry<<<grid_for(pb_.view.n + pb_.n_tri, 256), 256, 0, st_>>>(
            pb_.view.n, pb_.n_tri, pb_.view.tri_v, pb_.view.tri_area, x, w_.bad.ptr);
        SweepView s = pb_.view;
        s.x = const_cast<double4*>(x);
        uint64_t items = s.n + objective_items(pb_.counts);
        w_.term_e.reserve(items);
        launch_term_energy(s, pb_.counts, w_.term_e.ptr, st_);
        launch_sum_partial(w_.term_e.ptr, items, w_.partial.ptr, nullptr, 0, st_);
        k_nt_store<<<1, 256, 0, st_>>>(w_.partial.ptr, w_.scalars.ptr);
        CC_CUDA(cudaMemcpyAsync(w_.h_bad.ptr, w_.bad.ptr, sizeof(unsigned int), cudaMemcpyDeviceToHost, st_));
        double e = read_scalar();
        if (*w_.h_bad.ptr) return std::numeric_limits<double>::infinity();
        return e;
    }
    // Jacobi-preconditioned CG (System::pcg, src/solver.rs:189-224) into w_.d
    bool pcg(double shift, uint32_t limit, uint64_t& its) {
        diagonal(shift);
        const size_t m = m_;
        const int gb = grid_for(m, 256);
        CC_CUDA(cudaMemsetAsync(w_.d.ptr, 0, m * sizeof(double), st_));
        k_nt_negate<<<gb, 256, 0, st_>>>(m, w_.g.ptr, w_.r.ptr);
        k_nt_precond<<<gb, 256, 0, st_>>>(m, w_.r.ptr, w_.diag.ptr, w_.z.ptr);
        CC_CUDA(cudaMemcpyAsync(w_.p.ptr, w_.z.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st_));
        double rz = dot(w_.r.ptr, w_.z.ptr);
        double tol = 1e-5 * std::sqrt(dot(w_.r.ptr, w_.r.ptr));
        for (uint32_t it = 0; it < limit; ++it) {
            apply(shift);
            double curv = dot(w_.p.ptr, w_.ap.ptr);
            if (!std::isfinite(curv) || curv <= 0.0) {
                its = it + 1;
                return false;
            }
            double alpha = rz / curv;
            k_nt_cg_step<<<gb, 256, 0, st_>>>(m, alpha, w_.p.ptr, w_.ap.ptr, w_.d.ptr, w_.r.ptr);
            if (std::sqrt(dot(w_.r.ptr, w_.r.ptr)) <= tol) {
                its = it + 1;
                return true;
            }
            k_nt_precond<<<gb, 256, 0, st_>>>(m, w_.r.ptr, w_.diag.ptr, w_.z.ptr);
            double next = dot(w_.r.ptr, w_.z.ptr);
            double beta = next / rz;
            k_nt_direction<<<gb, 256, 0, st_>>>(m, w_.z.ptr, beta, w_.p.ptr);
            rz = next;
        }
        its = limit;
        return true;
    }
    // ap = H p + shift p by central differences of the exact gradient
    void apply(double shift) {
        double pmax = absmax(w_.p.ptr);
        if (!(pmax > 0.0)) {
            CC_CUDA(cudaMemsetAsync(w_.ap.ptr, 0, m_ * sizeof(double), st_));
            return;
        }
        double h = 1e-7 / pmax;
        move(w_.x.ptr, w_.p.ptr, h, w_.probe.ptr);
        gradient(w_.probe.ptr, w_.gp.ptr);
        move(w_.x.ptr, w_.p.ptr, -h, w_.probe.ptr);
        gradient(w_.probe.ptr, w_.gm.ptr);
        k_nt_fd<<<grid_for(m_, 256), 256, 0, st_>>>(m_, w_.gp.ptr, w_.gm.ptr, 0.5 / h, w_.p.ptr, shift, w_.ap.ptr);
    }

    NewtonProblem pb_;
    cudaStream_t st_;
    size_t m_ = 0;
    NewtonScratch w_;
};

}  // namespace

NewtonResult newton_solve(const NewtonProblem& pb, const double4* x_start, uint32_t newton_iterations,
                          uint32_t pcg_iterations, double abs_tol, double rel_tol, double4* x_out, double* gy2,
                          cudaStream_t st) {
    Newton nt(pb, st);
    NewtonResult r = nt.run(x_start, newton_iterations, pcg_iterations, abs_tol, rel_tol);
    CC_CUDA(cudaMemcpyAsync(x_out, r.x, pb.n_all * sizeof(double4), cudaMemcpyDeviceToDevice, st));
    r.x = nullptr;
    if (gy2) *gy2 = nt.gradient_sq_at(pb.y_all);
    CC_CUDA(cudaStreamSynchronize(st));
    return r;
}

}  // namespace cc
