// FP64 Newton reference step on the GPU (newton.cu).
#pragma once
#include "sweep.cuh"

namespace cc {

struct NewtonProblem {
    SweepView view;        // static terms, pinned, the step's target and inertia, the frozen contacts
    uint32_t n_all = 0;    // cloth + fixed obstacle vertices
    uint32_t n_free = 0;   // unpinned cloth vertices
    uint32_t n_tri = 0;
    ObjectiveCounts counts{};
    const double4* y_all = nullptr;  // [n_all] inertial target, fixed obstacle after it
};

struct NewtonResult {
    double4* x = nullptr;
    bool converged = false;
    uint32_t iterations = 0;
    uint64_t pcg_iterations = 0;
    double residual_rms = 0, objective = 0, gradient_sq = 0;
};

// Newton from x_start ([n_all], fixed part = obstacle); the result goes to
// x_out ([n_all]); *gy2 (if given) = |grad E(y)|^2 over free vertices.
NewtonResult newton_solve(const NewtonProblem& pb, const double4* x_start, uint32_t newton_iterations,
                          uint32_t pcg_iterations, double abs_tol, double rel_tol, double4* x_out, double* gy2,
                          cudaStream_t st);

}  // namespace cc
