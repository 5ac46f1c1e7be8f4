// Learned initial guess: per-vertex features, a 24-64-64-64-3 GELU MLP that
// predicts the correction of the adaptive guess, and its training kernels
// (forward, backward, Adam). No reference counterpart: the reference starts
// every step from Prediction::guess (src/vbd/prediction.rs:15-41); the
// learned guess replaces it only when its step energy is lower.
#pragma once
#include <cuda_fp16.h>

#include "sweep.cuh"

namespace cc {

constexpr int kMlpIn = 24;
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 3;
// parameter block (floats): W1[64][24] b1[64] W2[64][64] b2[64] W3[64][64]
// b3[64] W4[3][64] b4[3]; W[out][in], y = W x + b
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpHidden;
constexpr int kOffW4 = kOffB3 + kMlpHidden;
constexpr int kOffB4 = kOffW4 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kOffB4 + kMlpOut;  // 10,115

// Inputs of the feature kernel (all device pointers, moving vertices).
struct FeatureView {
    uint32_t n;
    const double4* x0;      // step-start positions
    const double4* v0;      // step-start velocities
    const double4* guess;   // adaptive guess
    const double4* target;  // inertial target y
    const uint8_t* pinned;
    const double* masses;
    double mean_mass;
    const uint32_t* ring_off;  // triangle 1-ring, CSR [n+1]
    const uint32_t* ring;
    const uint32_t* inc_off;  // static incidence (packed terms)
    const uint32_t* inc;
    const int4* tri_v;
    const double4* tri_coef;
    ContactsView contacts;
    double query_radius;
    double relaxation;
    double dt;
    double unit;  // displacement unit |g| dt^2
    const uint32_t* row;  // [n] output row of each free vertex
    const double4* prev_corr;      // [n] last step's x_end - adaptive guess
    int history;                   // host side of the adaptive-guess history test
    const unsigned int* mismatch;  // device side (state edited since the last step)
};

// out[row[v]][24] for every free vertex v.
void launch_features(const FeatureView& f, float* out, cudaStream_t st);
// Learned guess, clipped to the OGC ball like the warm start
// (src/vbd.rs:316-324): alt[v] = clip(guess[v] + alpha * unit * corr[row[v]]);
// pinned vertices copy x0. Counts clipped vertices into *clipped.
void launch_learned_warm_start(const FeatureView& f, const float* corr, double alpha, double4* alt,
                               unsigned int* clipped, cudaStream_t st);
// targets[row[v]] = (x[v] - guess[v]) / unit for free vertices.
void launch_targets(const FeatureView& f, const double4* x, float* targets, cudaStream_t st);

// MLP parameters with their Adam state, all on the device.
class Mlp {
   public:
    explicit Mlp(uint64_t seed);
    void set_params(const float* host, cudaStream_t st);
    void get_params(float* host, cudaStream_t st) const;
    const float* params() const { return p_.ptr; }
    // out[n][3] = MLP(features[n][24]): precision 0 = FP32 CUDA cores,
    // 1 = FP16 operands with FP32 accumulation on the tensor cores.
    void forward(const float* features, uint64_t n, float* out, int precision, cudaStream_t st);
    // Gradient of L = (1/n) sum_s |MLP(f_s) - t_s|^2 over the n samples listed
    // in `index` (or 0..n-1 when null) into grads[kMlpParams]; *loss = L.
    void gradients(const float* features, const float* targets, const uint32_t* index, uint64_t n, float* grads,
                   float* loss, cudaStream_t st);
    // Adam (Kingma & Ba 2015) with bias correction, one step.
    void adam(const float* grads, float lr, float beta1, float beta2, float eps, cudaStream_t st);
    float* grad_buffer() { return g_.ptr; }
    float* loss_buffer() { return loss_.ptr; }
    uint64_t adam_steps() const { return t_; }

    // error word of the last tensor-core forward (1 = a bounded wait gave up)
    unsigned int read_error(cudaStream_t st);

   private:
    DBuf<float> p_, m_, v_, g_, loss_, partial_;
    DBuf<__half> w16_;  // FP16 copies of W1..W4 in the tensor-core operand layout
    DBuf<unsigned int> err_;
    bool w16_valid_ = false;
    uint64_t t_ = 0;
    void refresh_half(cudaStream_t st);
    void forward_tc(const float* features, uint64_t n, float* out, cudaStream_t st);
};

}  // namespace cc
