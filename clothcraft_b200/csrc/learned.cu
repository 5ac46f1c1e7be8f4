// Learned initial guess: features, MLP inference and training kernels.
//
// Features (24 per free vertex, computed at the start of a step from the
// state, the adaptive guess, the inertial target and the step's OGC
// detection; `u` = |g| dt^2 is the displacement unit):
//   0-2   (y - x0) / u                      inertial displacement
//   3-5   (guess - x0) / u                  adaptive guess (prediction.rs)
//   6-8   mean over the 1-ring of the neighbours' guess displacement, minus own
//   9-11  (mean 1-ring position - x0) / mean 1-ring edge length
//   12-14 unit area-weighted normal of the incident triangles
//   15    100 * mean Green strain trace (E_ww + E_ff) of incident triangles
//   16    100 * mean |E_wf| shear of incident triangles
//   17    100 * max principal fibre strain max(E_ww, E_ff)
//   18    OGC nearest distance / query radius (radius / relaxation / rq)
//   19    contact terms incident to the vertex / 4 (capped at 16)
//   20-22 last step's correction (x_end - adaptive guess) / u, 0 without history
//   23    1 - ring size / 6
// The network maps them to a correction c; the learned guess is
// guess + u * c, clipped to the vertex's OGC ball.
#include <cuda_fp16.h>

#include <cmath>
#include <vector>

#include "learned.cuh"

namespace cc {

// GELU, tanh form (Hendrycks & Gimpel 2016): 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
__device__ __forceinline__ float gelu_f(float z) {
    const float c0 = 0.7978845608028654f, c1 = 0.044715f;
    float t = tanhf(c0 * (z + c1 * z * z * z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ void gelu_fg(float z, float& a, float& da) {
    const float c0 = 0.7978845608028654f, c1 = 0.044715f;
    float t = tanhf(c0 * (z + c1 * z * z * z));
    a = 0.5f * z * (1.0f + t);
    da = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * c0 * (1.0f + 3.0f * c1 * z * z);
}

// ------------------------------------------------------------- features
__global__ void k_features(FeatureView f, float* out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < f.n; v += gridDim.x * blockDim.x) {
        if (f.pinned[v]) continue;
        float* o = out + (size_t)f.row[v] * kMlpIn;
        const double iu = 1.0 / f.unit;
        d3 x = ld3(f.x0, v), y = ld3(f.target, v), g = ld3(f.guess, v);
        d3 dy = (y - x) * iu, dg = (g - x) * iu;
        d3 nb_dg = mk(0, 0, 0), nb_x = mk(0, 0, 0);
        double elen = 0.0;
        uint32_t r0 = f.ring_off[v], r1 = f.ring_off[v + 1];
        for (uint32_t k = r0; k < r1; ++k) {
            uint32_t u = f.ring[k];
            d3 xu = ld3(f.x0, u);
            nb_x = nb_x + xu;
            elen += len(xu - x);
            nb_dg = nb_dg + (ld3(f.guess, u) - xu) * iu;
        }
        uint32_t cnt = r1 - r0;
        d3 rel = mk(0, 0, 0), lap = mk(0, 0, 0);
        if (cnt) {
            double ic = 1.0 / (double)cnt;
            rel = nb_dg * ic - dg;
            double el = elen * ic;
            lap = (nb_x * ic - x) * (1.0 / fmax(el, 1e-12));
        }
        d3 nrm = mk(0, 0, 0);
        double tr = 0.0, shs = 0.0, mx = -1e30;
        uint32_t nt = 0;
        for (uint32_t k = f.inc_off[v]; k < f.inc_off[v + 1]; ++k) {
            uint32_t ent = f.inc[k];
            if ((ent >> 30) != TERM_TRI) continue;
            uint32_t t = ent & 0x0fffffffu;
            int4 tv = f.tri_v[t];
            double4 cf = f.tri_coef[t];
            d3 a = ld3(f.x0, (uint32_t)tv.x), b = ld3(f.x0, (uint32_t)tv.y), c = ld3(f.x0, (uint32_t)tv.z);
            d3 ds0 = b - a, ds1 = c - a;
            nrm = nrm + cross(ds0, ds1);
            d3 w = ds0 * cf.x + ds1 * cf.y;
            d3 q = ds0 * cf.z + ds1 * cf.w;
            double ew = 0.5 * (dot(w, w) - 1.0), ef = 0.5 * (dot(q, q) - 1.0);
            tr += ew + ef;
            shs += fabs(dot(w, q));
            mx = fmax(mx, fmax(ew, ef));
            ++nt;
        }
        double nl = len(nrm);
        if (nl > 0.0) nrm = nrm * (1.0 / nl);
        if (nt) {
            tr /= (double)nt;
            shs /= (double)nt;
        } else {
            mx = 0.0;
        }
        double dmin = f.contacts.radii[v] / f.relaxation / f.query_radius;
        uint32_t nc = f.contacts.inc_off[v + 1] - f.contacts.inc_off[v];
        d3 pc = mk(0, 0, 0);
        if (f.history && *f.mismatch == 0) pc = ld3(f.prev_corr, v) * iu;
        double feat[kMlpIn] = {dy.x,
                               dy.y,
                               dy.z,
                               dg.x,
                               dg.y,
                               dg.z,
                               rel.x,
                               rel.y,
                               rel.z,
                               lap.x,
                               lap.y,
                               lap.z,
                               nrm.x,
                               nrm.y,
                               nrm.z,
                               100.0 * tr,
                               100.0 * shs,
                               100.0 * mx,
                               fmin(dmin, 1.0),
                               (double)min(nc, 16u) * 0.25,
                               pc.x,
                               pc.y,
                               pc.z,
                               1.0 - (double)cnt / 6.0};
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) o[k] = (float)feat[k];
    }
}

void launch_features(const FeatureView& f, float* out, cudaStream_t st) {
    if (f.n == 0) return;
    k_features<<<grid_for(f.n, 128), 128, 0, st>>>(f, out);
}

__global__ void k_learned_warm_start(FeatureView f, const float* corr, double alpha, double4* alt,
                                     unsigned int* clipped) {
    unsigned int cnt = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < f.n; v += gridDim.x * blockDim.x) {
        if (f.pinned[v]) {
            alt[v] = f.x0[v];
            continue;
        }
        const float* c = corr + (size_t)f.row[v] * kMlpOut;
        d3 p = ld3(f.guess, v) + mk((double)c[0], (double)c[1], (double)c[2]) * (f.unit * alpha);
        if (!isfin(p)) p = ld3(f.guess, v);  // a non-finite prediction falls back per vertex
        d3 ctr = ld3(f.contacts.centers, v);
        d3 d = p - ctr;
        double l = len(d);
        double b = f.contacts.radii[v];
        if (l > b) {  // ContactSet::truncate (src/ogc/world.rs:91-100)
            p = ctr + d * (b / l);
            ++cnt;
        }
        st3(alt, v, p);
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(clipped, cnt);
}

void launch_learned_warm_start(const FeatureView& f, const float* corr, double alpha, double4* alt,
                               unsigned int* clipped, cudaStream_t st) {
    if (f.n == 0) return;
    k_learned_warm_start<<<grid_for(f.n, 256), 256, 0, st>>>(f, corr, alpha, alt, clipped);
}

__global__ void k_targets(FeatureView f, const double4* x, float* targets) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < f.n; v += gridDim.x * blockDim.x) {
        if (f.pinned[v]) continue;
        d3 c = (ld3(x, v) - ld3(f.guess, v)) * (1.0 / f.unit);
        float* o = targets + (size_t)f.row[v] * kMlpOut;
        o[0] = (float)c.x;
        o[1] = (float)c.y;
        o[2] = (float)c.z;
    }
}

void launch_targets(const FeatureView& f, const double4* x, float* targets, cudaStream_t st) {
    if (f.n == 0) return;
    k_targets<<<grid_for(f.n, 256), 256, 0, st>>>(f, x, targets);
}

// ------------------------------------------------------- FP32 inference
// One sample per thread. Weights and biases in shared memory (read as
// warp-wide broadcasts); each layer's input lives in registers and its output
// goes to a per-thread column of shared memory (conflict-free).
constexpr int kFwdBlock = 128;

template <int IN>
__device__ __forceinline__ void dense_gelu(const float* __restrict__ W, const float* __restrict__ b, const float* in,
                                           float* out_col) {
#pragma unroll 1
    for (int i = 0; i < kMlpHidden; i += 2) {
        float a0 = b[i], a1 = b[i + 1];
#pragma unroll
        for (int j = 0; j < IN; ++j) {
            a0 = fmaf(W[i * IN + j], in[j], a0);
            a1 = fmaf(W[(i + 1) * IN + j], in[j], a1);
        }
        out_col[i * kFwdBlock] = gelu_f(a0);
        out_col[(i + 1) * kFwdBlock] = gelu_f(a1);
    }
}

__global__ void __launch_bounds__(kFwdBlock) k_mlp_forward_f32(const float* __restrict__ P, const float* __restrict__ F,
                                                                 uint64_t n, float* __restrict__ out) {
    extern __shared__ float sm[];
    float* w = sm;                       // kMlpParams
    float* act = sm + kMlpParams + 1;    // [64][kFwdBlock]
    for (int i = threadIdx.x; i < kMlpParams; i += kFwdBlock) w[i] = P[i];
    __syncthreads();
    float* col = act + threadIdx.x;
    for (uint64_t s0 = (uint64_t)blockIdx.x * kFwdBlock; s0 < n; s0 += (uint64_t)gridDim.x * kFwdBlock) {
        uint64_t s = s0 + threadIdx.x;
        bool live = s < n;
        float x[kMlpIn];
#pragma unroll
        for (int j = 0; j < kMlpIn; ++j) x[j] = live ? F[s * kMlpIn + j] : 0.0f;
        dense_gelu<kMlpIn>(w + kOffW1, w + kOffB1, x, col);
        float h[kMlpHidden];
#pragma unroll
        for (int j = 0; j < kMlpHidden; ++j) h[j] = col[j * kFwdBlock];
        dense_gelu<kMlpHidden>(w + kOffW2, w + kOffB2, h, col);
#pragma unroll
        for (int j = 0; j < kMlpHidden; ++j) h[j] = col[j * kFwdBlock];
        dense_gelu<kMlpHidden>(w + kOffW3, w + kOffB3, h, col);
#pragma unroll
        for (int j = 0; j < kMlpHidden; ++j) h[j] = col[j * kFwdBlock];
        if (live) {
#pragma unroll
            for (int k = 0; k < kMlpOut; ++k) {
                float a = w[kOffB4 + k];
#pragma unroll
                for (int j = 0; j < kMlpHidden; ++j) a = fmaf(w[kOffW4 + k * kMlpHidden + j], h[j], a);
                out[s * kMlpOut + k] = a;
            }
        }
    }
}

// ------------------------------------------------------------- training
// One CTA of 128 threads processes tiles of 64 samples: forward (two threads
// per sample, 32 units each), loss gradient, back-propagation, and the
// weight gradients of the tile (sum over its samples) added to the CTA's own
// row of `partial`; k_mlp_reduce then sums the rows in a fixed order.
constexpr int kTile = 64;
constexpr int kPitch = kTile + 1;  // row pitch: unit-major rows, one column per sample
constexpr int kTrainBlock = 128;
constexpr int kTrainFloats = kMlpIn * kPitch + 6 * kMlpHidden * kPitch + 2 * kMlpHidden * kPitch + kMlpOut * kPitch;

__device__ __forceinline__ void add_partial(float* row, int p, float v) { row[p] += v; }

// dW[o][i] += sum_s D[o][s] * A[i][s]; db[o] += sum_s D[o][s]
__device__ __forceinline__ void weight_grads(const float* D, const float* A, int outs, int ins, int valid, float* row,
                                             int offW, int offB) {
    int entries = outs * ins + outs;
    for (int e = threadIdx.x; e < entries; e += kTrainBlock) {
        float acc = 0.0f;
        if (e < outs * ins) {
            int o = e / ins, i = e - o * ins;
            const float* d = D + o * kPitch;
            const float* a = A + i * kPitch;
            for (int s = 0; s < valid; ++s) acc = fmaf(d[s], a[s], acc);
            add_partial(row, offW + e, acc);
        } else {
            int o = e - outs * ins;
            const float* d = D + o * kPitch;
            for (int s = 0; s < valid; ++s) acc += d[s];
            add_partial(row, offB + o, acc);
        }
    }
}

// forward of one hidden layer for sample s, units [u0, u0+32)
template <int IN>
__device__ __forceinline__ void fwd_half(const float* __restrict__ P, int offW, int offB, const float* in_rows, int s,
                                         int u0, float* A, float* G) {
    float x[IN];
#pragma unroll
    for (int j = 0; j < IN; ++j) x[j] = in_rows[j * kPitch + s];
#pragma unroll 1
    for (int i = u0; i < u0 + 32; ++i) {
        float z = P[offB + i];
        const float* wr = P + offW + i * IN;
#pragma unroll
        for (int j = 0; j < IN; ++j) z = fmaf(wr[j], x[j], z);
        float a, da;
        gelu_fg(z, a, da);
        A[i * kPitch + s] = a;
        G[i * kPitch + s] = da;
    }
}

// delta of a hidden layer: Dout[i][s] = G[i][s] * sum_o W[o][i] Din[o][s], i in [u0, u0+32)
template <int OUTS>
__device__ __forceinline__ void bwd_half(const float* __restrict__ P, int offW, const float* Din, const float* G, int s,
                                         int u0, float* Dout) {
    float d[OUTS];
#pragma unroll
    for (int o = 0; o < OUTS; ++o) d[o] = Din[o * kPitch + s];
#pragma unroll 1
    for (int i = u0; i < u0 + 32; ++i) {
        float acc = 0.0f;
#pragma unroll
        for (int o = 0; o < OUTS; ++o) acc = fmaf(P[offW + o * kMlpHidden + i], d[o], acc);
        Dout[i * kPitch + s] = G[i * kPitch + s] * acc;
    }
}

__global__ void __launch_bounds__(kTrainBlock) k_mlp_train_tile(const float* __restrict__ P, const float* __restrict__ F,
                                                                  const float* __restrict__ T,
                                                                  const uint32_t* __restrict__ index, uint64_t n,
                                                                  float inv_n, float* partial) {
    extern __shared__ float sm[];
    float* X = sm;                                // [24][pitch]
    float* A1 = X + kMlpIn * kPitch;              // [64][pitch] activations
    float* G1 = A1 + kMlpHidden * kPitch;         // [64][pitch] GELU derivatives
    float* A2 = G1 + kMlpHidden * kPitch;
    float* G2 = A2 + kMlpHidden * kPitch;
    float* A3 = G2 + kMlpHidden * kPitch;
    float* G3 = A3 + kMlpHidden * kPitch;
    float* Da = G3 + kMlpHidden * kPitch;         // [64][pitch] deltas (ping)
    float* Db = Da + kMlpHidden * kPitch;         // (pong)
    float* D4 = Db + kMlpHidden * kPitch;         // [3][pitch]
    float* row = partial + (size_t)blockIdx.x * (kMlpParams + 1);
    const int s = threadIdx.x & (kTile - 1);
    const int half = threadIdx.x >> 6;  // 0 or 1
    const uint64_t tiles = (n + kTile - 1) / kTile;
    float loss = 0.0f;
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint64_t base = tile * kTile;
        int valid = (int)(n - base < (uint64_t)kTile ? n - base : (uint64_t)kTile);
        // inputs (zero columns past the end)
        for (int e = threadIdx.x; e < kMlpIn * kTile; e += kTrainBlock) {
            int ss = e / kMlpIn, j = e - ss * kMlpIn;
            float v = 0.0f;
            if (ss < valid) {
                uint64_t id = index ? index[base + ss] : base + ss;
                v = F[id * kMlpIn + j];
            }
            X[j * kPitch + ss] = v;
        }
        __syncthreads();
        fwd_half<kMlpIn>(P, kOffW1, kOffB1, X, s, half * 32, A1, G1);
        __syncthreads();
        fwd_half<kMlpHidden>(P, kOffW2, kOffB2, A1, s, half * 32, A2, G2);
        __syncthreads();
        fwd_half<kMlpHidden>(P, kOffW3, kOffB3, A2, s, half * 32, A3, G3);
        __syncthreads();
        // output layer and dL/dout = 2 (out - t) / n (zero past the end)
        if (half == 0) {
            float h[kMlpHidden];
#pragma unroll
            for (int j = 0; j < kMlpHidden; ++j) h[j] = A3[j * kPitch + s];
            uint64_t id = s < valid ? (index ? index[base + s] : base + s) : 0;
#pragma unroll
            for (int k = 0; k < kMlpOut; ++k) {
                float o = P[kOffB4 + k];
#pragma unroll
                for (int j = 0; j < kMlpHidden; ++j) o = fmaf(P[kOffW4 + k * kMlpHidden + j], h[j], o);
                float d = 0.0f;
                if (s < valid) {
                    float r = o - T[id * kMlpOut + k];
                    loss += r * r;
                    d = 2.0f * r * inv_n;
                }
                D4[k * kPitch + s] = d;
            }
        }
        __syncthreads();
        weight_grads(D4, A3, kMlpOut, kMlpHidden, valid, row, kOffW4, kOffB4);
        bwd_half<kMlpOut>(P, kOffW4, D4, G3, s, half * 32, Da);
        __syncthreads();
        weight_grads(Da, A2, kMlpHidden, kMlpHidden, valid, row, kOffW3, kOffB3);
        bwd_half<kMlpHidden>(P, kOffW3, Da, G2, s, half * 32, Db);
        __syncthreads();
        weight_grads(Db, A1, kMlpHidden, kMlpHidden, valid, row, kOffW2, kOffB2);
        bwd_half<kMlpHidden>(P, kOffW2, Db, G1, s, half * 32, Da);
        __syncthreads();
        weight_grads(Da, X, kMlpHidden, kMlpIn, valid, row, kOffW1, kOffB1);
        __syncthreads();
    }
    // loss: fixed-order block sum into the last slot of the row
    __shared__ float red[kTrainBlock];
    red[threadIdx.x] = loss;
    __syncthreads();
    for (int o = kTrainBlock / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) row[kMlpParams] = red[0] * inv_n;
}

__global__ void k_mlp_reduce(const float* partial, int rows, float* grads, float* loss) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= kMlpParams; p += gridDim.x * blockDim.x) {
        float a = 0.0f;
        for (int r = 0; r < rows; ++r) a += partial[(size_t)r * (kMlpParams + 1) + p];
        if (p < kMlpParams) grads[p] = a;
        else *loss = a;
    }
}

__global__ void k_adam(float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// ---------------------------------------------------------------- Mlp
namespace {
uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }
}  // namespace

Mlp::Mlp(uint64_t seed) {
    // Glorot-uniform weights (bound sqrt(6 / (fan_in + fan_out))), zero
    // biases; the output layer is scaled by 0.1 so the first corrections
    // are small.
    std::vector<float> h(kMlpParams, 0.0f);
    uint64_t st = seed;
    auto fill = [&](int off, int outs, int ins, double scale) {
        double b = std::sqrt(6.0 / (double)(ins + outs)) * scale;
        for (int k = 0; k < outs * ins; ++k) h[off + k] = (float)((2.0 * uniform01(st) - 1.0) * b);
    };
    fill(kOffW1, kMlpHidden, kMlpIn, 1.0);
    fill(kOffW2, kMlpHidden, kMlpHidden, 1.0);
    fill(kOffW3, kMlpHidden, kMlpHidden, 1.0);
    fill(kOffW4, kMlpOut, kMlpHidden, 0.1);
    p_.upload(h, nullptr);
    for (auto* b : {&m_, &v_, &g_}) {
        b->reserve(kMlpParams);
        b->zero(kMlpParams, nullptr);
    }
    loss_.reserve(1);
    loss_.zero(1, nullptr);
    CC_CUDA(cudaStreamSynchronize(nullptr));
}

void Mlp::set_params(const float* host, cudaStream_t st) {
    CC_CUDA(cudaMemcpyAsync(p_.ptr, host, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
    CC_CUDA(cudaMemsetAsync(m_.ptr, 0, kMlpParams * sizeof(float), st));
    CC_CUDA(cudaMemsetAsync(v_.ptr, 0, kMlpParams * sizeof(float), st));
    CC_CUDA(cudaStreamSynchronize(st));
    t_ = 0;
    w16_valid_ = false;
}

void Mlp::get_params(float* host, cudaStream_t st) const {
    CC_CUDA(cudaMemcpyAsync(host, p_.ptr, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
}

void Mlp::forward(const float* features, uint64_t n, float* out, int precision, cudaStream_t st) {
    if (n == 0) return;
    if (precision == 1) {
        forward_tc(features, n, out, st);
        return;
    }
    size_t smem = (kMlpParams + 1 + kMlpHidden * kFwdBlock) * sizeof(float);
    allow_dynamic_smem(k_mlp_forward_f32, smem);
    uint64_t blocks = (n + kFwdBlock - 1) / kFwdBlock;
    unsigned grid = (unsigned)std::min<uint64_t>(blocks, 148ull * 4ull);
    k_mlp_forward_f32<<<grid, kFwdBlock, smem, st>>>(p_.ptr, features, n, out);
    CC_CUDA(cudaGetLastError());
}

void Mlp::gradients(const float* features, const float* targets, const uint32_t* index, uint64_t n, float* grads,
                    float* loss, cudaStream_t st) {
    if (n == 0) throw Failure{CC_ERR_INVALID_ARGUMENT, "MLP gradients need at least one sample"};
    size_t smem = (size_t)kTrainFloats * sizeof(float);
    allow_dynamic_smem(k_mlp_train_tile, smem);
    uint64_t tiles = (n + kTile - 1) / kTile;
    int rows = (int)std::min<uint64_t>(tiles, 148ull);
    partial_.reserve((size_t)rows * (kMlpParams + 1));
    CC_CUDA(cudaMemsetAsync(partial_.ptr, 0, (size_t)rows * (kMlpParams + 1) * sizeof(float), st));
    k_mlp_train_tile<<<rows, kTrainBlock, smem, st>>>(p_.ptr, features, targets, index, n, 1.0f / (float)n,
                                                      partial_.ptr);
    k_mlp_reduce<<<(kMlpParams + 256) / 256, 256, 0, st>>>(partial_.ptr, rows, grads, loss);
    CC_CUDA(cudaGetLastError());
}

void Mlp::adam(const float* grads, float lr, float beta1, float beta2, float eps, cudaStream_t st) {
    ++t_;
    float c1 = 1.0f - (float)std::pow((double)beta1, (double)t_);
    float c2 = 1.0f - (float)std::pow((double)beta2, (double)t_);
    k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(p_.ptr, m_.ptr, v_.ptr, grads, lr, beta1, beta2, eps, c1, c2);
    CC_CUDA(cudaGetLastError());
    w16_valid_ = false;
}

}  // namespace cc
