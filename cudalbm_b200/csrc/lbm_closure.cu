// lbm_closure.cu -- the learned closure (lbm_closure_*, lbm_trainer_*,
// lbm_mlp_*, lbm_perturb_velocity, lbm_filter_2to1 of include/lbm_b200.h).
//
// A per-node MLP predicts a correction dtau to the relaxation time of an
// under-resolved run.  Pieces:
//   * training data: a fine run (perturbed initial velocities) is box-filtered
//     2:1 onto the coarse grid at coarse times t and t+1 (two fine steps),
//     with its non-equilibrium stresses rescaled to the coarse lattice;
//     the coarse solver advances the filtered state F(t) one plain step to C;
//     the target at each interior node is the dtau for which the node's
//     collision would have produced F(t+1) instead of C, to first order:
//         C(omega) = (1 - omega) pre + omega eq  =>  dC/domega = -neq_post / (1 - omega)
//         domega   = -(1 - omega) (r . neq_post) / (neq_post . neq_post),  r = F(t+1) - C
//     over the six second-order moments, dtau = 1 / (omega + domega) - tau0;
//   * training: FP32 forward/backward kernels on CUDA cores (one thread per
//     sample, then one thread per parameter summing over the CTA's samples),
//     Adam on the device, mean squared error on standardised targets;
//   * inference: mlp_infer_kernel (lbm_mlp.cuh, tensor cores) writes dtau for
//     every node from the current moments, then closure_kernel steps with it.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "lbm_b200.h"
#include "lbm_handle.hpp"
#include "lbm_mlp.cuh"
#include "lbm_step.cuh"

static_assert(sizeof(lbm_mlp) == sizeof(lbm::MlpParams), "lbm_mlp must mirror lbm::MlpParams");

namespace {

using lbm::kMlpHidden;
using lbm::kMlpIn;
using lbm::kMlpWeights;
using lbm::MlpDevice;
using lbm::MlpParams;

lbm_status fail(lbm_status s, const std::string &m) { return lbm::record_error(s, m); }

__host__ __device__ inline uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// uniform in [-1, 1) from a 64-bit hash (24 random bits)
__device__ inline float hash_sym(uint64_t h) { return float(int64_t(h >> 40) - (1ll << 23)) * (1.0f / float(1 << 23)); }

dim3 grid_for(size_t n) { return dim3(unsigned(std::min<size_t>((n + 255) / 256, size_t(148) * 16))); }

// ------------------------------------------------------- data kernels
// u, v, w (stored as 3u) of interior nodes += 3 * amplitude * U[-1, 1).
__global__ void perturb_kernel(float *m, int nx, int ny, int nz, float amp3, uint64_t seed)
{
    const size_t N = size_t(nx) * ny * nz;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / (size_t(nx) * ny));
        if (lbm::node_type(x, y, z, nx, ny, nz))
            continue;
        for (int c = 1; c <= 3; c++)
            m[size_t(c) * N + i] += amp3 * hash_sym(splitmix64(seed * 0x100000001B3ull + i * 4 + c));
    }
}

// Coarse node (X, Y, Z) from fine nodes (2X + a, 2Y + b, 2Z + c): the mean of
// rho - 1 and 3u, and for the second-order moments the mean of their
// equilibrium part (u_a u_b in stored units, which keeps the subgrid part
// mean(u_a u_b) - mean(u_a) mean(u_b)) plus kappa times the mean of their
// non-equilibrium part, which the coarse lattice carries kappa times larger
// (grid-refinement rescaling, see lbm_filter_2to1).
__global__ void filter_kernel(float *coarse, const float *fine, int nx, int ny, int nz, float kappa)
{
    const size_t Nc = size_t(nx) * ny * nz, Nf = Nc * 8;
    const int fx = 2 * nx, fy = 2 * ny;
    for (size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < Nc; j += size_t(gridDim.x) * blockDim.x) {
        const int x = int(j % nx), y = int((j / nx) % ny), z = int(j / (size_t(nx) * ny));
        float sum[10] = {}, eq[6] = {};
        for (int c = 0; c < 2; c++)
            for (int b = 0; b < 2; b++)
                for (int a = 0; a < 2; a++) {
                    const size_t i = size_t(2 * x + a) + size_t(fx) * (size_t(2 * y + b) + size_t(fy) * size_t(2 * z + c));
                    float m[10];
                    for (int k = 0; k < 10; k++)
                        m[k] = fine[size_t(k) * Nf + i];
                    for (int k = 0; k < 10; k++)
                        sum[k] += m[k];
                    eq[0] += 0.5f * m[1] * m[1];
                    eq[1] += m[1] * m[2];
                    eq[2] += m[1] * m[3];
                    eq[3] += 0.5f * m[2] * m[2];
                    eq[4] += m[2] * m[3];
                    eq[5] += 0.5f * m[3] * m[3];
                }
        for (int k = 0; k < 4; k++)
            coarse[size_t(k) * Nc + j] = sum[k] * 0.125f;
        for (int k = 0; k < 6; k++)
            coarse[size_t(4 + k) * Nc + j] = (eq[k] + kappa * (sum[4 + k] - eq[k])) * 0.125f;
    }
}

// kappa = 2 (tau_c / tau_f) (1 - omega_c) / (1 - omega_f): the ratio of the
// stored (post-collision) non-equilibrium moments on the two lattices for the
// same flow.  Pre-collision they scale with tau * S, S per lattice step twice
// as large on the coarse lattice (dt_c = 2 dt_f at equal lattice velocity);
// the collision multiplies them by (1 - omega).
float refinement_kappa(const lbm_handle *fine, const lbm_handle *coarse)
{
    return 2.0f * (coarse->tau / fine->tau) * (1.0f - coarse->omega) / (1.0f - fine->omega);
}

// Sample selection and target of node i (see the file header); false if the
// node gives no sample (boundary, off-stride, too little non-equilibrium
// stress for a stable ratio, or an unusable relaxation rate).
struct TargetArgs {
    const float *f0, *f1, *c;
    const double *acc;  // per node (sum r.neq, sum neq.neq) over a window of transitions, or null
    int nx, ny, nz;
    unsigned stride;
    float omega, tau0, r_ii, r_ij;
    double min_den;
};
// One transition's least-squares terms at node i: r . neq and neq . neq over
// the six second-order moments (r = F(t+1) - C, neq = C's non-equilibrium part).
__device__ void transition_terms(const TargetArgs &a, size_t i, size_t N, double &num, double &den)
{
    float cm[10];
    for (int k = 0; k < 10; k++)
        cm[k] = a.c[size_t(k) * N + i];
    const float u = cm[1], v = cm[2], w = cm[3];
    const float eq[6] = {0.5f * u * u, u * v, u * w, 0.5f * v * v, v * w, 0.5f * w * w};
    num = 0.0;
    den = 0.0;
    for (int k = 0; k < 6; k++) {
        const double neq = double(cm[4 + k]) - double(eq[k]);
        const double r = double(a.f1[size_t(4 + k) * N + i] - cm[4 + k]);
        num += r * neq;
        den += neq * neq;
    }
}
__device__ bool node_target(const TargetArgs &a, size_t i, float &dtau)
{
    const size_t N = size_t(a.nx) * a.ny * a.nz;
    if (i >= N || i % a.stride)
        return false;
    const int x = int(i % a.nx), y = int((i / a.nx) % a.ny), z = int(i / (size_t(a.nx) * a.ny));
    if (lbm::node_type(x, y, z, a.nx, a.ny, a.nz))
        return false;
    double num, den;
    if (a.acc) {
        num = a.acc[2 * i];
        den = a.acc[2 * i + 1];
    } else {
        transition_terms(a, i, N, num, den);
    }
    if (!(den > a.min_den))
        return false;
    const double w_new = double(a.omega) - double(1.0f - a.omega) * num / den;
    if (!(w_new > 0.0) || !(w_new < 2.0))
        return false;
    dtau = float(1.0 / w_new - double(a.tau0));
    return isfinite(dtau);
}

// Adds one transition's terms to the window sums of every interior node.
__global__ void accumulate_terms_kernel(TargetArgs a, double *acc)
{
    const size_t N = size_t(a.nx) * a.ny * a.nz;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % a.nx), y = int((i / a.nx) % a.ny), z = int(i / (size_t(a.nx) * a.ny));
        if (lbm::node_type(x, y, z, a.nx, a.ny, a.nz))
            continue;
        double num, den;
        transition_terms(a, i, N, num, den);
        acc[2 * i] += num;
        acc[2 * i + 1] += den;
    }
}

// Samples are stored in node order, whatever the scheduling: CTA b owns the
// nodes [b * kChunk, (b + 1) * kChunk); pass 1 counts its samples, the host
// turns the counts into offsets, pass 2 writes them with in-CTA ranks from
// warp ballots.
constexpr int kSampleCta = 256;
constexpr size_t kChunk = 8 * kSampleCta;

__global__ void __launch_bounds__(kSampleCta) count_samples_kernel(TargetArgs a, unsigned *counts)
{
    const size_t base = size_t(blockIdx.x) * kChunk;
    unsigned n = 0;
    for (size_t r = 0; r < kChunk; r += kSampleCta) {
        float d;
        n += node_target(a, base + r + threadIdx.x, d);
    }
    for (int o = 16; o > 0; o >>= 1)
        n += __shfl_down_sync(0xffffffffu, n, o);
    __shared__ unsigned warp_n[kSampleCta / 32];
    if ((threadIdx.x & 31) == 0)
        warp_n[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < kSampleCta / 32; w++)
            t += warp_n[w];
        counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kSampleCta) write_samples_kernel(TargetArgs a, const unsigned long long *offsets,
                                                                   float *feat, float *targ, unsigned long long cap)
{
    __shared__ unsigned warp_n[kSampleCta / 32];
    const size_t N = size_t(a.nx) * a.ny * a.nz;
    const size_t base = size_t(blockIdx.x) * kChunk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long next = offsets[blockIdx.x];
    for (size_t r = 0; r < kChunk; r += kSampleCta) {
        const size_t i = base + r + threadIdx.x;
        float dtau = 0.0f;
        const bool ok = node_target(a, i, dtau);
        const unsigned ballot = __ballot_sync(0xffffffffu, ok);
        if (lane == 0)
            warp_n[warp] = __popc(ballot);
        __syncthreads();
        unsigned before = 0, total = 0;
        for (int w = 0; w < kSampleCta / 32; w++) {
            before += w < warp ? warp_n[w] : 0u;
            total += warp_n[w];
        }
        const unsigned long long slot = next + before + __popc(ballot & ((1u << lane) - 1u));
        if (ok && slot < cap) {
            float m[10], fv[kMlpIn];
            for (int k = 0; k < 10; k++)
                m[k] = a.f0[size_t(k) * N + i];
            lbm::node_features(m, a.r_ii, a.r_ij, fv);
            for (int k = 0; k < kMlpIn; k++)
                feat[slot * kMlpIn + k] = fv[k];
            targ[slot] = dtau;
        }
        next += total;
        __syncthreads();
    }
}

// ----------------------------------------------------- training kernels
// d gelu / dz of the tanh form
__device__ __forceinline__ float gelu_grad(float z)
{
    const float t = tanhf(lbm::kGeluA * fmaf(lbm::kGeluB * z * z, z, z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * lbm::kGeluA * fmaf(3.0f * lbm::kGeluB, z * z, 1.0f);
}

// Mean squared error gradient over a batch.  Sample s of the batch is
// first + s (sequential) or hash(seed, s) % n (random).  Phase 1: one thread
// per sample, forward and backward, per-sample factors into shared memory;
// phase 2: one thread per parameter sums its products over the CTA's samples
// and adds them to grad (FP32 atomics).
constexpr int kTrainCta = 128;
struct TrainSmem {
    MlpParams p;
    float xs[kTrainCta][kMlpIn];
    float h1[kTrainCta][kMlpHidden], h2[kTrainCta][kMlpHidden];
    float dz1[kTrainCta][kMlpHidden], dz2[kTrainCta][kMlpHidden];
    float dy[kTrainCta];
};

__global__ void __launch_bounds__(kTrainCta) grad_kernel(const float *feat, const float *targ, uint64_t n,
                                                         uint64_t first, uint64_t batch, uint64_t seed, int random,
                                                         const MlpParams *params, float *partial, double *loss_partial)
{
    extern __shared__ __align__(16) unsigned char raw[];
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(raw);
    const int t = threadIdx.x;
    for (int i = t; i < int(sizeof(MlpParams) / 4); i += kTrainCta)
        reinterpret_cast<float *>(&S.p)[i] = reinterpret_cast<const float *>(params)[i];
    __syncthreads();
    const uint64_t s = uint64_t(blockIdx.x) * kTrainCta + t;
    float xs[kMlpIn], z1[kMlpHidden], h1[kMlpHidden], z2[kMlpHidden], h2[kMlpHidden];
    float dy = 0.0f, e2 = 0.0f;
    if (s < batch) {
        const uint64_t idx = random ? splitmix64(seed ^ (s * 0xD6E8FEB86659FD93ull)) % n : first + s;
        for (int k = 0; k < kMlpIn; k++)
            xs[k] = (feat[idx * kMlpIn + k] - S.p.in_mean[k]) * S.p.in_scale[k];
        const float y = lbm::mlp_forward_f32(S.p, xs, z1, h1, z2, h2);
        const float ts = fminf(fmaxf(targ[idx], S.p.dtau_lo), S.p.dtau_hi) / S.p.out_scale;
        const float e = y - ts;
        e2 = e * e;
        dy = 2.0f * e / float(batch);
    } else {
        for (int k = 0; k < kMlpIn; k++)
            xs[k] = 0.0f;
        for (int j = 0; j < kMlpHidden; j++)
            z1[j] = h1[j] = z2[j] = h2[j] = 0.0f;
    }
    float dz2[kMlpHidden];
    for (int j = 0; j < kMlpHidden; j++)
        dz2[j] = dy * S.p.w3[j] * gelu_grad(z2[j]);
    for (int k = 0; k < kMlpHidden; k++) {
        float a = 0.0f;
        for (int j = 0; j < kMlpHidden; j++)
            a = fmaf(dz2[j], S.p.w2[j * kMlpHidden + k], a);
        S.dz1[t][k] = a * gelu_grad(z1[k]);
        S.h1[t][k] = h1[k];
        S.h2[t][k] = h2[k];
        S.dz2[t][k] = dz2[k];
    }
    for (int k = 0; k < kMlpIn; k++)
        S.xs[t][k] = xs[k];
    S.dy[t] = dy;
    // CTA sum of the squared errors, in a fixed order
    double e2d = double(e2);
    for (int o = 16; o > 0; o >>= 1)
        e2d += __shfl_down_sync(0xffffffffu, e2d, o);
    __shared__ double warp_e2[kTrainCta / 32];
    if ((t & 31) == 0)
        warp_e2[t >> 5] = e2d;
    __syncthreads();
    if (t == 0) {
        double sum = 0.0;
        for (int w = 0; w < kTrainCta / 32; w++)
            sum += warp_e2[w];
        loss_partial[blockIdx.x] = sum;
    }
    // phase 2: parameter p (the lbm_mlp weight order w1, b1, w2, b2, w3, b3)
    for (int p = t; p < kMlpWeights; p += kTrainCta) {
        float acc = 0.0f;
        int q = p;
        if (q < kMlpHidden * kMlpIn) {
            const int j = q / kMlpIn, i = q % kMlpIn;
            for (int r = 0; r < kTrainCta; r++)
                acc = fmaf(S.dz1[r][j], S.xs[r][i], acc);
        } else if ((q -= kMlpHidden * kMlpIn) < kMlpHidden) {
            for (int r = 0; r < kTrainCta; r++)
                acc += S.dz1[r][q];
        } else if ((q -= kMlpHidden) < kMlpHidden * kMlpHidden) {
            const int j = q / kMlpHidden, k = q % kMlpHidden;
            for (int r = 0; r < kTrainCta; r++)
                acc = fmaf(S.dz2[r][j], S.h1[r][k], acc);
        } else if ((q -= kMlpHidden * kMlpHidden) < kMlpHidden) {
            for (int r = 0; r < kTrainCta; r++)
                acc += S.dz2[r][q];
        } else if ((q -= kMlpHidden) < kMlpHidden) {
            for (int r = 0; r < kTrainCta; r++)
                acc = fmaf(S.dy[r], S.h2[r][q], acc);
        } else {
            for (int r = 0; r < kTrainCta; r++)
                acc += S.dy[r];
        }
        partial[size_t(blockIdx.x) * kMlpWeights + p] = acc;
    }
}

// Sum of the CTAs' partial gradients (and losses), in CTA order.
__global__ void reduce_partials_kernel(const float *partial, const double *loss_partial, int ctas, float *grad,
                                       double *loss)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kMlpWeights) {
        float s = 0.0f;
        for (int b = 0; b < ctas; b++)
            s += partial[size_t(b) * kMlpWeights + p];
        grad[p] = s;
    }
    if (p == 0) {
        double l = 0.0;
        for (int b = 0; b < ctas; b++)
            l += loss_partial[b];
        *loss = l;
    }
}

// Adam (Kingma & Ba 2015) over the kMlpWeights leading floats of MlpParams.
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, float lr, float c1, float c2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpWeights)
        return;
    const float b1 = 0.9f, b2 = 0.999f;
    m[p] = b1 * m[p] + (1.0f - b1) * g[p];
    v[p] = b2 * v[p] + (1.0f - b2) * g[p] * g[p];
    w[p] -= lr * (m[p] * c1) / (sqrtf(v[p] * c2) + 1e-8f);
}

// FP32 forward over host-provided features: raw network output y.
__global__ void forward_kernel(const float *feat, uint64_t n, const MlpParams *params, float *y)
{
    __shared__ MlpParams P;
    for (int i = threadIdx.x; i < int(sizeof(MlpParams) / 4); i += blockDim.x)
        reinterpret_cast<float *>(&P)[i] = reinterpret_cast<const float *>(params)[i];
    __syncthreads();
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s < n; s += uint64_t(gridDim.x) * blockDim.x) {
        float xs[kMlpIn], z1[kMlpHidden], h1[kMlpHidden], z2[kMlpHidden], h2[kMlpHidden];
        for (int k = 0; k < kMlpIn; k++)
            xs[k] = (feat[s * kMlpIn + k] - P.in_mean[k]) * P.in_scale[k];
        y[s] = lbm::mlp_forward_f32(P, xs, z1, h1, z2, h2);
    }
}

// ------------------------------------------------------------- helpers
MlpDevice device_copy(const MlpParams &p, float tau0)
{
    MlpDevice d{};
    for (int n = 0; n < kMlpHidden; n++) {
        for (int k = 0; k < kMlpIn; k++)
            d.w1[lbm::umma_index(n, k, kMlpHidden)] = __float2half_rn(p.w1[n * kMlpIn + k]);
        for (int k = 0; k < kMlpHidden; k++)
            d.w2[lbm::umma_index(n, k, kMlpHidden)] = __float2half_rn(p.w2[n * kMlpHidden + k]);
    }
    std::memcpy(d.b1, p.b1, sizeof(d.b1));
    std::memcpy(d.b2, p.b2, sizeof(d.b2));
    std::memcpy(d.w3, p.w3, sizeof(d.w3));
    d.b3 = p.b3;
    std::memcpy(d.in_scale, p.in_scale, sizeof(d.in_scale));
    for (int k = 0; k < kMlpIn; k++)
        d.in_shift[k] = -p.in_mean[k] * p.in_scale[k];
    std::memcpy(d.in_lo, p.in_lo, sizeof(d.in_lo));
    std::memcpy(d.in_hi, p.in_hi, sizeof(d.in_hi));
    d.out_scale = p.out_scale;
    d.dtau_lo = p.dtau_lo;
    d.dtau_hi = p.dtau_hi;
    d.r_ii = 1.0f / (2.0f * 4.5f * tau0);
    d.r_ij = 1.0f / (2.0f * 9.0f * tau0);
    return d;
}

lbm_status launch_infer(const float *src, size_t N, const MlpDevice &net, float *out, unsigned *err, bool from_moments,
                        bool raw_y, cudaStream_t stream, int device)
{
    void *fn = from_moments ? (raw_y ? (void *)&lbm::mlp_infer_kernel<true, true> : (void *)&lbm::mlp_infer_kernel<true, false>)
                            : (raw_y ? (void *)&lbm::mlp_infer_kernel<false, true> : (void *)&lbm::mlp_infer_kernel<false, false>);
    static_assert(lbm::MlpSmem::BYTES <= lbm::MlpSmem::LAUNCH_BYTES, "layout");
    // the shared-memory attribute and the SM count, once per kernel and
    // device (these calls are far slower than a launch)
    struct Known {
        const void *fn;
        int device, sms;
    };
    static std::mutex mu;
    static std::vector<Known> known;
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (const Known &k : known)
            if (k.fn == fn && k.device == device)
                sms = k.sms;
        if (sms == 0) {
            LBM_CUDA_RETURN(
                cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lbm::MlpSmem::LAUNCH_BYTES));
            LBM_CUDA_RETURN(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
            known.push_back({fn, device, sms});
        }
    }
    const size_t tiles = (N + 127) / 128;
    // persistent: one wave of the CTAs the register budget keeps resident
    // (at most 8 per SM by shared memory, so their 32 tensor-memory columns
    // each fit the SM's 512)
    const unsigned grid = unsigned(std::min<size_t>(tiles, size_t(sms) * lbm::kMlpCtasPerSm));
    uint64_t timeout = 2000000000ull;
    MlpDevice net_arg = net;
    void *args[] = {&src, &N, &net_arg, &out, &err, &timeout};
    LBM_CUDA_RETURN(cudaLaunchKernel(fn, dim3(grid), dim3(128), args, lbm::MlpSmem::LAUNCH_BYTES, stream));
    return LBM_OK;
}

bool pick_closure(int Q, int tx, int ty, int stages, int npb, void *&fn, size_t &smem)
{
#define LBM_CLOSURE_SHAPE(QQ, TXX)                                                                             \
    if (Q == QQ && tx == TXX && ty == 8 && stages == 2 && npb == 1) {                                        \
        fn = reinterpret_cast<void *>(&lbm::closure_kernel<QQ, TXX, 8, 2, 1, 3>);                             \
        smem = lbm::SmemLayout<QQ, TXX, 8, 2, 1, float>::bytes;                                              \
        return true;                                                                                         \
    }
    LBM_CLOSURE_SHAPE(19, 32)
    LBM_CLOSURE_SHAPE(19, 16)
    LBM_CLOSURE_SHAPE(19, 8)
    LBM_CLOSURE_SHAPE(27, 32)
    LBM_CLOSURE_SHAPE(27, 16)
    LBM_CLOSURE_SHAPE(27, 8)
#undef LBM_CLOSURE_SHAPE
    return false;
}

// The closure kernel with the network fused in, for a handle's kernel shape
// (tiles of 128 or 256 threads); false: the shape has none.
bool pick_closure_fused(int Q, int tx, int ty, int stages, int npb, void *&fn, size_t &smem)
{
#define LBM_FUSED_SHAPE(QQ, TXX, MINB)                                                                        \
    if (Q == QQ && tx == TXX && ty == 8 && stages == 2 && npb == 1) {                                       \
        fn = reinterpret_cast<void *>(&lbm::closure_fused_kernel<QQ, TXX, 8, 2, 1, MINB>);                   \
        smem = lbm::FusedLayout<QQ, TXX, 8, 2, 1>::bytes;                                                   \
        return true;                                                                                        \
    }
    LBM_FUSED_SHAPE(19, 32, 2)
    LBM_FUSED_SHAPE(19, 16, 4)
    LBM_FUSED_SHAPE(27, 32, 2)
    LBM_FUSED_SHAPE(27, 16, 4)
#undef LBM_FUSED_SHAPE
    return false;
}
// shared memory of the fused shapes against the CTAs per SM their launch bounds assume
static_assert(2 * (lbm::FusedLayout<27, 32, 8, 2, 1>::bytes + 1024) <= 228 * 1024, "fused 32x8: 2 CTAs per SM");
static_assert(4 * (lbm::FusedLayout<27, 16, 8, 2, 1>::bytes + 1024) <= 228 * 1024, "fused 16x8: 4 CTAs per SM");

}  // namespace

// ------------------------------------------------------------ trainer
struct lbm_trainer {
    int device = 0;
    uint64_t cap = 0;
    float *feat = nullptr, *targ = nullptr;
    uint64_t n = 0;            // samples stored (at most cap)
    float *scratch = nullptr;  // F(t) copy and filtered F(t+1) of the coarse grid
    unsigned *counts = nullptr;            // per-CTA sample counts of one lbm_trainer_add
    unsigned long long *offsets = nullptr;  // and their offsets
    size_t count_slots = 0;
    size_t scratch_floats = 0;
    cudaStream_t stream = nullptr;
};

namespace lbm {

// One step of a handle with the closure: dtau from the current moments on
// the tensor cores, then the closure step kernel.
lbm_status closure_step(lbm_handle *h)
{
    void *ffn = nullptr;
    size_t fsmem = 0;
    if (h->closure_fused && h->closure_every == 1 &&
        pick_closure_fused(h->Q, h->launcher.tx, h->launcher.ty, h->launcher.stages, h->launcher.pop_buffers, ffn,
                           fsmem)) {
        // the network inside the step kernel: no dtau array, one launch
        struct Known {
            const void *fn;
            int device;
        };
        static std::mutex mu;
        static std::vector<Known> known;
        {
            std::lock_guard<std::mutex> lock(mu);
            bool seen = false;
            for (const Known &k : known)
                seen |= (k.fn == ffn && k.device == h->cfg.device);
            if (!seen) {
                LBM_CUDA_RETURN(cudaFuncSetAttribute(ffn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(fsmem)));
                known.push_back({ffn, h->cfg.device});
            }
        }
        StepParams<float, float> p{};
        const int nxt = h->cur ^ 1;
        p.out = static_cast<float *>(h->m[nxt]);
        p.nx = int(h->cfg.nx);
        p.ny = int(h->cfg.ny);
        p.nz = int(h->cfg.nz);
        p.zc = h->zc;
        p.z_lo = 0;
        p.z_hi = p.nz;
        p.rx = Relax{h->omega, h->t_omega, h->omega_d2, h->tau, h->cfg.u_inf};
        p.fault = h->err;
        p.timeout_ns = 2000000000ull;
        MlpDevice net = *h->mlp;
        const dim3 block(h->launcher.tx, h->launcher.ty);
        const dim3 grid(unsigned((h->cfg.nx + h->launcher.tx - 1) / h->launcher.tx),
                        unsigned((h->cfg.ny + h->launcher.ty - 1) / h->launcher.ty),
                        unsigned((h->cfg.nz + h->zc - 1) / h->zc));
        void *args[] = {&h->tmap[h->cur], &p, &net};
        LBM_CUDA_RETURN(cudaLaunchKernel(ffn, grid, block, args, fsmem, h->stream));
        h->closure_steps++;
        h->dtau_current = false;
        h->last_input_kept = true;
        h->cur = nxt;
        h->t += 1;
        h->launches += 1;
        return LBM_OK;
    }
    if (h->closure_steps++ % uint64_t(h->closure_every) == 0) {
        lbm_status s = launch_infer(static_cast<const float *>(h->m[h->cur]), h->N, *h->mlp, h->dtau,
                                    &h->err->flags, true, false, h->stream, h->cfg.device);
        if (s != LBM_OK)
            return s;
        h->launches += 1;
        h->dtau_current = true;
    }
    void *fn = nullptr;
    size_t smem = 0;
    if (!pick_closure(h->Q, h->launcher.tx, h->launcher.ty, h->launcher.stages, h->launcher.pop_buffers, fn, smem))
        return fail(LBM_ERR_STATE, "closure: the handle's kernel shape has no closure variant");
    StepParams<float, float> p{};
    const int nxt = h->cur ^ 1;
    p.out = static_cast<float *>(h->m[nxt]);
    p.nx = int(h->cfg.nx);
    p.ny = int(h->cfg.ny);
    p.nz = int(h->cfg.nz);
    p.zc = h->zc;
    p.z_lo = 0;
    p.z_hi = p.nz;
    p.rx = Relax{h->omega, h->t_omega, h->omega_d2, h->tau, h->cfg.u_inf};
    p.fault = h->err;
    p.timeout_ns = 2000000000ull;
    p.dtau = h->dtau;
    const dim3 block(h->launcher.tx, h->launcher.ty);
    const dim3 grid(unsigned((h->cfg.nx + h->launcher.tx - 1) / h->launcher.tx),
                    unsigned((h->cfg.ny + h->launcher.ty - 1) / h->launcher.ty),
                    unsigned((h->cfg.nz + h->zc - 1) / h->zc));
    void *args[] = {&h->tmap[h->cur], &p};
    LBM_CUDA_RETURN(cudaLaunchKernel(fn, grid, block, args, smem, h->stream));
    h->cur = nxt;
    h->t += 1;
    h->launches += 1;
    return LBM_OK;
}

}  // namespace lbm

extern "C" {

lbm_status lbm_perturb_velocity(lbm_handle *h, float amplitude, uint64_t seed)
{
    if (!h)
        return fail(LBM_ERR_ARG, "null handle");
    if (h->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_ARG, "lbm_perturb_velocity: FP32 storage only");
    LBM_CUDA_RETURN(cudaSetDevice(h->cfg.device));
    perturb_kernel<<<grid_for(h->N), 256, 0, h->stream>>>(static_cast<float *>(h->m[h->cur]), int(h->cfg.nx),
                                                          int(h->cfg.ny), int(h->cfg.nz), 3.0f * amplitude, seed);
    LBM_CUDA_RETURN(cudaGetLastError());
    h->launches += 1;
    LBM_CUDA_RETURN(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_filter_2to1(lbm_handle *fine, lbm_handle *coarse)
{
    if (!fine || !coarse)
        return fail(LBM_ERR_ARG, "null handle");
    if (fine->cfg.nx != 2 * coarse->cfg.nx || fine->cfg.ny != 2 * coarse->cfg.ny || fine->cfg.nz != 2 * coarse->cfg.nz)
        return fail(LBM_ERR_ARG, "lbm_filter_2to1: the fine mesh must be twice the coarse mesh in every direction");
    if (fine->storage != LBM_STORAGE_F32 || coarse->storage != LBM_STORAGE_F32 || fine->cfg.device != coarse->cfg.device)
        return fail(LBM_ERR_ARG, "lbm_filter_2to1: FP32 storage on one device");
    LBM_CUDA_RETURN(cudaSetDevice(fine->cfg.device));
    LBM_CUDA_RETURN(cudaStreamSynchronize(fine->stream));
    filter_kernel<<<grid_for(coarse->N), 256, 0, coarse->stream>>>(
        static_cast<float *>(coarse->m[coarse->cur]), static_cast<const float *>(fine->m[fine->cur]),
        int(coarse->cfg.nx), int(coarse->cfg.ny), int(coarse->cfg.nz), refinement_kappa(fine, coarse));
    LBM_CUDA_RETURN(cudaGetLastError());
    coarse->launches += 1;
    LBM_CUDA_RETURN(cudaStreamSynchronize(coarse->stream));
    return LBM_OK;
}

lbm_status lbm_trainer_create(int32_t device, uint64_t capacity, lbm_trainer **out)
{
    if (!out || capacity == 0)
        return fail(LBM_ERR_ARG, "lbm_trainer_create: null output or zero capacity");
    *out = nullptr;
    LBM_CUDA_RETURN(cudaSetDevice(device));
    lbm_trainer *t = new lbm_trainer();
    t->device = device;
    t->cap = capacity;
    if (cudaMalloc(&t->feat, capacity * kMlpIn * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&t->targ, capacity * sizeof(float)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) != cudaSuccess) {
        lbm_trainer_destroy(t);
        return fail(LBM_ERR_NOMEM, "lbm_trainer_create: cannot allocate the sample buffers");
    }
    *out = t;
    return LBM_OK;
}

lbm_status lbm_trainer_destroy(lbm_trainer *t)
{
    if (!t)
        return LBM_OK;
    cudaSetDevice(t->device);
    if (t->stream)
        cudaStreamSynchronize(t->stream);
    for (void *p : {static_cast<void *>(t->feat), static_cast<void *>(t->targ), static_cast<void *>(t->counts),
                    static_cast<void *>(t->offsets), static_cast<void *>(t->scratch)})
        if (p)
            cudaFree(p);
    if (t->stream)
        cudaStreamDestroy(t->stream);
    delete t;
    return LBM_OK;
}

}  // extern "C"

namespace {

TargetArgs target_args(const lbm_handle *coarse, const float *f0, const float *f1, uint32_t stride, float min_neq,
                       uint32_t window)
{
    TargetArgs a;
    a.f0 = f0;
    a.f1 = f1;
    a.c = static_cast<const float *>(coarse->m[coarse->cur]);
    a.acc = nullptr;
    a.nx = int(coarse->cfg.nx);
    a.ny = int(coarse->cfg.ny);
    a.nz = int(coarse->cfg.nz);
    a.stride = stride;
    a.omega = coarse->omega;
    a.tau0 = coarse->tau;
    a.r_ii = 1.0f / (2.0f * 4.5f * coarse->tau);
    a.r_ij = 1.0f / (2.0f * 9.0f * coarse->tau);
    // the threshold is on the RMS non-equilibrium stress of a transition
    a.min_den = std::max(1e-24, 6.0 * double(min_neq) * double(min_neq)) * double(window);
    return a;
}

// Count, then write, the samples of targets a (node order) after the stored ones.
lbm_status store_samples(lbm_trainer *t, lbm_handle *coarse, const TargetArgs &a, uint64_t *total)
{
    const size_t N = coarse->N;
    const size_t ctas = (N + kChunk - 1) / kChunk;
    if (t->count_slots < ctas) {
        cudaFree(t->counts);
        cudaFree(t->offsets);
        t->counts = nullptr;
        t->offsets = nullptr;
        t->count_slots = 0;
        LBM_CUDA_RETURN(cudaMalloc(&t->counts, ctas * sizeof(unsigned)));
        LBM_CUDA_RETURN(cudaMalloc(&t->offsets, ctas * sizeof(unsigned long long)));
        t->count_slots = ctas;
    }
    count_samples_kernel<<<unsigned(ctas), kSampleCta, 0, coarse->stream>>>(a, t->counts);
    LBM_CUDA_RETURN(cudaGetLastError());
    std::vector<unsigned> counts(ctas);
    std::vector<unsigned long long> offsets(ctas);
    LBM_CUDA_RETURN(cudaMemcpyAsync(counts.data(), t->counts, ctas * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                    coarse->stream));
    LBM_CUDA_RETURN(cudaStreamSynchronize(coarse->stream));
    unsigned long long run = t->n;
    for (size_t b = 0; b < ctas; b++) {
        offsets[b] = run;
        run += counts[b];
    }
    LBM_CUDA_RETURN(cudaMemcpyAsync(t->offsets, offsets.data(), ctas * sizeof(unsigned long long),
                                    cudaMemcpyHostToDevice, coarse->stream));
    write_samples_kernel<<<unsigned(ctas), kSampleCta, 0, coarse->stream>>>(a, t->offsets, t->feat, t->targ, t->cap);
    LBM_CUDA_RETURN(cudaGetLastError());
    LBM_CUDA_RETURN(cudaStreamSynchronize(coarse->stream));
    coarse->launches += 3;
    t->n = std::min<uint64_t>(run, t->cap);
    if (total)
        *total = t->n;
    return LBM_OK;
}

}  // namespace

extern "C" {

lbm_status lbm_trainer_add(lbm_trainer *t, lbm_handle *coarse, lbm_handle *fine_next, uint32_t stride, float min_neq,
                           uint64_t *total)
{
    if (!t || !coarse || !fine_next || stride == 0)
        return fail(LBM_ERR_ARG, "lbm_trainer_add: null argument or zero stride");
    if (coarse->closure || coarse->cfg.function_objects || coarse->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_ARG, "lbm_trainer_add: the coarse handle must run the plain FP32 method without function objects");
    if (fine_next->cfg.nx != 2 * coarse->cfg.nx || fine_next->cfg.ny != 2 * coarse->cfg.ny ||
        fine_next->cfg.nz != 2 * coarse->cfg.nz || fine_next->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_ARG, "lbm_trainer_add: the fine mesh must be twice the coarse mesh (FP32)");
    if (coarse->cfg.device != t->device || fine_next->cfg.device != t->device)
        return fail(LBM_ERR_ARG, "lbm_trainer_add: handles on another device");
    LBM_CUDA_RETURN(cudaSetDevice(t->device));
    const size_t N = coarse->N;
    if (t->scratch_floats < 20 * N) {
        if (t->scratch)
            cudaFree(t->scratch);
        t->scratch = nullptr;
        t->scratch_floats = 0;
        LBM_CUDA_RETURN(cudaMalloc(&t->scratch, 20 * N * sizeof(float)));
        t->scratch_floats = 20 * N;
    }
    float *f0 = t->scratch, *f1 = t->scratch + 10 * N;
    LBM_CUDA_RETURN(cudaStreamSynchronize(fine_next->stream));
    LBM_CUDA_RETURN(cudaStreamSynchronize(coarse->stream));
    LBM_CUDA_RETURN(cudaMemcpyAsync(f0, coarse->m[coarse->cur], 10 * N * sizeof(float), cudaMemcpyDeviceToDevice,
                                    coarse->stream));
    filter_kernel<<<grid_for(N), 256, 0, coarse->stream>>>(f1, static_cast<const float *>(fine_next->m[fine_next->cur]),
                                                           int(coarse->cfg.nx), int(coarse->cfg.ny), int(coarse->cfg.nz),
                                                           refinement_kappa(fine_next, coarse));
    LBM_CUDA_RETURN(cudaGetLastError());
    lbm_status s = lbm_step(coarse, 1);
    if (s != LBM_OK)
        return s;
    TargetArgs a = target_args(coarse, f0, f1, stride, min_neq, 1);
    return store_samples(t, coarse, a, total);
}

lbm_status lbm_trainer_add_window(lbm_trainer *t, lbm_handle *coarse, lbm_handle *fine, uint32_t window,
                                  uint32_t stride, float min_neq, uint64_t *total)
{
    if (!t || !coarse || !fine || stride == 0 || window == 0)
        return fail(LBM_ERR_ARG, "lbm_trainer_add_window: null argument, zero stride or zero window");
    if (coarse->closure || coarse->cfg.function_objects || coarse->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_ARG, "lbm_trainer_add_window: the coarse handle must run the plain FP32 method without function objects");
    if (fine->closure || fine->cfg.nx != 2 * coarse->cfg.nx || fine->cfg.ny != 2 * coarse->cfg.ny ||
        fine->cfg.nz != 2 * coarse->cfg.nz || fine->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_ARG, "lbm_trainer_add_window: the fine mesh must be twice the coarse mesh (plain FP32)");
    if (coarse->cfg.device != t->device || fine->cfg.device != t->device)
        return fail(LBM_ERR_ARG, "lbm_trainer_add_window: handles on another device");
    LBM_CUDA_RETURN(cudaSetDevice(t->device));
    const size_t N = coarse->N;
    // F(t) (the features), F(t+j+1), and the per-node window sums (2 doubles)
    const size_t need = 24 * N;
    if (t->scratch_floats < need) {
        if (t->scratch)
            cudaFree(t->scratch);
        t->scratch = nullptr;
        t->scratch_floats = 0;
        LBM_CUDA_RETURN(cudaMalloc(&t->scratch, need * sizeof(float)));
        t->scratch_floats = need;
    }
    float *fstart = t->scratch, *f1 = t->scratch + 10 * N;
    double *acc = reinterpret_cast<double *>(t->scratch + 20 * N);
    LBM_CUDA_RETURN(cudaStreamSynchronize(fine->stream));
    LBM_CUDA_RETURN(cudaStreamSynchronize(coarse->stream));
    LBM_CUDA_RETURN(cudaMemcpyAsync(fstart, coarse->m[coarse->cur], 10 * N * sizeof(float), cudaMemcpyDeviceToDevice,
                                    coarse->stream));
    LBM_CUDA_RETURN(cudaMemsetAsync(acc, 0, 2 * N * sizeof(double), coarse->stream));
    const int nx = int(coarse->cfg.nx), ny = int(coarse->cfg.ny), nz = int(coarse->cfg.nz);
    const float kappa = refinement_kappa(fine, coarse);
    for (uint32_t j = 0; j < window; j++) {
        // the coarse handle holds F(t+j); the fine run advances one coarse step
        lbm_status s = lbm_step(fine, 2);
        if (s != LBM_OK)
            return s;
        LBM_CUDA_RETURN(cudaStreamSynchronize(fine->stream));
        filter_kernel<<<grid_for(N), 256, 0, coarse->stream>>>(f1, static_cast<const float *>(fine->m[fine->cur]), nx,
                                                               ny, nz, kappa);
        LBM_CUDA_RETURN(cudaGetLastError());
        if ((s = lbm_step(coarse, 1)) != LBM_OK)  // C: one coarse step from F(t+j)
            return s;
        TargetArgs a = target_args(coarse, fstart, f1, stride, min_neq, window);
        accumulate_terms_kernel<<<grid_for(N), 256, 0, coarse->stream>>>(a, acc);
        LBM_CUDA_RETURN(cudaGetLastError());
        coarse->launches += 2;
        if (j + 1 < window)  // the next transition starts from the filtered F(t+j+1)
            LBM_CUDA_RETURN(cudaMemcpyAsync(coarse->m[coarse->cur], f1, 10 * N * sizeof(float),
                                            cudaMemcpyDeviceToDevice, coarse->stream));
    }
    TargetArgs a = target_args(coarse, fstart, f1, stride, min_neq, window);
    a.acc = acc;
    return store_samples(t, coarse, a, total);
}

lbm_status lbm_trainer_samples(lbm_trainer *t, uint64_t first, uint64_t count, float *features, float *targets,
                               uint64_t *total)
{
    if (!t)
        return fail(LBM_ERR_ARG, "null trainer");
    LBM_CUDA_RETURN(cudaSetDevice(t->device));
    const uint64_t n = t->n;
    if (total)
        *total = n;
    if (count == 0)
        return LBM_OK;
    if (first + count > n)
        return fail(LBM_ERR_ARG, "lbm_trainer_samples: range beyond the stored samples");
    if (features)
        LBM_CUDA_RETURN(cudaMemcpy(features, t->feat + first * kMlpIn, count * kMlpIn * sizeof(float),
                                   cudaMemcpyDeviceToHost));
    if (targets)
        LBM_CUDA_RETURN(cudaMemcpy(targets, t->targ + first, count * sizeof(float), cudaMemcpyDeviceToHost));
    return LBM_OK;
}

lbm_status lbm_trainer_gradient(lbm_trainer *t, const lbm_mlp *net, uint64_t first, uint64_t count, lbm_mlp *grad,
                                double *loss)
{
    if (!t || !net || !grad || count == 0)
        return fail(LBM_ERR_ARG, "null argument or empty range");
    uint64_t n = 0;
    lbm_status s = lbm_trainer_samples(t, 0, 0, nullptr, nullptr, &n);
    if (s != LBM_OK)
        return s;
    if (first + count > n)
        return fail(LBM_ERR_ARG, "lbm_trainer_gradient: range beyond the stored samples");
    const unsigned ctas = unsigned((count + kTrainCta - 1) / kTrainCta);
    MlpParams *dp = nullptr;
    float *dg = nullptr, *dpart = nullptr;
    double *dl = nullptr, *dlpart = nullptr;
    auto release = [&]() {
        cudaFree(dp);
        cudaFree(dg);
        cudaFree(dl);
        cudaFree(dpart);
        cudaFree(dlpart);
    };
    if (cudaMalloc(&dp, sizeof(MlpParams)) != cudaSuccess || cudaMalloc(&dg, sizeof(MlpParams)) != cudaSuccess ||
        cudaMalloc(&dl, sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dpart, size_t(ctas) * kMlpWeights * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dlpart, ctas * sizeof(double)) != cudaSuccess) {
        release();
        return fail(LBM_ERR_NOMEM, "lbm_trainer_gradient: no device memory");
    }
    cudaMemcpy(dp, net, sizeof(MlpParams), cudaMemcpyHostToDevice);
    cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(TrainSmem)));
    grad_kernel<<<ctas, kTrainCta, sizeof(TrainSmem), t->stream>>>(t->feat, t->targ, n, first, count, 0, 0, dp,
                                                                   dpart, dlpart);
    reduce_partials_kernel<<<(kMlpWeights + 255) / 256, 256, 0, t->stream>>>(dpart, dlpart, int(ctas), dg, dl);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(t->stream);
    if (e == cudaSuccess) {
        std::memset(grad, 0, sizeof(*grad));
        e = cudaMemcpy(grad, dg, kMlpWeights * sizeof(float), cudaMemcpyDeviceToHost);
    }
    double l = 0.0;
    if (e == cudaSuccess)
        e = cudaMemcpy(&l, dl, sizeof(double), cudaMemcpyDeviceToHost);
    release();
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("lbm_trainer_gradient: ") + cudaGetErrorString(e));
    if (loss)
        *loss = l / double(count);
    return LBM_OK;
}

lbm_status lbm_trainer_fit(lbm_trainer *t, const lbm_train_options *opt, lbm_mlp *net, lbm_train_report *rep)
{
    if (!t || !opt || !net)
        return fail(LBM_ERR_ARG, "null argument");
    if (opt->batch <= 0 || opt->steps <= 0 || !(opt->lr > 0.0f) || !(opt->dtau_hi > opt->dtau_lo))
        return fail(LBM_ERR_ARG, "lbm_trainer_fit: batch, steps, lr must be positive and dtau_lo < dtau_hi");
    uint64_t n = 0;
    lbm_status s = lbm_trainer_samples(t, 0, 0, nullptr, nullptr, &n);
    if (s != LBM_OK)
        return s;
    if (n < 16)
        return fail(LBM_ERR_STATE, "lbm_trainer_fit: fewer than 16 samples");
    // normalisation and ranges on the host (deterministic)
    std::vector<float> F(n * kMlpIn), T(n);
    if ((s = lbm_trainer_samples(t, 0, n, F.data(), T.data(), nullptr)) != LBM_OK)
        return s;
    MlpParams P{};
    for (int k = 0; k < kMlpIn; k++) {
        double sum = 0.0, sq = 0.0;
        float lo = F[k], hi = F[k];
        for (uint64_t i = 0; i < n; i++) {
            const double v = F[i * kMlpIn + k];
            sum += v;
            sq += v * v;
            lo = std::min(lo, F[i * kMlpIn + k]);
            hi = std::max(hi, F[i * kMlpIn + k]);
        }
        const double mean = sum / double(n), var = std::max(sq / double(n) - mean * mean, 0.0);
        P.in_mean[k] = float(mean);
        P.in_scale[k] = var > 0.0 ? float(1.0 / std::sqrt(var)) : 1.0f;
        P.in_lo[k] = lo;
        P.in_hi[k] = hi;
    }
    double tsum = 0.0, tsq = 0.0;
    for (uint64_t i = 0; i < n; i++) {
        const double v = std::min(std::max(T[i], opt->dtau_lo), opt->dtau_hi);
        tsum += v;
        tsq += v * v;
    }
    const double tvar = std::max(tsq / double(n) - (tsum / double(n)) * (tsum / double(n)), 0.0);
    P.out_scale = float(tvar > 0.0 ? std::sqrt(tvar + (tsum / double(n)) * (tsum / double(n))) : 1.0);
    P.dtau_lo = opt->dtau_lo;
    P.dtau_hi = opt->dtau_hi;
    // Glorot-uniform initial weights, zero biases
    std::mt19937_64 rng(opt->seed);
    auto uni = [&](float a) { return float((double(rng() >> 11) * 0x1.0p-53 * 2.0 - 1.0) * a); };
    const float a1 = std::sqrt(6.0f / (kMlpIn + kMlpHidden)), a2 = std::sqrt(6.0f / (2 * kMlpHidden)),
                a3 = std::sqrt(6.0f / (kMlpHidden + 1));
    for (float &w : P.w1)
        w = uni(a1);
    for (float &w : P.w2)
        w = uni(a2);
    for (float &w : P.w3)
        w = uni(a3);
    LBM_CUDA_RETURN(cudaSetDevice(t->device));
    const uint64_t B = uint64_t(opt->batch);
    const unsigned blocks = unsigned((B + kTrainCta - 1) / kTrainCta);
    MlpParams *dp = nullptr;
    float *dg = nullptr, *dm = nullptr, *dv = nullptr, *dpart = nullptr;
    double *dl = nullptr, *dlpart = nullptr;
    auto release = [&]() {
        cudaFree(dp);
        cudaFree(dg);
        cudaFree(dm);
        cudaFree(dv);
        cudaFree(dl);
        cudaFree(dpart);
        cudaFree(dlpart);
    };
    if (cudaMalloc(&dp, sizeof(MlpParams)) != cudaSuccess || cudaMalloc(&dg, kMlpWeights * 4) != cudaSuccess ||
        cudaMalloc(&dm, kMlpWeights * 4) != cudaSuccess || cudaMalloc(&dv, kMlpWeights * 4) != cudaSuccess ||
        cudaMalloc(&dl, sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dpart, size_t(blocks) * kMlpWeights * 4) != cudaSuccess ||
        cudaMalloc(&dlpart, blocks * sizeof(double)) != cudaSuccess) {
        release();
        return fail(LBM_ERR_NOMEM, "lbm_trainer_fit: no device memory");
    }
    cudaMemcpy(dp, &P, sizeof(P), cudaMemcpyHostToDevice);
    cudaMemset(dm, 0, kMlpWeights * 4);
    cudaMemset(dv, 0, kMlpWeights * 4);
    cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(TrainSmem)));
    double first_loss = -1.0, last_loss = 0.0;
    const int window = std::max(1, std::min(opt->steps / 10, 100));
    double acc = 0.0;
    int acc_n = 0;
    for (int step = 0; step < opt->steps; step++) {
        grad_kernel<<<blocks, kTrainCta, sizeof(TrainSmem), t->stream>>>(
            t->feat, t->targ, n, 0, B, splitmix64(opt->seed + 0x51ED27ull * uint64_t(step + 1)), 1, dp, dpart, dlpart);
        reduce_partials_kernel<<<(kMlpWeights + 255) / 256, 256, 0, t->stream>>>(dpart, dlpart, int(blocks), dg, dl);
        const float c1 = 1.0f / (1.0f - std::pow(0.9f, float(step + 1)));
        const float c2 = 1.0f / (1.0f - std::pow(0.999f, float(step + 1)));
        adam_kernel<<<(kMlpWeights + 255) / 256, 256, 0, t->stream>>>(reinterpret_cast<float *>(dp), dg, dm, dv,
                                                                       opt->lr, c1, c2);
        if (step < window || step >= opt->steps - window) {
            double l = 0.0;
            cudaMemcpyAsync(&l, dl, sizeof(double), cudaMemcpyDeviceToHost, t->stream);
            cudaStreamSynchronize(t->stream);
            acc += l / double(B);
            if (++acc_n == window) {
                if (first_loss < 0.0)
                    first_loss = acc / window;
                else
                    last_loss = acc / window;
                acc = 0.0;
                acc_n = 0;
            }
        }
    }
    cudaError_t e = cudaStreamSynchronize(t->stream);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpy(&P, dp, sizeof(P), cudaMemcpyDeviceToHost);
    release();
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("lbm_trainer_fit: ") + cudaGetErrorString(e));
    std::memcpy(net, &P, sizeof(P));
    if (rep) {
        rep->samples = n;
        rep->steps = uint64_t(opt->steps);
        rep->loss_first = first_loss;
        rep->loss_last = last_loss;
        rep->target_rms = P.out_scale;
    }
    return LBM_OK;
}

lbm_status lbm_mlp_infer(int32_t device, const lbm_mlp *net, const float *features, uint64_t n, float *y,
                         int32_t tensor_cores)
{
    if (!net || !features || !y || n == 0)
        return fail(LBM_ERR_ARG, "null argument or no samples");
    LBM_CUDA_RETURN(cudaSetDevice(device));
    MlpParams P;
    std::memcpy(&P, net, sizeof(P));
    float *df = nullptr, *dy = nullptr;
    void *dn = nullptr;
    unsigned *derr = nullptr;
    auto release = [&]() {
        cudaFree(df);
        cudaFree(dy);
        cudaFree(dn);
        cudaFree(derr);
    };
    if (cudaMalloc(&df, n * kMlpIn * 4) != cudaSuccess || cudaMalloc(&dy, n * 4) != cudaSuccess ||
        cudaMalloc(&dn, std::max(sizeof(MlpDevice), sizeof(MlpParams))) != cudaSuccess ||
        cudaMalloc(&derr, 4) != cudaSuccess) {
        release();
        return fail(LBM_ERR_NOMEM, "lbm_mlp_infer: no device memory");
    }
    cudaMemcpy(df, features, n * kMlpIn * 4, cudaMemcpyHostToDevice);
    cudaMemset(derr, 0, 4);
    lbm_status s = LBM_OK;
    if (tensor_cores) {
        s = launch_infer(df, n, device_copy(P, 1.0f), dy, derr, false, true, nullptr, device);
    } else {
        cudaMemcpy(dn, &P, sizeof(P), cudaMemcpyHostToDevice);
        forward_kernel<<<grid_for(n), 256>>>(df, n, static_cast<const MlpParams *>(dn), dy);
    }
    cudaError_t e = cudaDeviceSynchronize();
    unsigned flags = 0;
    if (e == cudaSuccess)
        e = cudaMemcpy(y, dy, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&flags, derr, 4, cudaMemcpyDeviceToHost);
    release();
    if (s != LBM_OK)
        return s;
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("lbm_mlp_infer: ") + cudaGetErrorString(e));
    if (flags)
        return fail(LBM_ERR_TIMEOUT, "lbm_mlp_infer: a tensor-core MMA did not complete in time");
    return LBM_OK;
}

lbm_status lbm_closure_set(lbm_handle *h, const lbm_mlp *net)
{
    if (!h)
        return fail(LBM_ERR_ARG, "null handle");
    LBM_CUDA_RETURN(cudaSetDevice(h->cfg.device));
    if (!net) {
        h->closure = false;
        return LBM_OK;
    }
    if (h->cfg.function_objects || h->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_ARG, "lbm_closure_set: the closure runs with FP32 storage and no function objects");
    if (!(net->dtau_lo <= net->dtau_hi) || !(h->tau + net->dtau_lo > 0.5f))
        return fail(LBM_ERR_ARG, "lbm_closure_set: need dtau_lo <= dtau_hi and tau + dtau_lo > 0.5");
    void *fn;
    size_t smem;
    if (!pick_closure(h->Q, h->launcher.tx, h->launcher.ty, h->launcher.stages, h->launcher.pop_buffers, fn, smem)) {
        // move to the closure's kernel shape (same results, other tiling)
        const int tx = h->cfg.nx % 32 == 0 ? 32 : (h->cfg.nx % 16 == 0 ? 16 : 8);
        lbm_status s = lbm::retile(h, tx, 8, 2, 1, h->zc);
        if (s != LBM_OK)
            return s;
        pick_closure(h->Q, h->launcher.tx, h->launcher.ty, h->launcher.stages, h->launcher.pop_buffers, fn, smem);
    }
    LBM_CUDA_RETURN(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    if (!h->dtau) {
        LBM_CUDA_RETURN(cudaMalloc(&h->dtau, h->N * sizeof(float)));
        h->device_bytes += h->N * sizeof(float);
        LBM_CUDA_RETURN(cudaMemsetAsync(h->dtau, 0, h->N * sizeof(float), h->stream));
    }
    if (!h->mlp)
        h->mlp = new MlpDevice();
    MlpParams P;
    std::memcpy(&P, net, sizeof(P));
    *h->mlp = device_copy(P, h->tau);
    h->closure = true;
    h->closure_steps = 0;
    return LBM_OK;
}

lbm_status lbm_closure_fused(lbm_handle *h, int32_t on)
{
    if (!h)
        return fail(LBM_ERR_ARG, "lbm_closure_fused: null handle");
    h->closure_fused = on != 0;
    return LBM_OK;
}

lbm_status lbm_closure_refresh(lbm_handle *h, int32_t every)
{
    if (!h || every < 1)
        return fail(LBM_ERR_ARG, "lbm_closure_refresh: null handle or interval below 1");
    h->closure_every = every;
    h->closure_steps = 0;
    return LBM_OK;
}

lbm_status lbm_closure_dtau(lbm_handle *h, float *host, size_t count)
{
    if (!h || !host)
        return fail(LBM_ERR_ARG, "null argument");
    if (!h->dtau)
        return fail(LBM_ERR_STATE, "lbm_closure_dtau: no closure on this handle");
    if (count != h->N)
        return fail(LBM_ERR_ARG, "lbm_closure_dtau: count must be the node count");
    LBM_CUDA_RETURN(cudaSetDevice(h->cfg.device));
    if (!h->dtau_current) {
        // the last step evaluated the network inside the step kernel: the
        // same network on that step's input state (the other moment buffer,
        // while nothing has overwritten it) gives its dtau bit for bit;
        // otherwise the state has been replaced since, and the network on
        // the current state gives the dtau the next step will use
        const void *src = h->last_input_kept ? h->m[h->cur ^ 1] : h->m[h->cur];
        lbm_status s = launch_infer(static_cast<const float *>(src), h->N, *h->mlp, h->dtau, &h->err->flags, true,
                                    false, h->stream, h->cfg.device);
        if (s != LBM_OK)
            return s;
        h->launches += 1;
        h->dtau_current = true;
    }
    LBM_CUDA_RETURN(cudaMemcpyAsync(host, h->dtau, count * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    LBM_CUDA_RETURN(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

}  // extern "C"
