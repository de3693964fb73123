// lbm_mlp.cuh -- the learned closure's per-node network on sm_100a.
//
// Network (fixed shape): 16 features -> 32 -> 32 -> 1, GELU after both hidden
// layers in its tanh form (Hendrycks & Gimpel 2016):
//     gelu(x) = 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).  Features of a node, from its stored (post-collision)
// moments m: the 10 moments themselves and the six strain-rate components
// 3 (u_a u_b - m_ab) / (2 scale tau0) (the strain-rate function object's
// formula); each standardised as (f - mean) * scale.  Output y; the closure
// adds dtau = clamp(out_scale * y, dtau_lo, dtau_hi) to the node's relaxation
// time, or nothing when any raw feature lies outside the range seen in
// training (the plain collision is the fallback).
//
// Two evaluations:
//   * mlp_forward_f32: FP32 on CUDA cores (training, reference path);
//   * mlp_infer_kernel: tensor cores.  A CTA of 128 threads takes 128 nodes
//     (one per thread = one row of M = 128): each thread writes its features
//     in FP16 into shared memory in the UMMA canonical K-major layout, one
//     thread issues tcgen05.mma (kind::f16, FP32 accumulators in tensor
//     memory) for 16 -> 32, every warp reads its 32 rows back with
//     tcgen05.ld, applies bias + GELU, writes FP16 activations for 32 -> 32
//     (two K = 16 MMAs into the same 32 tensor-memory columns), reads back,
//     and finishes the 32 -> 1 layer on CUDA cores; the next tile's node
//     values are loaded meanwhile.  Weights are FP16 (converted once on the host into the operand
//     layout), accumulation FP32.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_step.cuh"

namespace lbm {

constexpr int kMlpIn = 16, kMlpHidden = 32;

// FP32 network parameters and normalisation (the C ABI's lbm_mlp layout).
struct MlpParams {
    float w1[kMlpHidden * kMlpIn], b1[kMlpHidden];          // [out][in]
    float w2[kMlpHidden * kMlpHidden], b2[kMlpHidden];
    float w3[kMlpHidden], b3;
    float in_mean[kMlpIn], in_scale[kMlpIn];
    float in_lo[kMlpIn], in_hi[kMlpIn];
    float out_scale, dtau_lo, dtau_hi;
};
constexpr int kMlpWeights = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpHidden + 1;

// Device copy for the tensor-core path: FP16 weights already in the operand
// layout (umma_index), FP32 vectors.
struct MlpDevice {
    __half w1[kMlpHidden * kMlpIn];
    __half w2[kMlpHidden * kMlpHidden];
    float b1[kMlpHidden], b2[kMlpHidden], w3[kMlpHidden], b3;
    float in_scale[kMlpIn], in_shift[kMlpIn], in_lo[kMlpIn], in_hi[kMlpIn];  // x = f * scale + shift
    float out_scale, dtau_lo, dtau_hi;
    float r_ii, r_ij;  // 1 / (2 * 4.5 * tau0), 1 / (2 * 9 * tau0) for the strain-rate features
};

// Element (row, k) of a rows x K FP16 operand in the K-major, no-swizzle
// canonical layout: core matrices of 8 rows x 8 elements (16 B per row,
// 128 B each), consecutive along the rows (stride 128 B, the descriptor's
// SBO), K-chunks of 8 a whole row-extent apart (rows/8 * 128 B, the LBO).
__host__ __device__ constexpr int umma_index(int row, int k, int rows)
{
    return ((k >> 3) * (rows >> 3) + (row >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

constexpr float kGeluA = 0.79788456080286536f, kGeluB = 0.044715f;  // sqrt(2/pi), cubic coefficient

// accurate tanh (training and the FP32 path)
__device__ __forceinline__ float gelu(float x)
{
    return 0.5f * x * (1.0f + tanhf(kGeluA * fmaf(kGeluB * x * x, x, x)));
}
// hardware tanh (tanh.approx.f32; its error is below the FP16 rounding of
// the activations that follow) for the tensor-core path
__device__ __forceinline__ float gelu_fast(float x)
{
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(kGeluA * fmaf(kGeluB * x * x, x, x)));
    return 0.5f * x * (1.0f + t);
}

// One row (one node) of an FP16 operand in umma_index layout: K values, stored
// as K/8 16-byte vectors (consecutive rows are consecutive 16-byte slots of a
// core matrix, so a warp's stores do not conflict).
template <int K>
__device__ __forceinline__ void store_row_f16(__half *base, int row, const float *v)
{
#pragma unroll
    for (int c = 0; c < K / 8; c++) {
        __align__(16) __half2 h[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            h[j] = __floats2half2_rn(v[8 * c + 2 * j], v[8 * c + 2 * j + 1]);
        *reinterpret_cast<uint4 *>(base + umma_index(row, 8 * c, 128)) = *reinterpret_cast<const uint4 *>(h);
    }
}

// The 16 raw features of a node from its 10 stored moments (rho - 1, 3u, ...).
// Products and sums are rounded separately (no contraction), so a host
// restatement in FP32 reproduces them exactly.
__device__ __forceinline__ void node_features(const float *m, float r_ii, float r_ij, float *f)
{
#pragma unroll
    for (int k = 0; k < 10; k++)
        f[k] = m[k];
    const float u = m[1], v = m[2], w = m[3];
    const float uu[6] = {__fmul_rn(u, u), __fmul_rn(u, v), __fmul_rn(u, w),
                         __fmul_rn(v, v), __fmul_rn(v, w), __fmul_rn(w, w)};
    const int mi[6] = {4, 5, 6, 7, 8, 9};
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const float r = (c == 0 || c == 3 || c == 5) ? r_ii : r_ij;
        f[10 + c] = __fmul_rn(__fmul_rn(3.0f, __fsub_rn(uu[c], m[mi[c]])), r);
    }
}

// 1 if every raw feature lies inside [lo, hi].
template <typename P>
__device__ __forceinline__ bool in_range(const float *f, const P &p)
{
    bool ok = true;
#pragma unroll
    for (int k = 0; k < kMlpIn; k++)
        ok &= (f[k] >= p.in_lo[k]) & (f[k] <= p.in_hi[k]);
    return ok;
}

// FP32 forward on CUDA cores; also returns the hidden activations the
// backward pass needs (pre-activations z1, z2 and activations h1, h2).
__device__ __forceinline__ float mlp_forward_f32(const MlpParams &p, const float *xs, float *z1, float *h1, float *z2,
                                                 float *h2)
{
#pragma unroll 4
    for (int j = 0; j < kMlpHidden; j++) {
        float a = p.b1[j];
#pragma unroll
        for (int k = 0; k < kMlpIn; k++)
            a = fmaf(p.w1[j * kMlpIn + k], xs[k], a);
        z1[j] = a;
        h1[j] = gelu(a);
    }
    float y = p.b3;
#pragma unroll 4
    for (int j = 0; j < kMlpHidden; j++) {
        float a = p.b2[j];
#pragma unroll
        for (int k = 0; k < kMlpHidden; k++)
            a = fmaf(p.w2[j * kMlpHidden + k], h1[k], a);
        z2[j] = a;
        h2[j] = gelu(a);
        y = fmaf(p.w3[j], h2[j], y);
    }
    return y;
}

// ------------------------------------------------------------ tcgen05 PTX
// Shared-memory operand descriptor, K-major, no swizzle (sm_100 format:
// start >> 4 in bits 0-13, LBO >> 4 in 16-29, SBO >> 4 in 32-45, version 1
// in bits 46-47, layout type 0).
__device__ __forceinline__ uint64_t umma_desc(const void *smem_start, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    const uint64_t a = (smem_u32(smem_start) >> 4) & 0x3FFFu;
    return a | (uint64_t((lbo_bytes >> 4) & 0x3FFFu) << 16) | (uint64_t((sbo_bytes >> 4) & 0x3FFFu) << 32) |
           (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: D FP32 (bit 4), A and B FP16
// (formats 0), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
template <int M, int N>
__host__ __device__ constexpr uint32_t umma_idesc_f16_f32()
{
    static_assert(M == 128 && N % 16 == 0 && N >= 16 && N <= 256, "shape");
    return (1u << 4) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// One MMA, issued by the threads with `pred` (exactly one thread of the CTA):
// D[tmem] (+)= A[smem] * B[smem]^T.
__device__ __forceinline__ void umma_f16_if(bool pred, uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                            uint32_t idesc, bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "setp.ne.u32 q, %5, 0;\n\t"
        "@p tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, q;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(unsigned(pred)), "r"(unsigned(accumulate))
        : "memory");
}
// Make `bar` track completion of this thread's earlier MMAs (one arrival).
__device__ __forceinline__ void umma_commit_if(bool pred, uint64_t *bar)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "@p tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}" ::"r"(smem_u32(bar)),
        "r"(unsigned(pred))
        : "memory");
}
__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
// Whole-warp tensor-memory allocation (columns a power of two >= 32); the
// base address is written to shared memory.
__device__ __forceinline__ void tmem_alloc_warp(uint32_t *smem_result, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_result)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 32 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld_32cols(uint32_t taddr, float *v)
{
    __syncwarp();  // .sync.aligned: the lanes may leave a bounded wait at different times
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++)
        v[j] = __uint_as_float(r[j]);
}

// ------------------------------------------------------- inference kernel
// Shared memory of mlp_infer_kernel (byte offsets; operands 128 B aligned).
struct MlpSmem {
    static constexpr int W1 = 0;                          // 32 x 16 FP16, 1 KB
    static constexpr int W2 = W1 + kMlpHidden * kMlpIn * 2;   // 32 x 32 FP16, 2 KB
    static constexpr int A1 = W2 + kMlpHidden * kMlpHidden * 2;  // 128 x 16 FP16, 4 KB
    static constexpr int A2 = A1 + 128 * kMlpIn * 2;          // 128 x 32 FP16, 8 KB
    static constexpr int BAR = A2 + 128 * kMlpHidden * 2;     // mbarrier
    static constexpr int TMEM = BAR + 8;                      // allocated tensor-memory address
    static constexpr int FLAG = TMEM + 4;                     // abort flag
    static constexpr int BYTES = FLAG + 4;
    // shared memory requested per CTA: with at most 14 CTAs on an SM (227 KB),
    // their 14 x 32 tensor-memory columns never exceed the SM's 512
    static constexpr int LAUNCH_BYTES = 16 * 1024;
    // leading (K-chunk) byte offsets of the operands; the stride between
    // 8-row groups is 128 B for all of them
    static constexpr uint32_t LBO_W = (kMlpHidden / 8) * 128, LBO_A = (128 / 8) * 128, SBO = 128;
};

enum : unsigned { ERR_MMA_TIMEOUT = 2u };

// The network is a kernel parameter (constant bank: its uniform values feed
// instructions directly).  Source of a node's 16 raw features: stored moments [10][N] (FROM_MOMENTS)
// or a feature array [N][16].  Output dtau[N] (clamped, 0 where the inputs
// leave the training range), or the raw network output y[N] (RAW_Y).
template <bool FROM_MOMENTS, bool RAW_Y>
__global__ void __launch_bounds__(128, 8) mlp_infer_kernel(const float *src, size_t N,
                                                           const __grid_constant__ MlpDevice net, float *out,
                                                           unsigned *err, uint64_t timeout_ns)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __half *w1 = reinterpret_cast<__half *>(sm + MlpSmem::W1);
    __half *w2 = reinterpret_cast<__half *>(sm + MlpSmem::W2);
    __half *a1 = reinterpret_cast<__half *>(sm + MlpSmem::A1);
    __half *a2 = reinterpret_cast<__half *>(sm + MlpSmem::A2);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + MlpSmem::BAR);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + MlpSmem::TMEM);
    int *flag = reinterpret_cast<int *>(sm + MlpSmem::FLAG);
    const int tid = threadIdx.x, warp = tid >> 5;
    const bool leader = tid == 0;

    // weights (already in operand layout) into shared memory
    for (int i = tid; i < kMlpHidden * kMlpIn; i += 128)
        w1[i] = net.w1[i];
    for (int i = tid; i < kMlpHidden * kMlpHidden; i += 128)
        w2[i] = net.w2[i];
    mbar_init_if(leader, bar);
    fence_mbar_init_if(leader);
    *flag = 0;
    __syncwarp();
    if (warp == 0)
        tmem_alloc_warp(tmem_slot, 32);  // 32 FP32 columns: layer 1, then layer 2
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    cta_sync();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = uint32_t(warp * 32) << 16;
    constexpr uint32_t idesc = umma_idesc_f16_f32<128, kMlpHidden>();
    const uint64_t d_w1 = umma_desc(w1, MlpSmem::LBO_W, MlpSmem::SBO);
    const uint64_t d_a1 = umma_desc(a1, MlpSmem::LBO_A, MlpSmem::SBO);
    unsigned phase = 0;

    const size_t tiles = (N + 127) / 128;
    // node values of the next tile are loaded while the current one computes
    auto load = [&](size_t tile, float *v) {
        const size_t node = tile * 128 + tid;
        if (tile < tiles && node < N) {
            if constexpr (FROM_MOMENTS) {
#pragma unroll
                for (int k = 0; k < 10; k++)
                    v[k] = src[size_t(k) * N + node];
            } else {
#pragma unroll
                for (int k = 0; k < kMlpIn; k++)
                    v[k] = src[node * kMlpIn + k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < kMlpIn; k++)
                v[k] = 0.0f;
        }
    };
    constexpr int NV = FROM_MOMENTS ? 10 : kMlpIn;
    float next[kMlpIn];
    load(blockIdx.x, next);
    for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const size_t node = tile * 128 + tid;
        const bool valid = node < N;
        float f[kMlpIn];
        if constexpr (FROM_MOMENTS) {
            node_features(next, net.r_ii, net.r_ij, f);
        } else {
#pragma unroll
            for (int k = 0; k < kMlpIn; k++)
                f[k] = next[k];
        }
        (void)NV;
        load(tile + gridDim.x, next);
        const bool inside = valid && in_range(f, net);
        // layer 1 operand: this thread's row of standardised features
#pragma unroll
        for (int k = 0; k < kMlpIn; k++)
            f[k] = fmaf(f[k], net.in_scale[k], net.in_shift[k]);
        store_row_f16<kMlpIn>(a1, tid, f);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        cta_sync();
        tc_fence_after();
        umma_f16_if(leader, tmem, d_a1, d_w1, idesc, false);
        umma_commit_if(leader, bar);
        if (!mbar_wait_bounded(bar, phase, timeout_ns)) {
            atomicOr(err, ERR_MMA_TIMEOUT);
            *flag = 1;
        }
        phase ^= 1u;
        tc_fence_after();
        float h[kMlpHidden];
        tmem_ld_32cols(tmem + lane_base, h);
#pragma unroll
        for (int j = 0; j < kMlpHidden; j++)
            h[j] = gelu_fast(h[j] + net.b1[j]);
        store_row_f16<kMlpHidden>(a2, tid, h);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        // every thread has read its layer-1 accumulators (tcgen05.wait::ld):
        // layer 2 may overwrite the same columns
        tc_fence_before();
        cta_sync();
        if (*flag)
            break;
        tc_fence_after();
        // layer 2: K = 32 as two K = 16 steps
#pragma unroll
        for (int s = 0; s < 2; s++)
            umma_f16_if(leader, tmem, umma_desc(a2 + s * 2 * (MlpSmem::LBO_A / 2), MlpSmem::LBO_A, MlpSmem::SBO),
                        umma_desc(w2 + s * 2 * (MlpSmem::LBO_W / 2), MlpSmem::LBO_W, MlpSmem::SBO), idesc, s > 0);
        umma_commit_if(leader, bar);
        if (!mbar_wait_bounded(bar, phase, timeout_ns)) {
            atomicOr(err, ERR_MMA_TIMEOUT);
            *flag = 1;
        }
        phase ^= 1u;
        tc_fence_after();
        tmem_ld_32cols(tmem + lane_base, h);
        float y = net.b3;
#pragma unroll
        for (int j = 0; j < kMlpHidden; j++)
            y = fmaf(net.w3[j], gelu_fast(h[j] + net.b2[j]), y);
        if (valid) {
            if constexpr (RAW_Y)
                out[node] = y;
            else
                out[node] = inside ? fminf(fmaxf(net.out_scale * y, net.dtau_lo), net.dtau_hi) : 0.0f;
        }
        tc_fence_before();
        cta_sync();
        if (*flag)
            break;
    }
    if (*flag) {
        // an MMA did not complete in time: give it a bounded chance to
        // finish before its tensor memory is released
        (void)mbar_wait_bounded(bar, phase ^ 1u, 1000000ull);
    }
    tc_fence_before();
    cta_sync();
    tc_fence_after();
    if (warp == 0)
        tmem_dealloc_warp(tmem, 32);
}

}  // namespace lbm
