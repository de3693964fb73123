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
//   * mlp_infer_kernel: the two hidden layers on the tensor cores.  A CTA of
//     128 threads takes 128 nodes (one per thread = one row of M = 128): each
//     thread writes its standardised features in FP16 into shared memory in
//     the UMMA canonical K-major layout, one thread issues tcgen05.mma
//     (kind::f16, FP32 accumulators in tensor memory), every warp reads its
//     32 rows back with tcgen05.ld, adds the biases in FP32, applies GELU in
//     packed FP16 (two values per instruction, tanh.approx.f16x2) and writes
//     the FP16 activations as the layer-2 operand; the 32 -> 1 layer runs on
//     CUDA cores in FP32 from the FP16 activations.  An MMA costs the tensor
//     pipe about the same time for any N up to 128 (measured: ~126 cycles
//     per M = 128, K = 16 instruction, back to back), so the kernel issues the
//     fewest: one for layer 1 (K = 16), two for layer 2 (K = 32).  Weights are
//     FP16 (converted once on the host into the operand layout), biases and
//     accumulation FP32; the next tile's node values are loaded meanwhile.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_ptx.cuh"

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
    __half w1[kMlpHidden * kMlpIn];      // [32 out][16 in]
    __half w2[kMlpHidden * kMlpHidden];  // [32 out][32 in]
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
// Two FP32 values as FP16x2 (lo in the low half), rounded to nearest and
// saturated to the largest finite FP16 (so no infinity reaches the GELU).
__device__ __forceinline__ uint32_t pack_f16x2_sat(float lo, float hi)
{
    uint32_t d;
    asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// GELU of two FP16 values in packed FP16 arithmetic: x^2, a (1 + b x^2),
// x a (1 + b x^2), tanh.approx.f16x2, then 0.5 x + 0.5 x tanh.  Finite inputs
// give finite outputs (tanh saturates to +-1).
__device__ __forceinline__ uint32_t gelu_f16x2(uint32_t xu)
{
    const __half2 x = *reinterpret_cast<const __half2 *>(&xu);
    const __half2 a = __float2half2_rn(kGeluA), ab = __float2half2_rn(kGeluA * kGeluB);
    const __half2 u = __hmul2(x, __hfma2(__hmul2(x, x), ab, a));
    uint32_t t;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t *>(&u)));
    const __half2 hx = __hmul2(x, __float2half2_rn(0.5f));
    const __half2 g = __hfma2(hx, *reinterpret_cast<const __half2 *>(&t), hx);
    return *reinterpret_cast<const uint32_t *>(&g);
}

// 8 consecutive K values (4 packed pairs) of one row of an FP16 operand in
// umma_index layout with `rows` rows: one 16-byte store (consecutive rows are
// consecutive 16-byte slots of a core matrix, so a warp's stores do not conflict).
__device__ __forceinline__ void store_chunk_f16(__half *base, int row, int k0, int rows, uint32_t p0, uint32_t p1,
                                                uint32_t p2, uint32_t p3)
{
    *reinterpret_cast<uint4 *>(base + umma_index(row, k0, rows)) = make_uint4(p0, p1, p2, p3);
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

// Bounded mbarrier wait that sleeps in the barrier unit between checks
// (try_wait with a suspend-time hint, in ns) instead of spinning on it, so a
// waiting warp takes no issue slots from the warps that compute.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, unsigned parity, uint32_t hint_ns)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_sleep_bounded(uint64_t *bar, unsigned parity, uint64_t limit_ns)
{
    if (mbar_try_wait_sleep(bar, parity, 1000u))
        return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try_wait_sleep(bar, parity, 1000u))
            return true;
        if (global_ns() - t0 > limit_ns)
            return false;
    }
}

// ---------------------------------------------- network fused into a step
// The closure step kernel evaluates the network for the nodes of every plane
// it receives, one M = 128 tile per group of four warps (128 threads), with
// the same arithmetic as mlp_infer_kernel (so the same dtau, bit for bit):
//   plane p received:  each thread writes its node's standardised features
//                      (layer-1 operand row); after the CTA barrier the
//                      group's leader issues layer 1 (K = 16);
//   update of plane p-1: the group reads layer 2 of plane p-1 (issued one
//                      plane earlier) and derives the nodes' dtau;
//   after the update:  layer 1 of plane p is read back, biased, GELU'd and
//                      written as the layer-2 operand; after a group barrier
//                      the leader issues layer 2 (K = 32, two MMAs).
// The tensor-core latency hides behind the plane's reconstruction and
// update.  Layer 1 and layer 2 have separate operands and accumulators, so no
// step waits for an MMA other than the one whose result it reads.
struct FusedMlpSmem {
    static constexpr int W1 = 0;                                     // 32 x 16 FP16 (shared by the groups)
    static constexpr int W2 = W1 + kMlpHidden * kMlpIn * 2;          // 32 x 32 FP16
    static constexpr int GROUP0 = W2 + kMlpHidden * kMlpHidden * 2;  // first group's operands
    static constexpr int A1 = 0;                                     // 128 x 16 FP16 (group-relative)
    static constexpr int A2 = A1 + 128 * kMlpIn * 2;                 // 128 x 32 FP16
    static constexpr int GROUP_BYTES = A2 + 128 * kMlpHidden * 2;
    template <int NG>
    struct Of {
        static constexpr int BARS = GROUP0 + NG * GROUP_BYTES;  // two mbarriers per group
        static constexpr int TMEM = BARS + NG * 16;             // allocated tensor-memory address
        static constexpr int BYTES = TMEM + 16;
        static constexpr uint32_t COLS = NG == 1 ? 64 : 128;    // 64 columns per group, power of two
    };
    static constexpr uint32_t LBO_W = (kMlpHidden / 8) * 128, LBO_A = (128 / 8) * 128, SBO = 128;
};
static_assert(FusedMlpSmem::W2 % 128 == 0 && FusedMlpSmem::GROUP0 % 128 == 0 && FusedMlpSmem::A2 % 128 == 0 &&
                  FusedMlpSmem::GROUP_BYTES % 128 == 0,
              "operand alignment");

// Per-thread view of its group's network state.
struct FusedMlp {
    __half *w1, *w2;        // shared operands
    __half *a1, *a2;        // this group's operands
    uint64_t *bar1, *bar2;  // this group's MMA-completion barriers
    uint32_t tm1, tm2;      // this warp's lanes of the group's layer-1 / layer-2 accumulators
    uint32_t t1_issue, t2_issue;  // the accumulators' base addresses (for the MMA)
    int row;                // this thread's row of the group's tile
    int group;              // group index (named barrier group + 1)
    bool leader;            // issues the group's MMAs
    unsigned ph1, ph2;      // parities the next waits expect
    bool in_prev, in_cur;   // features in range: node updated next / node of this plane
};

// Layer-1 operand row from a node's stored moments; returns whether every
// raw feature lies in the training range.
__device__ __forceinline__ bool fused_features(FusedMlp &f, const MlpDevice &net, const float *m_stored)
{
    float x[kMlpIn];
    node_features(m_stored, net.r_ii, net.r_ij, x);
    const bool inside = in_range(x, net);
#pragma unroll
    for (int c = 0; c < kMlpIn / 8; c++) {
        uint32_t p[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            p[j] = pack_f16x2_sat(fmaf(x[8 * c + 2 * j], net.in_scale[8 * c + 2 * j], net.in_shift[8 * c + 2 * j]),
                                  fmaf(x[8 * c + 2 * j + 1], net.in_scale[8 * c + 2 * j + 1],
                                       net.in_shift[8 * c + 2 * j + 1]));
        store_chunk_f16(f.a1, f.row, 8 * c, 128, p[0], p[1], p[2], p[3]);
    }
    return inside;
}

// Layer 1 (16 -> 32) of the group's tile, by its leader, after the CTA barrier
// that follows the operand writes (each writer fenced them for the async proxy).
__device__ __forceinline__ void fused_issue_layer1(const FusedMlp &f)
{
    constexpr uint32_t idesc = umma_idesc_f16_f32<128, kMlpHidden>();
    tc_fence_after();
    umma_f16_if(f.leader, f.t1_issue, umma_desc(f.a1, FusedMlpSmem::LBO_A, FusedMlpSmem::SBO),
                umma_desc(f.w1, FusedMlpSmem::LBO_W, FusedMlpSmem::SBO), idesc, false);
    umma_commit_if(f.leader, f.bar1);
}

// Layer 1's accumulators -> bias, GELU -> layer-2 operand; group barrier;
// layer 2 (32 -> 32) by the leader.  False when the wait for layer 1 gave up
// (the MMA is then not issued; the caller aborts the CTA).
__device__ __forceinline__ bool fused_layer2(FusedMlp &f, const MlpDevice &net, uint64_t timeout_ns)
{
    constexpr uint32_t idesc = umma_idesc_f16_f32<128, kMlpHidden>();
    const bool ok = mbar_wait_sleep_bounded(f.bar1, f.ph1, timeout_ns);
    f.ph1 ^= 1u;
    tc_fence_after();
    float z[kMlpHidden];
    tmem_ld_32cols(f.tm1, z);
#pragma unroll
    for (int c = 0; c < kMlpHidden / 8; c++) {
        uint32_t p[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int i = 8 * c + 2 * j;
            p[j] = gelu_f16x2(pack_f16x2_sat(z[i] + net.b1[i], z[i + 1] + net.b1[i + 1]));
        }
        store_chunk_f16(f.a2, f.row, 8 * c, 128, p[0], p[1], p[2], p[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncwarp();
    asm volatile("bar.sync %0, 128;" ::"r"(f.group + 1) : "memory");
    tc_fence_after();
    const bool go = ok;  // a leader whose wait gave up issues nothing (the CTA then aborts)
    for (int s = 0; s < kMlpHidden / 16; s++)
        // one K-step of 16 spans two 8-wide K-chunks: 2 x LBO bytes = LBO halves
        umma_f16_if(f.leader && go, f.t2_issue,
                    umma_desc(f.a2 + s * FusedMlpSmem::LBO_A, FusedMlpSmem::LBO_A, FusedMlpSmem::SBO),
                    umma_desc(f.w2 + s * FusedMlpSmem::LBO_W, FusedMlpSmem::LBO_W, FusedMlpSmem::SBO), idesc, s > 0);
    umma_commit_if(f.leader && go, f.bar2);
    return ok;
}

// Layer 2's accumulators -> bias, GELU, the 32 -> 1 layer -> dtau of the node
// whose features were written one plane earlier (0 outside the training
// range).  ok = false when the wait gave up.
__device__ __forceinline__ float fused_dtau(FusedMlp &f, const MlpDevice &net, uint64_t timeout_ns, bool &ok)
{
    ok = mbar_wait_sleep_bounded(f.bar2, f.ph2, timeout_ns);
    f.ph2 ^= 1u;
    tc_fence_after();
    float z[kMlpHidden];
    tmem_ld_32cols(f.tm2, z);
    tc_fence_before();
    float y = net.b3;
#pragma unroll
    for (int i = 0; i < kMlpHidden; i += 2) {
        const uint32_t g = gelu_f16x2(pack_f16x2_sat(z[i] + net.b2[i], z[i + 1] + net.b2[i + 1]));
        const float2 h = __half22float2(*reinterpret_cast<const __half2 *>(&g));
        y = fmaf(net.w3[i], h.x, y);
        y = fmaf(net.w3[i + 1], h.y, y);
    }
    return f.in_prev ? fminf(fmaxf(net.out_scale * y, net.dtau_lo), net.dtau_hi) : 0.0f;
}

// ------------------------------------------------------- inference kernel
// Shared memory of mlp_infer_kernel (byte offsets; operands 128 B aligned).
struct MlpSmem {
    static constexpr int W1 = 0;                                 // 32 x 16 FP16, 1 KB
    static constexpr int W2 = W1 + kMlpHidden * kMlpIn * 2;      // 32 x 32 FP16, 2 KB
    static constexpr int A1 = W2 + kMlpHidden * kMlpHidden * 2;  // 128 x 16 FP16, 4 KB (features)
    static constexpr int A2 = A1 + 128 * kMlpIn * 2;             // 128 x 32 FP16, 8 KB (layer-1 activations)
    static constexpr int BAR = A2 + 128 * kMlpHidden * 2;        // mbarrier
    static constexpr int TMEM = BAR + 8;                         // allocated tensor-memory address
    static constexpr int BYTES = TMEM + 4;
    // shared memory requested per CTA: at most 13 CTAs fit an SM (228 KB,
    // 1 KB reserved each), and 13 x 32 tensor-memory columns fit its 512
    static constexpr int LAUNCH_BYTES = 16 * 1024;
    // leading (K-chunk) byte offsets: (rows / 8) x 128 B; the stride between
    // 8-row groups is 128 B for all operands
    static constexpr uint32_t LBO_W = (kMlpHidden / 8) * 128, LBO_A = (128 / 8) * 128, SBO = 128;
};
static_assert(MlpSmem::A1 % 128 == 0 && MlpSmem::A2 % 128 == 0 && MlpSmem::W2 % 128 == 0, "operand alignment");
static_assert(MlpSmem::BYTES <= MlpSmem::LAUNCH_BYTES &&
                  (228 * 1024 / (MlpSmem::LAUNCH_BYTES + 1024)) * 32 <= 512,
              "the CTAs shared memory admits to an SM must fit its tensor memory");

enum : unsigned { ERR_MMA_TIMEOUT = 2u };

#ifndef LBM_MLP_CTAS_PER_SM
#define LBM_MLP_CTAS_PER_SM 8
#endif
// CTAs per SM the register budget is sized for (the launch's grid is one wave of them)
constexpr int kMlpCtasPerSm = LBM_MLP_CTAS_PER_SM;

// The network is a kernel parameter (constant bank).  Source of a node's 16
// raw features: stored moments [10][N] (FROM_MOMENTS) or a feature array
// [N][16].  Output dtau[N] (clamped, 0 where the inputs leave the training
// range), or the raw network output y[N] (RAW_Y).
template <bool FROM_MOMENTS, bool RAW_Y>
__global__ void __launch_bounds__(128, kMlpCtasPerSm) mlp_infer_kernel(const float *src, size_t N,
                                                                       const __grid_constant__ MlpDevice net,
                                                                       float *out, unsigned *err, uint64_t timeout_ns)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __half *w1 = reinterpret_cast<__half *>(sm + MlpSmem::W1);
    __half *w2 = reinterpret_cast<__half *>(sm + MlpSmem::W2);
    __half *a1 = reinterpret_cast<__half *>(sm + MlpSmem::A1);
    __half *a2 = reinterpret_cast<__half *>(sm + MlpSmem::A2);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + MlpSmem::BAR);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + MlpSmem::TMEM);
    const int tid = threadIdx.x, warp = tid >> 5;
    const bool leader = tid == 0;

    // weights (already in operand layout) into shared memory, 4 B at a time
    // (the parameter block guarantees 4-byte alignment)
    {
        const uint32_t *g = reinterpret_cast<const uint32_t *>(net.w1);
        uint32_t *d = reinterpret_cast<uint32_t *>(sm + MlpSmem::W1);
        constexpr int n4 = (MlpSmem::A1 - MlpSmem::W1) / 4;  // w1 and w2 are contiguous in both
        static_assert(sizeof(net.w1) + sizeof(net.w2) == MlpSmem::A1 - MlpSmem::W1, "weights");
        for (int i = tid; i < n4; i += 128)
            d[i] = g[i];
    }
    mbar_init_if(leader, bar);
    fence_mbar_init_if(leader);
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
    unsigned phase = 0;
    bool failed = false;   // warp 0's MMA wait gave up
    bool aborted = false;  // uniform: from the barrier's OR-reduction
    // One layer: a barrier (the operand is written, the previous
    // accumulators are read), the K-steps (16 each) and their commit issued by
    // one thread, the completion awaited by warp 0 alone (bounded, sleeping)
    // while the other warps sleep in the second barrier, whose OR-reduction
    // tells every thread whether the wait gave up (false: stop).
    auto layer = [&](const __half *a, const __half *w, int ksteps) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        cta_sync();
        tc_fence_after();
        for (int s = 0; s < ksteps; s++)
            umma_f16_if(leader, tmem, umma_desc(a + s * MlpSmem::LBO_A, MlpSmem::LBO_A, MlpSmem::SBO),
                        umma_desc(w + s * MlpSmem::LBO_W, MlpSmem::LBO_W, MlpSmem::SBO), idesc, s > 0);
        umma_commit_if(leader, bar);
        if (warp == 0 && !mbar_wait_sleep_bounded(bar, phase, timeout_ns)) {
            if (leader)
                atomicOr(err, ERR_MMA_TIMEOUT);
            failed = true;
        }
        phase ^= 1u;
        __syncwarp();
        if (__syncthreads_or(failed)) {
            aborted = true;
            return false;
        }
        tc_fence_after();
        return true;
    };

    const size_t tiles = (N + 127) / 128;
    constexpr int NV = FROM_MOMENTS ? 10 : kMlpIn;  // values loaded per node
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
            for (int k = 0; k < NV; k++)
                v[k] = 0.0f;
        }
    };
    float next[NV];
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
        load(tile + gridDim.x, next);
        const bool inside = valid && in_range(f, net);
        // layer-1 operand: this thread's row of standardised features
#pragma unroll
        for (int c = 0; c < kMlpIn / 8; c++) {
            uint32_t p[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
                p[j] = pack_f16x2_sat(fmaf(f[8 * c + 2 * j], net.in_scale[8 * c + 2 * j], net.in_shift[8 * c + 2 * j]),
                                      fmaf(f[8 * c + 2 * j + 1], net.in_scale[8 * c + 2 * j + 1],
                                           net.in_shift[8 * c + 2 * j + 1]));
            store_chunk_f16(a1, tid, 8 * c, 128, p[0], p[1], p[2], p[3]);
        }
        // each layer starts at a barrier: the threads have read the previous
        // layer's accumulators (tcgen05.wait::ld) and written its operand
        if (!layer(a1, w1, kMlpIn / 16))  // 16 -> 32
            break;
        float z[kMlpHidden];
        tmem_ld_32cols(tmem + lane_base, z);
#pragma unroll
        for (int c = 0; c < kMlpHidden / 8; c++) {
            uint32_t p[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int i = 8 * c + 2 * j;
                p[j] = gelu_f16x2(pack_f16x2_sat(z[i] + net.b1[i], z[i + 1] + net.b1[i + 1]));
            }
            store_chunk_f16(a2, tid, 8 * c, 128, p[0], p[1], p[2], p[3]);
        }
        if (!layer(a2, w2, kMlpHidden / 16))  // 32 -> 32
            break;
        tmem_ld_32cols(tmem + lane_base, z);
        float y = net.b3;
#pragma unroll
        for (int i = 0; i < kMlpHidden; i += 2) {
            const uint32_t g = gelu_f16x2(pack_f16x2_sat(z[i] + net.b2[i], z[i + 1] + net.b2[i + 1]));
            const float2 h = __half22float2(*reinterpret_cast<const __half2 *>(&g));
            y = fmaf(net.w3[i], h.x, y);
            y = fmaf(net.w3[i + 1], h.y, y);
        }
        if (valid) {
            if constexpr (RAW_Y)
                out[node] = y;
            else
                out[node] = inside ? fminf(fmaxf(net.out_scale * y, net.dtau_lo), net.dtau_hi) : 0.0f;
        }
        // the next tile's first barrier orders this read before its MMAs
    }
    if (aborted) {
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
