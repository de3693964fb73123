// lbm_step.cuh -- the fused LBM time step for sm_100a (z-marching tiles).
//
// One CTA owns a TX x TY column tile of the x-y plane and a chunk of z-planes
// and marches up that chunk.  For every plane it
//   1. receives the plane's 10 moment fields -- tile plus a one-node ring --
//      from global memory by one TMA (cp.async.bulk.tensor.4d) into a
//      multi-stage shared-memory ring, completion tracked by an mbarrier;
//   2. reconstructs the populations of its nodes (and, on the ring, only the
//      ones that point into the tile) and writes the ones that move in x-y
//      into a double-buffered shared-memory plane;
//   3. after one __syncthreads, pulls f_q(x) = R_q(m(x - c_q)) for every
//      direction: x-y movers from shared memory, pure-z movers and the rest
//      population from registers of the previous/next plane;
//   4. updates the plane below (whose three source planes are now complete):
//      boundary or interior moments, scale, collide, store, and the fused
//      function objects S, k and their running means.
// No population ever goes to global memory: the reference's block-halo faces
// (src/blockHalo/halo.cuh) are replaced by the moment ring, which neighbour
// CTAs read at the same time from L2.
//
// Moments live in two global buffers (read A, write B, swap each step) laid
// out as [field][z][y][x] float32 -- x fastest, 10 fields of nx*ny*nz.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lbm_core.cuh"

namespace lbm {

// ------------------------------------------------------------ storage
// How the 10 moment fields are held in HBM.  FP32 stores the reference's
// values as they are.  The 16-bit formats store (value * scale[field]) with
// power-of-two scales (exact to apply and undo) that bring typical cavity
// magnitudes -- rho-1 ~ 1e-3, 3u ~ 0.1, 4.5 m_aa and 9 m_ab ~ 1e-2 -- near 1,
// away from the fp16 subnormal range; arithmetic stays FP32.  XPAD is the
// left padding of a TMA box so that its x start is 16-byte aligned.
template <typename ST>
struct Storage;

template <>
struct Storage<float> {
    static constexpr int BYTES = 4, XPAD = 4;
    __host__ __device__ static constexpr float scale(int) { return 1.0f; }
    __device__ static float load(float v, int) { return v; }
    __device__ static float store(float v, int) { return v; }
};

template <>
struct Storage<__half> {
    static constexpr int BYTES = 2, XPAD = 8;
    __host__ __device__ static constexpr float scale(int k) { return (k >= 1 && k <= 3) ? 8.0f : 64.0f; }
    __device__ static float load(__half v, int k) { return __half2float(v) * (1.0f / scale(k)); }
    __device__ static __half store(float v, int k) { return __float2half_rn(v * scale(k)); }
};

template <>
struct Storage<__nv_bfloat16> {
    static constexpr int BYTES = 2, XPAD = 8;
    __host__ __device__ static constexpr float scale(int) { return 1.0f; }
    __device__ static float load(__nv_bfloat16 v, int) { return __bfloat162float(v); }
    __device__ static __nv_bfloat16 store(float v, int) { return __float2bfloat16_rn(v); }
};

// ------------------------------------------------------------------ PTX
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after `limit_ns` and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int k = 0; k < 32; k++)
            if (mbar_try_wait(bar, parity))
                return true;
        if (global_ns() - t0 > limit_ns)
            return false;
    }
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ------------------------------------------------------------- params
enum : unsigned { ERR_TMA_TIMEOUT = 1u };

template <typename MeanT>
struct FOPtrs {
    float *S;            // [6][N] or null
    MeanT *SMean;        // [6][N] or null
    float *k;            // [N] or null
    MeanT *kMean;        // [N] or null
    MeanT *momentsMean;  // [10][N] or null
    MeanT inv_count;     // 1 / (t + 1), t the absolute step index
    StrainDiv sd;        // divisors of S and their reciprocals
};

// Global sums of one step's result, accumulated by every CTA (FP64).
struct MonitorSlot {
    double mass;                   // sum of rho
    double rho_u2;                 // sum of rho |u_stored|^2 (kinetic energy = this * 0.5 / 9)
    unsigned long long nonfinite;  // nodes with a NaN/Inf among their 10 stored moments
};

template <typename MeanT, typename ST = float>
struct StepParams {
    ST *out;           // [10][N] moments after the step
    MonitorSlot *mon;  // per-step sums (monitored kernels only)
    int nx, ny, nz;
    int zc;            // z-planes per CTA
    Relax rx;
    FOPtrs<MeanT> fo;
    unsigned *err;
    uint64_t timeout_ns;
};

template <int TX, int TY, typename ST = float>
struct TileGeom {
    static constexpr int XPAD = Storage<ST>::XPAD;  // TMA box starts XPAD nodes left (16 B alignment)
    static constexpr int TXP = TX + 2 * XPAD;       // staged row length
    static constexpr int RY = TY + 2;               // staged rows (ring included)
    static constexpr int PLANE_FLOATS = 10 * RY * TXP;  // elements of one staged plane
    static constexpr int PLANE_BYTES = PLANE_FLOATS * Storage<ST>::BYTES;
    static constexpr int PX = TX + 2, PY = TY + 2;  // population plane incl. ring
    static constexpr int RING = 2 * (TX + 2) + 2 * TY;
    static_assert(PLANE_BYTES % 128 == 0, "stage size must keep 128 B alignment");
};

// NPB population planes: 2 lets consecutive planes overlap with one barrier
// per plane; 1 saves shared memory (more CTAs per SM) at a second barrier.
template <int Q, int TX, int TY, int NSTAGE, int NPB = 2, typename ST = float>
struct SmemLayout {
    using G = TileGeom<TX, TY, ST>;
    static constexpr int NXY = XY<Q>::N;
    static constexpr size_t bar_off = 0;
    static constexpr size_t stage_off = 128;
    static constexpr size_t pop_off = stage_off + size_t(NSTAGE) * G::PLANE_BYTES;
    static constexpr size_t pop_floats = size_t(NXY) * G::PY * G::PX;
    static constexpr size_t bytes = pop_off + NPB * pop_floats * 4;
};

// directions grouped by cz: U (cz = +1), S (cz = 0, rest included), D (cz = -1)
template <int Q>
struct ZGroups {
    static constexpr int NU = count_cz<Q>(1), NS = count_cz<Q>(0), ND = count_cz<Q>(-1);
};

// Compile-time loop helper: calls f(IC<i>{}) for i in [B, E).
template <int V>
struct IC {
    static constexpr int value = V;
};
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F &&f)
{
    if constexpr (B < E) {
        f(IC<B>{});
        static_for<B + 1, E>(f);
    }
}

// Reconstruct the x-y movers of ring node (rx, ry) that point into the tile
// (those with the given sign of cx or cy) and store them into pop plane pb.
template <int Q, int TX, int TY, int AXIS, int SIGN, typename ST>
__device__ __forceinline__ void ring_pops(const ST *sm, float *pb, int rx, int ry)
{
    using G = TileGeom<TX, TY, ST>;
    float m[10];
#pragma unroll
    for (int k = 0; k < 10; k++)
        m[k] = Storage<ST>::load(sm[(k * G::RY + ry + 1) * G::TXP + rx + G::XPAD], k);
    m[0] = m[0] + 1.0f;
    const RecPre r = rec_pre<Q>(m);
    static_for<0, XY<Q>::N>([&](auto s) {
        constexpr int q = XY<Q>::q(decltype(s)::value);
        constexpr int c = AXIS == 0 ? cx_of(q) : cy_of(q);
        if constexpr (c == SIGN)
            pb[(decltype(s)::value * G::PY + ry + 1) * G::PX + rx + 1] = rec_q<Q, q>(r, m);
    });
}

// ---------------------------------------------------------------- kernel
template <int Q, int TX, int TY, int NSTAGE, bool FO, typename MeanT, bool MON = false, int NPB = 2, int MINB = 2,
          typename ST = float>
__global__ void __launch_bounds__(TX *TY, MINB)
    step_kernel(const __grid_constant__ CUtensorMap tmap_in, const StepParams<MeanT, ST> p)
{
    using G = TileGeom<TX, TY, ST>;
    using L = SmemLayout<Q, TX, TY, NSTAGE, NPB, ST>;
    using ZG = ZGroups<Q>;
    constexpr int NXY = XY<Q>::N;

    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);
    ST *stages = reinterpret_cast<ST *>(smem + L::stage_off);
    float *pops = reinterpret_cast<float *>(smem + L::pop_off);
    __shared__ int s_abort;

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int lin = ty * TX + tx;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * p.zc;
    const int z1 = min(z0 + p.zc, p.nz);
    const int nplanes = z1 - z0 + 2;  // planes z0-1 .. z1
    const int x = x0 + tx, y = y0 + ty;
    const bool own = (x < p.nx) && (y < p.ny);
    const size_t N = size_t(p.nx) * p.ny * p.nz;
    const size_t plane = size_t(p.nx) * p.ny;

    if (lin == 0) {
        prefetch_tmap(&tmap_in);
        for (int s = 0; s < NSTAGE; s++)
            mbar_init(&bars[s], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    if (lin == 0) {
        for (int s = 0; s < NSTAGE && s < nplanes; s++) {
            mbar_expect_tx(&bars[s], G::PLANE_BYTES);
            tma_load_4d(stages + s * G::PLANE_FLOATS, &tmap_in, x0 - G::XPAD, y0 - 1, z0 - 1 + s, 0, &bars[s]);
        }
    }

    // populations held in registers between planes
    float U2[ZG::NU], U1[ZG::NU], S1[ZG::NS];  // U(p-2), U(p-1), S(p-1)
    double mon_mass = 0.0, mon_ke = 0.0;
    unsigned mon_bad = 0;

    for (int i = 0; i < nplanes; i++) {
        const int pz = z0 - 1 + i;  // plane being received
        const int stage = i % NSTAGE;
        const unsigned parity = (i / NSTAGE) & 1;
        ST *sm = stages + stage * G::PLANE_FLOATS;
        float *pb = pops + (NPB == 2 ? (i & 1) : 0) * L::pop_floats;

        // running means of the node updated in this iteration (plane pz-1),
        // loaded early so the latency hides behind the reconstruction
        const int zu = pz - 1;
        const bool upd = (i >= 2) && own;
        const size_t iu = size_t(zu) * plane + size_t(y) * p.nx + x;
        MeanT sm_old[6], km_old = MeanT(0);
        if constexpr (FO) {
            if (upd) {
                if (p.fo.SMean) {
#pragma unroll
                    for (int c = 0; c < 6; c++)
                        sm_old[c] = p.fo.SMean[c * N + iu];
                }
                if (p.fo.kMean)
                    km_old = p.fo.kMean[iu];
            }
        }

        if (!mbar_wait_bounded(&bars[stage], parity, p.timeout_ns)) {
            atomicOr(p.err, ERR_TMA_TIMEOUT);
            s_abort = 1;
        }

        // own node: reconstruct all directions
        float U0[ZG::NU], S0[ZG::NS], D0[ZG::ND];
        {
            float m[10];
#pragma unroll
            for (int k = 0; k < 10; k++)
                m[k] = Storage<ST>::load(sm[(k * G::RY + ty + 1) * G::TXP + tx + G::XPAD], k);
            m[0] = m[0] + 1.0f;
            const RecPre r = rec_pre<Q>(m);
            static_for<0, NXY>([&](auto s) {
                constexpr int q = XY<Q>::q(decltype(s)::value);
                pb[(decltype(s)::value * G::PY + ty + 1) * G::PX + tx + 1] = rec_q<Q, q>(r, m);
            });
            U0[zslot<Q>(5)] = rec_q<Q, 5>(r, m);
            D0[zslot<Q>(6)] = rec_q<Q, 6>(r, m);
            S0[zslot<Q>(0)] = rec_q<Q, 0>(r, m);
        }
        // ring nodes: only the directions that enter the tile
        if (lin < G::RING) {
            int r = lin;
            if (r < TX + 2) {
                ring_pops<Q, TX, TY, 1, +1, ST>(sm, pb, r - 1, -1);
            } else if ((r -= TX + 2) < TX + 2) {
                ring_pops<Q, TX, TY, 1, -1, ST>(sm, pb, r - 1, TY);
            } else if ((r -= TX + 2) < TY) {
                ring_pops<Q, TX, TY, 0, +1, ST>(sm, pb, -1, r);
            } else {
                r -= TY;
                ring_pops<Q, TX, TY, 0, -1, ST>(sm, pb, TX, r);
            }
        }
        __syncthreads();
        if (s_abort)
            break;

        // the stage is consumed: refill it with plane i + NSTAGE
        if (lin == 0 && i + NSTAGE < nplanes) {
            fence_proxy_async();
            mbar_expect_tx(&bars[stage], G::PLANE_BYTES);
            tma_load_4d(sm, &tmap_in, x0 - G::XPAD, y0 - 1, pz + NSTAGE, 0, &bars[stage]);
        }

        // pull the down-movers (cz = -1) that land on plane pz-1
        static_for<0, NXY>([&](auto s) {
            constexpr int q = XY<Q>::q(decltype(s)::value);
            if constexpr (cz_of(q) == -1)
                D0[zslot<Q>(q)] = pb[(decltype(s)::value * G::PY + ty + 1 - cy_of(q)) * G::PX + tx + 1 - cx_of(q)];
        });

        if (i >= 2) {
            // update plane zu = pz - 1 from U(pz-2), S(pz-1), D(pz)
            float f[Q];
            static_for<0, Q>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                constexpr int c = cz_of(q);
                if constexpr (c == 1) f[q] = U2[zslot<Q>(q)];
                if constexpr (c == 0) f[q] = S1[zslot<Q>(q)];
                if constexpr (c == -1) f[q] = D0[zslot<Q>(q)];
            });
            if (own) {
                const unsigned type = node_type(x, y, zu, p.nx, p.ny, p.nz);
                float m[10];
                node_update<Q>(f, type, p.rx, m);
                ST *o = p.out + iu;
                o[0] = Storage<ST>::store(m[0] - 1.0f, 0);
#pragma unroll
                for (int k = 1; k < 10; k++)
                    o[k * N] = Storage<ST>::store(m[k], k);
                if constexpr (MON) {
                    mon_mass += double(m[0]);
                    mon_ke += double(m[0] * ((m[1] * m[1] + m[2] * m[2]) + m[3] * m[3]));
                    const float chk = (((m[0] + m[1]) + (m[2] + m[3])) + ((m[4] + m[5]) + (m[6] + m[7]))) + (m[8] + m[9]);
                    mon_bad += !isfinite(chk);
                }
                if constexpr (FO) {
                    if (p.fo.S || p.fo.SMean) {
                        float s6[6];
                        strain_rate(m, p.fo.sd, s6);
                        if (p.fo.S) {
#pragma unroll
                            for (int c = 0; c < 6; c++)
                                p.fo.S[c * N + iu] = s6[c];
                        }
                        if (p.fo.SMean) {
#pragma unroll
                            for (int c = 0; c < 6; c++)
                                p.fo.SMean[c * N + iu] = time_average<MeanT>(sm_old[c], MeanT(s6[c]), p.fo.inv_count);
                        }
                    }
                    if (p.fo.k || p.fo.kMean) {
                        const float ke = kinetic(m[1], m[2], m[3]);
                        if (p.fo.k)
                            p.fo.k[iu] = ke;
                        if (p.fo.kMean)
                            p.fo.kMean[iu] = time_average<MeanT>(km_old, MeanT(ke), p.fo.inv_count);
                    }
                    if (p.fo.momentsMean) {
                        m[0] = m[0] - 1.0f;
#pragma unroll
                        for (int c = 0; c < 10; c++) {
                            MeanT *a = p.fo.momentsMean + c * N + iu;
                            *a = time_average<MeanT>(*a, MeanT(m[c]), p.fo.inv_count);
                        }
                    }
                }
            }
        }

        // keep this plane's same-plane and up-movers for the next updates
        static_for<0, NXY>([&](auto s) {
            constexpr int q = XY<Q>::q(decltype(s)::value);
            if constexpr (cz_of(q) == 0)
                S0[zslot<Q>(q)] = pb[(decltype(s)::value * G::PY + ty + 1 - cy_of(q)) * G::PX + tx + 1 - cx_of(q)];
            if constexpr (cz_of(q) == 1)
                U0[zslot<Q>(q)] = pb[(decltype(s)::value * G::PY + ty + 1 - cy_of(q)) * G::PX + tx + 1 - cx_of(q)];
        });
#pragma unroll
        for (int k = 0; k < ZG::NU; k++) {
            U2[k] = U1[k];
            U1[k] = U0[k];
        }
#pragma unroll
        for (int k = 0; k < ZG::NS; k++)
            S1[k] = S0[k];
        if constexpr (NPB == 1)
            __syncthreads();  // the single population plane is rewritten next iteration
    }

    if constexpr (MON) {
        // CTA sums, then one FP64 atomic per quantity
        for (int o = 16; o > 0; o >>= 1) {
            mon_mass += __shfl_down_sync(0xffffffffu, mon_mass, o);
            mon_ke += __shfl_down_sync(0xffffffffu, mon_ke, o);
            mon_bad += __shfl_down_sync(0xffffffffu, mon_bad, o);
        }
        __shared__ double s_mon[2][TX * TY / 32];
        __shared__ unsigned s_bad[TX * TY / 32];
        const int lane = lin & 31, wid = lin >> 5;
        if (lane == 0) {
            s_mon[0][wid] = mon_mass;
            s_mon[1][wid] = mon_ke;
            s_bad[wid] = mon_bad;
        }
        __syncthreads();
        if (lin == 0) {
            double a = 0.0, b = 0.0;
            unsigned long long c = 0;
            for (int w = 0; w < TX * TY / 32; w++) {
                a += s_mon[0][w];
                b += s_mon[1][w];
                c += s_bad[w];
            }
            atomicAdd(&p.mon->mass, a);
            atomicAdd(&p.mon->rho_u2, b);
            atomicAdd(&p.mon->nonfinite, c);
        }
    }

    if (s_abort) {
        // give TMA copies still in flight a bounded chance to land before exit
        if (lin == 0)
            for (int s = 0; s < NSTAGE; s++)
                (void)mbar_wait_bounded(&bars[s], 0, 1000000ull);
    }
}

}  // namespace lbm
