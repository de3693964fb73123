// lbm_step.cuh -- the fused LBM time step for sm_100a (z-marching tiles).
//
// One CTA owns a TX x TY column tile of the x-y plane and a chunk of z-planes
// and marches up that chunk.  For every plane it
//   1. receives the plane's 10 moment fields -- tile plus a one-node ring --
//      from global memory by one TMA (cp.async.bulk.tensor.4d) into a
//      multi-stage shared-memory ring, completion tracked by an mbarrier;
//   2. reconstructs the populations of its nodes (and, on the ring, only the
//      ones that point into the tile) and writes the ones that move in x-y
//      into a shared-memory population plane (one or two buffers), grouped
//      by in-plane step (cx, cy): per group one float cell for the
//      down-mover and one float2 cell for the same-plane and up-movers;
//   3. after a CTA barrier, pulls f_q(x) = R_q(m(x - c_q)) for every
//      direction: x-y movers from shared memory, pure-z movers and the rest
//      population from registers of the previous/next plane;
//   4. updates the plane below (whose three source planes are now complete):
//      boundary or interior moments, scale, collide, store, and the fused
//      function objects S, k and their running means (and, in the closure
//      kernels, the relaxation time from the learned network).
// No population ever goes to global memory: the reference's block-halo faces
// (src/blockHalo/halo.cuh) are replaced by the moment ring, which neighbour
// CTAs read at the same time from L2.
//
// Moments live in two global buffers (read A, write B, swap each step) laid
// out as [field][z][y][x] -- x fastest, 10 fields of nx*ny*nz, in the storage
// format (FP32, or FP16/BF16: see Storage).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lbm_core.cuh"
#include "lbm_mlp.cuh"
#include "lbm_ptx.cuh"

namespace lbm {

// ------------------------------------------------------------ storage
// How the 10 moment fields are held in HBM.  FP32 stores the reference's
// values as they are.  FP16 stores value * SC with one power-of-two scale for
// every field (exact to apply and undo), which lifts typical cavity magnitudes
// -- rho-1 ~ 1e-3, 3u ~ 0.1, 4.5 m_aa and 9 m_ab ~ 1e-2 -- out of the FP16
// subnormal range; BF16 has FP32's exponent range and stores the values as
// they are.  Arithmetic stays FP32.  Because the scale is one power of two,
// the step kernel never applies it: it reconstructs the populations from the
// scaled moments with scaled constants and scales the collision's output
// constants instead (see rec_pre / scale_collide), which rounds exactly as the
// unscaled arithmetic would, so loading and storing a moment is one
// conversion.  load/store (with the scale) serve the other kernels.  XPAD is
// the left padding of a TMA box so that its x start is 16-byte aligned.
template <typename ST>
struct Storage;

template <>
struct Storage<float> {
    static constexpr int BYTES = 4, XPAD = 4;
    static constexpr int SCI = 1;
    static constexpr float SC = float(SCI);
    __host__ __device__ static constexpr float scale(int) { return SC; }
    __device__ static float load(float v, int) { return v; }
    __device__ static float store(float v, int) { return v; }
    __device__ static float load_raw(float v) { return v; }
    __device__ static float store_raw(float v) { return v; }
};

template <>
struct Storage<__half> {
    static constexpr int BYTES = 2, XPAD = 8;
    static constexpr int SCI = 64;
    static constexpr float SC = float(SCI);
    __host__ __device__ static constexpr float scale(int) { return SC; }
    __device__ static float load(__half v, int) { return __half2float(v) * (1.0f / SC); }
    __device__ static __half store(float v, int) { return __float2half_rn(v * SC); }
    __device__ static float load_raw(__half v) { return __half2float(v); }
    __device__ static __half store_raw(float v) { return __float2half_rn(v); }
};

template <>
struct Storage<__nv_bfloat16> {
    static constexpr int BYTES = 2, XPAD = 8;
    static constexpr int SCI = 1;
    static constexpr float SC = float(SCI);
    __host__ __device__ static constexpr float scale(int) { return SC; }
    __device__ static float load(__nv_bfloat16 v, int) { return __bfloat162float(v); }
    __device__ static __nv_bfloat16 store(float v, int) { return __float2bfloat16_rn(v); }
    __device__ static float load_raw(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static __nv_bfloat16 store_raw(float v) { return __float2bfloat16_rn(v); }
};

// rho from a stored rho - 1 (scaled by SC): one rounding, as rho0 + value.
template <typename ST>
__device__ __forceinline__ float rho_of_stored(float v)
{
    if constexpr (Storage<ST>::SC == 1.0f)
        return v + 1.0f;
    else
        return fmaf(v, 1.0f / Storage<ST>::SC, 1.0f);
}
// The stored value of rho: SC (rho - 1), rounded once.
template <typename ST>
__device__ __forceinline__ float stored_of_rho(float rho)
{
    if constexpr (Storage<ST>::SC == 1.0f)
        return rho - 1.0f;
    else
        return fmaf(rho, Storage<ST>::SC, -Storage<ST>::SC);
}

// ------------------------------------------------------------- params
enum : unsigned { ERR_TMA_TIMEOUT = 1u };

// Device-side error record of the step kernels: flag bits, and where the
// first failure happened (the first CTA to fail fills in the details).
struct StepFault {
    unsigned flags;              // ERR_* bits
    unsigned recorded;           // set once the details below are valid
    int block[3];                // blockIdx of the CTA
    int item, mesh;              // batch work item and mesh-table row (-1 outside batches)
    int plane;                   // plane index within the work item (0 = plane z0-1)
    unsigned seq;                // planes the CTA had received before this one
    unsigned slot, parity;       // stage slot waited on and the phase parity expected
    unsigned long long barrier;  // raw 64-bit mbarrier word when the wait gave up
};

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
    int z_lo, z_hi;    // planes this launch updates: CTA bz takes [z_lo + bz zc, min(z_lo + (bz+1) zc, z_hi))
    Relax rx;
    FOPtrs<MeanT> fo;
    StepFault *fault;
    uint64_t timeout_ns;
    const float *dtau;  // per-node relaxation-time correction (closure kernels only)
};
// The host fills one block type for every storage format (the output is a
// pointer), so the layouts must agree; FP32- and FP64-mean blocks differ only
// inside the function-object fields.
using StepParamsF32 = StepParams<float, float>;
using StepParamsF16 = StepParams<float, __half>;
using StepParamsBF16 = StepParams<float, __nv_bfloat16>;
using StepParamsF64Means = StepParams<double, float>;
static_assert(sizeof(StepParamsF32) == sizeof(StepParamsF16) && sizeof(StepParamsF32) == sizeof(StepParamsBF16) &&
                  offsetof(StepParamsF32, dtau) == offsetof(StepParamsF16, dtau) &&
                  offsetof(StepParamsF32, dtau) == offsetof(StepParamsBF16, dtau),
              "parameter block layout must not depend on the storage type");
static_assert(offsetof(StepParamsF32, fault) == offsetof(StepParamsF64Means, fault) &&
                  offsetof(StepParamsF32, timeout_ns) == offsetof(StepParamsF64Means, timeout_ns) &&
                  offsetof(StepParamsF32, dtau) == offsetof(StepParamsF64Means, dtau),
              "fields after the function-object block at the same offsets for both mean precisions");

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

// The x-y movers grouped by their in-plane step (cx, cy): group g holds the
// directions with that step and cz = -1 (D), 0 (S), +1 (U), whichever the
// lattice has (D3Q27: all three in every group; D3Q19: all three on the axes,
// S alone on the diagonals).  In the population plane a group's (S, U) pair
// is one float2 cell and its D one float cell, so a node stores and a
// neighbour pulls a whole group with two shared-memory accesses.
__host__ __device__ constexpr int group_cx(int g)
{
    constexpr int t[8] = {1, -1, 0, 0, 1, -1, 1, -1};
    return t[g];
}
__host__ __device__ constexpr int group_cy(int g)
{
    constexpr int t[8] = {0, 0, 1, -1, 1, -1, -1, 1};
    return t[g];
}
// direction q of lattice Q with step (cx, cy, cz), or -1
template <int Q>
__host__ __device__ constexpr int q_of_step(int cx, int cy, int cz)
{
    for (int q = 0; q < Q; q++)
        if (cx_of(q) == cx && cy_of(q) == cy && cz_of(q) == cz)
            return q;
    return -1;
}
template <int Q>
struct PopGroups {
    static constexpr int NG = 8;
    __host__ __device__ static constexpr int qD(int g) { return q_of_step<Q>(group_cx(g), group_cy(g), -1); }
    __host__ __device__ static constexpr int qS(int g) { return q_of_step<Q>(group_cx(g), group_cy(g), 0); }
    __host__ __device__ static constexpr int qU(int g) { return q_of_step<Q>(group_cx(g), group_cy(g), 1); }
    // cells: groups with U first (float2 planes), then S-only groups (float
    // planes), then the D planes; offsets in floats, in units of one plane
    __host__ __device__ static constexpr int n_su()
    {
        int n = 0;
        for (int g = 0; g < NG; g++)
            n += qU(g) >= 0;
        return n;
    }
    __host__ __device__ static constexpr int su_plane(int g)  // float2 plane index, groups with U
    {
        int n = 0;
        for (int h = 0; h < g; h++)
            n += qU(h) >= 0;
        return n;
    }
    __host__ __device__ static constexpr int s_plane(int g)  // float plane index (after the float2 planes)
    {
        int n = 2 * n_su();
        for (int h = 0; h < g; h++)
            n += qU(h) < 0;
        return n;
    }
    __host__ __device__ static constexpr int d_plane(int g)  // float plane index
    {
        int n = 2 * n_su();
        for (int h = 0; h < NG; h++)
            n += qU(h) < 0;
        for (int h = 0; h < g; h++)
            n += qD(h) >= 0;
        return n;
    }
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

// Population-plane offsets (floats) of group g's cells at plane cell `cell`
// (compile-time plane offsets).
template <int Q, int TX, int TY, typename ST>
struct PopCell {
    using G = TileGeom<TX, TY, ST>;
    using PG = PopGroups<Q>;
    static constexpr int PLANE = G::PY * G::PX;
    template <int g>
    __device__ static int su(int cell)
    {
        constexpr int off = 2 * PG::su_plane(g) * PLANE;
        return off + 2 * cell;
    }
    template <int g>
    __device__ static int s(int cell)
    {
        constexpr int off = PG::s_plane(g) * PLANE;
        return off + cell;
    }
    template <int g>
    __device__ static int d(int cell)
    {
        constexpr int off = PG::d_plane(g) * PLANE;
        return off + cell;
    }
};

// Store the x-y movers of group g reconstructed at plane cell `cell`.
template <int Q, int TX, int TY, typename ST, int g>
__device__ __forceinline__ void store_group(float *pb, int cell, const RecPre &r, const float *m)
{
    using PG = PopGroups<Q>;
    using C = PopCell<Q, TX, TY, ST>;
    constexpr int qs = PG::qS(g), qu = PG::qU(g), qd = PG::qD(g);
    if constexpr (qu >= 0)
        *reinterpret_cast<float2 *>(pb + C::template su<g>(cell)) = make_float2(rec_q<Q, qs>(r, m), rec_q<Q, qu>(r, m));
    else
        pb[C::template s<g>(cell)] = rec_q<Q, qs>(r, m);
    if constexpr (qd >= 0)
        pb[C::template d<g>(cell)] = rec_q<Q, qd>(r, m);
}

// Reconstruct the x-y movers of ring node (rx, ry) that point into the tile
// (the groups with the given sign of cx or cy) and store them into pop plane pb.
template <int Q, int TX, int TY, int AXIS, int SIGN, typename ST>
__device__ __forceinline__ void ring_pops(const ST *sm, float *pb, int rx, int ry)
{
    using G = TileGeom<TX, TY, ST>;
    float m[10];
#pragma unroll
    for (int k = 0; k < 10; k++)
        m[k] = Storage<ST>::load_raw(sm[(k * G::RY + ry + 1) * G::TXP + rx + G::XPAD]);
    m[0] = rho_of_stored<ST>(m[0]);
    const RecPre r = rec_pre<Q, Storage<ST>::SCI>(m);
    const int cell = (ry + 1) * G::PX + rx + 1;
    static_for<0, PopGroups<Q>::NG>([&](auto gc) {
        constexpr int g = decltype(gc)::value;
        constexpr int c = AXIS == 0 ? group_cx(g) : group_cy(g);
        if constexpr (c == SIGN)
            store_group<Q, TX, TY, ST, g>(pb, cell, r, m);
    });
}

// ---------------------------------------------------------------- kernel
// Shared memory of a step CTA: mbarriers, TMA stage ring, population plane(s).
template <typename ST>
struct CtaSmem {
    uint64_t *bars;
    ST *stages;
    float *pops;
};
template <int Q, int TX, int TY, int NSTAGE, int NPB, typename ST>
__device__ __forceinline__ CtaSmem<ST> cta_smem(unsigned char *smem)
{
    using L = SmemLayout<Q, TX, TY, NSTAGE, NPB, ST>;
    return {reinterpret_cast<uint64_t *>(smem + L::bar_off), reinterpret_cast<ST *>(smem + L::stage_off),
            reinterpret_cast<float *>(smem + L::pop_off)};
}

// Per-thread monitor sums (monitored kernels only).
struct MonAcc {
    double mass = 0.0, ke = 0.0;
    unsigned bad = 0;
};

static __device__ __noinline__ void record_fault(StepFault *f, unsigned flag, int item, int mesh, int plane, unsigned seq,
                                          unsigned slot, unsigned parity, const uint64_t *bar)
{
    atomicOr(&f->flags, flag);
    if (atomicCAS(&f->recorded, 0u, 2u) == 0u) {
        f->block[0] = blockIdx.x;
        f->block[1] = blockIdx.y;
        f->block[2] = blockIdx.z;
        f->item = item;
        f->mesh = mesh;
        f->plane = plane;
        f->seq = seq;
        f->slot = slot;
        f->parity = parity;
        f->barrier = *reinterpret_cast<const volatile unsigned long long *>(bar);
        __threadfence();
        atomicExch(&f->recorded, 1u);
    }
}

// ---------------------------------------------------------- checked build
// With LBM_CHECKED (the separately built checked library, the stand-in for a
// memory checker on this hardware) the step kernels verify every shared-
// memory index, global node index and TMA coordinate before they use it.  A
// failed check sets ERR_BOUNDS in the fault record, with the check's number
// in `slot` and the place (block, item, plane), replaces a shared-memory
// index by 0 and skips a global store, so nothing outside the buffers is
// touched; lbm_synchronize then reports LBM_ERR_STATE.  The ordinary build
// compiles the checks away.
enum : unsigned { ERR_BOUNDS = 4u };
enum : unsigned { CHK_TMA_X = 1, CHK_TMA_PLANE = 2, CHK_STAGE = 3, CHK_POP = 4, CHK_NODE = 5, CHK_PTR = 6 };

static __device__ __noinline__ void record_bounds(StepFault *f, unsigned code, int item, int mesh, int plane,
                                                  unsigned seq)
{
    atomicOr(&f->flags, ERR_BOUNDS);
    if (atomicCAS(&f->recorded, 0u, 2u) == 0u) {
        f->block[0] = blockIdx.x;
        f->block[1] = blockIdx.y;
        f->block[2] = blockIdx.z;
        f->item = item;
        f->mesh = mesh;
        f->plane = plane;
        f->seq = seq;
        f->slot = code;
        f->parity = 0;
        f->barrier = 0;
        __threadfence();
        atomicExch(&f->recorded, 1u);
    }
}

#ifdef LBM_CHECKED
// cond holds, or the failure is recorded (false)
#define LBM_CHK(cond, code, plane) \
    ((cond) ? true : (record_bounds(p.fault, (code), item, mesh, (plane), g0 + unsigned(plane)), false))
// idx if 0 <= idx < limit, else 0 (and the failure recorded)
#define LBM_IDX(idx, limit, plane) (LBM_CHK((idx) >= 0 && (idx) < (limit), CHK_POP, plane) ? (idx) : 0)
#else
#define LBM_CHK(cond, code, plane) true
#define LBM_IDX(idx, limit, plane) (idx)
#endif

// One work item: tile (bx, by) of the x-y plane, z-chunk bz of the mesh that
// p and tmap describe.  The planes a CTA receives are numbered g0, g0+1, ...
// across all the items it processes, so that the stage slot (g % NSTAGE), the
// phase of its mbarrier ((g / NSTAGE) & 1) and the population plane (g & 1)
// keep cycling from one item to the next; the mbarriers are initialised once
// per CTA.  Returns false, uniformly across the CTA, when a TMA wait timed
// out (the error flag is then set).
//
// CLM selects the relaxation: 0 the plain collision; 1 the learned closure
// with dtau read per node from p.dtau; 2 the learned closure with the network
// evaluated in this kernel (mlp: the thread's group state, net: the network;
// see FusedMlp), the same dtau as mode 1 after mlp_infer_kernel, bit for bit.
// FO selects the function objects: 0 none; 1 those whose pointers in p.fo
// are set (checked per field at run time); 2 exactly S, SMean, k and kMean
// (the checks resolved at compile time, which measured 3% faster).
template <int Q, int TX, int TY, int NSTAGE, int FO, typename MeanT, bool MON, int NPB, typename ST, int CLM = 0>
__device__ __forceinline__ bool march_chunk(const CUtensorMap *tmap, const StepParams<MeanT, ST> &p, int bx, int by,
                                            int bz, unsigned g0, const CtaSmem<ST> &sh, int *s_abort, MonAcc &acc,
                                            int item = -1, int mesh = -1, FusedMlp *mlp = nullptr,
                                            const MlpDevice *net = nullptr)
{
    using G = TileGeom<TX, TY, ST>;
    using L = SmemLayout<Q, TX, TY, NSTAGE, NPB, ST>;
    using ZG = ZGroups<Q>;
    uint64_t *const bars = sh.bars;
    ST *const stages = sh.stages;
    float *const pops = sh.pops;

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int lin = ty * TX + tx;
    const int x0 = bx * TX, y0 = by * TY;
    const int z0 = p.z_lo + bz * p.zc;
    const int z1 = min(z0 + p.zc, p.z_hi);
    const int nplanes = z1 - z0 + 2;  // planes z0-1 .. z1
    const int x = x0 + tx, y = y0 + ty;
    const bool own = (x < p.nx) && (y < p.ny);
    const size_t N = size_t(p.nx) * p.ny * p.nz;
    const uint32_t plane32 = uint32_t(p.nx) * uint32_t(p.ny);
    const uint32_t row32 = uint32_t(y) * uint32_t(p.nx) + uint32_t(x);
    // node class bits of x and y (normalVector.cuh:321-334); z is added per plane
    const unsigned type_xy = (x == 0 ? WEST : 0u) | (x == p.nx - 1 ? EAST : 0u) | (y == 0 ? SOUTH : 0u) |
                             (y == p.ny - 1 ? NORTH : 0u);
    using PG = PopGroups<Q>;
    using C = PopCell<Q, TX, TY, ST>;
    static_assert(PG::d_plane(PG::NG) == XY<Q>::N, "population-plane groups cover the x-y movers");
    constexpr bool FO4 = FO == 2;  // S, SMean, k, kMean present, momentsMean absent
    const int my_cell = (ty + 1) * G::PX + tx + 1;
    constexpr int PCELLS = G::PX * G::PY;  // cells of one population-plane group
#ifdef LBM_CHECKED
    {
        // the TMA box starts 16-byte aligned in x; the item's planes lie in
        // the mesh; the staged plane holds this thread's row and column; the
        // output and function-object buffers the kernel writes exist
        (void)LBM_CHK(((x0 - G::XPAD) * Storage<ST>::BYTES) % 16 == 0, CHK_TMA_X, 0);
        (void)LBM_CHK(z0 >= 0 && z0 < z1 && z1 <= p.nz && z0 >= p.z_lo && z1 <= p.z_hi, CHK_TMA_PLANE, 0);
        (void)LBM_CHK(ty + 1 < G::RY && tx + G::XPAD < G::TXP, CHK_STAGE, 0);
        (void)LBM_CHK(p.out != nullptr && (!MON || p.mon != nullptr) &&
                          (!FO4 || (p.fo.S && p.fo.SMean && p.fo.k && p.fo.kMean)),
                      CHK_PTR, 0);
    }
#endif

    // first planes of the item (the slots were last read by ordinary loads)
#pragma unroll
    for (int s = 0; s < NSTAGE; s++) {
        const unsigned slot = (g0 + s) % NSTAGE;
        tma_issue_if(lin == 0 && s < nplanes, stages + slot * G::PLANE_FLOATS, tmap, x0 - G::XPAD, y0 - 1, z0 - 1 + s,
                     0, &bars[slot], G::PLANE_BYTES);
    }

    // Populations held in registers between planes: the up-movers of the
    // two previous planes (UA for even i, UB for odd i) and the same-plane
    // movers of the previous plane (S1).  The iteration for plane i reads
    // U(i-2) from its set and S(i-1) in the update, then overwrites both
    // with U(i) and S(i): without function objects the loop runs two planes
    // per trip and no population is moved between registers.
    float UA[ZG::NU], UB[ZG::NU], S1[ZG::NS];

    // U2 holds U(i-2) on entry; U(i) is written into Unew (which may be U2
    // itself: the update has read U2 before the plane's up-movers are pulled)
    auto plane_step = [&](const int i, float(&U2)[ZG::NU], float(&Unew)[ZG::NU]) -> bool {
        const int pz = z0 - 1 + i;  // plane being received
        const unsigned g = g0 + i;
        const int stage = g % NSTAGE;
        const unsigned parity = (g / NSTAGE) & 1;
        ST *sm = stages + stage * G::PLANE_FLOATS;
        float *pb = pops + (NPB == 2 ? (g & 1) : 0) * L::pop_floats;

        // running means of the node updated in this iteration (plane pz-1),
        // loaded early so the latency hides behind the reconstruction
        const int zu = pz - 1;
        const bool upd = (i >= 2) && own;
        // node offset within a field (32 bits: lbm_create keeps every mesh
        // below 2^32 nodes) against per-field base pointers, which are the
        // same for the whole CTA
        const uint32_t iu = uint32_t(zu) * plane32 + row32;
        MeanT sm_old[6], km_old = MeanT(0);
        float dtau = 0.0f;
        // this thread updates a node in this iteration (checked build: one in
        // this launch's planes and in the mesh); only such threads touch the
        // node's global fields
        const bool upd_node = upd && own && LBM_CHK(zu >= p.z_lo && zu < p.z_hi && size_t(iu) < N, CHK_NODE, i);
        if constexpr (CLM == 1) {
            if (upd_node)
                dtau = p.dtau[iu];
        }
        // the network runs for the planes this CTA updates (z0 .. z1-1)
        const bool net_plane = (i >= 1) && (i <= nplanes - 2);
        if constexpr (FO != 0) {
            if (upd_node) {
                if (FO4 || p.fo.SMean) {
#pragma unroll
                    for (int c = 0; c < 6; c++)
                        sm_old[c] = (p.fo.SMean + c * N)[iu];
                }
                if (FO4 || p.fo.kMean)
                    km_old = p.fo.kMean[iu];
            }
        }

        if (!mbar_wait_bounded(&bars[stage], parity, p.timeout_ns)) {
            record_fault(p.fault, ERR_TMA_TIMEOUT, item, mesh, i, g0 + i, stage, parity, &bars[stage]);
            *s_abort = 1;
        }

        // own node: reconstruct all directions
        float D0[ZG::ND];
        float own_up, own_rest;  // the pure-z up-mover and the rest population, kept for the next planes
        {
            float m[10];
#pragma unroll
            for (int k = 0; k < 10; k++)
                m[k] = Storage<ST>::load_raw(sm[(k * G::RY + ty + 1) * G::TXP + tx + G::XPAD]);
            if constexpr (CLM == 2) {
                // this node's network features, from the stored values
                if (net_plane) {
                    mlp->in_cur = fused_features(*mlp, *net, m) && own;
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                }
            }
            m[0] = rho_of_stored<ST>(m[0]);
            const RecPre r = rec_pre<Q, Storage<ST>::SCI>(m);
            const int cell = LBM_IDX(my_cell, PCELLS, i);
            static_for<0, PG::NG>([&](auto gc) { store_group<Q, TX, TY, ST, decltype(gc)::value>(pb, cell, r, m); });
            own_up = rec_q<Q, 5>(r, m);
            D0[zslot<Q>(6)] = rec_q<Q, 6>(r, m);
            own_rest = rec_q<Q, 0>(r, m);
        }
#ifdef LBM_CHECKED
        {
            // every ring node this thread reconstructs lies on the ring
            int rx = -2, ry = -2;
            if (TX == 32) {
                const int w = lin >> 5, l = lin & 31;
                if (w == 0) { rx = l; ry = -1; }
                else if (w == 1) { rx = l; ry = TY; }
                else if (w == 2 && l < TY + 2) { rx = -1; ry = l - 1; }
                else if (w == 3 && l < TY + 2) { rx = TX; ry = l - 1; }
            } else if (lin < G::RING) {
                int r = lin;
                if (r < TX + 2) { rx = r - 1; ry = -1; }
                else if ((r -= TX + 2) < TX + 2) { rx = r - 1; ry = TY; }
                else if ((r -= TX + 2) < TY) { rx = -1; ry = r; }
                else { rx = TX; ry = r - TY; }
            }
            if (rx != -2)
                (void)LBM_CHK(rx >= -1 && rx <= TX && ry >= -1 && ry <= TY && (rx == -1 || rx == TX || ry == -1 || ry == TY),
                              CHK_POP, i);
        }
#endif
        // ring nodes: only the directions that enter the tile.  With 32-wide
        // tiles each side goes to one warp (the bottom and top rows, x = 0..31,
        // to warps 0 and 1; the left and right columns, corners included, to
        // warps 2 and 3), so no warp runs two sides one after the other.
        if constexpr (TX == 32) {
            const int w = lin >> 5, l = lin & 31;
            if (w == 0) {
                ring_pops<Q, TX, TY, 1, +1, ST>(sm, pb, l, -1);
            } else if (w == 1) {
                ring_pops<Q, TX, TY, 1, -1, ST>(sm, pb, l, TY);
            } else if (w == 2) {
                if (l < TY + 2)
                    ring_pops<Q, TX, TY, 0, +1, ST>(sm, pb, -1, l - 1);
            } else if (w == 3) {
                if (l < TY + 2)
                    ring_pops<Q, TX, TY, 0, -1, ST>(sm, pb, TX, l - 1);
            }
        } else if (lin < G::RING) {
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
        if constexpr (CLM == 2)
            tc_fence_before();
        cta_sync();
        if (*s_abort)
            return false;
        if constexpr (CLM == 2) {
            if (net_plane)
                fused_issue_layer1(*mlp);
        }

        // the stage is consumed: refill it with plane i + NSTAGE
        (void)LBM_CHK(!(lin == 0 && i + NSTAGE < nplanes) || (pz + NSTAGE <= p.nz && pz + NSTAGE <= z1), CHK_TMA_PLANE, i);
        tma_issue_if(lin == 0 && i + NSTAGE < nplanes, sm, tmap, x0 - G::XPAD, y0 - 1, pz + NSTAGE, 0, &bars[stage],
                     G::PLANE_BYTES);

        // pull the down-movers (cz = -1) that land on plane pz-1
        static_for<0, PG::NG>([&](auto gc) {
            constexpr int g = decltype(gc)::value;
            constexpr int qd = PG::qD(g);
            constexpr int off = group_cy(g) * G::PX + group_cx(g);
            if constexpr (qd >= 0) {
                constexpr int sd = zslot<Q>(qd);
                D0[sd] = pb[C::template d<g>(LBM_IDX(my_cell - off, PCELLS, i))];
            }
        });

        if (i >= 2) {
            if constexpr (CLM == 2) {
                // dtau of the nodes updated now: layer 2 of the previous plane
                bool ok = true;
                dtau = fused_dtau(*mlp, *net, *s_abort ? 1000000ull : p.timeout_ns, ok);
                if (!ok) {
                    record_fault(p.fault, ERR_MMA_TIMEOUT, item, mesh, i, g0 + i, 2u, mlp->ph2 ^ 1u, mlp->bar2);
                    *s_abort = 1;
                }
            }
            // update plane zu = pz - 1 from U(pz-2), S(pz-1), D(pz)
            float f[Q];
            static_for<0, Q>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                constexpr int c = cz_of(q);
                if constexpr (c == 1) f[q] = U2[zslot<Q>(q)];
                if constexpr (c == 0) f[q] = S1[zslot<Q>(q)];
                if constexpr (c == -1) f[q] = D0[zslot<Q>(q)];
            });
            if (upd_node) {
                const unsigned type = type_xy | (zu == 0 ? BACK : 0u) | (zu == p.nz - 1 ? FRONT : 0u);
                float m[10];
                if constexpr (CLM != 0) {
                    // interior nodes relax with tau0 + dtau; omega as the host
                    // derives it from tau, so dtau = 0 gives the plain bits
                    Relax r = p.rx;
                    if (!type) {
                        r.omega = __fdiv_rn(1.0f, __fadd_rn(p.rx.tau, dtau));
                        r.t_omega = __fsub_rn(1.0f, r.omega);
                        r.omega_d2 = __fmul_rn(r.omega, 0.5f);
                    }
                    node_update<Q>(f, type, r, m);
                } else {
                    node_update<Q, Storage<ST>::SCI>(f, type, p.rx, m);
                }
                // m[1..9] come out of the collision scaled by SC, m[0] is rho
                p.out[iu] = Storage<ST>::store_raw(stored_of_rho<ST>(m[0]));
#pragma unroll
                for (int k = 1; k < 10; k++)
                    (p.out + k * N)[iu] = Storage<ST>::store_raw(m[k]);
                if constexpr (Storage<ST>::SC != 1.0f && (MON || FO != 0)) {
                    // the monitor and the function objects take the moments unscaled
#pragma unroll
                    for (int k = 1; k < 10; k++)
                        m[k] = m[k] * (1.0f / Storage<ST>::SC);
                }
                if constexpr (MON) {
                    acc.mass += double(m[0]);
                    acc.ke += double(m[0] * ((m[1] * m[1] + m[2] * m[2]) + m[3] * m[3]));
                    const float chk = (((m[0] + m[1]) + (m[2] + m[3])) + ((m[4] + m[5]) + (m[6] + m[7]))) + (m[8] + m[9]);
                    acc.bad += !isfinite(chk);
                }
                if constexpr (FO != 0) {
                    if (FO4 || p.fo.S || p.fo.SMean) {
                        float s6[6];
                        strain_rate(m, p.fo.sd, s6);
                        if (FO4 || p.fo.S) {
#pragma unroll
                            for (int c = 0; c < 6; c++)
                                (p.fo.S + c * N)[iu] = s6[c];
                        }
                        if (FO4 || p.fo.SMean) {
#pragma unroll
                            for (int c = 0; c < 6; c++)
                                (p.fo.SMean + c * N)[iu] = time_average<MeanT>(sm_old[c], MeanT(s6[c]), p.fo.inv_count);
                        }
                    }
                    if (FO4 || p.fo.k || p.fo.kMean) {
                        const float ke = kinetic(m[1], m[2], m[3]);
                        if (FO4 || p.fo.k)
                            p.fo.k[iu] = ke;
                        if (FO4 || p.fo.kMean)
                            p.fo.kMean[iu] = time_average<MeanT>(km_old, MeanT(ke), p.fo.inv_count);
                    }
                    if (!FO4 && p.fo.momentsMean) {
                        m[0] = m[0] - 1.0f;
#pragma unroll
                        for (int c = 0; c < 10; c++) {
                            MeanT *a = p.fo.momentsMean + c * N + iu;  // (rare path)
                            *a = time_average<MeanT>(*a, MeanT(m[c]), p.fo.inv_count);
                        }
                    }
                }
            }
        }

        if constexpr (CLM == 2) {
            // layer 1 of this plane -> layer-2 operand; layer 2 issued
            if (net_plane) {
                if (!fused_layer2(*mlp, *net, *s_abort ? 1000000ull : p.timeout_ns)) {
                    record_fault(p.fault, ERR_MMA_TIMEOUT, item, mesh, i, g0 + i, 1u, mlp->ph1 ^ 1u, mlp->bar1);
                    *s_abort = 1;
                }
                mlp->in_prev = mlp->in_cur;
            }
        }

        // keep this plane's same-plane and up-movers for the next updates
        static_for<0, PG::NG>([&](auto gc) {
            constexpr int g = decltype(gc)::value;
            constexpr int off = group_cy(g) * G::PX + group_cx(g);
            constexpr int qs = PG::qS(g), qu = PG::qU(g);
            constexpr int ss = zslot<Q>(qs);
            const int cell = LBM_IDX(my_cell - off, PCELLS, i);
            if constexpr (qu >= 0) {
                constexpr int su_slot = zslot<Q>(qu);
                const float2 su = *reinterpret_cast<const float2 *>(pb + C::template su<g>(cell));
                S1[ss] = su.x;
                Unew[su_slot] = su.y;
            } else {
                S1[ss] = pb[C::template s<g>(cell)];
            }
        });
        Unew[zslot<Q>(5)] = own_up;
        S1[zslot<Q>(0)] = own_rest;
        if constexpr (NPB == 1)
            cta_sync();  // the single population plane is rewritten next iteration
        return true;
    };

    if constexpr (FO != 0 || CLM == 2) {
        // with the function objects or the fused network the body is large:
        // one plane per trip, the up-mover sets rotated by register moves
        // (two unrolled copies of these bodies measured slower)
        // (UA: U(i-2), UB: U(i-1); the new set rotates in with two moves per
        // direction)
        for (int i = 0; i < nplanes; i++) {
            float U0[ZG::NU];
            if (!plane_step(i, UA, U0))
                return false;
#pragma unroll
            for (int k = 0; k < ZG::NU; k++) {
                UA[k] = UB[k];
                UB[k] = U0[k];
            }
        }
    } else {
        for (int i = 0; i < nplanes; i += 2) {
            if (!plane_step(i, UA, UA))
                return false;
            if (i + 1 < nplanes && !plane_step(i + 1, UB, UB))
                return false;
        }
    }
    return true;
}

// CTA sums of the monitor, then one FP64 atomic per quantity.
template <int NT>
__device__ __forceinline__ void monitor_flush(MonAcc a, MonitorSlot *mon, int lin)
{
    for (int o = 16; o > 0; o >>= 1) {
        a.mass += __shfl_down_sync(0xffffffffu, a.mass, o);
        a.ke += __shfl_down_sync(0xffffffffu, a.ke, o);
        a.bad += __shfl_down_sync(0xffffffffu, a.bad, o);
    }
    __shared__ double s_mon[2][NT / 32];
    __shared__ unsigned s_bad[NT / 32];
    const int lane = lin & 31, wid = lin >> 5;
    if (lane == 0) {
        s_mon[0][wid] = a.mass;
        s_mon[1][wid] = a.ke;
        s_bad[wid] = a.bad;
    }
    cta_sync();
    if (lin == 0) {
        double m = 0.0, k = 0.0;
        unsigned long long c = 0;
        for (int w = 0; w < NT / 32; w++) {
            m += s_mon[0][w];
            k += s_mon[1][w];
            c += s_bad[w];
        }
        atomicAdd(&mon->mass, m);
        atomicAdd(&mon->rho_u2, k);
        atomicAdd(&mon->nonfinite, c);
    }
}

template <int NSTAGE>
__device__ __forceinline__ void init_barriers(uint64_t *bars, bool pred)
{
#pragma unroll
    for (int s = 0; s < NSTAGE; s++)
        mbar_init_if(pred, &bars[s]);
    fence_mbar_init_if(pred);
}

// After a timeout: give TMA copies still in flight a bounded chance to land
// before the CTA exits (both phases are polled, each for at most 1 ms).
template <int NSTAGE>
__device__ __forceinline__ void drain_after_abort(uint64_t *bars)
{
    for (int s = 0; s < NSTAGE; s++)
        for (unsigned ph = 0; ph < 2; ph++)
            (void)mbar_wait_bounded(&bars[s], ph, 1000000ull);
}

// One step of one mesh: CTA (bx, by, bz) of the grid marches its work item.
template <int Q, int TX, int TY, int NSTAGE, int FO, typename MeanT, bool MON = false, int NPB = 2, int MINB = 2,
          typename ST = float>
__global__ void __launch_bounds__(TX *TY, MINB)
    step_kernel(const __grid_constant__ CUtensorMap tmap_in, const StepParams<MeanT, ST> p)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_abort;
    const CtaSmem<ST> sh = cta_smem<Q, TX, TY, NSTAGE, NPB, ST>(smem);
    const int lin = threadIdx.y * TX + threadIdx.x;
    init_barriers<NSTAGE>(sh.bars, lin == 0);
    s_abort = 0;
    cta_sync();
    MonAcc acc;
    march_chunk<Q, TX, TY, NSTAGE, FO, MeanT, MON, NPB, ST>(&tmap_in, p, blockIdx.x, blockIdx.y, blockIdx.z, 0u, sh,
                                                            &s_abort, acc);
    if constexpr (MON)
        monitor_flush<TX * TY>(acc, p.mon, lin);
    if (s_abort && lin == 0)
        drain_after_abort<NSTAGE>(sh.bars);
}

// One step with the learned closure: as step_kernel (no function objects,
// FP32 storage), each interior node relaxing with tau0 + p.dtau[node].
template <int Q, int TX, int TY, int NSTAGE, int NPB, int MINB>
__global__ void __launch_bounds__(TX *TY, MINB)
    closure_kernel(const __grid_constant__ CUtensorMap tmap_in, const StepParams<float, float> p)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_abort;
    const CtaSmem<float> sh = cta_smem<Q, TX, TY, NSTAGE, NPB, float>(smem);
    const int lin = threadIdx.y * TX + threadIdx.x;
    init_barriers<NSTAGE>(sh.bars, lin == 0);
    s_abort = 0;
    cta_sync();
    MonAcc acc;
    march_chunk<Q, TX, TY, NSTAGE, false, float, false, NPB, float, 1>(&tmap_in, p, blockIdx.x, blockIdx.y,
                                                                       blockIdx.z, 0u, sh, &s_abort, acc);
    if (s_abort && lin == 0)
        drain_after_abort<NSTAGE>(sh.bars);
}

// Shared-memory offset of the fused network's operands (after the step's
// own layout, 128-byte aligned) and the total for a closure_fused_kernel CTA.
template <int Q, int TX, int TY, int NSTAGE, int NPB>
struct FusedLayout {
    using L = SmemLayout<Q, TX, TY, NSTAGE, NPB, float>;
    static constexpr int NG = TX * TY / 128;
    static constexpr size_t mlp_off = (L::bytes + 127) / 128 * 128;
    static constexpr size_t bytes = mlp_off + FusedMlpSmem::Of<NG>::BYTES;
};

// One step with the learned closure, the network evaluated in the kernel
// (march_chunk mode 2): FP32 storage, no function objects; every interior
// node relaxes with tau0 + dtau from the network on its moments at the start
// of the step -- the result of mlp_infer_kernel followed by closure_kernel,
// bit for bit, without the per-node dtau array.  Tiles of 128 or 256
// threads (one or two network groups).
template <int Q, int TX, int TY, int NSTAGE, int NPB, int MINB>
__global__ void __launch_bounds__(TX *TY, MINB)
    closure_fused_kernel(const __grid_constant__ CUtensorMap tmap_in, const StepParams<float, float> p,
                         const __grid_constant__ MlpDevice net)
{
    constexpr int NT = TX * TY;
    static_assert(NT % 128 == 0 && NT <= 256, "one or two groups of four warps");
    using FL = FusedLayout<Q, TX, TY, NSTAGE, NPB>;
    using MS = FusedMlpSmem;
    using MG = FusedMlpSmem::Of<FL::NG>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_abort;
    const CtaSmem<float> sh = cta_smem<Q, TX, TY, NSTAGE, NPB, float>(smem);
    unsigned char *ms = smem + FL::mlp_off;
    const int lin = threadIdx.y * TX + threadIdx.x;
    const int warp = lin >> 5, grp = lin >> 7;
    {
        // FP16 weights (already in the operand layout) into shared memory
        const uint32_t *g = reinterpret_cast<const uint32_t *>(net.w1);
        uint32_t *d = reinterpret_cast<uint32_t *>(ms + MS::W1);
        constexpr int n4 = (MS::GROUP0 - MS::W1) / 4;
        static_assert(sizeof(net.w1) + sizeof(net.w2) == MS::GROUP0 - MS::W1, "weights");
        for (int k = lin; k < n4; k += NT)
            d[k] = g[k];
    }
    uint64_t *mbars = reinterpret_cast<uint64_t *>(ms + MG::BARS);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(ms + MG::TMEM);
#pragma unroll
    for (int s = 0; s < NSTAGE; s++)
        mbar_init_if(lin == 0, &sh.bars[s]);
#pragma unroll
    for (int b = 0; b < 2 * FL::NG; b++)
        mbar_init_if(lin == 0, &mbars[b]);
    fence_mbar_init_if(lin == 0);
    s_abort = 0;
    if (warp == 0)
        tmem_alloc_warp(tslot, MG::COLS);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the weights, for the MMAs
    tc_fence_before();
    cta_sync();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    FusedMlp f;
    f.w1 = reinterpret_cast<__half *>(ms + MS::W1);
    f.w2 = reinterpret_cast<__half *>(ms + MS::W2);
    f.a1 = reinterpret_cast<__half *>(ms + MS::GROUP0 + grp * MS::GROUP_BYTES + MS::A1);
    f.a2 = reinterpret_cast<__half *>(ms + MS::GROUP0 + grp * MS::GROUP_BYTES + MS::A2);
    f.bar1 = &mbars[2 * grp];
    f.bar2 = &mbars[2 * grp + 1];
    f.t1_issue = tbase + uint32_t(grp * 64);  // columns: layer 1 at +0, layer 2 at +32
    f.t2_issue = f.t1_issue + 32u;
    const uint32_t lanes = uint32_t((warp & 3) * 32) << 16;
    f.tm1 = f.t1_issue + lanes;
    f.tm2 = f.t2_issue + lanes;
    f.row = lin & 127;
    f.group = grp;
    f.leader = (lin & 127) == 0;
    f.ph1 = f.ph2 = 0u;
    f.in_prev = f.in_cur = false;
    MonAcc acc;
    march_chunk<Q, TX, TY, NSTAGE, false, float, false, NPB, float, 2>(&tmap_in, p, blockIdx.x, blockIdx.y,
                                                                       blockIdx.z, 0u, sh, &s_abort, acc, -1, -1,
                                                                       &f, &net);
    if (s_abort) {
        if (lin == 0)
            drain_after_abort<NSTAGE>(sh.bars);
        if (f.leader) {
            // MMAs possibly still in flight: a bounded chance to finish
            // before their tensor memory is released
            for (unsigned ph = 0; ph < 2; ph++) {
                (void)mbar_wait_bounded(f.bar1, ph, 1000000ull);
                (void)mbar_wait_bounded(f.bar2, ph, 1000000ull);
            }
        }
    }
    tc_fence_before();
    cta_sync();
    tc_fence_after();
    if (warp == 0)
        tmem_dealloc_warp(tbase, MG::COLS);
}

// ------------------------------------------------------------ batches
// Many independent meshes advanced by one launch per step: a persistent grid
// (as many CTAs as fit on the GPU at once) takes work items -- one tile and
// z-chunk of one mesh each -- from a global counter until all are done.
// Items are numbered mesh by mesh in the order of the mesh table, which the
// host sorts so that the biggest items come first.
struct BatchMesh {
    float *m[2];          // moment buffers [10][nz][ny][nx] (FP32)
    int nx, ny, nz, zc;   // mesh and z-planes per work item
    int tiles_x, tiles_y; // tiles per x-y plane
    int item_begin;       // first work item of this mesh
    int cur;              // buffer that holds the state when flip == 0
    Relax rx;
};

struct BatchParams {
    const BatchMesh *mesh;   // [nmesh], item_begin ascending
    const CUtensorMap *tmap; // [2 * nmesh]: buffer b of mesh i at 2 i + b (global memory)
    int nmesh, items;
    unsigned *next;          // next unclaimed work item
    unsigned *done;          // CTAs that have finished; the last one resets both counters
    StepFault *fault;
    uint64_t timeout_ns;
    int persistent;          // 1: CTAs claim items from *next; 0: one item per CTA, item = blockIdx.x
};

// Acquire a tensor map that was written to global memory by a copy from the
// host before the launch, for use by the tensor-map proxy.  The writer is the
// host, so the fence takes system scope.
__device__ __forceinline__ void tmap_acquire_if(bool pred, const CUtensorMap *map)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "@p fence.proxy.tensormap::generic.acquire.sys [%0], 128;\n\t}" ::"l"(reinterpret_cast<uint64_t>(map)),
        "r"(unsigned(pred))
        : "memory");
}

template <int Q, int TX, int TY, int NSTAGE, int NPB, int MINB>
__global__ void __launch_bounds__(TX *TY, MINB) batch_kernel(const BatchParams bp, const int flip)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_abort, s_item;
    const CtaSmem<float> sh = cta_smem<Q, TX, TY, NSTAGE, NPB, float>(smem);
    const int lin = threadIdx.y * TX + threadIdx.x;
    init_barriers<NSTAGE>(sh.bars, lin == 0);
    s_abort = 0;
    MonAcc acc;
    unsigned g = 0;  // planes received so far by this CTA
    for (int round = 0;; round++) {
        // s_item is rewritten only after every thread has passed a barrier
        // inside march_chunk, i.e. after all of them have read it
        if (lin < 32) {
            // warp 0 claims the item together (the shuffle keeps it converged)
            unsigned v = 0;
            if (bp.persistent) {
                if (lin == 0)
                    v = atomicAdd(bp.next, 1u);
                v = __shfl_sync(0xffffffffu, v, 0);
            } else {
                v = round == 0 ? blockIdx.x : unsigned(bp.items);
            }
            if (lin == 0)
                s_item = int(v);
        }
        cta_sync();
        const int item = s_item;
        if (item >= bp.items)
            break;
        int lo = 0, hi = bp.nmesh - 1;  // last mesh with item_begin <= item
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (bp.mesh[mid].item_begin <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        const BatchMesh &bm = bp.mesh[lo];
        const int in = bm.cur ^ flip;
        StepParams<float, float> p{};
        p.out = bm.m[in ^ 1];
        p.mon = nullptr;
        p.nx = bm.nx;
        p.ny = bm.ny;
        p.nz = bm.nz;
        p.zc = bm.zc;
        p.z_lo = 0;
        p.z_hi = bm.nz;
        p.rx = bm.rx;
        p.fault = bp.fault;
        p.timeout_ns = bp.timeout_ns;
        const int local = item - bm.item_begin;
        const int bx = local % bm.tiles_x, rest = local / bm.tiles_x;
        const int by = rest % bm.tiles_y, bz = rest / bm.tiles_y;
        const CUtensorMap *map = bp.tmap + 2 * lo + in;
        tmap_acquire_if(lin == 0, map);
        if (!march_chunk<Q, TX, TY, NSTAGE, false, float, false, NPB, float>(map, p, bx, by, bz, g, sh, &s_abort, acc,
                                                                            item, lo))
            break;
        g += unsigned(min(p.zc, p.nz - bz * p.zc) + 2);
    }
    if (lin == 0) {
        if (s_abort)
            drain_after_abort<NSTAGE>(sh.bars);
        __threadfence();
        if (atomicAdd(bp.done, 1u) == gridDim.x - 1) {
            *bp.next = 0;
            *bp.done = 0;
        }
    }
}

}  // namespace lbm
