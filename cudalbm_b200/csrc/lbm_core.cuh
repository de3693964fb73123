// lbm_core.cuh -- per-node arithmetic of the moment-representation LBM step.
//
// Device functions shared by the step kernels: the lattice tables, the
// regularised reconstruction of populations from the 10 scaled moments, the
// interior moment sums, the wet-node boundary moments of the closed lid-driven
// cavity, the scaling and the second-order collision, and the run-time
// function objects.  Each follows the reference's expression order so that
// nvcc rounds it the same way:
//
//   reconstruction     src/velocitySet/D3Q19.cuh:311-374, D3Q27.cuh:248-331
//   moment sums        src/velocitySet/velocitySet.cuh:337-438 (right folds)
//   incoming mask      src/velocitySet/velocitySet.cuh:204-220
//   boundary moments   src/boundaryConditions/boundaryConditions.cuh:99-554
//   node classes       src/boundaryConditions/normalVector.cuh:73-335
//   scale              src/velocitySet/velocitySet.cuh:130-142
//   collision          src/collision/secondOrder.cuh:93-105
//   S, k, time means   src/functionObjects/strainRateTensor.cuh:71-90,
//                      kineticEnergy.cuh:72-85, functionObjects.cuh:79-97
#pragma once

#include <cstdint>

namespace lbm {

// ---------------------------------------------------------------- lattice
// D3Q27 ordering; its first 19 directions are D3Q19.
__host__ __device__ constexpr int cx_of(int q)
{
    constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[q];
}
__host__ __device__ constexpr int cy_of(int q)
{
    constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return t[q];
}
__host__ __device__ constexpr int cz_of(int q)
{
    constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[q];
}

// Directions that move in the x-y plane (exchanged through shared memory by
// the z-marching kernel): every q except rest (0) and the pure-z pair (5, 6).
template <int Q>
struct XY {
    static constexpr int N = Q - 3;
    __host__ __device__ static constexpr int q(int s) { return s < 4 ? s + 1 : s + 3; }
};

// Number of directions with a given cz (the rest direction counts as cz = 0).
template <int Q>
__host__ __device__ constexpr int count_cz(int c)
{
    int n = 0;
    for (int q = 0; q < Q; q++)
        n += (cz_of(q) == c);
    return n;
}
// Position of q among the directions sharing its cz value (ascending q).
template <int Q>
__host__ __device__ constexpr int zslot(int q)
{
    int n = 0;
    for (int r = 0; r < q; r++)
        n += (cz_of(r) == cz_of(q));
    return n;
}
template <int Q>
__host__ __device__ constexpr int q_of_zslot(int c, int s)
{
    for (int q = 0; q < Q; q++)
        if (cz_of(q) == c && zslot<Q>(q) == s)
            return q;
    return -1;
}

struct Consts {
    static constexpr float cs2 = static_cast<float>(1.0 / 3.0);
};

// Weight class of q: 0 rest, 1 axis, 2 face diagonal, 3 body diagonal.
__host__ __device__ constexpr int wclass(int q)
{
    return (cx_of(q) != 0) + (cy_of(q) != 0) + (cz_of(q) != 0);
}
template <int Q>
__host__ __device__ constexpr float weight(int cls)
{
    return Q == 19 ? (cls == 0 ? static_cast<float>(1.0 / 3.0) : cls == 1 ? static_cast<float>(1.0 / 18.0) : static_cast<float>(1.0 / 36.0))
                   : (cls == 0 ? static_cast<float>(8.0 / 27.0) : cls == 1 ? static_cast<float>(2.0 / 27.0)
                      : cls == 2 ? static_cast<float>(1.0 / 54.0) : static_cast<float>(1.0 / 216.0));
}

// ------------------------------------------------------ reconstruction
// Bracketing per direction, as written in the reference:
//   rhow * (((((pics2 +- u) +- v) +- w) + m_xx) + m_yy ...  +- m_ab)
//   body diagonals: ... + m_zz) +- (m_xy +- m_xz +- m_yz)
struct RecPre {
    float pics2;
    float rhow[4];
};

// m[0] is rho; m[1..9] are the stored moments times SC = SCI, a power of two
// (1 for the reference's values).  Every term of a population's bracket then
// carries the factor SC and the weight carries 1/SC: each rounding is the
// unscaled one scaled by an exact power of two, so the populations are the
// same bits for every SC.
template <int Q, int SCI = 1>
__device__ __forceinline__ RecPre rec_pre(const float *m)
{
    constexpr float SC = float(SCI);
    RecPre r;
    r.pics2 = SC - Consts::cs2 * (m[4] + m[7] + m[9]);
    r.rhow[0] = m[0] * (weight<Q>(0) / SC);
    r.rhow[1] = m[0] * (weight<Q>(1) / SC);
    r.rhow[2] = m[0] * (weight<Q>(2) / SC);
    r.rhow[3] = m[0] * (weight<Q>(3) / SC);
    return r;
}

template <int Q, int q>
__device__ __forceinline__ float rec_q(const RecPre &r, const float *m)
{
    constexpr int cx = cx_of(q), cy = cy_of(q), cz = cz_of(q);
    constexpr int nnz = (cx != 0) + (cy != 0) + (cz != 0);
    if constexpr (q == 0) {
        return r.rhow[0] * r.pics2;
    } else {
        float s = r.pics2;
        if constexpr (cx > 0) s = s + m[1];
        if constexpr (cx < 0) s = s - m[1];
        if constexpr (cy > 0) s = s + m[2];
        if constexpr (cy < 0) s = s - m[2];
        if constexpr (cz > 0) s = s + m[3];
        if constexpr (cz < 0) s = s - m[3];
        if constexpr (cx != 0) s = s + m[4];
        if constexpr (cy != 0) s = s + m[7];
        if constexpr (cz != 0) s = s + m[9];
        if constexpr (nnz == 2) {
            if constexpr (cx != 0 && cy != 0) {
                if constexpr (cx * cy > 0) s = s + m[5]; else s = s - m[5];
            }
            if constexpr (cx != 0 && cz != 0) {
                if constexpr (cx * cz > 0) s = s + m[6]; else s = s - m[6];
            }
            if constexpr (cy != 0 && cz != 0) {
                if constexpr (cy * cz > 0) s = s + m[8]; else s = s - m[8];
            }
        }
        if constexpr (nnz == 3) {
            constexpr int sxy = cx * cy, s6 = sxy * cx * cz, s8 = sxy * cy * cz;
            float g;
            if constexpr (s6 > 0) g = m[5] + m[6]; else g = m[5] - m[6];
            if constexpr (s8 > 0) g = g + m[8]; else g = g - m[8];
            if constexpr (sxy > 0) s = s + g; else s = s - g;
        }
        return r.rhow[nnz] * s;
    }
}

// ------------------------------------------------------- moment sums
// sum over q (ascending, nonzero weight c_a c_b) of c_a c_b f_q, evaluated as
// the reference's unary right fold: E0 + (E1 + (... + (E_{n-2} + E_{n-1}))).
// A, B in {-1 (none), 0 (x), 1 (y), 2 (z)}.
__host__ __device__ constexpr int cdir(int a, int q)
{
    return a < 0 ? 1 : (a == 0 ? cx_of(q) : (a == 1 ? cy_of(q) : cz_of(q)));
}

template <int Q, int A, int B, int q>
__device__ __forceinline__ float fold_from(const float *f)
{
    if constexpr (q >= Q) {
        return 0.0f;  // never used as a value: see has_term
    } else {
        constexpr int c = cdir(A, q) * cdir(B, q);
        // find next q with nonzero coefficient
        constexpr int nq = [] {
            int r = q + 1;
            while (r < Q && cdir(A, r) * cdir(B, r) == 0) r++;
            return r;
        }();
        if constexpr (c == 0) {
            return fold_from<Q, A, B, nq>(f);
        } else {
            const float e = (c > 0) ? f[q] : -f[q];
            if constexpr (nq >= Q)
                return e;
            else
                return e + fold_from<Q, A, B, nq>(f);
        }
    }
}

// node class bits (normalVector.cuh:321-334)
enum : unsigned { WEST = 0x01, EAST = 0x02, SOUTH = 0x04, NORTH = 0x08, BACK = 0x10, FRONT = 0x20 };

__device__ __forceinline__ unsigned node_type(int x, int y, int z, int nx, int ny, int nz)
{
    return (x == 0 ? WEST : 0u) | (x == nx - 1 ? EAST : 0u) | (y == 0 ? SOUTH : 0u) | (y == ny - 1 ? NORTH : 0u) |
           (z == 0 ? BACK : 0u) | (z == nz - 1 ? FRONT : 0u);
}

// Bit q set if direction q has the given sign along the given axis.
template <int AXIS, int SIGN>
__host__ __device__ constexpr unsigned dir_mask()
{
    unsigned m = 0;
    for (int q = 0; q < 27; q++) {
        const int c = AXIS == 0 ? cx_of(q) : (AXIS == 1 ? cy_of(q) : cz_of(q));
        if (c == SIGN)
            m |= 1u << q;
    }
    return m;
}

// Directions that stream into a node of class t from outside the domain
// (the complement of incomingSwitch, velocitySet.cuh:204-220).
__device__ __forceinline__ unsigned unknown_dirs(unsigned t)
{
    return ((t & EAST) ? dir_mask<0, -1>() : 0u) | ((t & WEST) ? dir_mask<0, 1>() : 0u) |
           ((t & NORTH) ? dir_mask<1, -1>() : 0u) | ((t & SOUTH) ? dir_mask<1, 1>() : 0u) |
           ((t & FRONT) ? dir_mask<2, -1>() : 0u) | ((t & BACK) ? dir_mask<2, 1>() : 0u);
}

// The reference sums incomingSwitch*f_q with incomingSwitch in {0, 1}.  A zero
// term leaves a right fold's value unchanged, so zeroing the unknown f_q and
// folding as for an interior node gives the same bits as the masked sums.
template <int Q, int q = 0>
__device__ __forceinline__ void zero_unknown(float *f, unsigned unknown)
{
    if constexpr (q < Q) {
        f[q] = ((unknown >> q) & 1u) ? 0.0f : f[q];
        zero_unknown<Q, q + 1>(f, unknown);
    }
}

// The ten raw sums the moments are built from: sum f, sum f c_a, sum f c_a c_b.
template <int Q>
__device__ __forceinline__ void moment_folds(const float *f, float *s)
{
    s[0] = fold_from<Q, -1, -1, 0>(f);
    s[1] = fold_from<Q, 0, -1, 0>(f);
    s[2] = fold_from<Q, 1, -1, 0>(f);
    s[3] = fold_from<Q, 2, -1, 0>(f);
    s[4] = fold_from<Q, 0, 0, 0>(f);
    s[5] = fold_from<Q, 0, 1, 0>(f);
    s[6] = fold_from<Q, 0, 2, 0>(f);
    s[7] = fold_from<Q, 1, 1, 0>(f);
    s[8] = fold_from<Q, 1, 2, 0>(f);
    s[9] = fold_from<Q, 2, 2, 0>(f);
}

struct Relax {
    float omega, t_omega, omega_d2, tau, u_lid;
};

// Interior moments (unscaled) from the folds: velocitySet.cuh:398-417.
__device__ __forceinline__ void interior_moments(const float *s, float *mom)
{
    mom[0] = s[0];
    const float inv_rho = 1.0f / mom[0];
    mom[1] = s[1] * inv_rho;
    mom[2] = s[2] * inv_rho;
    mom[3] = s[3] * inv_rho;
    mom[4] = (s[4] * inv_rho) - Consts::cs2;
    mom[5] = s[5] * inv_rho;
    mom[6] = s[6] * inv_rho;
    mom[7] = (s[7] * inv_rho) - Consts::cs2;
    mom[8] = s[8] * inv_rho;
    mom[9] = (s[9] * inv_rho) - Consts::cs2;
}

// Wet-node boundary moments (unscaled), boundaryConditions.cuh:99-533, from
// the folds of the known populations (s[0] = rho_I, s[5,6,8] = the raw
// c_a c_b sums whose quotients by rho_I are the reference's m_ab_I).
template <int Q>
__device__ __forceinline__ void boundary_moments(const float *s, unsigned t, const Relax &rx, float *mom)
{
    const float rho_I = s[0];
    const float inv_rho_I = 1.0f / rho_I;
    const float omega = rx.omega;
    const float U = rx.u_lid;

    {
        const float nB = static_cast<float>(__popc(t & 0x3Fu));
        // U<alpha>: only the North wall moves (U_North = {u_inf, 0, 0}); the
        // mean over the node's nB walls.  A zero numerator gives +0 for every
        // nB, so only the North lid divides (the zero quotients are written
        // as such: a zero numerator sends the IEEE division to its slow path)
        mom[1] = (t & NORTH) ? U / nB : 0.0f;
        mom[2] = 0.0f;
        mom[3] = 0.0f;
        mom[4] = mom[1] * mom[1];
    }
    mom[7] = 0.0f;
    mom[9] = 0.0f;

#define LBM_MXY_I (s[5] * inv_rho_I)
#define LBM_MXZ_I (s[6] * inv_rho_I)
#define LBM_MYZ_I (s[8] * inv_rho_I)
    switch (t) {
    case SOUTH | WEST | BACK:
    case SOUTH | WEST | FRONT:
    case SOUTH | EAST | BACK:
    case SOUTH | EAST | FRONT:
        if constexpr (Q == 19)
            mom[0] = 12.0f * rho_I / 7.0f;
        else
            mom[0] = 216.0f * rho_I / 125.0f;
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    case SOUTH | WEST: {
        const float mxy_I = LBM_MXY_I;
        mom[0] = 36.0f * (rho_I - mxy_I * rho_I + mxy_I * rho_I * omega) / (24.0f + omega);
        mom[5] = (36.0f * mxy_I * rho_I - mom[0]) / (9.0f * mom[0]);
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    }
    case SOUTH | EAST: {
        const float mxy_I = LBM_MXY_I;
        mom[0] = -36.0f * (-rho_I - mxy_I * rho_I + mxy_I * rho_I * omega) / (24.0f + omega);
        mom[5] = (36.0f * mxy_I * rho_I + mom[0]) / (9.0f * mom[0]);
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    }
    case WEST | BACK:
    case EAST | FRONT: {
        const float mxz_I = LBM_MXZ_I;
        const float rho = 36.0f * (rho_I - mxz_I * rho_I + mxz_I * rho_I * omega) / (24.0f + omega);
        const float mxz = (36.0f * mxz_I * rho_I - rho) / (9.0f * rho);
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = mxz;
        mom[8] = 0.0f;
        return;
    }
    case WEST | FRONT:
    case EAST | BACK: {
        const float mxz_I = LBM_MXZ_I;
        const float rho = -36.0f * (-rho_I - mxz_I * rho_I + mxz_I * rho_I * omega) / (24.0f + omega);
        const float mxz = (36.0f * mxz_I * rho_I + rho) / (9.0f * rho);
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = mxz;
        mom[8] = 0.0f;
        return;
    }
    case SOUTH | BACK: {
        const float myz_I = LBM_MYZ_I;
        const float rho = 36.0f * (rho_I - myz_I * rho_I + myz_I * rho_I * omega) / (24.0f + omega);
        const float myz = (36.0f * myz_I * rho_I - rho) / (9.0f * rho);
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = myz;
        return;
    }
    case SOUTH | FRONT: {
        const float myz_I = LBM_MYZ_I;
        const float rho = -36.0f * (-rho_I - myz_I * rho_I + myz_I * rho_I * omega) / (24.0f + omega);
        const float myz = (36.0f * myz_I * rho_I + rho) / (9.0f * rho);
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = myz;
        return;
    }
    case WEST:
    case EAST: {
        const float mxy_I = LBM_MXY_I;
        const float mxz_I = LBM_MXZ_I;
        const float rho = 6.0f * rho_I / 5.0f;
        mom[0] = rho;
        mom[5] = 2.0f * mxy_I * rho_I / rho;
        mom[6] = 2.0f * mxz_I * rho_I / rho;
        mom[8] = 0.0f;
        return;
    }
    case SOUTH: {
        const float mxy_I = LBM_MXY_I;
        const float myz_I = LBM_MYZ_I;
        const float rho = 6.0f * rho_I / 5.0f;
        mom[0] = rho;
        mom[5] = 2.0f * mxy_I * rho_I / rho;
        mom[6] = 0.0f;
        mom[8] = 2.0f * myz_I * rho_I / rho;
        return;
    }
    case BACK:
    case FRONT: {
        const float mxz_I = LBM_MXZ_I;
        const float myz_I = LBM_MYZ_I;
        const float rho = 6.0f * rho_I / 5.0f;
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = 2.0f * mxz_I * rho_I / rho;
        mom[8] = 2.0f * myz_I * rho_I / rho;
        return;
    }
    case NORTH: {
        const float mxy_I = LBM_MXY_I;
        const float myz_I = LBM_MYZ_I;
        const float rho = 6.0f * rho_I / 5.0f;
        mom[0] = rho;
        mom[5] = (6.0f * mxy_I * rho_I - U * rho) / (3.0f * rho);
        mom[6] = 0.0f;
        mom[8] = 2.0f * myz_I * rho_I / rho;
        return;
    }
    case NORTH | WEST | BACK:
    case NORTH | WEST | FRONT:
        mom[0] = -24.0f * rho_I / (-14.0f - 8.0f * U + 9.0f * U * U);
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    case NORTH | EAST | BACK:
    case NORTH | EAST | FRONT:
        mom[0] = -24.0f * rho_I / (-14.0f + 8.0f * U + 9.0f * U * U);
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    case NORTH | BACK: {
        const float myz_I = LBM_MYZ_I;
        const float rho = 72.0f * (-rho_I - myz_I * rho_I + myz_I * rho_I * omega) / (-48.0f - 2.0f * omega + 3.0f * U * U * omega);
        const float myz = (72.0f * myz_I * rho_I + 2.0f * rho - 3.0f * U * U * rho) / (18.0f * rho);
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = myz;
        return;
    }
    case NORTH | FRONT: {
        const float myz_I = LBM_MYZ_I;
        const float rho = -72.0f * (rho_I - myz_I * rho_I + myz_I * rho_I * omega) / (-48.0f - 2.0f * omega + 3.0f * U * U * omega);
        const float myz = (72.0f * myz_I * rho_I - 2.0f * rho + 3.0f * U * U * rho) / (18.0f * rho);
        mom[0] = rho;
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = myz;
        return;
    }
    case NORTH | EAST: {
        const float mxy_I = LBM_MXY_I;
        const float rho = 36.0f * (rho_I - mxy_I * rho_I + mxy_I * rho_I * omega) /
                          (24.0f - 18.0f * U - 18.0f * U * U + omega + 3.0f * U * omega + 3.0f * U * U * omega);
        const float mxy = (36.0f * mxy_I * rho_I - rho - 3.0f * U * rho - 3.0f * U * U * rho) / (9.0f * rho);
        mom[0] = rho;
        mom[5] = mxy;
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    }
    case NORTH | WEST: {
        const float mxy_I = LBM_MXY_I;
        const float rho = -36.0f * (-rho_I - mxy_I * rho_I + mxy_I * rho_I * omega) /
                          (24.0f + 18.0f * U - 18.0f * U * U + omega - 3.0f * U * omega + 3.0f * U * U * omega);
        const float mxy = (36.0f * mxy_I * rho_I + rho - 3.0f * U * rho + 3.0f * U * U * rho) / (9.0f * rho);
        mom[0] = rho;
        mom[5] = mxy;
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    }
    default:
        // not a boundary class (unreachable: every one of the 26 is listed)
        mom[0] = rho_I;
        mom[5] = 0.0f;
        mom[6] = 0.0f;
        mom[8] = 0.0f;
        return;
    }
#undef LBM_MXY_I
#undef LBM_MXZ_I
#undef LBM_MYZ_I
}

// velocitySet::scale followed by secondOrder::collide.  With SC = SCI != 1 (a
// power of two) the output comes out multiplied by SC: the scale factors take
// SC and the quadratic terms' coefficients 1/SC, each product being the
// unscaled one times SC exactly.
template <int SCI = 1>
__device__ __forceinline__ void scale_collide(float *m, const Relax &rx)
{
    constexpr float SC = float(SCI);
    m[1] = (3.0f * SC) * (m[1]);
    m[2] = (3.0f * SC) * (m[2]);
    m[3] = (3.0f * SC) * (m[3]);
    m[4] = (4.5f * SC) * (m[4]);
    m[5] = (9.0f * SC) * (m[5]);
    m[6] = (9.0f * SC) * (m[6]);
    m[7] = (4.5f * SC) * (m[7]);
    m[8] = (9.0f * SC) * (m[8]);
    m[9] = (4.5f * SC) * (m[9]);

    const float od2 = SC == 1.0f ? rx.omega_d2 : rx.omega_d2 * (1.0f / SC);
    const float om = SC == 1.0f ? rx.omega : rx.omega * (1.0f / SC);
    m[4] = rx.t_omega * m[4] + od2 * (m[1]) * (m[1]);
    m[7] = rx.t_omega * m[7] + od2 * (m[2]) * (m[2]);
    m[9] = rx.t_omega * m[9] + od2 * (m[3]) * (m[3]);

    m[5] = rx.t_omega * m[5] + om * (m[1]) * (m[2]);
    m[6] = rx.t_omega * m[6] + om * (m[1]) * (m[3]);
    m[8] = rx.t_omega * m[8] + om * (m[2]) * (m[3]);
}

// Full node update from the streamed populations f[Q] (in direction order).
// Returns the stored (post-collision) moments with rho still including rho0.
// f is clobbered (unknown directions of boundary nodes are zeroed).
template <int Q, int SCI = 1>
__device__ __forceinline__ void node_update(float *f, unsigned type, const Relax &rx, float *m)
{
    if (type)
        zero_unknown<Q>(f, unknown_dirs(type));
    float s[10];
    moment_folds<Q>(f, s);
    if (type)
        boundary_moments<Q>(s, type, rx, m);
    else
        interior_moments(s, m);
    scale_collide<SCI>(m, rx);
}

// ------------------------------------------------------- function objects
// x / d rounded to nearest, for d > 0 and r = RN(1/d): q = RN(x r), the
// remainder e = x - d q is exact by FMA, and RN(q + e r) is the correctly
// rounded quotient (P. Markstein, "Computation of elementary functions on the
// IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990) as long as
// nothing underflows or overflows: numerators must lie in [2^-64, 2^64) in
// magnitude or be +0; div_unsafe(x) >= 128 flags the others, which
// div_exact() handles.  Both are checked against IEEE division for every
// float numerator by tests/cuda/div_exhaustive.cu.
__device__ __forceinline__ float div_by_recip(float x, float d, float r)
{
    const float q = x * r;
    const float e = fmaf(-d, q, x);
    return fmaf(e, r, q);
}
__device__ __forceinline__ unsigned div_unsafe(float x)
{
    // >= 128 when outside the window; +0 (bit pattern 0) counts as inside:
    // div_by_recip returns +0 for it, the correctly rounded +0 / d
    const unsigned b = __float_as_uint(x);
    return b ? ((b >> 23) & 0xffu) - 63u : 0u;
}

// x / d rounded to nearest-even for any float x and d in [1, 2^40) with
// r = RN(1/d), using only multiplies and FMAs (no divide instruction):
//  * zeros, infinities and NaN: x * r has the right value and sign;
//  * |x| in [2^-64, 2^64): div_by_recip;
//  * |x| >= 2^64: scale by 2^-96 (exact), divide, scale back (exact, or the
//    same overflow to infinity as the IEEE quotient);
//  * |x| < 2^-64 with a normal quotient: scale by 2^96, divide, scale back;
//  * subnormal quotient: the result is n * 2^-149 with n = round-half-even of
//    X / d, X = |x| * 2^149 (an integer-valued float below 2^23 d): q = RN(X/d)
//    cannot cross a half-integer (those are representable), so rint(q) is n
//    unless q is itself a half-integer, where the sign of the exact remainder
//    X - d q decides.
__device__ __forceinline__ float div_exact(float x, float d, float r)
{
    const unsigned ex = (__float_as_uint(x) >> 23) & 0xffu;
    if (ex - 63u < 128u)
        return div_by_recip(x, d, r);
    if (x == 0.0f || ex == 0xffu)
        return x * r;
    const float ax = fabsf(x);
    float y;
    if (ex >= 191u) {
        y = div_by_recip(ax * 0x1p-96f, d, r) * 0x1p96f;
    } else {
        const float ys = div_by_recip(ax * 0x1p96f, d, r);
        if (ys >= 0x1p-30f) {
            y = ys * 0x1p-96f;
        } else {
            const float X = ax * 0x1p100f * 0x1p49f;
            const float q = div_by_recip(X, d, r);
            const float fl = floorf(q);
            float n = rintf(q);
            if (q - fl == 0.5f) {
                const float e = fmaf(-d, q, X);
                n = e > 0.0f ? fl + 1.0f : (e < 0.0f ? fl : n);
            }
            y = n * 0x1p-100f * 0x1p-49f;
        }
    }
    return copysignf(y, x);
}

// Divisors of the strain-rate tensor (strainRateTensor.cuh:71-90):
// 2 * scale_ii * tau and 2 * scale_ij * tau, with their reciprocals.
struct StrainDiv {
    float d_ii, r_ii, d_ij, r_ij;
};

// S_ab = 3 (u_a u_b - m_ab) / (2 scale tau) for the six components
// (xx, xy, xz, yy, yz, zz) of the stored moments m (u = m[1..3]).
// The roundings are written out (intrinsics) as the reference's compiled
// kernel performs them -- 3 * fma(u_a, u_b, -m_ab) -- so that no contraction
// or sharing of u_a u_b with other formulas in this kernel can change them
// (tests/test_reference_rounding.py checks the form on the reference's
// golden outputs).
__device__ __forceinline__ void strain_rate(const float *m, const StrainDiv &sd, float *S)
{
    const float u = m[1], v = m[2], w = m[3];
    float x[6];
    x[0] = __fmul_rn(3.0f, __fmaf_rn(u, u, -m[4]));
    x[1] = __fmul_rn(3.0f, __fmaf_rn(u, v, -m[5]));
    x[2] = __fmul_rn(3.0f, __fmaf_rn(u, w, -m[6]));
    x[3] = __fmul_rn(3.0f, __fmaf_rn(v, v, -m[7]));
    x[4] = __fmul_rn(3.0f, __fmaf_rn(v, w, -m[8]));
    x[5] = __fmul_rn(3.0f, __fmaf_rn(w, w, -m[9]));
    const unsigned worst = max(max(max(div_unsafe(x[0]), div_unsafe(x[1])), max(div_unsafe(x[2]), div_unsafe(x[3]))),
                               max(div_unsafe(x[4]), div_unsafe(x[5])));
    if (worst < 128u) {
        S[0] = div_by_recip(x[0], sd.d_ii, sd.r_ii);
        S[1] = div_by_recip(x[1], sd.d_ij, sd.r_ij);
        S[2] = div_by_recip(x[2], sd.d_ij, sd.r_ij);
        S[3] = div_by_recip(x[3], sd.d_ii, sd.r_ii);
        S[4] = div_by_recip(x[4], sd.d_ij, sd.r_ij);
        S[5] = div_by_recip(x[5], sd.d_ii, sd.r_ii);
    } else {
        S[0] = div_exact(x[0], sd.d_ii, sd.r_ii);
        S[1] = div_exact(x[1], sd.d_ij, sd.r_ij);
        S[2] = div_exact(x[2], sd.d_ij, sd.r_ij);
        S[3] = div_exact(x[3], sd.d_ii, sd.r_ii);
        S[4] = div_exact(x[4], sd.d_ij, sd.r_ij);
        S[5] = div_exact(x[5], sd.d_ii, sd.r_ii);
    }
}
__device__ __forceinline__ float kinetic(float u, float v, float w)
{
    // sqrtf((u*u) + (v*v) + (w*w)) * 0.5 as the reference's kernel rounds it:
    // v*v alone, then u*u and w*w each fused into the sum (intrinsics, so the
    // form does not depend on this kernel's other uses of the products).  A
    // node at rest (+0, the sum of squares is never -0) skips the square
    // root: sqrtf(+0) * 0.5 = +0, and a zero argument takes sqrtf's slow path
    const float s = __fmaf_rn(w, w, __fmaf_rn(u, u, __fmul_rn(v, v)));
    return s == 0.0f ? 0.0f : __fmul_rn(sqrtf(s), 0.5f);
}
template <typename T>
__device__ __forceinline__ T time_average(T mean, T f, T inv)
{
    return mean + (f - mean) * inv;
}

}  // namespace lbm
