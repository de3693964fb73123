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

template <int Q>
__device__ __forceinline__ float weight_rho(float rho, int cls);

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

// Moments in registers: m[0] = rho (with the +1 offset applied), m[1..3] =
// 3u, m[4,7,9] = 4.5 m_aa, m[5,6,8] = 9 m_ab (the reference's scaled units).
struct Moments {
    float m[10];
};

// ------------------------------------------------------ reconstruction
// Bracketing per direction, as written in the reference:
//   rhow * (((((pics2 +- u) +- v) +- w) + m_xx) + m_yy ...  +- m_ab)
//   body diagonals: ... + m_zz) +- (m_xy +- m_xz +- m_yz)
struct RecPre {
    float pics2;
    float rhow[4];
};

template <int Q>
__device__ __forceinline__ RecPre rec_pre(const float *m)
{
    RecPre r;
    r.pics2 = 1.0f - Consts::cs2 * (m[4] + m[7] + m[9]);
    r.rhow[0] = m[0] * weight<Q>(0);
    r.rhow[1] = m[0] * weight<Q>(1);
    r.rhow[2] = m[0] * weight<Q>(2);
    r.rhow[3] = m[0] * weight<Q>(3);
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

// Masked variant for boundary nodes: directions that would stream in from
// outside the domain contribute 0 (reference: incomingSwitch * f_q).
__device__ __forceinline__ bool is_known(int q, unsigned type);

template <int Q, int A, int B, int q>
__device__ __forceinline__ float fold_masked(const float *f, const float *mask)
{
    if constexpr (q >= Q) {
        return 0.0f;
    } else {
        constexpr int c = cdir(A, q) * cdir(B, q);
        constexpr int nq = [] {
            int r = q + 1;
            while (r < Q && cdir(A, r) * cdir(B, r) == 0) r++;
            return r;
        }();
        if constexpr (c == 0) {
            return fold_masked<Q, A, B, nq>(f, mask);
        } else {
            const float e = (c > 0) ? mask[q] * f[q] : -mask[q] * f[q];
            if constexpr (nq >= Q)
                return e;
            else
                return e + fold_masked<Q, A, B, nq>(f, mask);
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

// 1.0f if f_q is known at a node of this class, 0.0f if it streams in from
// outside the domain.
template <int q>
__device__ __forceinline__ float known_switch(unsigned t)
{
    constexpr int cx = cx_of(q), cy = cy_of(q), cz = cz_of(q);
    const bool cond_x = ((t & EAST) && cx < 0) || ((t & WEST) && cx > 0);
    const bool cond_y = ((t & NORTH) && cy < 0) || ((t & SOUTH) && cy > 0);
    const bool cond_z = ((t & FRONT) && cz < 0) || ((t & BACK) && cz > 0);
    return static_cast<float>(!(cond_x | cond_y | cond_z));
}

template <int Q, int q = 0>
__device__ __forceinline__ void fill_mask(float *mask, unsigned t)
{
    if constexpr (q < Q) {
        mask[q] = known_switch<q>(t);
        fill_mask<Q, q + 1>(mask, t);
    }
}

struct Relax {
    float omega, t_omega, omega_d2, tau, u_lid;
};

// Interior moments (unscaled): velocitySet.cuh:398-417.
template <int Q>
__device__ __forceinline__ void interior_moments(const float *f, float *mom)
{
    mom[0] = fold_from<Q, -1, -1, 0>(f);
    const float inv_rho = 1.0f / mom[0];
    mom[1] = fold_from<Q, 0, -1, 0>(f) * inv_rho;
    mom[2] = fold_from<Q, 1, -1, 0>(f) * inv_rho;
    mom[3] = fold_from<Q, 2, -1, 0>(f) * inv_rho;
    mom[4] = (fold_from<Q, 0, 0, 0>(f) * inv_rho) - Consts::cs2;
    mom[5] = fold_from<Q, 0, 1, 0>(f) * inv_rho;
    mom[6] = fold_from<Q, 0, 2, 0>(f) * inv_rho;
    mom[7] = (fold_from<Q, 1, 1, 0>(f) * inv_rho) - Consts::cs2;
    mom[8] = fold_from<Q, 1, 2, 0>(f) * inv_rho;
    mom[9] = (fold_from<Q, 2, 2, 0>(f) * inv_rho) - Consts::cs2;
}

// Wet-node boundary moments (unscaled), boundaryConditions.cuh:99-533.
template <int Q>
__device__ __forceinline__ void boundary_moments(const float *f, unsigned t, const Relax &rx, float *mom)
{
    float mask[Q];
    fill_mask<Q>(mask, t);
    const float rho_I = fold_masked<Q, -1, -1, 0>(f, mask);
    const float inv_rho_I = 1.0f / rho_I;
    const float omega = rx.omega;
    const float U = rx.u_lid;

    {
        const float nB = static_cast<float>(__popc(t & 0x3Fu));
        // U<alpha>: only the North wall moves (U_North = {u_inf, 0, 0})
        mom[1] = ((t & NORTH) ? U : 0.0f) / nB;
        mom[2] = 0.0f / nB;
        mom[3] = 0.0f / nB;
        mom[4] = mom[1] * mom[1];
    }
    mom[7] = 0.0f;
    mom[9] = 0.0f;

#define LBM_MXY_I (fold_masked<Q, 0, 1, 0>(f, mask) * inv_rho_I)
#define LBM_MXZ_I (fold_masked<Q, 0, 2, 0>(f, mask) * inv_rho_I)
#define LBM_MYZ_I (fold_masked<Q, 1, 2, 0>(f, mask) * inv_rho_I)
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

// velocitySet::scale followed by secondOrder::collide.
__device__ __forceinline__ void scale_collide(float *m, const Relax &rx)
{
    m[1] = 3.0f * (m[1]);
    m[2] = 3.0f * (m[2]);
    m[3] = 3.0f * (m[3]);
    m[4] = 4.5f * (m[4]);
    m[5] = 9.0f * (m[5]);
    m[6] = 9.0f * (m[6]);
    m[7] = 4.5f * (m[7]);
    m[8] = 9.0f * (m[8]);
    m[9] = 4.5f * (m[9]);

    m[4] = rx.t_omega * m[4] + rx.omega_d2 * (m[1]) * (m[1]);
    m[7] = rx.t_omega * m[7] + rx.omega_d2 * (m[2]) * (m[2]);
    m[9] = rx.t_omega * m[9] + rx.omega_d2 * (m[3]) * (m[3]);

    m[5] = rx.t_omega * m[5] + rx.omega * (m[1]) * (m[2]);
    m[6] = rx.t_omega * m[6] + rx.omega * (m[1]) * (m[3]);
    m[8] = rx.t_omega * m[8] + rx.omega * (m[2]) * (m[3]);
}

// Full node update from the streamed populations f[Q] (in direction order).
// Returns the stored (post-collision) moments with rho still including rho0.
template <int Q>
__device__ __forceinline__ void node_update(const float *f, unsigned type, const Relax &rx, float *m)
{
    if (type)
        boundary_moments<Q>(f, type, rx, m);
    else
        interior_moments<Q>(f, m);
    scale_collide(m, rx);
}

// ------------------------------------------------------- function objects
__device__ __forceinline__ float strain_diag(float ua, float ub, float mab, float tau)
{
    return 3.0f * ((ua * ub) - mab) / (2.0f * 4.5f * tau);
}
__device__ __forceinline__ float strain_off(float ua, float ub, float mab, float tau)
{
    return 3.0f * ((ua * ub) - mab) / (2.0f * 9.0f * tau);
}
__device__ __forceinline__ float kinetic(float u, float v, float w)
{
    return sqrtf((u * u) + (v * v) + (w * w)) * 0.5f;
}
template <typename T>
__device__ __forceinline__ T time_average(T mean, T f, T inv)
{
    return mean + (f - mean) * inv;
}

}  // namespace lbm
