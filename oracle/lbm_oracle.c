/*
 * lbm_oracle.c -- CPU restatement of cudaLBM's moment-representation LBM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * solver in cudalbm_b200/csrc: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it.  The product never calls it.
 *
 * It restates, in plain C with OpenMP over z-planes, what the reference's
 * fused kernel (applications/momentBasedD3Q19/momentBasedD3Q19.cuh:88-189 and
 * applications/momentBasedD3Q27/momentBasedD3Q27.cuh:88-186) computes per node
 * and per step, in global (x, y, z) indexing:
 *
 *   m(t+1, x) = Collide(Scale(BC_or_Moments(x, { f_q = R_q(m(t, x - c_q)) })))
 *
 * where R_q is the regularised reconstruction of population q from the 10
 * scaled moments.  The reference moves populations between nodes through
 * shared memory (src/streaming/streaming.cuh:89-154) and between 8^3 blocks
 * through global halo faces (src/blockHalo/halo.cuh:171-494); both deliver
 * exactly R_q(m(t, x - c_q)) to node x.  Populations that would come from
 * outside the domain only reach boundary nodes, where the reference multiplies
 * them by 0 (src/velocitySet/velocitySet.cuh:204-220), so they are 0 here.
 *
 * The arithmetic type is REAL (double by default; -DORACLE_REAL=float builds
 * the diagnostic single-precision variant).  Expressions keep the reference's
 * association order (left-to-right sums in the reconstruction, right folds in
 * the moment sums) so that the float variant rounds like the reference except
 * where nvcc contracts a multiply-add into an FMA.
 *
 * Parity pin: tests/test_oracle_golden.py checks this oracle against .LBMBin
 * outputs of the reference executables themselves (the .npz files in
 * tests/golden, made by
 * tests/golden/make_golden.py on a B200).
 *
 * Field layout: m[f * N + (z * ny + y) * nx + x], f = 0..9 in the order
 * rho, u, v, w, m_xx, m_xy, m_xz, m_yy, m_yz, m_zz (reference
 * src/globalFunctions.cuh:482-494); rho is stored as rho - 1 and the other
 * moments in the reference's scaled units (velocitySet.cuh:130-142).
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
typedef ORACLE_REAL real;

#ifdef ORACLE_FLOAT_SUFFIX
#define API(name) name##_f32
#else
#define API(name) name
#endif

/* D3Q27 velocity ordering; the first 19 entries are D3Q19
 * (src/velocitySet/D3Q19.cuh:172-304, src/velocitySet/D3Q27.cuh:166-241). */
static const int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
static const int CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
static const int CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

typedef struct oracle_params {
    int q;            /* 19 or 27 */
    int64_t nx, ny, nz;
    /* relaxation constants, as the reference uploads them
     * (src/latticeMesh/latticeMesh.cuh:177-201) */
    double omega, t_omega, omega_d2, tau;
    double u_lid;     /* U_North[0] = u_inf */
} oracle_params;

enum { W_ = 0x01, E_ = 0x02, S_ = 0x04, N_ = 0x08, B_ = 0x10, F_ = 0x20 };

/* node class bitmask, src/boundaryConditions/normalVector.cuh:321-334 */
int API(oracle_node_type)(int64_t x, int64_t y, int64_t z, int64_t nx, int64_t ny, int64_t nz)
{
    return (x == 0) * W_ | (x == nx - 1) * E_ | (y == 0) * S_ | (y == ny - 1) * N_ | (z == 0) * B_ | (z == nz - 1) * F_;
}

static real weight(int q, int Q)
{
    /* D3Q19.cuh:98-150, D3Q27.cuh:98-144 */
    if (Q == 19)
        return q == 0 ? (real)(1.0 / 3.0) : (q <= 6 ? (real)(1.0 / 18.0) : (real)(1.0 / 36.0));
    return q == 0 ? (real)(8.0 / 27.0) : (q <= 6 ? (real)(2.0 / 27.0) : (q <= 18 ? (real)(1.0 / 54.0) : (real)(1.0 / 216.0)));
}

/* Population q reconstructed from scaled moments m (rho = m[0] including the
 * +1 offset), D3Q19.cuh:311-374 and D3Q27.cuh:248-331.  Terms are added in
 * the reference's order: first-order (u, v, w), diagonal (xx, yy, zz), then
 * the off-diagonal term(s). */
static real reconstruct_q(int q, int Q, const real *m)
{
    const real cs2 = (real)(1.0 / 3.0);
    const real pics2 = (real)1.0 - cs2 * ((m[4] + m[7]) + m[9]);
    const real rhow = m[0] * weight(q, Q);
    const int cx = CX[q], cy = CY[q], cz = CZ[q];
    if (q == 0)
        return rhow * pics2;
    real s = pics2;
    if (cx) s = cx > 0 ? s + m[1] : s - m[1];
    if (cy) s = cy > 0 ? s + m[2] : s - m[2];
    if (cz) s = cz > 0 ? s + m[3] : s - m[3];
    if (cx) s = s + m[4];
    if (cy) s = s + m[7];
    if (cz) s = s + m[9];
    const int nnz = (cx != 0) + (cy != 0) + (cz != 0);
    if (nnz == 2) {
        if (cx && cy) s = (cx * cy > 0) ? s + m[5] : s - m[5];
        if (cx && cz) s = (cx * cz > 0) ? s + m[6] : s - m[6];
        if (cy && cz) s = (cy * cz > 0) ? s + m[8] : s - m[8];
    } else if (nnz == 3) {
        const int sxy = cx * cy, s6 = sxy * cx * cz, s8 = sxy * cy * cz;
        real g = m[5];
        g = s6 > 0 ? g + m[6] : g - m[6];
        g = s8 > 0 ? g + m[8] : g - m[8];
        s = sxy > 0 ? s + g : s - g;
    }
    return rhow * s;
}

void API(oracle_reconstruct)(int Q, const real *m, real *f)
{
    for (int q = 0; q < Q; q++)
        f[q] = reconstruct_q(q, Q, m);
}

/* incomingSwitch (velocitySet.cuh:204-220): 1 if population q is known at a
 * node of class `type`, 0 if it would stream in from outside the domain. */
static int known(int q, int type)
{
    const int cx = CX[q], cy = CY[q], cz = CZ[q];
    const int in_x = ((type & E_) && cx < 0) || ((type & W_) && cx > 0);
    const int in_y = ((type & N_) && cy < 0) || ((type & S_) && cy > 0);
    const int in_z = ((type & F_) && cz < 0) || ((type & B_) && cz > 0);
    return !(in_x || in_y || in_z);
}

/* sum_q mask_q * ca_q * cb_q * f_q over the q with nonzero ca*cb, as the
 * reference's fold expression evaluates it: a right fold in ascending q
 * (velocitySet.cuh:370-396).  a, b in {-1: none, 0: x, 1: y, 2: z}. */
static real moment_sum(const real *f, int Q, int a, int b, int type)
{
    const int *C[3] = {CX, CY, CZ};
    int idx[27], coef[27], n = 0;
    for (int q = 0; q < Q; q++) {
        const int ca = a < 0 ? 1 : C[a][q];
        const int cb = b < 0 ? 1 : C[b][q];
        if (ca * cb != 0) {
            idx[n] = q;
            coef[n] = ca * cb;
            n++;
        }
    }
    real s = 0;
    int first = 1;
    for (int k = n - 1; k >= 0; k--) {
        const int q = idx[k];
        real term = coef[k] > 0 ? f[q] : -f[q];
        if (type >= 0 && !known(q, type))
            term = (real)0 * term;
        if (first) {
            s = term;
            first = 0;
        } else {
            s = term + s;
        }
    }
    return s;
}

/* Interior moments, velocitySet.cuh:398-417 (unscaled: m_aa minus cs2). */
static void interior_moments(const real *f, int Q, real *mom)
{
    const real cs2 = (real)(1.0 / 3.0);
    mom[0] = moment_sum(f, Q, -1, -1, -1);
    const real inv_rho = (real)1 / mom[0];
    mom[1] = moment_sum(f, Q, 0, -1, -1) * inv_rho;
    mom[2] = moment_sum(f, Q, 1, -1, -1) * inv_rho;
    mom[3] = moment_sum(f, Q, 2, -1, -1) * inv_rho;
    mom[4] = (moment_sum(f, Q, 0, 0, -1) * inv_rho) - cs2;
    mom[5] = moment_sum(f, Q, 0, 1, -1) * inv_rho;
    mom[6] = moment_sum(f, Q, 0, 2, -1) * inv_rho;
    mom[7] = (moment_sum(f, Q, 1, 1, -1) * inv_rho) - cs2;
    mom[8] = moment_sum(f, Q, 1, 2, -1) * inv_rho;
    mom[9] = (moment_sum(f, Q, 2, 2, -1) * inv_rho) - cs2;
}

/* Wet-node regularised boundary moments for the closed cavity with a moving
 * North lid, src/boundaryConditions/boundaryConditions.cuh:99-554.  Writes the
 * unscaled moments (rho, u, v, w, m_xx, m_xy, m_xz, m_yy, m_yz, m_zz). */
static void boundary_moments(const real *f, int Q, int type, real omega, real U, real *mom)
{
    const real rho_I = moment_sum(f, Q, -1, -1, type);
    const real inv_rho_I = (real)1 / rho_I;
    const int nb = !!(type & W_) + !!(type & E_) + !!(type & S_) + !!(type & N_) + !!(type & B_) + !!(type & F_);
    /* U<alpha> (boundaryConditions.cuh:543-554): only U_North is nonzero */
    mom[1] = ((type & N_) ? U : (real)0) / (real)nb;
    mom[2] = (real)0;
    mom[3] = (real)0;
    mom[4] = mom[1] * mom[1];
    mom[7] = (real)0;
    mom[9] = (real)0;
    real rho = 0, mxy = 0, mxz = 0, myz = 0;
#define MXY_I (moment_sum(f, Q, 0, 1, type) * inv_rho_I)
#define MXZ_I (moment_sum(f, Q, 0, 2, type) * inv_rho_I)
#define MYZ_I (moment_sum(f, Q, 1, 2, type) * inv_rho_I)
    switch (type) {
    case S_ | W_ | B_:
    case S_ | W_ | F_:
    case S_ | E_ | B_:
    case S_ | E_ | F_:
        rho = Q == 19 ? (real)12 * rho_I / (real)7 : (real)216 * rho_I / (real)125;
        break;
    case S_ | W_: {
        const real a = MXY_I;
        rho = (real)36 * (rho_I - a * rho_I + a * rho_I * omega) / ((real)24 + omega);
        mxy = ((real)36 * a * rho_I - rho) / ((real)9 * rho);
    } break;
    case S_ | E_: {
        const real a = MXY_I;
        rho = -(real)36 * (-rho_I - a * rho_I + a * rho_I * omega) / ((real)24 + omega);
        mxy = ((real)36 * a * rho_I + rho) / ((real)9 * rho);
    } break;
    case W_ | B_:
    case E_ | F_: {
        const real a = MXZ_I;
        rho = (real)36 * (rho_I - a * rho_I + a * rho_I * omega) / ((real)24 + omega);
        mxz = ((real)36 * a * rho_I - rho) / ((real)9 * rho);
    } break;
    case W_ | F_:
    case E_ | B_: {
        const real a = MXZ_I;
        rho = -(real)36 * (-rho_I - a * rho_I + a * rho_I * omega) / ((real)24 + omega);
        mxz = ((real)36 * a * rho_I + rho) / ((real)9 * rho);
    } break;
    case S_ | B_: {
        const real a = MYZ_I;
        rho = (real)36 * (rho_I - a * rho_I + a * rho_I * omega) / ((real)24 + omega);
        myz = ((real)36 * a * rho_I - rho) / ((real)9 * rho);
    } break;
    case S_ | F_: {
        const real a = MYZ_I;
        rho = -(real)36 * (-rho_I - a * rho_I + a * rho_I * omega) / ((real)24 + omega);
        myz = ((real)36 * a * rho_I + rho) / ((real)9 * rho);
    } break;
    case W_:
    case E_: {
        const real a = MXY_I, b = MXZ_I;
        rho = (real)6 * rho_I / (real)5;
        mxy = (real)2 * a * rho_I / rho;
        mxz = (real)2 * b * rho_I / rho;
    } break;
    case S_: {
        const real a = MXY_I, b = MYZ_I;
        rho = (real)6 * rho_I / (real)5;
        mxy = (real)2 * a * rho_I / rho;
        myz = (real)2 * b * rho_I / rho;
    } break;
    case B_:
    case F_: {
        const real a = MXZ_I, b = MYZ_I;
        rho = (real)6 * rho_I / (real)5;
        mxz = (real)2 * a * rho_I / rho;
        myz = (real)2 * b * rho_I / rho;
    } break;
    case N_: {
        const real a = MXY_I, b = MYZ_I;
        rho = (real)6 * rho_I / (real)5;
        mxy = ((real)6 * a * rho_I - U * rho) / ((real)3 * rho);
        myz = (real)2 * b * rho_I / rho;
    } break;
    case N_ | W_ | B_:
    case N_ | W_ | F_:
        rho = -(real)24 * rho_I / (-(real)14 - (real)8 * U + (real)9 * U * U);
        break;
    case N_ | E_ | B_:
    case N_ | E_ | F_:
        rho = -(real)24 * rho_I / (-(real)14 + (real)8 * U + (real)9 * U * U);
        break;
    case N_ | B_: {
        const real a = MYZ_I;
        rho = (real)72 * (-rho_I - a * rho_I + a * rho_I * omega) /
              (-(real)48 - (real)2 * omega + (real)3 * U * U * omega);
        myz = ((real)72 * a * rho_I + (real)2 * rho - (real)3 * U * U * rho) / ((real)18 * rho);
    } break;
    case N_ | F_: {
        const real a = MYZ_I;
        rho = -(real)72 * (rho_I - a * rho_I + a * rho_I * omega) /
              (-(real)48 - (real)2 * omega + (real)3 * U * U * omega);
        myz = ((real)72 * a * rho_I - (real)2 * rho + (real)3 * U * U * rho) / ((real)18 * rho);
    } break;
    case N_ | E_: {
        const real a = MXY_I;
        rho = (real)36 * (rho_I - a * rho_I + a * rho_I * omega) /
              ((real)24 - (real)18 * U - (real)18 * U * U + omega + (real)3 * U * omega + (real)3 * U * U * omega);
        mxy = ((real)36 * a * rho_I - rho - (real)3 * U * rho - (real)3 * U * U * rho) / ((real)9 * rho);
    } break;
    case N_ | W_: {
        const real a = MXY_I;
        rho = -(real)36 * (-rho_I - a * rho_I + a * rho_I * omega) /
              ((real)24 + (real)18 * U - (real)18 * U * U + omega - (real)3 * U * omega + (real)3 * U * U * omega);
        mxy = ((real)36 * a * rho_I + rho - (real)3 * U * rho + (real)3 * U * U * rho) / ((real)9 * rho);
    } break;
    default:
        /* unreachable for a boundary node: every one of the 26 classes is listed */
        rho = rho_I;
        break;
    }
#undef MXY_I
#undef MXZ_I
#undef MYZ_I
    mom[0] = rho;
    mom[5] = mxy;
    mom[6] = mxz;
    mom[8] = myz;
}

/* velocitySet::scale (velocitySet.cuh:130-142) then secondOrder::collide
 * (src/collision/secondOrder.cuh:93-105). */
static void scale_and_collide(real *m, real omega, real t_omega, real omega_d2)
{
    m[1] = (real)3 * m[1];
    m[2] = (real)3 * m[2];
    m[3] = (real)3 * m[3];
    m[4] = (real)4.5 * m[4];
    m[5] = (real)9 * m[5];
    m[6] = (real)9 * m[6];
    m[7] = (real)4.5 * m[7];
    m[8] = (real)9 * m[8];
    m[9] = (real)4.5 * m[9];
    m[4] = t_omega * m[4] + omega_d2 * m[1] * m[1];
    m[7] = t_omega * m[7] + omega_d2 * m[2] * m[2];
    m[9] = t_omega * m[9] + omega_d2 * m[3] * m[3];
    m[5] = t_omega * m[5] + omega * m[1] * m[2];
    m[6] = t_omega * m[6] + omega * m[1] * m[3];
    m[8] = t_omega * m[8] + omega * m[2] * m[3];
}

/* One node update: gather the streamed populations, compute the moments
 * (boundary or interior), scale and collide.  `out` gets the stored values
 * (rho - 1, scaled moments). */
static void update_node(const oracle_params *p, const real *m_in, int64_t x, int64_t y, int64_t z, real *out)
{
    const int Q = p->q;
    const int64_t nx = p->nx, ny = p->ny, nz = p->nz, N = nx * ny * nz;
    real f[27];
    for (int q = 0; q < Q; q++) {
        const int64_t sx = x - CX[q], sy = y - CY[q], sz = z - CZ[q];
        if (sx < 0 || sx >= nx || sy < 0 || sy >= ny || sz < 0 || sz >= nz) {
            f[q] = 0;
            continue;
        }
        const int64_t s = (sz * ny + sy) * nx + sx;
        real m[10];
        for (int k = 0; k < 10; k++)
            m[k] = (real)m_in[k * N + s];
        m[0] = m[0] + (real)1;
        f[q] = reconstruct_q(q, Q, m);
    }
    const int type = API(oracle_node_type)(x, y, z, nx, ny, nz);
    real mom[10];
    if (type)
        boundary_moments(f, Q, type, (real)p->omega, (real)p->u_lid, mom);
    else
        interior_moments(f, Q, mom);
    scale_and_collide(mom, (real)p->omega, (real)p->t_omega, (real)p->omega_d2);
    mom[0] = mom[0] - (real)1;
    for (int k = 0; k < 10; k++)
        out[k] = mom[k];
}

/* One time step over the whole mesh: m_in -> m_out (distinct buffers). */
void API(oracle_step)(const oracle_params *p, const real *m_in, real *m_out)
{
    const int64_t nx = p->nx, ny = p->ny, nz = p->nz, N = nx * ny * nz;
#pragma omp parallel for schedule(static) collapse(2)
    for (int64_t z = 0; z < nz; z++)
        for (int64_t y = 0; y < ny; y++)
            for (int64_t x = 0; x < nx; x++) {
                real out[10];
                update_node(p, m_in, x, y, z, out);
                const int64_t i = (z * ny + y) * nx + x;
                for (int k = 0; k < 10; k++)
                    m_out[k * N + i] = out[k];
            }
}

/* Run-time function objects for the moments m after step t (absolute step
 * index t, as passed by the reference's time loop):
 *   S  (6 comp.)  src/functionObjects/strainRateTensor.cuh:71-90
 *   k             src/functionObjects/kineticEnergy.cuh:72-85
 *   means         functionObjects.cuh:79-97 with invNewCount = 1/(t+1)
 * Any output pointer may be NULL.  The means are updated in place.
 * The reference evaluates these in float with float tau and float
 * 1/(t+1) (strainRateTensor.cuh:332); they are evaluated in REAL here. */
void API(oracle_function_objects)(const oracle_params *p, const real *m, int64_t t, real *S, real *SMean, real *k,
                                  real *kMean, real *momentsMean)
{
    const int64_t N = p->nx * p->ny * p->nz;
    const real tau = (real)p->tau;
    const real inv = (real)1 / (real)(t + 1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        const real u = m[1 * N + i], v = m[2 * N + i], w = m[3 * N + i];
        const real mxx = m[4 * N + i], mxy = m[5 * N + i], mxz = m[6 * N + i];
        const real myy = m[7 * N + i], myz = m[8 * N + i], mzz = m[9 * N + i];
        real s[6];
        s[0] = (real)3 * ((u * u) - mxx) / ((real)2 * (real)4.5 * tau);
        s[1] = (real)3 * ((u * v) - mxy) / ((real)2 * (real)9 * tau);
        s[2] = (real)3 * ((u * w) - mxz) / ((real)2 * (real)9 * tau);
        s[3] = (real)3 * ((v * v) - myy) / ((real)2 * (real)4.5 * tau);
        s[4] = (real)3 * ((v * w) - myz) / ((real)2 * (real)9 * tau);
        s[5] = (real)3 * ((w * w) - mzz) / ((real)2 * (real)4.5 * tau);
        const real ke = (real)sqrt((double)((u * u) + (v * v) + (w * w))) * (real)0.5;
        for (int c = 0; c < 6; c++) {
            if (S) S[c * N + i] = s[c];
            if (SMean) SMean[c * N + i] = SMean[c * N + i] + (s[c] - SMean[c * N + i]) * inv;
        }
        if (k) k[i] = ke;
        if (kMean) kMean[i] = kMean[i] + (ke - kMean[i]) * inv;
        if (momentsMean)
            for (int c = 0; c < 10; c++)
                momentsMean[c * N + i] = momentsMean[c * N + i] + (m[c * N + i] - momentsMean[c * N + i]) * inv;
    }
}

/* Initial moments from per-region values, src/array/hostArray.cuh:304-359.
 * region[f * 7 + r], r = internalField, North, South, East, West, Front, Back,
 * already scaled as src/boundaryConditions/boundaryValue.cuh:147-254 does.
 * The reference evaluates this in float (scalar_t) and so does this function;
 * note its Front value applies at z == 0 and Back at z == nz - 1. */
void API(oracle_initial_moments)(const oracle_params *p, const float *region, real *m)
{
    const int64_t nx = p->nx, ny = p->ny, nz = p->nz, N = nx * ny * nz;
    for (int f = 0; f < 10; f++) {
        const float *r = region + 7 * f;
        for (int64_t z = 0; z < nz; z++)
            for (int64_t y = 0; y < ny; y++)
                for (int64_t x = 0; x < nx; x++) {
                    const int w = x == 0, e = x == nx - 1, s = y == 0, n = y == ny - 1, fr = z == 0, b = z == nz - 1;
                    const int count = w + e + s + n + fr + b;
                    const float sum = ((float)w * r[4]) + ((float)e * r[3]) + ((float)s * r[2]) + ((float)n * r[1]) +
                                      ((float)fr * r[5]) + ((float)b * r[6]);
                    m[f * N + (z * ny + y) * nx + x] = (real)(count > 0 ? sum / (float)count : r[0]);
                }
    }
}

/* Convenience loop: run n steps from absolute step t0, ping-ponging between
 * a and b (result ends in a), updating function objects after every step the
 * way the reference's time loop does (momentBasedD3Q19.cu:104-137). */
void API(oracle_run)(const oracle_params *p, real *a, real *b, int64_t t0, int64_t n, real *S, real *SMean, real *k,
                     real *kMean, real *momentsMean)
{
    const int64_t N = p->nx * p->ny * p->nz;
    for (int64_t t = t0; t < t0 + n; t++) {
        API(oracle_step)(p, a, b);
        for (int64_t i = 0; i < 10 * N; i++)
            a[i] = b[i];
        if (S || SMean || k || kMean || momentsMean)
            API(oracle_function_objects)(p, a, t, S, SMean, k, kMean, momentsMean);
    }
}

int API(oracle_real_bytes)(void) { return (int)sizeof(real); }
