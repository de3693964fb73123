// lbm_variants.cuh -- the compiled step-kernel variants and how to launch them.
//
// Each translation unit variants_*.cu instantiates one group of variants of
// lbm::step_kernel (lattice x storage format) and exposes a pick_* function
// that returns the launcher for a requested tiling; splitting them keeps the
// build parallel.  lbm_capi.cu only sees the Launcher records.
#pragma once

#include <cstddef>

namespace lbm {

struct Launcher {
    void *fn = nullptr;      // plain step
    void *fn_mon = nullptr;  // step that also accumulates the per-step monitor sums
    size_t smem = 0;
    int tx = 0, ty = 0, stages = 0, pop_buffers = 2;
};

// Every compiled kernel variant: (lattice, tile x, tile y, TMA stages,
// population-plane code, storage).  Population-plane code 1 = one plane,
// 3 CTAs/SM; 2 = two planes, 2 CTAs/SM; 4 = one plane, 4 CTAs/SM.  Storage
// codes: 0 FP32, 1 FP16, 2 BF16.
struct Variant {
    int Q, tx, ty, stages, npb, storage;
};
constexpr Variant kVariants[] = {
    {19, 32, 8, 2, 1, 0}, {19, 32, 8, 3, 1, 0}, {19, 32, 8, 3, 2, 0}, {19, 32, 8, 2, 2, 0}, {19, 32, 8, 2, 4, 0},
    {19, 16, 8, 2, 1, 0}, {19, 8, 8, 2, 1, 0},  {27, 32, 8, 2, 1, 0}, {27, 32, 8, 2, 2, 0}, {27, 16, 8, 2, 1, 0},
    {27, 8, 8, 2, 1, 0},  {19, 32, 8, 2, 1, 1}, {19, 32, 8, 3, 1, 1}, {19, 16, 8, 2, 1, 1}, {27, 32, 8, 2, 1, 1},
    {27, 16, 8, 2, 1, 1}, {19, 32, 8, 2, 1, 2}, {19, 32, 8, 3, 1, 2}, {19, 16, 8, 2, 1, 2}, {27, 32, 8, 2, 1, 2},
    {27, 16, 8, 2, 1, 2}, {19, 32, 8, 2, 4, 1}, {19, 32, 8, 2, 4, 2}};

// fo: the handle's function-object bits (LBM_FO_*).
bool pick_q19_f32(int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out);
bool pick_q27_f32(int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out);
bool pick_f16(int Q, int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out);
bool pick_bf16(int Q, int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out);

#ifdef __CUDACC__
template <int Q, int TX, int TY, int NS, int FO, typename MeanT, bool MON, int NPB, int MINB, typename ST>
void *kernel_fn()
{
    return reinterpret_cast<void *>(&step_kernel<Q, TX, TY, NS, FO, MeanT, MON, NPB, MINB, ST>);
}

// The function-object kernel for a set of function objects: none; exactly
// S, SMean, k and kMean (code 2: no run-time checks); any other set (code 1).
constexpr unsigned kFoFour = 0x0Fu;  // LBM_FO_S | LBM_FO_SMEAN | LBM_FO_K | LBM_FO_KMEAN

template <int Q, int TX, int TY, int NS, int NPB, int MINB, typename ST, int FO>
void pick_means(Launcher &l, int mean_bits)
{
    if (mean_bits == 64) {
        l.fn = kernel_fn<Q, TX, TY, NS, FO, double, false, NPB, MINB, ST>();
        l.fn_mon = kernel_fn<Q, TX, TY, NS, FO, double, true, NPB, MINB, ST>();
    } else {
        l.fn = kernel_fn<Q, TX, TY, NS, FO, float, false, NPB, MINB, ST>();
        l.fn_mon = kernel_fn<Q, TX, TY, NS, FO, float, true, NPB, MINB, ST>();
    }
}

template <int Q, int TX, int TY, int NS, int NPB, int MINB, typename ST>
Launcher pick_fo(unsigned fo, int mean_bits)
{
    Launcher l;
    l.tx = TX;
    l.ty = TY;
    l.stages = NS;
    l.pop_buffers = NPB;
    l.smem = SmemLayout<Q, TX, TY, NS, NPB, ST>::bytes;
    if (!fo) {
        l.fn = kernel_fn<Q, TX, TY, NS, 0, float, false, NPB, MINB, ST>();
        l.fn_mon = kernel_fn<Q, TX, TY, NS, 0, float, true, NPB, MINB, ST>();
    } else if (fo == kFoFour) {
        pick_means<Q, TX, TY, NS, NPB, MINB, ST, 2>(l, mean_bits);
    } else {
        pick_means<Q, TX, TY, NS, NPB, MINB, ST, 1>(l, mean_bits);
    }
    return l;
}

#define LBM_VARIANT(QQ, TXX, TYY, NSS, NPBCODE, NPB, MINB, ST)                                  \
    if (Q == QQ && tx == TXX && ty == TYY && stages == NSS && npb == NPBCODE) {                 \
        out = pick_fo<QQ, TXX, TYY, NSS, NPB, MINB, ST>(fo, mean_bits);                          \
        out.pop_buffers = NPBCODE;                                                              \
        return true;                                                                            \
    }
#endif

}  // namespace lbm
