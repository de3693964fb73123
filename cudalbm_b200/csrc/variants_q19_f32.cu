// variants_q19_f32.cu -- step-kernel instantiations (see lbm_variants.cuh).
#include "lbm_step.cuh"
#include "lbm_variants.cuh"

namespace lbm {

bool pick_q19_f32(int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out)
{
    constexpr int Q = 19;
    LBM_VARIANT(19, 32, 8, 2, 1, 1, 3, float)
    LBM_VARIANT(19, 32, 8, 3, 1, 1, 3, float)
    LBM_VARIANT(19, 32, 8, 3, 2, 2, 2, float)
    LBM_VARIANT(19, 32, 8, 2, 2, 2, 2, float)
    LBM_VARIANT(19, 32, 8, 2, 4, 1, 4, float)
    LBM_VARIANT(19, 16, 8, 2, 1, 1, 3, float)
    LBM_VARIANT(19, 8, 8, 2, 1, 1, 3, float)
    return false;
}

}  // namespace lbm
