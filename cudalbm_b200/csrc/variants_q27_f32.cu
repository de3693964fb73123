// variants_q27_f32.cu -- step-kernel instantiations (see lbm_variants.cuh).
#include "lbm_step.cuh"
#include "lbm_variants.cuh"

namespace lbm {

bool pick_q27_f32(int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out)
{
    constexpr int Q = 27;
    LBM_VARIANT(27, 32, 8, 2, 1, 1, 3, float)
    LBM_VARIANT(27, 32, 8, 2, 2, 2, 2, float)
    LBM_VARIANT(27, 16, 8, 2, 1, 1, 3, float)
    LBM_VARIANT(27, 8, 8, 2, 1, 1, 3, float)
    return false;
}

}  // namespace lbm
