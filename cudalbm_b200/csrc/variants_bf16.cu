// variants_bf16.cu -- step-kernel instantiations (see lbm_variants.cuh).
#include "lbm_step.cuh"
#include "lbm_variants.cuh"

namespace lbm {

bool pick_bf16(int Q, int tx, int ty, int stages, int npb, unsigned fo, int mean_bits, Launcher &out)
{
    LBM_VARIANT(19, 32, 8, 2, 1, 1, 3, __nv_bfloat16)
    LBM_VARIANT(19, 32, 8, 2, 4, 1, 4, __nv_bfloat16)
    LBM_VARIANT(19, 32, 8, 3, 1, 1, 3, __nv_bfloat16)
    LBM_VARIANT(19, 16, 8, 2, 1, 1, 3, __nv_bfloat16)
    LBM_VARIANT(27, 32, 8, 2, 1, 1, 3, __nv_bfloat16)
    LBM_VARIANT(27, 16, 8, 2, 1, 1, 3, __nv_bfloat16)
    return false;
}

}  // namespace lbm
