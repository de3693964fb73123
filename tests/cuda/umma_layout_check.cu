// Host-side checks of the tensor-core operand layout constants of
// cudalbm_b200/csrc/lbm_mlp.cuh (built with nvcc, run on the CPU).
#include <cstdint>
#include <vector>

#include "lbm_mlp.cuh"

namespace {

// 0 if umma_index(row, k, rows) is the K-major no-swizzle canonical layout
// (8 x 8 core matrices of 16-byte rows; 8-row groups SBO = 128 B apart;
// K-chunks of 8 LBO = rows / 8 * 128 B apart) and a bijection onto
// [0, rows * K); otherwise a code naming the first failure.
int check_operand(int rows, int K, uint32_t lbo)
{
    std::vector<int> seen(size_t(rows) * K, 0);
    for (int r = 0; r < rows; r++)
        for (int k = 0; k < K; k++) {
            const int i = lbm::umma_index(r, k, rows);
            if (i < 0 || i >= rows * K)
                return 1;
            if (seen[size_t(i)]++)
                return 2;
            const uint32_t bytes = uint32_t(i) * 2u;
            const uint32_t want = uint32_t(k / 8) * lbo + uint32_t(r / 8) * lbm::MlpSmem::SBO + uint32_t(r % 8) * 16u +
                                  uint32_t(k % 8) * 2u;
            if (bytes != want)
                return 3;
        }
    return 0;
}

}  // namespace

extern "C" int umma_layout_check(uint32_t *idesc_n32)
{
    using lbm::MlpSmem;
    *idesc_n32 = lbm::umma_idesc_f16_f32<128, lbm::kMlpHidden>();
    if (int e = check_operand(128, lbm::kMlpIn, MlpSmem::LBO_A))
        return 10 + e;  // layer-1 operand: features
    if (int e = check_operand(128, lbm::kMlpHidden, MlpSmem::LBO_A))
        return 20 + e;  // layer-2 operand: hidden activations
    if (int e = check_operand(lbm::kMlpHidden, lbm::kMlpIn, MlpSmem::LBO_W))
        return 30 + e;  // w1
    if (int e = check_operand(lbm::kMlpHidden, lbm::kMlpHidden, MlpSmem::LBO_W))
        return 40 + e;  // w2
    // shared-memory regions: 128-byte aligned, in order, sized as the operands
    const int regions[][2] = {{MlpSmem::W1, lbm::kMlpHidden * lbm::kMlpIn * 2},
                              {MlpSmem::W2, lbm::kMlpHidden * lbm::kMlpHidden * 2},
                              {MlpSmem::A1, 128 * lbm::kMlpIn * 2},
                              {MlpSmem::A2, 128 * lbm::kMlpHidden * 2}};
    int end = 0;
    for (const auto &g : regions) {
        if (g[0] % 128 || g[0] < end)
            return 60;
        end = g[0] + g[1];
    }
    if (MlpSmem::BAR < end || MlpSmem::BAR % 8 || MlpSmem::BYTES > MlpSmem::LAUNCH_BYTES)
        return 61;
    // the weight block copied into shared memory is the struct's leading bytes
    if (sizeof(lbm::MlpDevice::w1) + sizeof(lbm::MlpDevice::w2) != size_t(MlpSmem::A1 - MlpSmem::W1))
        return 62;
    return 0;
}
