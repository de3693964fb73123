// Exhaustive check of lbm::div_exact (the step kernel's division by the
// uniform strain-rate divisor) against IEEE division on the GPU: every float
// bit pattern is used as the numerator (NaNs must give NaN).  Also counts,
// per exponent of the numerator, where the unguarded Markstein step alone
// would differ, and fails if any numerator the strain rate's guard
// (div_unsafe) lets through to div_by_recip alone is among them.
// Built and called by tests/test_gpu_division.py.
#include <cuda_runtime.h>

#include "lbm_core.cuh"

__global__ void div_check(float d, float r, unsigned long long *bad, unsigned *first, unsigned long long *hist)
{
    unsigned long long n = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < (1ull << 32);
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned bits = (unsigned)i;
        const float x = __uint_as_float(bits);
        const float b = __fdiv_rn(x, d);
        if (isnan(b)) {  // NaN in, NaN out: payloads may differ
            if (!isnan(lbm::div_exact(x, d, r)))
                n++;
            continue;
        }
        const float a = lbm::div_exact(x, d, r);
        if (__float_as_uint(a) != __float_as_uint(b)) {
            n++;
            atomicMin(first, bits);
        }
        const float u = lbm::div_by_recip(x, d, r);
        if (isfinite(x) && __float_as_uint(u) != __float_as_uint(b)) {
            atomicAdd(&hist[(bits >> 23) & 0xffu], 1ull);
            // the strain rate's dispatch: a numerator div_unsafe() passes
            // is divided by div_by_recip alone, so that must be exact too
            if (lbm::div_unsafe(x) < 128u) {
                n++;
                atomicMin(first, bits);
            }
        }
    }
    if (n)
        atomicAdd(bad, n);
}

extern "C" int div_exhaustive(float d, unsigned long long *bad_out, unsigned *first_out, unsigned long long *hist_out)
{
    unsigned long long *bad, *hist;
    unsigned *first;
    if (cudaMalloc(&bad, 8) != cudaSuccess || cudaMalloc(&first, 4) != cudaSuccess ||
        cudaMalloc(&hist, 256 * 8) != cudaSuccess)
        return 1;
    cudaMemset(bad, 0, 8);
    cudaMemset(hist, 0, 256 * 8);
    cudaMemset(first, 0xff, 4);
    const float r = 1.0f / d;  // host float division: RN(1/d)
    div_check<<<148 * 8, 256>>>(d, r, bad, first, hist);
    if (cudaDeviceSynchronize() != cudaSuccess)
        return 2;
    cudaMemcpy(bad_out, bad, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(first_out, first, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hist_out, hist, 256 * 8, cudaMemcpyDeviceToHost);
    cudaFree(bad);
    cudaFree(first);
    cudaFree(hist);
    return 0;
}
