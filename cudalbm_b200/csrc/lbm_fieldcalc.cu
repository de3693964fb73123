// lbm_fieldcalc.cu -- fieldCalculate's containsNaN / spatialMean on the device.
//
// The reference's fieldCalculate reads each saved time's ten moment fields
// to the host and loops over them there (applications/fieldCalculate/
// fieldCalculate.cuh:74-170): a field "contains NaN" if any value is NaN
// (std::isnan; infinities do not count), and its spatial mean is the float
// sum of its values in global node order (x fastest, fileInput.cuh:777-820
// de-interleaves the block-tiled file into that order), added left to right
// from 0 and divided by float(nodes).  Here both run on the GPU:
//
//  * stats_kernel / stats_finish_kernel: NaN count and an FP64 sum per field,
//    a grid-wide reduction in a fixed order (repeatable bit for bit), the
//    accurate mean the solver's monitor also reports;
//  * ordered_sum_kernel: the reference's left-to-right float sum, which
//    rounds after every addition and so cannot be reassociated.  One warp per
//    field: all 32 lanes fetch the next chunk (1024 values, global order,
//    gathered from either layout) while lane 0 adds the current one from
//    shared memory, so the sum runs at the FADD latency with the loads hidden.
//    Its printed value is what the reference prints, digit for digit.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "lbm_b200.h"
#include "lbm_handle.hpp"

namespace {

constexpr int kStatsThreads = 256;
constexpr int kStatsBlocksPerField = 256;
constexpr int kOrderedChunk = 1024;  // values per warp round, 32 per lane

__device__ __forceinline__ size_t tiled_address(int x, int y, size_t z, int nbx, int nby)
{
    const size_t tx = x & 7, ty = y & 7, tz = z & 7, bx = x >> 3, by = y >> 3, bz = z >> 3;
    return tx + 8 * (ty + 8 * (tz + 8 * (bx + size_t(nbx) * (by + size_t(nby) * bz))));
}

// grid (kStatsBlocksPerField, fields): partial FP64 sums and NaN counts per block
__global__ void __launch_bounds__(kStatsThreads) stats_kernel(const float *fields, size_t N, double *part_sum,
                                                                unsigned long long *part_nan)
{
    const float *f = fields + size_t(blockIdx.y) * N;
    double s = 0.0;
    unsigned long long nan = 0;
    for (size_t i = blockIdx.x * size_t(kStatsThreads) + threadIdx.x; i < N; i += size_t(gridDim.x) * kStatsThreads) {
        const float v = f[i];
        if (isnan(v))
            nan++;
        else
            s += double(v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        nan += __shfl_down_sync(0xffffffffu, nan, o);
    }
    __shared__ double ws[kStatsThreads / 32];
    __shared__ unsigned long long wn[kStatsThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        ws[warp] = s;
        wn[warp] = nan;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        unsigned long long n = 0;
        for (int w = 0; w < kStatsThreads / 32; w++) {
            t += ws[w];
            n += wn[w];
        }
        part_sum[size_t(blockIdx.y) * gridDim.x + blockIdx.x] = t;
        part_nan[size_t(blockIdx.y) * gridDim.x + blockIdx.x] = n;
    }
}

// one thread per field: the blocks' partials in block order
__global__ void stats_finish_kernel(const double *part_sum, const unsigned long long *part_nan, int blocks,
                                    int fields, size_t N, double *mean, unsigned long long *nan)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= fields)
        return;
    double t = 0.0;
    unsigned long long n = 0;
    for (int b = 0; b < blocks; b++) {
        t += part_sum[size_t(k) * blocks + b];
        n += part_nan[size_t(k) * blocks + b];
    }
    mean[k] = t / double(N);
    nan[k] = n;
}

// one warp per field (blockIdx.x): the left-to-right float sum in global order
__global__ void __launch_bounds__(32) ordered_sum_kernel(const float *fields, size_t N, int nx, int ny, int tiled,
                                                         float *mean_ref)
{
    __shared__ float chunk[kOrderedChunk];
    const float *f = fields + size_t(blockIdx.x) * N;
    const int lane = threadIdx.x;
    const size_t chunks = (N + kOrderedChunk - 1) / kOrderedChunk;
    float r[kOrderedChunk / 32];
    // global index g = c * kOrderedChunk + 32 j + lane; in the tiled layout its
    // (x, y, z) is split once per chunk and advanced by 32 nodes per j
    auto fetch = [&](size_t c) {
        size_t g = c * kOrderedChunk + lane;
        const size_t row = g / size_t(nx);
        int x = int(g - row * size_t(nx)), y = int(row % size_t(ny));
        size_t z = row / size_t(ny);
#pragma unroll
        for (int j = 0; j < kOrderedChunk / 32; j++) {
            r[j] = g < N ? __ldg(f + (tiled ? tiled_address(x, y, z, nx >> 3, ny >> 3) : g)) : 0.0f;
            g += 32;
            x += 32;
            while (x >= nx) {
                x -= nx;
                if (++y == ny) {
                    y = 0;
                    ++z;
                }
            }
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int j = 0; j < kOrderedChunk / 32; j++)
            chunk[j * 32 + lane] = r[j];
    };
    fetch(0);
    stage();
    __syncwarp();
    float sum = 0.0f;
    for (size_t c = 0; c < chunks; c++) {
        if (c + 1 < chunks)
            fetch(c + 1);  // in flight while lane 0 adds chunk c
        if (lane == 0) {
            const int n = int(c + 1 < chunks ? kOrderedChunk : N - c * kOrderedChunk);
            for (int i = 0; i < n; i++)
                sum = __fadd_rn(sum, chunk[i]);
        }
        __syncwarp();
        if (c + 1 < chunks)
            stage();
        __syncwarp();
    }
    if (lane == 0)
        mean_ref[blockIdx.x] = __fdiv_rn(sum, float(N));
}

}  // namespace

extern "C" {

lbm_status lbm_field_statistics(int32_t device, const float *fields, int64_t nx, int64_t ny, int64_t nz,
                                int32_t nfields, lbm_order order, int32_t *nan_count, float *mean_ref,
                                double *mean)
{
    if (!fields || !nan_count || !mean_ref || !mean)
        return lbm::record_error(LBM_ERR_ARG, "lbm_field_statistics: null argument");
    if (nx <= 0 || ny <= 0 || nz <= 0 || nfields <= 0 || nfields > 65535)
        return lbm::record_error(LBM_ERR_ARG, "lbm_field_statistics: empty mesh or field count out of range");
    if (order != LBM_ORDER_GLOBAL && order != LBM_ORDER_TILED)
        return lbm::record_error(LBM_ERR_ARG, "lbm_field_statistics: unknown order");
    if (order == LBM_ORDER_TILED && (nx % 8 || ny % 8 || nz % 8))
        return lbm::record_error(LBM_ERR_ARG, "lbm_field_statistics: the tiled order needs multiples of 8");
    if (nx > (1 << 30) || ny > (1 << 30))
        return lbm::record_error(LBM_ERR_ARG, "lbm_field_statistics: mesh dimension too large");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return lbm::record_error(LBM_ERR_ARG, "lbm_field_statistics: device ordinal out of range");
    LBM_CUDA_RETURN(cudaSetDevice(device));
    const size_t N = size_t(nx) * size_t(ny) * size_t(nz);
    const size_t bytes = N * size_t(nfields) * sizeof(float);
    const int blocks = kStatsBlocksPerField;
    const size_t parts = size_t(blocks) * size_t(nfields);
    float *d_fields = nullptr, *d_ref = nullptr;
    double *d_part = nullptr, *d_mean = nullptr;
    unsigned long long *d_pnan = nullptr, *d_nan = nullptr;
    cudaStream_t st = nullptr;
    auto release = [&]() {
        if (st)
            cudaStreamSynchronize(st);
        cudaFree(d_fields);
        cudaFree(d_ref);
        cudaFree(d_part);
        cudaFree(d_mean);
        cudaFree(d_pnan);
        cudaFree(d_nan);
        if (st)
            cudaStreamDestroy(st);
    };
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMalloc(&d_fields, bytes);
    if (e == cudaSuccess)
        e = cudaMalloc(&d_ref, size_t(nfields) * sizeof(float));
    if (e == cudaSuccess)
        e = cudaMalloc(&d_part, parts * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMalloc(&d_mean, size_t(nfields) * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMalloc(&d_pnan, parts * sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMalloc(&d_nan, size_t(nfields) * sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_fields, fields, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        stats_kernel<<<dim3(blocks, unsigned(nfields)), kStatsThreads, 0, st>>>(d_fields, N, d_part, d_pnan);
        stats_finish_kernel<<<(nfields + 127) / 128, 128, 0, st>>>(d_part, d_pnan, blocks, nfields, N, d_mean, d_nan);
        ordered_sum_kernel<<<unsigned(nfields), 32, 0, st>>>(d_fields, N, int(nx), int(ny),
                                                             order == LBM_ORDER_TILED ? 1 : 0, d_ref);
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> nan(static_cast<size_t>(nfields));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nan.data(), d_nan, nan.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(mean, d_mean, size_t(nfields) * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(mean_ref, d_ref, size_t(nfields) * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    release();
    if (e != cudaSuccess)
        return lbm::record_error(e == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,
                                 std::string("lbm_field_statistics: ") + cudaGetErrorString(e));
    for (int32_t k = 0; k < nfields; k++)
        nan_count[k] = nan[size_t(k)] > 0x7fffffffull ? 0x7fffffff : int32_t(nan[size_t(k)]);
    return LBM_OK;
}

}  // extern "C"
