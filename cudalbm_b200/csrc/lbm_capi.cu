// lbm_capi.cu -- implementation of the C ABI in include/lbm_b200.h.
//
// Owns the device state of one cavity (two moment buffers, the function-object
// accumulators, the TMA descriptors and a stream), dispatches the fused step
// kernel of lbm_step.cuh and provides the device-side helpers around it:
// initial state from region values, host<->device transfers in either node
// order, and double-precision global reductions.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "casefile.hpp"
#include "lbm_b200.h"
#include "lbm_handle.hpp"
#include "lbm_mlp.cuh"
#include "lbm_step.cuh"
#include "lbmbin.hpp"
#include "postprocess.hpp"
#include "lbm_variants.cuh"

namespace {

thread_local std::string g_last_error;

lbm_status fail(lbm_status s, const std::string &msg)
{
    g_last_error = msg;
    return s;
}

#define LBM_CUDA(call)                                                                                        \
    do {                                                                                                      \
        cudaError_t e_ = (call);                                                                              \
        if (e_ != cudaSuccess)                                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,                      \
                        std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + std::to_string((int)e_) + ")"); \
    } while (0)

// ---------------------------------------------------------------- kernels
template <typename ST>
__global__ void init_regions_kernel(ST *m, int nx, int ny, int nz, const float *region)
{
    // src/array/hostArray.cuh:304-359, evaluated in float as the reference does
    // (its "front" is z == 0 and "back" z == nz-1 there).
    const size_t N = size_t(nx) * ny * nz;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / (size_t(nx) * ny));
        const bool w = x == 0, e = x == nx - 1, s = y == 0, n = y == ny - 1, fr = z == 0, b = z == nz - 1;
        const int count = w + e + s + n + fr + b;
#pragma unroll
        for (int f = 0; f < 10; f++) {
            const float *r = region + 7 * f;
            const float sum = (float(w) * r[4]) + (float(e) * r[3]) + (float(s) * r[2]) + (float(n) * r[1]) +
                              (float(fr) * r[5]) + (float(b) * r[6]);
            m[f * N + i] = lbm::Storage<ST>::store(count > 0 ? sum / float(count) : r[0], f);
        }
    }
}

__device__ __forceinline__ size_t tiled_index(int x, int y, int z, int nbx, int nby)
{
    const int tx = x & 7, ty = y & 7, tz = z & 7, bx = x >> 3, by = y >> 3, bz = z >> 3;
    return size_t(tx) + 8 * (size_t(ty) + 8 * (size_t(tz) + 8 * (size_t(bx) + size_t(nbx) * (size_t(by) + size_t(nby) * bz))));
}

// One moment field between host values (reference convention, order/type of
// the host buffer) and the device storage format of field k.
template <typename ST, typename H>
__global__ void moment_in_kernel(ST *dst, const H *src, int k, int nx, int ny, int nz, int tiled)
{
    const size_t N = size_t(nx) * ny * nz;
    const int nbx = nx / 8, nby = ny / 8;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / (size_t(nx) * ny));
        const size_t j = tiled ? tiled_index(x, y, z, nbx, nby) : i;
        dst[i] = lbm::Storage<ST>::store(float(src[j]), k);
    }
}
template <typename ST, typename H>
__global__ void moment_out_kernel(H *dst, const ST *src, int k, int nx, int ny, int nz, int tiled)
{
    const size_t N = size_t(nx) * ny * nz;
    const int nbx = nx / 8, nby = ny / 8;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / (size_t(nx) * ny));
        const size_t j = tiled ? tiled_index(x, y, z, nbx, nby) : i;
        dst[j] = H(lbm::Storage<ST>::load(src[i], k));
    }
}

// Planes of the 10 moment fields between a contiguous FP32 staging block
// ([field][cnt nodes]) and the device storage format at node offset `off` of
// every field (lbm_run_streamed with 16-bit storage); blockIdx.y = field.
template <typename ST>
__global__ void planes_in_kernel(ST *m, const float *stage, size_t N, size_t off, size_t cnt)
{
    const int k = blockIdx.y;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < cnt; i += size_t(gridDim.x) * blockDim.x)
        m[size_t(k) * N + off + i] = lbm::Storage<ST>::store(stage[size_t(k) * cnt + i], k);
}
template <typename ST>
__global__ void planes_out_kernel(float *stage, const ST *m, size_t N, size_t off, size_t cnt)
{
    const int k = blockIdx.y;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < cnt; i += size_t(gridDim.x) * blockDim.x)
        stage[size_t(k) * cnt + i] = lbm::Storage<ST>::load(m[size_t(k) * N + off + i], k);
}

// dst (device layout, global order) <- src (one field of nodes, given order/type)
template <typename S, typename D>
__global__ void gather_in_kernel(D *dst, const S *src, int nx, int ny, int nz, int tiled)
{
    const size_t N = size_t(nx) * ny * nz;
    const int nbx = nx / 8, nby = ny / 8;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / (size_t(nx) * ny));
        const size_t j = tiled ? tiled_index(x, y, z, nbx, nby) : i;
        dst[i] = D(src[j]);
    }
}
template <typename S, typename D>
__global__ void scatter_out_kernel(D *dst, const S *src, int nx, int ny, int nz, int tiled)
{
    const size_t N = size_t(nx) * ny * nz;
    const int nbx = nx / 8, nby = ny / 8;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / (size_t(nx) * ny));
        const size_t j = tiled ? tiled_index(x, y, z, nbx, nby) : i;
        dst[j] = D(src[i]);
    }
}

// Cut plane normal to `axis` between node planes i0 and i1 with weight w
// (linear interpolation, no contraction into FMA so that host and device
// round alike); out[v][a + na*b] with (a, b) = (y, z), (x, z) or (x, y).
template <typename T>
__device__ __forceinline__ float plane_value(const T *src, size_t N, int v, size_t node)
{
    if constexpr (std::is_same_v<T, float> || std::is_same_v<T, double>)
        return float(src[size_t(v) * N + node]);
    else
        return lbm::Storage<T>::load(src[size_t(v) * N + node], v);
}
template <typename T>
__global__ void cut_plane_kernel(float *out, const T *src, int nvars, int nx, int ny, int nz, int axis, int i0, int i1,
                                 float w)
{
    const size_t N = size_t(nx) * ny * nz;
    const int na = axis == 0 ? ny : nx, nb = axis == 2 ? ny : nz;
    const size_t per = size_t(na) * nb;
    for (size_t j = blockIdx.x * size_t(blockDim.x) + threadIdx.x; j < per * nvars; j += size_t(gridDim.x) * blockDim.x) {
        const int v = int(j / per);
        const int a = int(j % per % na), b = int(j % per / na);
        auto node = [&](int i) {
            const int x = axis == 0 ? i : a, y = axis == 0 ? a : (axis == 1 ? i : b), z = axis == 2 ? i : b;
            return size_t(x) + size_t(nx) * (size_t(y) + size_t(ny) * z);
        };
        const float f0 = plane_value(src, N, v, node(i0)), f1 = plane_value(src, N, v, node(i1));
        out[j] = __fadd_rn(__fmul_rn(1.0f - w, f0), __fmul_rn(w, f1));
    }
}

// Self-test of the failure path: every thread waits, with the step kernels'
// bounded wait, on an mbarrier that nothing arrives on; the wait gives up
// after timeout_ns and the fault is recorded as in the step kernels.  No
// copy or other asynchronous operation is in flight.
__global__ void wait_timeout_kernel(lbm::StepFault *fault, uint64_t timeout_ns)
{
    __shared__ __align__(8) uint64_t bar;
    lbm::mbar_init_if(threadIdx.x == 0, &bar);
    lbm::fence_mbar_init_if(threadIdx.x == 0);
    __syncthreads();
    if (!lbm::mbar_wait_bounded(&bar, 0u, timeout_ns))
        lbm::record_fault(fault, lbm::ERR_TMA_TIMEOUT, -1, -1, 0, 0u, 0u, 0u, &bar);
}

template <typename ST>
__global__ void reduce_kernel(const ST *m, size_t N, double *acc, unsigned long long *bad)
{
    using S = lbm::Storage<ST>;
    double mass = 0.0, ke = 0.0;
    unsigned long long nb = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x) {
        const double rho = double(S::load(m[i], 0)) + 1.0;
        const double u = double(S::load(m[N + i], 1)) / 3.0, v = double(S::load(m[2 * N + i], 2)) / 3.0,
                     w = double(S::load(m[3 * N + i], 3)) / 3.0;
        mass += rho;
        ke += 0.5 * rho * (u * u + v * v + w * w);
#pragma unroll
        for (int f = 0; f < 10; f++)
            nb += !isfinite(S::load(m[f * N + i], f));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mass += __shfl_down_sync(0xffffffffu, mass, o);
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        nb += __shfl_down_sync(0xffffffffu, nb, o);
    }
    __shared__ double s_m[32], s_k[32];
    __shared__ unsigned long long s_b[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s_m[wid] = mass;
        s_k[wid] = ke;
        s_b[wid] = nb;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        mass = lane < nw ? s_m[lane] : 0.0;
        ke = lane < nw ? s_k[lane] : 0.0;
        nb = lane < nw ? s_b[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            mass += __shfl_down_sync(0xffffffffu, mass, o);
            ke += __shfl_down_sync(0xffffffffu, ke, o);
            nb += __shfl_down_sync(0xffffffffu, nb, o);
        }
        if (lane == 0) {
            atomicAdd(&acc[0], mass);
            atomicAdd(&acc[1], ke);
            atomicAdd(bad, nb);
        }
    }
}

// --------------------------------------------------------- kernel table
using lbm::StepParams;

using lbm::Launcher;
using lbm::Variant;
using lbm::kVariants;

bool pick_launcher(int Q, int tx, int ty, int stages, int npb, int storage, unsigned fo, int mean_bits, Launcher &out)
{
    if (storage == 1)
        return lbm::pick_f16(Q, tx, ty, stages, npb, fo, mean_bits, out);
    if (storage == 2)
        return lbm::pick_bf16(Q, tx, ty, stages, npb, fo, mean_bits, out);
    return Q == 19 ? lbm::pick_q19_f32(tx, ty, stages, npb, fo, mean_bits, out)
                   : lbm::pick_q27_f32(tx, ty, stages, npb, fo, mean_bits, out);
}

// Default tiling for a mesh: widest tile whose width divides nx, z-chunks
// sized so that the grid holds several waves of CTAs on 148 SMs.
void default_tiling(int Q, int64_t nx, int64_t ny, int64_t nz, int &tx, int &ty, int &zc, int &stages)
{
    (void)Q;
    tx = (nx % 32 == 0) ? 32 : (nx % 16 == 0 ? 16 : 8);
    ty = 8;
    stages = 2;
    const int64_t tiles = ((nx + tx - 1) / tx) * ((ny + ty - 1) / ty);
    int64_t c = nz;
    while (c > 16 && tiles * ((nz + c - 1) / c) < 8 * 148)
        c = (c + 1) / 2;
    zc = int(c);
}

using lbm::EncodeTiledFn;

EncodeTiledFn get_encode()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

}  // namespace

namespace {

template <typename T>
lbm_status dev_alloc(lbm_handle *h, T **p, size_t count)
{
    LBM_CUDA(cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T)));
    h->device_bytes += count * sizeof(T);
    return LBM_OK;
}

lbm_status make_tmap(lbm_handle *h, int which)
{
    EncodeTiledFn enc = get_encode();
    if (!enc)
        return fail(LBM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const auto &c = h->cfg;
    const int XPAD = h->storage ? lbm::Storage<__half>::XPAD : lbm::Storage<float>::XPAD;
    const cuuint64_t e = h->esz;
    cuuint64_t dims[4] = {cuuint64_t(c.nx), cuuint64_t(c.ny), cuuint64_t(c.nz), 10};
    cuuint64_t strides[3] = {cuuint64_t(c.nx) * e, cuuint64_t(c.nx) * c.ny * e, cuuint64_t(h->N) * e};
    cuuint32_t box[4] = {cuuint32_t(h->launcher.tx + 2 * XPAD), cuuint32_t(h->launcher.ty + 2), 1, 10};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = h->storage == 1   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                   : h->storage == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                     : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = enc(&h->tmap[which], dt, 4, h->m[which], dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(LBM_ERR_CUDA, "cuTensorMapEncodeTiled failed with CUresult " + std::to_string(int(r)));
    return LBM_OK;
}

int nvars_of(lbm_field_set s)
{
    switch (s) {
    case LBM_FIELDS_MOMENTS: return 10;
    case LBM_FIELDS_S: return 6;
    case LBM_FIELDS_SMEAN: return 6;
    case LBM_FIELDS_K: return 1;
    case LBM_FIELDS_KMEAN: return 1;
    case LBM_FIELDS_MOMENTSMEAN: return 10;
    }
    return -1;
}

// device pointer and element type (0 float, 1 double) of a field set
lbm_status field_ptr(lbm_handle *h, lbm_field_set s, void **p, int *is_double)
{
    const bool md = h->cfg.mean_bits == 64;
    *is_double = 0;
    switch (s) {
    case LBM_FIELDS_MOMENTS: *p = h->m[h->cur]; break;
    case LBM_FIELDS_S: *p = h->S; break;
    case LBM_FIELDS_SMEAN: *p = h->SMean; *is_double = md; break;
    case LBM_FIELDS_K: *p = h->k; break;
    case LBM_FIELDS_KMEAN: *p = h->kMean; *is_double = md; break;
    case LBM_FIELDS_MOMENTSMEAN: *p = h->momentsMean; *is_double = md; break;
    default: return fail(LBM_ERR_ARG, "unknown field set");
    }
    if (!*p)
        return fail(LBM_ERR_STATE, "field set not enabled for this handle (see function_objects)");
    return LBM_OK;
}

lbm_status ensure_scratch(lbm_handle *h, size_t bytes)
{
    if (h->scratch_bytes >= bytes)
        return LBM_OK;
    if (h->scratch) {
        cudaFree(h->scratch);
        h->device_bytes -= h->scratch_bytes;
        h->scratch = nullptr;
        h->scratch_bytes = 0;
    }
    LBM_CUDA(cudaMalloc(&h->scratch, bytes));
    h->scratch_bytes = bytes;
    h->device_bytes += bytes;
    return LBM_OK;
}

// How one field set moves between host values and the device buffer.
struct Xfer {
    size_t hsz;   // bytes per host value
    bool direct;  // one plain copy: same order, type and values on both sides
};
Xfer xfer_of(const lbm_handle *h, lbm_field_set set, lbm_dtype dtype, int is_double, lbm_order order)
{
    const size_t hsz = dtype == LBM_F64 ? 8 : 4;
    const bool moments = set == LBM_FIELDS_MOMENTS;
    const size_t dsz = moments ? h->esz : (is_double ? 8 : 4);
    return {hsz, order == LBM_ORDER_GLOBAL && hsz == dsz && (!moments || h->storage == 0)};
}

// The copy stream, its events and two scratch halves of `half` bytes.
lbm_status ensure_xfer(lbm_handle *h, size_t half)
{
    if (!h->xstream)
        LBM_CUDA(cudaStreamCreateWithFlags(&h->xstream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++) {
        if (!h->xe_copied[b])
            LBM_CUDA(cudaEventCreateWithFlags(&h->xe_copied[b], cudaEventDisableTiming));
        if (!h->xe_converted[b])
            LBM_CUDA(cudaEventCreateWithFlags(&h->xe_converted[b], cudaEventDisableTiming));
    }
    return ensure_scratch(h, 2 * half);
}

dim3 grid_1d(size_t N);

// Field v of a set: host values in `src` (order and type of the call) ->
// device field, on the handle stream.
lbm_status convert_in(lbm_handle *h, lbm_field_set set, lbm_dtype dtype, int is_double, void *dptr, int v,
                      const void *src, int tiled)
{
    const int nx = int(h->cfg.nx), ny = int(h->cfg.ny), nz = int(h->cfg.nz);
    const dim3 g = grid_1d(h->N);
    cudaStream_t st = h->stream;
    const bool f64 = dtype == LBM_F64;
    if (set == LBM_FIELDS_MOMENTS) {
        // moments go through the storage format (FP32 / FP16 / BF16)
        char *dst = static_cast<char *>(dptr) + size_t(v) * h->N * h->esz;
        if (h->storage == 1) {
            if (f64)
                moment_in_kernel<<<g, 256, 0, st>>>(reinterpret_cast<__half *>(dst), static_cast<const double *>(src), v, nx, ny, nz, tiled);
            else
                moment_in_kernel<<<g, 256, 0, st>>>(reinterpret_cast<__half *>(dst), static_cast<const float *>(src), v, nx, ny, nz, tiled);
        } else if (h->storage == 2) {
            if (f64)
                moment_in_kernel<<<g, 256, 0, st>>>(reinterpret_cast<__nv_bfloat16 *>(dst), static_cast<const double *>(src), v, nx, ny, nz, tiled);
            else
                moment_in_kernel<<<g, 256, 0, st>>>(reinterpret_cast<__nv_bfloat16 *>(dst), static_cast<const float *>(src), v, nx, ny, nz, tiled);
        } else {
            if (f64)
                moment_in_kernel<<<g, 256, 0, st>>>(reinterpret_cast<float *>(dst), static_cast<const double *>(src), v, nx, ny, nz, tiled);
            else
                moment_in_kernel<<<g, 256, 0, st>>>(reinterpret_cast<float *>(dst), static_cast<const float *>(src), v, nx, ny, nz, tiled);
        }
    } else if (f64) {
        if (is_double)
            gather_in_kernel<double, double><<<g, 256, 0, st>>>(static_cast<double *>(dptr) + v * h->N, static_cast<const double *>(src), nx, ny, nz, tiled);
        else
            gather_in_kernel<double, float><<<g, 256, 0, st>>>(static_cast<float *>(dptr) + v * h->N, static_cast<const double *>(src), nx, ny, nz, tiled);
    } else {
        if (is_double)
            gather_in_kernel<float, double><<<g, 256, 0, st>>>(static_cast<double *>(dptr) + v * h->N, static_cast<const float *>(src), nx, ny, nz, tiled);
        else
            gather_in_kernel<float, float><<<g, 256, 0, st>>>(static_cast<float *>(dptr) + v * h->N, static_cast<const float *>(src), nx, ny, nz, tiled);
    }
    LBM_CUDA(cudaGetLastError());
    h->launches += 1;
    return LBM_OK;
}

// Field v of a set: device field -> host values in `dst` (order and type of
// the call), on the handle stream.
lbm_status convert_out(lbm_handle *h, lbm_field_set set, lbm_dtype dtype, int is_double, const void *dptr, int v,
                       void *dst, int tiled)
{
    const int nx = int(h->cfg.nx), ny = int(h->cfg.ny), nz = int(h->cfg.nz);
    const dim3 g = grid_1d(h->N);
    cudaStream_t st = h->stream;
    const bool f64 = dtype == LBM_F64;
    const bool moments = set == LBM_FIELDS_MOMENTS;
    const size_t dsz = moments ? h->esz : (is_double ? 8 : 4);
    const char *src = static_cast<const char *>(dptr) + size_t(v) * h->N * dsz;
    if (moments) {
        if (h->storage == 1) {
            if (f64)
                moment_out_kernel<<<g, 256, 0, st>>>(static_cast<double *>(dst), reinterpret_cast<const __half *>(src), v, nx, ny, nz, tiled);
            else
                moment_out_kernel<<<g, 256, 0, st>>>(static_cast<float *>(dst), reinterpret_cast<const __half *>(src), v, nx, ny, nz, tiled);
        } else if (h->storage == 2) {
            if (f64)
                moment_out_kernel<<<g, 256, 0, st>>>(static_cast<double *>(dst), reinterpret_cast<const __nv_bfloat16 *>(src), v, nx, ny, nz, tiled);
            else
                moment_out_kernel<<<g, 256, 0, st>>>(static_cast<float *>(dst), reinterpret_cast<const __nv_bfloat16 *>(src), v, nx, ny, nz, tiled);
        } else {
            if (f64)
                moment_out_kernel<<<g, 256, 0, st>>>(static_cast<double *>(dst), reinterpret_cast<const float *>(src), v, nx, ny, nz, tiled);
            else
                moment_out_kernel<<<g, 256, 0, st>>>(static_cast<float *>(dst), reinterpret_cast<const float *>(src), v, nx, ny, nz, tiled);
        }
    } else if (f64) {
        if (is_double)
            scatter_out_kernel<double, double><<<g, 256, 0, st>>>(static_cast<double *>(dst), reinterpret_cast<const double *>(src), nx, ny, nz, tiled);
        else
            scatter_out_kernel<float, double><<<g, 256, 0, st>>>(static_cast<double *>(dst), reinterpret_cast<const float *>(src), nx, ny, nz, tiled);
    } else {
        if (is_double)
            scatter_out_kernel<double, float><<<g, 256, 0, st>>>(static_cast<float *>(dst), reinterpret_cast<const double *>(src), nx, ny, nz, tiled);
        else
            scatter_out_kernel<float, float><<<g, 256, 0, st>>>(static_cast<float *>(dst), reinterpret_cast<const float *>(src), nx, ny, nz, tiled);
    }
    LBM_CUDA(cudaGetLastError());
    h->launches += 1;
    return LBM_OK;
}

dim3 grid_1d(size_t N)
{
    return dim3(unsigned(std::min<size_t>((N + 255) / 256, size_t(148) * 16)));
}

// Parameter blocks carry FP64 running means only for the kernels that keep
// them: function objects on and mean_bits 64 (pick_fo); every other kernel
// takes the FP32-mean block.
bool means_f64(const lbm_handle *h)
{
    return h->cfg.function_objects != 0 && h->cfg.mean_bits == 64;
}

template <typename MeanT>
lbm_status launch_step(lbm_handle *h, bool monitored = false)
{
    if (h->closure) {
        if (monitored)
            return fail(LBM_ERR_STATE, "monitored steps are not available with the learned closure");
        return lbm::closure_step(h);
    }
    // the parameter block has the same layout for every storage type (the
    // output is a pointer); it is filled once here as the FP32 instance
    StepParams<MeanT> p{};
    const int nxt = h->cur ^ 1;
    p.out = static_cast<float *>(h->m[nxt]);
    p.mon = h->mon;
    p.nx = int(h->cfg.nx);
    p.ny = int(h->cfg.ny);
    p.nz = int(h->cfg.nz);
    p.zc = h->zc;
    p.z_lo = 0;
    p.z_hi = p.nz;
    p.rx = lbm::Relax{h->omega, h->t_omega, h->omega_d2, h->tau, h->cfg.u_inf};
    p.fo.S = h->S;
    p.fo.SMean = static_cast<MeanT *>(h->SMean);
    p.fo.k = h->k;
    p.fo.kMean = static_cast<MeanT *>(h->kMean);
    p.fo.momentsMean = static_cast<MeanT *>(h->momentsMean);
    // invNewCount = 1 / (timeStep + 1) in scalar_t (strainRateTensor.cuh:332)
    if constexpr (std::is_same_v<MeanT, float>)
        p.fo.inv_count = 1.0f / static_cast<float>(h->t + 1);
    else
        p.fo.inv_count = 1.0 / static_cast<double>(h->t + 1);
    // divisors 2*4.5*tau and 2*9*tau in float as the reference evaluates them;
    // the host's float division is IEEE, so the reciprocals are RN(1/d)
    p.fo.sd.d_ii = 2.0f * 4.5f * h->tau;
    p.fo.sd.d_ij = 2.0f * 9.0f * h->tau;
    p.fo.sd.r_ii = 1.0f / p.fo.sd.d_ii;
    p.fo.sd.r_ij = 1.0f / p.fo.sd.d_ij;
    p.fault = h->err;
    p.timeout_ns = 2000000000ull;
    const dim3 block(h->launcher.tx, h->launcher.ty);
    const dim3 grid(unsigned((h->cfg.nx + h->launcher.tx - 1) / h->launcher.tx),
                    unsigned((h->cfg.ny + h->launcher.ty - 1) / h->launcher.ty),
                    unsigned((h->cfg.nz + h->zc - 1) / h->zc));
    void *args[] = {&h->tmap[h->cur], &p};
    LBM_CUDA(cudaLaunchKernel(monitored ? h->launcher.fn_mon : h->launcher.fn, grid, block, args, h->launcher.smem,
                              h->stream));
    h->cur = nxt;
    h->t += 1;
    h->launches += 1;
    return LBM_OK;
}

// Step t of the planes [z_lo, z_hi) only, reading buffer `in` and writing the
// other one (lbm_run_streamed); mon: the step's monitor slot or null.  The
// handle's step counter and buffer index are left alone.
template <typename MeanT>
lbm_status launch_slab(lbm_handle *h, int in, int64_t t, int z_lo, int z_hi, int zc, lbm::MonitorSlot *mon)
{
    StepParams<MeanT> p{};
    p.out = static_cast<float *>(h->m[in ^ 1]);
    p.mon = mon;
    p.nx = int(h->cfg.nx);
    p.ny = int(h->cfg.ny);
    p.nz = int(h->cfg.nz);
    p.zc = zc;
    p.z_lo = z_lo;
    p.z_hi = z_hi;
    p.rx = lbm::Relax{h->omega, h->t_omega, h->omega_d2, h->tau, h->cfg.u_inf};
    p.fo.S = h->S;
    p.fo.SMean = static_cast<MeanT *>(h->SMean);
    p.fo.k = h->k;
    p.fo.kMean = static_cast<MeanT *>(h->kMean);
    p.fo.momentsMean = static_cast<MeanT *>(h->momentsMean);
    if constexpr (std::is_same_v<MeanT, float>)
        p.fo.inv_count = 1.0f / static_cast<float>(t + 1);
    else
        p.fo.inv_count = 1.0 / static_cast<double>(t + 1);
    p.fo.sd.d_ii = 2.0f * 4.5f * h->tau;
    p.fo.sd.d_ij = 2.0f * 9.0f * h->tau;
    p.fo.sd.r_ii = 1.0f / p.fo.sd.d_ii;
    p.fo.sd.r_ij = 1.0f / p.fo.sd.d_ij;
    p.fault = h->err;
    p.timeout_ns = 2000000000ull;
    const dim3 block(h->launcher.tx, h->launcher.ty);
    const dim3 grid(unsigned((h->cfg.nx + h->launcher.tx - 1) / h->launcher.tx),
                    unsigned((h->cfg.ny + h->launcher.ty - 1) / h->launcher.ty), unsigned((z_hi - z_lo + zc - 1) / zc));
    void *args[] = {&h->tmap[in], &p};
    LBM_CUDA(cudaLaunchKernel(mon ? h->launcher.fn_mon : h->launcher.fn, grid, block, args, h->launcher.smem,
                              h->stream));
    h->launches += 1;
    return LBM_OK;
}

}  // namespace

namespace lbm {
// Lets other translation units of the library report through lbm_last_error().
lbm_status record_error(lbm_status s, const std::string &msg)
{
    return fail(s, msg);
}

EncodeTiledFn encode_tiled() { return get_encode(); }

lbm_status check_fault(const StepFault &f, const char *who)
{
    if (f.flags & ERR_BOUNDS) {
        // only the checked build (LBM_CHECKED) sets this flag
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s failed index check %u (block %d,%d,%d item %d mesh %d plane %d)", who,
                      f.slot, f.block[0], f.block[1], f.block[2], f.item, f.mesh, f.plane);
        return fail(LBM_ERR_STATE, buf);
    }
    if (f.flags & ERR_MMA_TIMEOUT)
        return fail(LBM_ERR_TIMEOUT, "the closure network timed out waiting for a tensor-core MMA");
    if (!(f.flags & ERR_TMA_TIMEOUT))
        return LBM_OK;
    std::string msg = std::string(who) + " timed out waiting for a TMA copy";
    if (f.recorded == 1) {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      " (block %d,%d,%d item %d mesh %d plane %d seq %u slot %u parity %u mbarrier 0x%016llx)",
                      f.block[0], f.block[1], f.block[2], f.item, f.mesh, f.plane, f.seq, f.slot, f.parity, f.barrier);
        msg += buf;
    }
    return fail(LBM_ERR_TIMEOUT, msg);
}

void destroy_handle(lbm_handle *h)
{
    if (!h)
        return;
    cudaSetDevice(h->cfg.device);
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    for (void *p : {h->m[0], h->m[1], static_cast<void *>(h->S), static_cast<void *>(h->k), h->SMean, h->kMean,
                    h->momentsMean, static_cast<void *>(h->err), static_cast<void *>(h->red),
                    static_cast<void *>(h->mon), h->scratch, static_cast<void *>(h->dtau),
                    static_cast<void *>(h->mon_steps)})
        if (p)
            cudaFree(p);
    if (h->dstream) {
        cudaStreamSynchronize(h->dstream);
        cudaStreamDestroy(h->dstream);
    }
    delete h->mlp;
    if (h->steps_graph)
        cudaGraphExecDestroy(h->steps_graph);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->xstream) {
        cudaStreamSynchronize(h->xstream);
        cudaStreamDestroy(h->xstream);
    }
    for (int b = 0; b < 2; b++) {
        if (h->xe_copied[b]) cudaEventDestroy(h->xe_copied[b]);
        if (h->xe_converted[b]) cudaEventDestroy(h->xe_converted[b]);
    }
    if (h->stream && h->own_stream)
        cudaStreamDestroy(h->stream);
    delete h;
}
}  // namespace lbm

extern "C" {

void lbm_config_default(lbm_config *c)
{
    std::memset(c, 0, sizeof(*c));
    c->lattice = 19;
    c->device = 0;
    c->nx = c->ny = c->nz = 64;
    c->Re = 100.0f;
    c->u_inf = 0.05f;
    c->function_objects = 0;
    c->mean_bits = 32;
    c->start_step = 0;
}

const char *lbm_last_error(void) { return g_last_error.c_str(); }

const char *lbm_status_string(lbm_status s)
{
    switch (s) {
    case LBM_OK: return "ok";
    case LBM_ERR_ARG: return "invalid argument";
    case LBM_ERR_CUDA: return "CUDA error";
    case LBM_ERR_NOMEM: return "out of memory";
    case LBM_ERR_TIMEOUT: return "device wait timed out";
    case LBM_ERR_IO: return "I/O error";
    case LBM_ERR_PARSE: return "parse error";
    case LBM_ERR_STATE: return "invalid state";
    case LBM_ERR_NONFINITE: return "non-finite value in solution";
    }
    return "unknown status";
}

int lbm_field_set_vars(lbm_field_set set) { return nvars_of(set); }

lbm_status lbm_create(const lbm_config *cfg, lbm_handle **out)
{
    g_last_error.clear();
    if (!cfg || !out)
        return fail(LBM_ERR_ARG, "null argument");
    *out = nullptr;
    const lbm_config &c = *cfg;
    if (c.lattice != 19 && c.lattice != 27)
        return fail(LBM_ERR_ARG, "lattice must be 19 or 27");
    if (c.nx <= 0 || c.ny <= 0 || c.nz <= 0 || c.nx % 8 || c.ny % 8 || c.nz % 8)
        return fail(LBM_ERR_ARG, "mesh dimensions must be positive multiples of 8 (block::nx() * nxBlocks() == nx)");
    if (c.nx > (1 << 30) || c.ny > (1 << 30) || c.nz > (1 << 30))
        return fail(LBM_ERR_ARG, "mesh dimension too large");
    // the step kernels address a node within a field with 32 bits (the FP32
    // state of 2^32 nodes would take 343 GB, beyond one GPU)
    if (uint64_t(c.nx) * uint64_t(c.ny) * uint64_t(c.nz) >= (uint64_t(1) << 32))
        return fail(LBM_ERR_ARG, "mesh too large: at most 2^32 - 1 nodes");
    if (!(c.Re > 0.0f) || !std::isfinite(c.u_inf))
        return fail(LBM_ERR_ARG, "Re must be positive and u_inf finite");
    if (c.mean_bits != 32 && c.mean_bits != 64)
        return fail(LBM_ERR_ARG, "mean_bits must be 32 or 64");
    if (c.function_objects & ~0x1Fu)
        return fail(LBM_ERR_ARG, "unknown function object bits");
    if (c.storage < 0 || c.storage > 2)
        return fail(LBM_ERR_ARG, "storage must be LBM_STORAGE_F32, LBM_STORAGE_F16 or LBM_STORAGE_BF16");

    int ndev = 0;
    LBM_CUDA(cudaGetDeviceCount(&ndev));
    if (c.device < 0 || c.device >= ndev)
        return fail(LBM_ERR_ARG, "device ordinal out of range (Number of GPUs requested is greater than the number available)");
    LBM_CUDA(cudaSetDevice(c.device));

    lbm_handle *h = new lbm_handle();
    h->cfg = c;
    h->Q = c.lattice;
    h->N = size_t(c.nx) * c.ny * c.nz;
    h->t = c.start_step;
    h->storage = c.storage;
    h->esz = c.storage ? 2 : 4;

    // relaxation constants in float, as the reference (latticeMesh.cuh:177-201)
    const float nu = c.u_inf * static_cast<float>(c.nx - 1) / c.Re;
    h->tau = 0.5f + 3.0f * nu;
    h->omega = 1.0f / h->tau;
    h->t_omega = 1.0f - h->omega;
    h->omega_d2 = h->omega * 0.5f;

    int tx, ty, zc, st;
    default_tiling(h->Q, c.nx, c.ny, c.nz, tx, ty, zc, st);
    if (c.tile_x) tx = c.tile_x;
    if (c.tile_y) ty = c.tile_y;
    if (c.z_chunk) zc = c.z_chunk;
    if (c.stages) st = c.stages;
    const unsigned fo = c.function_objects;
    const int npb = c.pop_buffers ? c.pop_buffers : 1;
    if (h->storage && tx == 8)
        tx = 16;
    if (!pick_launcher(h->Q, tx, ty, st, npb, h->storage, fo, c.mean_bits, h->launcher)) {
        delete h;
        return fail(LBM_ERR_ARG, "unsupported tile configuration");
    }
    h->zc = std::max(1, std::min<int>(zc, int(c.nz)));

    auto cleanup_fail = [&](lbm_status s) {
        std::string msg = g_last_error;
        lbm_destroy(h);
        g_last_error = msg;
        return s;
    };
    lbm_status s;
    LBM_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    LBM_CUDA(cudaEventCreate(&h->ev0));
    LBM_CUDA(cudaEventCreate(&h->ev1));
    for (int b = 0; b < 2; b++)
        if ((s = dev_alloc(h, reinterpret_cast<char **>(&h->m[b]), 10 * h->N * h->esz)) != LBM_OK)
            return cleanup_fail(s);
    const size_t msz = c.mean_bits == 64 ? 8 : 4;
    if (c.function_objects & LBM_FO_S)
        if ((s = dev_alloc(h, &h->S, 6 * h->N)) != LBM_OK) return cleanup_fail(s);
    if (c.function_objects & LBM_FO_K)
        if ((s = dev_alloc(h, &h->k, h->N)) != LBM_OK) return cleanup_fail(s);
    if (c.function_objects & LBM_FO_SMEAN)
        if ((s = dev_alloc(h, reinterpret_cast<char **>(&h->SMean), 6 * h->N * msz)) != LBM_OK) return cleanup_fail(s);
    if (c.function_objects & LBM_FO_KMEAN)
        if ((s = dev_alloc(h, reinterpret_cast<char **>(&h->kMean), h->N * msz)) != LBM_OK) return cleanup_fail(s);
    if (c.function_objects & LBM_FO_MOMENTSMEAN)
        if ((s = dev_alloc(h, reinterpret_cast<char **>(&h->momentsMean), 10 * h->N * msz)) != LBM_OK) return cleanup_fail(s);
    if ((s = dev_alloc(h, &h->err, 1)) != LBM_OK) return cleanup_fail(s);
    if ((s = dev_alloc(h, &h->red, 4)) != LBM_OK) return cleanup_fail(s);
    if ((s = dev_alloc(h, &h->mon, 1)) != LBM_OK) return cleanup_fail(s);
    for (int b = 0; b < 2; b++) {
        cudaMemsetAsync(h->m[b], 0, 10 * h->N * h->esz, h->stream);
    }
    if (h->S) cudaMemsetAsync(h->S, 0, 6 * h->N * 4, h->stream);
    if (h->k) cudaMemsetAsync(h->k, 0, h->N * 4, h->stream);
    if (h->SMean) cudaMemsetAsync(h->SMean, 0, 6 * h->N * msz, h->stream);
    if (h->kMean) cudaMemsetAsync(h->kMean, 0, h->N * msz, h->stream);
    if (h->momentsMean) cudaMemsetAsync(h->momentsMean, 0, 10 * h->N * msz, h->stream);
    cudaMemsetAsync(h->err, 0, sizeof(lbm::StepFault), h->stream);
    if (cudaGetLastError() != cudaSuccess)
        return cleanup_fail(fail(LBM_ERR_CUDA, "cudaMemsetAsync failed"));
    for (int b = 0; b < 2; b++)
        if ((s = make_tmap(h, b)) != LBM_OK)
            return cleanup_fail(s);
    for (void *fn : {h->launcher.fn, h->launcher.fn_mon})
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(h->launcher.smem)) != cudaSuccess)
            return cleanup_fail(fail(LBM_ERR_CUDA, "cannot reserve shared memory for the step kernel"));
    *out = h;
    return LBM_OK;
}

lbm_status lbm_destroy(lbm_handle *h)
{
    if (!h)
        return LBM_OK;
    if (h->batch)
        return fail(LBM_ERR_STATE, "this cavity belongs to a batch: destroy the batch instead");
    lbm::destroy_handle(h);
    return LBM_OK;
}

lbm_status lbm_init_regions(lbm_handle *h, const float region[70])
{
    if (!h || !region)
        return fail(LBM_ERR_ARG, "null argument");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    lbm_status s = ensure_scratch(h, 70 * sizeof(float));
    if (s != LBM_OK)
        return s;
    h->last_input_kept = false;  // the state is replaced (see lbm_closure_dtau)
    h->dtau_current = h->dtau_current && !h->closure;
    LBM_CUDA(cudaMemcpyAsync(h->scratch, region, 70 * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    const int nx = int(h->cfg.nx), ny = int(h->cfg.ny), nz = int(h->cfg.nz);
    const float *rg = static_cast<float *>(h->scratch);
    if (h->storage == 1)
        init_regions_kernel<<<grid_1d(h->N), 256, 0, h->stream>>>(static_cast<__half *>(h->m[h->cur]), nx, ny, nz, rg);
    else if (h->storage == 2)
        init_regions_kernel<<<grid_1d(h->N), 256, 0, h->stream>>>(static_cast<__nv_bfloat16 *>(h->m[h->cur]), nx, ny, nz, rg);
    else
        init_regions_kernel<<<grid_1d(h->N), 256, 0, h->stream>>>(static_cast<float *>(h->m[h->cur]), nx, ny, nz, rg);
    LBM_CUDA(cudaGetLastError());
    h->launches += 1;
    const size_t msz = h->cfg.mean_bits == 64 ? 8 : 4;
    if (h->S) cudaMemsetAsync(h->S, 0, 6 * h->N * 4, h->stream);
    if (h->k) cudaMemsetAsync(h->k, 0, h->N * 4, h->stream);
    if (h->SMean) cudaMemsetAsync(h->SMean, 0, 6 * h->N * msz, h->stream);
    if (h->kMean) cudaMemsetAsync(h->kMean, 0, h->N * msz, h->stream);
    if (h->momentsMean) cudaMemsetAsync(h->momentsMean, 0, 10 * h->N * msz, h->stream);
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_write_fields(lbm_handle *h, lbm_field_set set, const void *host, size_t count, lbm_dtype dtype,
                            lbm_order order)
{
    if (!h || !host)
        return fail(LBM_ERR_ARG, "null argument");
    const int nv = nvars_of(set);
    if (nv < 0)
        return fail(LBM_ERR_ARG, "unknown field set");
    if (count != size_t(nv) * h->N)
        return fail(LBM_ERR_ARG, "count must equal nvars * nx * ny * nz");
    if (order == LBM_ORDER_TILED && (h->cfg.nx % 8 || h->cfg.ny % 8 || h->cfg.nz % 8))
        return fail(LBM_ERR_ARG, "tiled order needs multiples of 8");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    void *dptr;
    int is_double;
    lbm_status s = field_ptr(h, set, &dptr, &is_double);
    if (s != LBM_OK)
        return s;
    if (set == LBM_FIELDS_MOMENTS) {
        h->last_input_kept = false;  // the state is replaced (see lbm_closure_dtau)
        h->dtau_current = h->dtau_current && !h->closure;
    }
    const Xfer x = xfer_of(h, set, dtype, is_double, order);
    if (x.direct) {
        // same values, order and type on both sides: one copy
        LBM_CUDA(cudaMemcpyAsync(dptr, host, size_t(nv) * h->N * x.hsz, cudaMemcpyHostToDevice, h->stream));
        LBM_CUDA(cudaStreamSynchronize(h->stream));
        return LBM_OK;
    }
    if ((s = ensure_xfer(h, h->N * x.hsz)) != LBM_OK)
        return s;
    // field v: host -> scratch half (v & 1) on the copy stream, then the
    // conversion kernel on the handle stream; the copy of v + 1 overlaps the
    // conversion of v, and a half is refilled only after its kernel has run
    LBM_CUDA(cudaEventRecord(h->xe_converted[0], h->stream));
    LBM_CUDA(cudaEventRecord(h->xe_converted[1], h->stream));
    for (int v = 0; v < nv; v++) {
        const int b = v & 1;
        char *half = static_cast<char *>(h->scratch) + size_t(b) * h->N * x.hsz;
        const char *src = static_cast<const char *>(host) + size_t(v) * h->N * x.hsz;
        LBM_CUDA(cudaStreamWaitEvent(h->xstream, h->xe_converted[b], 0));
        LBM_CUDA(cudaMemcpyAsync(half, src, h->N * x.hsz, cudaMemcpyHostToDevice, h->xstream));
        LBM_CUDA(cudaEventRecord(h->xe_copied[b], h->xstream));
        LBM_CUDA(cudaStreamWaitEvent(h->stream, h->xe_copied[b], 0));
        if ((s = convert_in(h, set, dtype, is_double, dptr, v, half, order == LBM_ORDER_TILED)) != LBM_OK)
            return s;
        LBM_CUDA(cudaEventRecord(h->xe_converted[b], h->stream));
    }
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_read_fields(lbm_handle *h, lbm_field_set set, void *host, size_t count, lbm_dtype dtype, lbm_order order)
{
    if (!h || !host)
        return fail(LBM_ERR_ARG, "null argument");
    const int nv = nvars_of(set);
    if (nv < 0)
        return fail(LBM_ERR_ARG, "unknown field set");
    if (count != size_t(nv) * h->N)
        return fail(LBM_ERR_ARG, "count must equal nvars * nx * ny * nz");
    if (order == LBM_ORDER_TILED && (h->cfg.nx % 8 || h->cfg.ny % 8 || h->cfg.nz % 8))
        return fail(LBM_ERR_ARG, "tiled order needs multiples of 8");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    void *dptr;
    int is_double;
    lbm_status s = field_ptr(h, set, &dptr, &is_double);
    if (s != LBM_OK)
        return s;
    const Xfer x = xfer_of(h, set, dtype, is_double, order);
    if (x.direct) {
        LBM_CUDA(cudaMemcpyAsync(host, dptr, size_t(nv) * h->N * x.hsz, cudaMemcpyDeviceToHost, h->stream));
        LBM_CUDA(cudaStreamSynchronize(h->stream));
        return LBM_OK;
    }
    if ((s = ensure_xfer(h, h->N * x.hsz)) != LBM_OK)
        return s;
    // field v: conversion kernel into scratch half (v & 1) on the handle
    // stream, then scratch -> host on the copy stream; the conversion of v + 1
    // overlaps the copy of v, and a half is rewritten only after its copy
    LBM_CUDA(cudaEventRecord(h->xe_copied[0], h->stream));
    LBM_CUDA(cudaEventRecord(h->xe_copied[1], h->stream));
    for (int v = 0; v < nv; v++) {
        const int b = v & 1;
        char *half = static_cast<char *>(h->scratch) + size_t(b) * h->N * x.hsz;
        char *dst = static_cast<char *>(host) + size_t(v) * h->N * x.hsz;
        LBM_CUDA(cudaStreamWaitEvent(h->stream, h->xe_copied[b], 0));
        if ((s = convert_out(h, set, dtype, is_double, dptr, v, half, order == LBM_ORDER_TILED)) != LBM_OK)
            return s;
        LBM_CUDA(cudaEventRecord(h->xe_converted[b], h->stream));
        LBM_CUDA(cudaStreamWaitEvent(h->xstream, h->xe_converted[b], 0));
        LBM_CUDA(cudaMemcpyAsync(dst, half, h->N * x.hsz, cudaMemcpyDeviceToHost, h->xstream));
        LBM_CUDA(cudaEventRecord(h->xe_copied[b], h->xstream));
    }
    LBM_CUDA(cudaStreamSynchronize(h->xstream));
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

}  // extern "C"

namespace {

// Plain steps (no function objects, no closure) repeat their launch
// parameters every two steps, so lbm_step replays a CUDA graph of
// kGraphSteps of them, captured from buffer 0: one graph launch instead of
// kGraphSteps kernel launches (the per-launch cost matters for small meshes).
constexpr uint64_t kGraphSteps = 16;

lbm_status ensure_steps_graph(lbm_handle *h)
{
    if (h->steps_graph)
        return LBM_OK;
    const int cur0 = h->cur;
    const int64_t t0 = h->t;
    const uint64_t l0 = h->launches;
    h->cur = 0;
    LBM_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    lbm_status s = LBM_OK;
    const bool md = means_f64(h);
    for (uint64_t i = 0; i < kGraphSteps && s == LBM_OK; i++)
        s = md ? launch_step<double>(h) : launch_step<float>(h);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->cur = cur0;
    h->t = t0;
    h->launches = l0;
    if (s != LBM_OK) {
        if (g)
            cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("step graph capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&h->steps_graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        h->steps_graph = nullptr;
        return fail(LBM_ERR_CUDA, std::string("step graph instantiation: ") + cudaGetErrorString(ei));
    }
    return LBM_OK;
}

void drop_steps_graph(lbm_handle *h)
{
    if (h->steps_graph) {
        cudaGraphExecDestroy(h->steps_graph);
        h->steps_graph = nullptr;
    }
}

}  // namespace

extern "C" {

lbm_status lbm_step(lbm_handle *h, uint64_t n)
{
    if (!h)
        return fail(LBM_ERR_ARG, "null handle");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    if (n == 0)
        return LBM_OK;
    const bool md = means_f64(h);
    const bool graphed = !h->cfg.function_objects && !h->closure && n >= kGraphSteps;
    if (graphed) {
        // built once per kernel variant, outside the timed span
        lbm_status s = ensure_steps_graph(h);
        if (s != LBM_OK)
            return s;
    }
    LBM_CUDA(cudaEventRecord(h->ev0, h->stream));
    uint64_t i = 0;
    if (graphed) {
        lbm_status s;
        if (h->cur != 0) {
            if ((s = md ? launch_step<double>(h) : launch_step<float>(h)) != LBM_OK)
                return s;
            i++;
        }
        for (; n - i >= kGraphSteps; i += kGraphSteps) {
            LBM_CUDA(cudaGraphLaunch(h->steps_graph, h->stream));
            h->t += int64_t(kGraphSteps);
            h->launches += kGraphSteps;
        }
    }
    for (; i < n; i++) {
        lbm_status s = md ? launch_step<double>(h) : launch_step<float>(h);
        if (s != LBM_OK)
            return s;
    }
    LBM_CUDA(cudaEventRecord(h->ev1, h->stream));
    h->timed = true;
    return LBM_OK;
}

lbm_status lbm_step_monitored(lbm_handle *h, uint64_t n, lbm_monitor *out)
{
    if (!h || (!out && n))
        return fail(LBM_ERR_ARG, "null argument");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    static_assert(sizeof(lbm_monitor) == sizeof(lbm::MonitorSlot), "monitor layout");
    if (n == 0)
        return LBM_OK;
    LBM_CUDA(cudaEventRecord(h->ev0, h->stream));
    const bool md = means_f64(h);
    for (uint64_t i = 0; i < n; i++) {
        LBM_CUDA(cudaMemsetAsync(h->mon, 0, sizeof(lbm::MonitorSlot), h->stream));
        lbm_status s = md ? launch_step<double>(h, true) : launch_step<float>(h, true);
        if (s != LBM_OK)
            return s;
        LBM_CUDA(cudaMemcpyAsync(&out[i], h->mon, sizeof(lbm::MonitorSlot), cudaMemcpyDeviceToHost, h->stream));
    }
    LBM_CUDA(cudaEventRecord(h->ev1, h->stream));
    h->timed = true;
    return LBM_OK;
}

lbm_status lbm_run_streamed(lbm_handle *h, const float *moments, uint64_t n, void *const out[6], lbm_monitor *mon,
                            const lbm_stream_opts *opts)
{
    if (!h || !moments || !out)
        return fail(LBM_ERR_ARG, "null argument");
    if (n == 0 || n > uint64_t(1) << 30)
        return fail(LBM_ERR_ARG, "lbm_run_streamed: n must be in [1, 2^30]");
    if (h->closure)
        return fail(LBM_ERR_STATE, "lbm_run_streamed: not available with the learned closure");
    const int P = opts && opts->slab > 0 ? opts->slab : 16;
    const int zc = opts && opts->z_chunk > 0 ? std::min(opts->z_chunk, P) : std::min(4, P);
    const int lead = opts && opts->lead > 0 ? opts->lead : 2;
    if (P > (1 << 20) || lead > (1 << 20))
        return fail(LBM_ERR_ARG, "lbm_run_streamed: slab or lead too large");
    // host buffers and the device field of every requested set
    struct Out {
        char *host;
        char *dev;
        size_t esz;
        int nv;
    };
    std::vector<Out> outs;
    for (int s = 0; s < 6; s++) {
        if (!out[s] || s == LBM_FIELDS_MOMENTS)
            continue;
        void *d = nullptr;
        int is_double = 0;
        lbm_status st = field_ptr(h, lbm_field_set(s), &d, &is_double);
        if (st != LBM_OK)
            return st;
        outs.push_back({static_cast<char *>(out[s]), static_cast<char *>(d), size_t(is_double ? 8 : 4),
                        nvars_of(lbm_field_set(s))});
    }
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->xstream)
        LBM_CUDA(cudaStreamCreateWithFlags(&h->xstream, cudaStreamNonBlocking));
    if (!h->dstream)
        LBM_CUDA(cudaStreamCreateWithFlags(&h->dstream, cudaStreamNonBlocking));
    if (mon && h->mon_steps_cap < n) {
        if (h->mon_steps) {
            cudaFree(h->mon_steps);
            h->device_bytes -= h->mon_steps_cap * sizeof(lbm::MonitorSlot);
            h->mon_steps = nullptr;
            h->mon_steps_cap = 0;
        }
        LBM_CUDA(cudaMalloc(&h->mon_steps, n * sizeof(lbm::MonitorSlot)));
        h->mon_steps_cap = n;
        h->device_bytes += n * sizeof(lbm::MonitorSlot);
    }
    const int nz = int(h->cfg.nz);
    const size_t plane = size_t(h->cfg.nx) * size_t(h->cfg.ny);
    const size_t pitch = h->N * sizeof(float);
    const int UP = std::min(P, 4);                                   // planes per upload chunk
    const int U = (nz + UP - 1) / UP;                                // upload chunks
    // 16-bit storage: the host values (FP32) pass through a staging block of
    // UP planes each way and a conversion kernel on the copy's own stream
    float *stage_up = nullptr, *stage_down = nullptr;
    if (h->storage != 0) {
        const size_t sb = 10 * size_t(UP) * plane;
        lbm_status ss = ensure_scratch(h, 2 * sb * sizeof(float));
        if (ss != LBM_OK)
            return ss;
        stage_up = static_cast<float *>(h->scratch);
        stage_down = stage_up + sb;
    }
    auto convert_planes = [&](bool in, float *stage, void *mbuf, size_t off, size_t cnt,
                              cudaStream_t cs) -> lbm_status {
        const dim3 g(unsigned(std::min<size_t>((cnt + 255) / 256, size_t(148) * 4)), 10);
        if (h->storage == 1) {
            if (in)
                planes_in_kernel<<<g, 256, 0, cs>>>(static_cast<__half *>(mbuf), stage, h->N, off, cnt);
            else
                planes_out_kernel<<<g, 256, 0, cs>>>(stage, static_cast<const __half *>(mbuf), h->N, off, cnt);
        } else {
            if (in)
                planes_in_kernel<<<g, 256, 0, cs>>>(static_cast<__nv_bfloat16 *>(mbuf), stage, h->N, off, cnt);
            else
                planes_out_kernel<<<g, 256, 0, cs>>>(stage, static_cast<const __nv_bfloat16 *>(mbuf), h->N, off,
                                                     cnt);
        }
        LBM_CUDA(cudaGetLastError());
        h->launches += 1;
        return LBM_OK;
    };
    const int in0 = h->cur;
    const int fin = int((uint64_t(in0) + n) & 1u);  // buffer of the final moments
    // A long job runs its first and last kSkew steps as skewed slabs (the
    // upload overlaps the first ones, the download the last ones) and the
    // steps between them as whole-mesh launches; a short one is one skewed
    // phase with both transfers.
    constexpr uint64_t kSkew = 16;
    const bool split = n > 2 * kSkew;
    std::vector<cudaEvent_t> evs;
    auto cleanup = [&] {
        for (cudaEvent_t e : evs)
            cudaEventDestroy(e);
    };
    auto new_event = [&](cudaEvent_t *e) -> lbm_status {
        if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess)
            return fail(LBM_ERR_CUDA, "lbm_run_streamed: event creation failed");
        evs.push_back(*e);
        return LBM_OK;
    };
    const bool md = means_f64(h);
    auto step_range = [&](uint64_t s, int64_t lo, int64_t hi, int zcl) -> lbm_status {
        const int in = int((uint64_t(in0) + s) & 1u);
        lbm::MonitorSlot *slot = mon ? h->mon_steps + s : nullptr;
        return md ? launch_slab<double>(h, in, h->t + int64_t(s), int(lo), int(hi), zcl, slot)
                  : launch_slab<float>(h, in, h->t + int64_t(s), int(lo), int(hi), zcl, slot);
    };
    std::vector<cudaEvent_t> up(size_t(U), nullptr);
    int waited = -1;  // upload chunks the compute stream has waited for
    // Steps [s0, s0 + m) as skewed slabs: slab j covers planes [bnd(j),
    // bnd(j+1)) at its first step and one plane lower at each following
    // step; the first slab is m + lead planes high, so that its own last
    // step already finishes planes, the others P, up to nz + m - 1.  With
    // `uploads`, slab j first waits for the chunk that holds plane bnd(j+1);
    // with `downloads`, the planes slab j finished go to the host after it.
    auto skewed = [&](uint64_t s0, uint64_t m, bool uploads, bool downloads) -> lbm_status {
        const int64_t F = int64_t(m) + lead;
        auto bnd = [&](int64_t j) -> int64_t { return j == 0 ? 0 : F + (j - 1) * int64_t(P); };
        const int64_t span = int64_t(nz) + int64_t(m) - 1;
        const int J = int(1 + (span > F ? (span - F + P - 1) / P : 0));
        for (int j = 0; j < J; j++) {
            if (uploads) {
                const int need = int(std::min<int64_t>(nz - 1, bnd(j + 1)) / UP);
                for (; waited < need; waited++)
                    LBM_CUDA(cudaStreamWaitEvent(h->stream, up[size_t(waited + 1)], 0));
            }
            for (uint64_t s = 0; s < m; s++) {
                const int64_t lo = std::max<int64_t>(0, bnd(j) - int64_t(s));
                const int64_t hi = std::min<int64_t>(nz, bnd(j + 1) - int64_t(s));
                if (lo >= hi)
                    continue;
                lbm_status ls = step_range(s0 + s, lo, hi, zc);
                if (ls != LBM_OK)
                    return ls;
            }
            if (!downloads)
                continue;
            // planes whose last step slab j completed
            const int64_t flo = std::max<int64_t>(0, bnd(j) - int64_t(m) + 1);
            const int64_t fhi = std::min<int64_t>(nz, bnd(j + 1) - int64_t(m) + 1);
            if (flo >= fhi)
                continue;
            cudaEvent_t done;
            lbm_status es = new_event(&done);
            if (es != LBM_OK)
                return es;
            LBM_CUDA(cudaEventRecord(done, h->stream));
            LBM_CUDA(cudaStreamWaitEvent(h->dstream, done, 0));
            const size_t z0 = size_t(flo), nzs = size_t(fhi - flo);
            char *host_m = static_cast<char *>(out[LBM_FIELDS_MOMENTS]);
            if (host_m && h->storage == 0) {
                const size_t off = z0 * plane * sizeof(float);
                LBM_CUDA(cudaMemcpy2DAsync(host_m + off, pitch, static_cast<const char *>(h->m[fin]) + off, pitch,
                                           nzs * plane * sizeof(float), 10, cudaMemcpyDeviceToHost, h->dstream));
            } else if (host_m) {
                for (size_t a = z0; a < z0 + nzs; a += size_t(UP)) {
                    const size_t b = std::min(z0 + nzs, a + size_t(UP));
                    const size_t off = a * plane, cnt = (b - a) * plane;
                    lbm_status cs = convert_planes(false, stage_down, h->m[fin], off, cnt, h->dstream);
                    if (cs != LBM_OK)
                        return cs;
                    LBM_CUDA(cudaMemcpy2DAsync(host_m + off * sizeof(float), pitch, stage_down,
                                               cnt * sizeof(float), cnt * sizeof(float), 10, cudaMemcpyDeviceToHost,
                                               h->dstream));
                }
            }
            for (const Out &o : outs) {
                const size_t off = z0 * plane * o.esz;
                LBM_CUDA(cudaMemcpy2DAsync(o.host + off, h->N * o.esz, o.dev + off, h->N * o.esz,
                                           nzs * plane * o.esz, size_t(o.nv), cudaMemcpyDeviceToHost, h->dstream));
            }
        }
        return LBM_OK;
    };
    lbm_status st = LBM_OK;
    auto run = [&]() -> lbm_status {
        cudaEvent_t start, end;
        lbm_status es = new_event(&start);
        if (es == LBM_OK)
            es = new_event(&end);
        for (size_t u = 0; u < up.size() && es == LBM_OK; u++)
            es = new_event(&up[u]);
        if (es != LBM_OK)
            return es;
        // the copies must not overtake work already queued on the handle
        LBM_CUDA(cudaEventRecord(start, h->stream));
        LBM_CUDA(cudaStreamWaitEvent(h->xstream, start, 0));
        LBM_CUDA(cudaStreamWaitEvent(h->dstream, start, 0));
        // uploads: chunk u = planes [u UP, (u+1) UP) of all 10 fields (small
        // chunks, so that the first slab starts early)
        char *dst0 = static_cast<char *>(h->m[in0]);
        for (int u = 0; u < U; u++) {
            const size_t z0 = size_t(u) * UP, z1 = std::min<size_t>(nz, z0 + UP);
            const size_t off = z0 * plane, cnt = (z1 - z0) * plane;
            const char *src = reinterpret_cast<const char *>(moments) + off * sizeof(float);
            if (h->storage == 0) {
                LBM_CUDA(cudaMemcpy2DAsync(dst0 + off * sizeof(float), pitch, src, pitch, cnt * sizeof(float), 10,
                                           cudaMemcpyHostToDevice, h->xstream));
            } else {
                LBM_CUDA(cudaMemcpy2DAsync(stage_up, cnt * sizeof(float), src, pitch, cnt * sizeof(float), 10,
                                           cudaMemcpyHostToDevice, h->xstream));
                lbm_status cs = convert_planes(true, stage_up, dst0, off, cnt, h->xstream);
                if (cs != LBM_OK)
                    return cs;
            }
            LBM_CUDA(cudaEventRecord(up[size_t(u)], h->xstream));
        }
        if (mon)
            LBM_CUDA(cudaMemsetAsync(h->mon_steps, 0, n * sizeof(lbm::MonitorSlot), h->stream));
        LBM_CUDA(cudaEventRecord(h->ev0, h->stream));
        lbm_status ps;
        if (!split) {
            ps = skewed(0, n, true, true);
        } else {
            ps = skewed(0, kSkew, true, false);
            for (uint64_t s = kSkew; ps == LBM_OK && s < n - kSkew; s++)
                ps = step_range(s, 0, nz, h->zc);
            if (ps == LBM_OK)
                ps = skewed(n - kSkew, kSkew, false, true);
        }
        if (ps != LBM_OK)
            return ps;
        LBM_CUDA(cudaEventRecord(h->ev1, h->stream));
        if (mon) {
            LBM_CUDA(cudaEventRecord(end, h->stream));
            LBM_CUDA(cudaStreamWaitEvent(h->dstream, end, 0));
            LBM_CUDA(cudaMemcpyAsync(mon, h->mon_steps, n * sizeof(lbm::MonitorSlot), cudaMemcpyDeviceToHost,
                                     h->dstream));
        }
        return LBM_OK;
    };
    st = run();
    // wait for everything queued, also after an error in the middle
    const cudaError_t e1 = cudaStreamSynchronize(h->dstream);
    const cudaError_t e2 = cudaStreamSynchronize(h->xstream);
    const cudaError_t e3 = cudaStreamSynchronize(h->stream);
    cleanup();
    if (st != LBM_OK)
        return st;
    for (cudaError_t e : {e1, e2, e3})
        if (e != cudaSuccess)
            return fail(LBM_ERR_CUDA, std::string("lbm_run_streamed: ") + cudaGetErrorString(e));
    h->cur = fin;
    h->t += int64_t(n);
    h->timed = true;
    h->last_input_kept = false;
    lbm::StepFault f{};
    LBM_CUDA(cudaMemcpy(&f, h->err, sizeof(f), cudaMemcpyDeviceToHost));
    return lbm::check_fault(f, "a step kernel");
}

lbm_status lbm_synchronize(lbm_handle *h)
{
    if (!h)
        return fail(LBM_ERR_ARG, "null handle");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    lbm::StepFault f{};
    LBM_CUDA(cudaMemcpy(&f, h->err, sizeof(f), cudaMemcpyDeviceToHost));
    return lbm::check_fault(f, "a step kernel");
}

lbm_status lbm_reduce(lbm_handle *h, double out[3])
{
    if (!h || !out)
        return fail(LBM_ERR_ARG, "null argument");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    LBM_CUDA(cudaMemsetAsync(h->red, 0, 4 * sizeof(double), h->stream));
    auto *dbad = reinterpret_cast<unsigned long long *>(h->red + 2);
    if (h->storage == 1)
        reduce_kernel<<<grid_1d(h->N), 256, 0, h->stream>>>(static_cast<const __half *>(h->m[h->cur]), h->N, h->red, dbad);
    else if (h->storage == 2)
        reduce_kernel<<<grid_1d(h->N), 256, 0, h->stream>>>(static_cast<const __nv_bfloat16 *>(h->m[h->cur]), h->N,
                                                             h->red, dbad);
    else
        reduce_kernel<<<grid_1d(h->N), 256, 0, h->stream>>>(static_cast<const float *>(h->m[h->cur]), h->N, h->red, dbad);
    LBM_CUDA(cudaGetLastError());
    h->launches += 1;
    double r[3];
    unsigned long long bad = 0;
    LBM_CUDA(cudaMemcpyAsync(r, h->red, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LBM_CUDA(cudaMemcpyAsync(&bad, h->red + 2, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    out[0] = r[0];
    out[1] = r[1];
    out[2] = double(bad);
    return LBM_OK;
}

lbm_status lbm_case_read(const char *dir, lbm_case *out)
{
    if (!dir || !out)
        return fail(LBM_ERR_ARG, "null argument");
    std::memset(out, 0, sizeof(*out));
    try {
        const lbm::ProgramControl pc = lbm::read_program_control(dir);
        if (pc.caseName.size() >= sizeof(out->case_name))
            return fail(LBM_ERR_PARSE, "caseName too long");
        std::strncpy(out->case_name, pc.caseName.c_str(), sizeof(out->case_name) - 1);
        out->Re = pc.Re;
        out->u_inf = pc.u_inf;
        out->n_time_steps = pc.nTimeSteps;
        out->save_interval = pc.saveInterval;
        out->info_interval = pc.infoInterval;
        const lbm::LatticeMesh m = lbm::read_lattice_mesh(dir);
        out->nx = m.nx;
        out->ny = m.ny;
        out->nz = m.nz;
        out->Lx = m.Lx;
        out->Ly = m.Ly;
        out->Lz = m.Lz;
        out->function_objects = lbm::read_function_objects(dir);
        const std::vector<uint64_t> t = lbm::time_indices(dir, pc.caseName);
        out->has_restart = !t.empty();
        out->latest_time = t.empty() ? 0 : t.back();
        if (t.empty()) {
            const std::array<float, 70> r = lbm::read_initial_conditions(dir);
            std::copy(r.begin(), r.end(), out->region);
        }
    } catch (const lbm::CaseError &e) {
        return fail(std::string(e.what()).find("not opened") != std::string::npos ? LBM_ERR_IO : LBM_ERR_PARSE, e.what());
    } catch (const std::exception &e) {
        return fail(LBM_ERR_PARSE, e.what());
    }
    return LBM_OK;
}

lbm_status lbm_lbmbin_write(const char *path, uint64_t nx, uint64_t ny, uint64_t nz, int32_t nvars,
                            const char *const *names, const float *values, uint64_t time_step, int32_t time_average)
{
    if (!path || !names || !values || nvars <= 0)
        return fail(LBM_ERR_ARG, "null or empty argument");
    try {
        std::vector<std::string> n(names, names + nvars);
        lbm::write_field_file(path, nx, ny, nz, n, values, time_step, time_average != 0);
    } catch (const std::exception &e) {
        return fail(LBM_ERR_IO, e.what());
    }
    return LBM_OK;
}

lbm_status lbm_vts_write(const char *path, uint64_t nx, uint64_t ny, uint64_t nz, const float L[3], int32_t nvars,
                         const char *const *names, const float *values)
{
    if (!path || !L || !names || !values || nvars <= 0 || nx == 0 || ny == 0 || nz == 0)
        return fail(LBM_ERR_ARG, "null or empty argument");
    try {
        const uint64_t n = nx * ny * nz;
        lbm::FieldSet f(static_cast<size_t>(nvars));
        for (int32_t v = 0; v < nvars; v++)
            f[v].assign(values + size_t(v) * n, values + size_t(v + 1) * n);
        lbm::write_vts(path, f, std::vector<std::string>(names, names + nvars), nx, ny, nz, L);
    } catch (const std::exception &e) {
        return fail(LBM_ERR_IO, e.what());
    }
    return LBM_OK;
}

lbm_status lbm_cut_plane(lbm_handle *h, lbm_field_set set, int32_t axis, float position, float *host_out, size_t count)
{
    if (!h || !host_out)
        return fail(LBM_ERR_ARG, "null argument");
    if (axis < 0 || axis > 2)
        return fail(LBM_ERR_ARG, "lbm_cut_plane: axis must be 0 (x), 1 (y) or 2 (z)");
    const int64_t dims[3] = {h->cfg.nx, h->cfg.ny, h->cfg.nz};
    const float index = static_cast<float>(dims[axis] - 1) * position;
    if (!(index >= 0.0f) || index > static_cast<float>(dims[axis] - 1))
        return fail(LBM_ERR_ARG, "lbm_cut_plane: position must lie in [0, 1]");
    const int nv = nvars_of(set);
    if (nv < 0)
        return fail(LBM_ERR_ARG, "unknown field set");
    const size_t na = size_t(axis == 0 ? h->cfg.ny : h->cfg.nx), nb = size_t(axis == 2 ? h->cfg.ny : h->cfg.nz);
    const size_t total = size_t(nv) * na * nb;
    if (count != total)
        return fail(LBM_ERR_ARG, "lbm_cut_plane: count must be " + std::to_string(total));
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    void *src = nullptr;
    int is_double = 0;
    lbm_status s = field_ptr(h, set, &src, &is_double);
    if (s != LBM_OK)
        return s;
    if ((s = ensure_scratch(h, total * sizeof(float))) != LBM_OK)
        return s;
    const int i0 = int(std::floor(index)), i1 = int(std::ceil(index));
    const float w = index - static_cast<float>(i0);
    float *dst = static_cast<float *>(h->scratch);
    const int nx = int(h->cfg.nx), ny = int(h->cfg.ny), nz = int(h->cfg.nz);
    const dim3 g = grid_1d(total);
    if (set == LBM_FIELDS_MOMENTS && h->storage == 1)
        cut_plane_kernel<<<g, 256, 0, h->stream>>>(dst, static_cast<const __half *>(src), nv, nx, ny, nz, axis, i0, i1, w);
    else if (set == LBM_FIELDS_MOMENTS && h->storage == 2)
        cut_plane_kernel<<<g, 256, 0, h->stream>>>(dst, static_cast<const __nv_bfloat16 *>(src), nv, nx, ny, nz, axis, i0,
                                                   i1, w);
    else if (is_double)
        cut_plane_kernel<<<g, 256, 0, h->stream>>>(dst, static_cast<const double *>(src), nv, nx, ny, nz, axis, i0, i1, w);
    else
        cut_plane_kernel<<<g, 256, 0, h->stream>>>(dst, static_cast<const float *>(src), nv, nx, ny, nz, axis, i0, i1, w);
    LBM_CUDA(cudaGetLastError());
    h->launches += 1;
    LBM_CUDA(cudaMemcpyAsync(host_out, dst, total * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_selftest_wait_timeout(int32_t device, uint64_t timeout_ns)
{
    if (timeout_ns == 0 || timeout_ns > 10000000000ull)
        return fail(LBM_ERR_ARG, "lbm_selftest_wait_timeout: timeout must be in (0, 10 s]");
    LBM_CUDA(cudaSetDevice(device));
    lbm::StepFault *d = nullptr;
    LBM_CUDA(cudaMalloc(&d, sizeof(*d)));
    cudaMemset(d, 0, sizeof(*d));
    wait_timeout_kernel<<<1, 64>>>(d, timeout_ns);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaDeviceSynchronize();
    lbm::StepFault f{};
    if (e == cudaSuccess)
        e = cudaMemcpy(&f, d, sizeof(f), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("lbm_selftest_wait_timeout: ") + cudaGetErrorString(e));
    return lbm::check_fault(f, "the self-test wait");
}

lbm_status lbm_host_alloc(size_t bytes, void **out)
{
    if (!out)
        return fail(LBM_ERR_ARG, "null argument");
    *out = nullptr;
    LBM_CUDA(cudaMallocHost(out, bytes));
    return LBM_OK;
}

lbm_status lbm_host_free(void *p)
{
    if (p)
        LBM_CUDA(cudaFreeHost(p));
    return LBM_OK;
}

// ------------------------------------------------------------- autotuner
namespace {

struct TuneKey {
    int Q;
    int64_t nx, ny, nz;
    uint32_t fo;
    int mean_bits;
    bool operator==(const TuneKey &o) const
    {
        return Q == o.Q && nx == o.nx && ny == o.ny && nz == o.nz && fo == o.fo && mean_bits == o.mean_bits;
    }
};
struct TuneEntry {
    TuneKey key;
    lbm_tuning best;
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune_cache;

const char *tune_cache_path()
{
    const char *p = std::getenv("LBM_B200_TUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

void load_tune_file()
{
    static bool loaded = false;
    if (loaded)
        return;
    loaded = true;
    const char *path = tune_cache_path();
    if (!path)
        return;
    FILE *f = std::fopen(path, "r");
    if (!f)
        return;
    TuneEntry e{};
    long long nx, ny, nz;
    unsigned fo;
    while (std::fscanf(f, "%d %lld %lld %lld %u %d %d %d %d %d %d %lf %d", &e.key.Q, &nx, &ny, &nz, &fo, &e.key.mean_bits,
                       &e.best.tile_x, &e.best.tile_y, &e.best.stages, &e.best.pop_buffers, &e.best.z_chunk,
                       &e.best.ms_per_step, &e.best.closure_fused) == 13) {
        e.key.nx = nx;
        e.key.ny = ny;
        e.key.nz = nz;
        e.key.fo = fo;
        g_tune_cache.push_back(e);
    }
    std::fclose(f);
}

void save_tune_entry(const TuneEntry &e)
{
    const char *path = tune_cache_path();
    if (!path)
        return;
    FILE *f = std::fopen(path, "a");
    if (!f)
        return;
    std::fprintf(f, "%d %lld %lld %lld %u %d %d %d %d %d %d %.6f %d\n", e.key.Q, (long long)e.key.nx, (long long)e.key.ny,
                 (long long)e.key.nz, e.key.fo, e.key.mean_bits, e.best.tile_x, e.best.tile_y, e.best.stages,
                 e.best.pop_buffers, e.best.z_chunk, e.best.ms_per_step, e.best.closure_fused);
    std::fclose(f);
}

// Switch the handle to another kernel variant (same results, other speed).
lbm_status apply_variant(lbm_handle *h, int tx, int ty, int stages, int npb, int zc)
{
    Launcher l;
    if (!pick_launcher(h->Q, tx, ty, stages, npb, h->storage, h->cfg.function_objects, h->cfg.mean_bits, l))
        return fail(LBM_ERR_ARG, "unsupported tile configuration");
    for (void *fn : {l.fn, l.fn_mon})
        LBM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(l.smem)));
    h->launcher = l;
    h->zc = std::max(1, std::min<int>(zc, int(h->cfg.nz)));
    drop_steps_graph(h);
    for (int b = 0; b < 2; b++) {
        lbm_status s = make_tmap(h, b);
        if (s != LBM_OK)
            return s;
    }
    return LBM_OK;
}

}  // namespace

}  // extern "C"
namespace lbm {
lbm_status retile(lbm_handle *h, int tx, int ty, int stages, int npb, int zc)
{
    return apply_variant(h, tx, ty, stages, npb, zc);
}
}  // namespace lbm
extern "C" {

lbm_status lbm_autotune(lbm_handle *h, int32_t trial_steps, lbm_tuning *out)
{
    if (!h)
        return fail(LBM_ERR_ARG, "null handle");
    LBM_CUDA(cudaSetDevice(h->cfg.device));
    if (trial_steps <= 0)
        trial_steps = 10;
    // the size class: lattice, mesh, function objects, mean precision, and
    // (in the high bits of the function-object word) the storage format and
    // whether a learned closure is set -- each has its own kernel shapes
    const uint32_t kClosureKey = 0x100u, kStorageShift = 9;
    const TuneKey key{h->Q, h->cfg.nx, h->cfg.ny, h->cfg.nz,
                      h->cfg.function_objects | (h->closure ? kClosureKey : 0u) |
                          (uint32_t(h->storage) << kStorageShift),
                      h->cfg.mean_bits};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        load_tune_file();
        for (const auto &e : g_tune_cache)
            if (e.key == key) {
                lbm_status s = apply_variant(h, e.best.tile_x, e.best.tile_y, e.best.stages, e.best.pop_buffers,
                                             e.best.z_chunk);
                if (s != LBM_OK)
                    return s;
                if (h->closure)
                    h->closure_fused = e.best.closure_fused != 0;
                if (out) {
                    *out = e.best;
                    out->from_cache = 1;
                }
                return LBM_OK;
            }
    }
    // back up the state the trials will advance
    const size_t msz = h->cfg.mean_bits == 64 ? 8 : 4;
    std::vector<std::pair<void *, size_t>> live = {{h->m[h->cur], 10 * h->N * h->esz}};
    if (h->S) live.push_back({h->S, 6 * h->N * 4});
    if (h->k) live.push_back({h->k, h->N * 4});
    if (h->SMean) live.push_back({h->SMean, 6 * h->N * msz});
    if (h->kMean) live.push_back({h->kMean, h->N * msz});
    if (h->momentsMean) live.push_back({h->momentsMean, 10 * h->N * msz});
    std::vector<void *> backup(live.size(), nullptr);
    auto release = [&]() {
        for (void *p : backup)
            if (p)
                cudaFree(p);
    };
    for (size_t i = 0; i < live.size(); i++) {
        if (cudaMalloc(&backup[i], live[i].second) != cudaSuccess) {
            release();
            return fail(LBM_ERR_NOMEM, "autotune: no room to back up the state");
        }
        cudaMemcpyAsync(backup[i], live[i].first, live[i].second, cudaMemcpyDeviceToDevice, h->stream);
    }
    const int cur0 = h->cur;
    const int64_t t0 = h->t;
    const uint64_t launches0 = h->launches;
    const uint64_t closure_steps0 = h->closure_steps;
    auto restore = [&]() {
        h->cur = cur0;
        h->t = t0;
        h->closure_steps = closure_steps0;
        h->last_input_kept = false;  // trial steps overwrote the other buffer
        h->dtau_current = false;     // and, on the separate path, dtau[]
        live[0].first = h->m[cur0];
        for (size_t i = 0; i < live.size(); i++)
            cudaMemcpyAsync(live[i].first, backup[i], live[i].second, cudaMemcpyDeviceToDevice, h->stream);
    };
    const bool md = means_f64(h);
    lbm_tuning best{};
    best.ms_per_step = 1e30;
    int tried = 0;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->cfg.device);
    for (const Variant &v : kVariants) {
        if (v.Q != h->Q || v.storage != h->storage || v.tx > h->cfg.nx || v.ty > h->cfg.ny)
            continue;
        if (h->closure && (v.stages != 2 || v.npb != 1))
            continue;  // shapes that have a closure kernel
        // z-chunks below 8 only for meshes too small to fill the GPU at 8
        // (such a chunk re-reads two planes for every 2-4 it updates)
        const int64_t tiles = ((h->cfg.nx + v.tx - 1) / v.tx) * ((h->cfg.ny + v.ty - 1) / v.ty);
        const bool small = tiles * ((h->cfg.nz + 7) / 8) < 4 * 148 * 3;
        // Candidates: powers of two, and chunk lengths whose grid is close to
        // a whole number of waves of resident CTAs (k waves for k = 1..12):
        // the last wave of a grid 9.2 waves long runs the GPU at a fifth of
        // its CTA slots.  Chunks need not divide nz (the last is shorter).
        std::vector<int> zcs = {2, 4, 8, 16, 32, 64};
        {
            Launcher l;
            int per_sm = 0;
            if (pick_launcher(h->Q, v.tx, v.ty, v.stages, v.npb, h->storage, h->cfg.function_objects,
                              h->cfg.mean_bits, l) &&
                cudaFuncSetAttribute(l.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(l.smem)) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, l.fn, v.tx * v.ty, l.smem) == cudaSuccess &&
                per_sm > 0) {
                const int64_t resident = int64_t(per_sm) * sms;
                for (int64_t k = 1; k <= 12; k++) {
                    const int64_t chunks = std::max<int64_t>(1, (k * resident + tiles / 2) / tiles);
                    const int zc = int((h->cfg.nz + chunks - 1) / chunks);
                    if (std::find(zcs.begin(), zcs.end(), zc) == zcs.end())
                        zcs.push_back(zc);
                }
            }
        }
        for (int zc : zcs) {
            if (zc > h->cfg.nz || (zc < 8 && !small))
                continue;
            lbm_status s = apply_variant(h, v.tx, v.ty, v.stages, v.npb, zc);
            if (s != LBM_OK) {
                release();
                return s;
            }
            for (int w = 0; w < 2 && s == LBM_OK; w++)
                s = md ? launch_step<double>(h) : launch_step<float>(h);
            cudaEventRecord(h->ev0, h->stream);
            for (int k = 0; k < trial_steps && s == LBM_OK; k++)
                s = md ? launch_step<double>(h) : launch_step<float>(h);
            cudaEventRecord(h->ev1, h->stream);
            float ms = 0.0f;
            if (s == LBM_OK && cudaEventSynchronize(h->ev1) == cudaSuccess &&
                cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) {
                const double per = double(ms) / trial_steps;
                if (per < best.ms_per_step) {
                    best.ms_per_step = per;
                    best.tile_x = v.tx;
                    best.tile_y = v.ty;
                    best.stages = v.stages;
                    best.pop_buffers = v.npb;
                    best.z_chunk = zc;
                }
                tried++;
            }
            restore();
            if (s != LBM_OK) {
                release();
                return s;
            }
        }
    }
    lbm_status s = tried ? apply_variant(h, best.tile_x, best.tile_y, best.stages, best.pop_buffers, best.z_chunk)
                         : fail(LBM_ERR_STATE, "autotune: no kernel variant fits this mesh");
    best.closure_fused = h->closure_fused ? 1 : 0;
    if (s == LBM_OK && h->closure) {
        // the learned closure's two evaluations on the chosen shape: the
        // network inside the step kernel, or a separate inference kernel
        double ms_mode[2] = {1e30, 1e30};
        for (int fused = 0; fused < 2 && s == LBM_OK; fused++) {
            h->closure_fused = fused != 0;
            for (int w = 0; w < 2 && s == LBM_OK; w++)
                s = md ? launch_step<double>(h) : launch_step<float>(h);
            cudaEventRecord(h->ev0, h->stream);
            for (int k = 0; k < trial_steps && s == LBM_OK; k++)
                s = md ? launch_step<double>(h) : launch_step<float>(h);
            cudaEventRecord(h->ev1, h->stream);
            float ms = 0.0f;
            if (s == LBM_OK && cudaEventSynchronize(h->ev1) == cudaSuccess &&
                cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess)
                ms_mode[fused] = double(ms) / trial_steps;
            restore();
            tried++;
        }
        h->closure_fused = ms_mode[1] <= ms_mode[0];
        best.closure_fused = h->closure_fused ? 1 : 0;
        best.ms_per_step = std::min(ms_mode[0], ms_mode[1]);
    }
    LBM_CUDA(cudaStreamSynchronize(h->stream));
    release();
    (void)launches0;
    h->timed = false;
    if (s != LBM_OK)
        return s;
    best.candidates = tried;
    best.from_cache = 0;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache.push_back({key, best});
        save_tune_entry({key, best});
    }
    if (out)
        *out = best;
    return LBM_OK;
}

lbm_status lbm_get_info(lbm_handle *h, lbm_info *info)
{
    if (!h || !info)
        return fail(LBM_ERR_ARG, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->step = h->t;
    info->nodes = int64_t(h->N);
    info->tau = h->tau;
    info->omega = h->omega;
    info->tile_x = h->launcher.tx;
    info->tile_y = h->launcher.ty;
    info->z_chunk = h->zc;
    info->stages = h->launcher.stages;
    info->device_bytes = h->device_bytes;
    info->kernel_launches = h->launches;
    if (h->timed) {
        float ms = 0.0f;
        if (cudaEventSynchronize(h->ev1) == cudaSuccess && cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess)
            info->last_step_ms = ms;
    }
    return LBM_OK;
}

}  // extern "C"
