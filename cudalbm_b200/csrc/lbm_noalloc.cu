// lbm_noalloc.cu -- global sums over the moments without allocating memory.
//
// Who needs this: programs that embed the solver but must not call
// cudaMalloc at the moment they want a diagnostic.  A host framework that has
// handed all device memory to its own caching allocator cannot grow it behind
// that allocator's back; a monitoring thread that samples a simulation whose
// buffers it does not own should not allocate (an allocation can synchronise
// the device or fail under memory pressure); code that keeps the solution in
// its own device arrays has no lbm_handle whose buffers lbm_reduce could use.
// lbm_reduce_moments_noalloc reduces any caller-owned array of moments and
// keeps its only scratch -- one partial sum per block of nodes -- in a fixed,
// statically sized device array of this file.
//
// The scratch is g_partials below: (kMaxPartials + 1) triples of doubles,
// 1.5 MiB, held on every GPU that loads this library until the process exits.
// Every call overwrites each slot it later reads, so nothing needs clearing,
// but all calls share the array: calls that overlap on the GPU (from two
// streams, or from host threads without ordering between them) race and must
// be serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "lbm_b200.h"

namespace lbm {
lbm_status record_error(lbm_status s, const std::string &msg);
}

namespace {

constexpr int kThreads = 256;
constexpr uint64_t kChunk = 16384;           // nodes summed by one block, in a fixed order
constexpr uint64_t kMaxPartials = 65536;     // blocks per call
constexpr uint64_t kMaxNodes = kChunk * kMaxPartials;  // 2^30 nodes (e.g. 1024^3)

struct Partial {
    double mass, ke, bad;
};

// The only scratch: per-block partials, then the final triple at [kMaxPartials].
static __device__ __align__(256) Partial g_partials[kMaxPartials + 1];

// messages go to the library's lbm_last_error() (lbm_capi.cu)
lbm_status fail(lbm_status s, const std::string &m)
{
    return lbm::record_error(s, m);
}

// Deterministic block sum: fixed pairing in shared memory.
__device__ void block_sum(Partial &p)
{
    __shared__ double sm[3][kThreads];
    const int t = threadIdx.x;
    sm[0][t] = p.mass;
    sm[1][t] = p.ke;
    sm[2][t] = p.bad;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (t < s) {
            sm[0][t] += sm[0][t + s];
            sm[1][t] += sm[1][t + s];
            sm[2][t] += sm[2][t + s];
        }
        __syncthreads();
    }
    p = {sm[0][0], sm[1][0], sm[2][0]};
}

__global__ void __launch_bounds__(kThreads) partial_sums(const float *m, uint64_t n, Partial *scratch)
{
    const uint64_t b0 = uint64_t(blockIdx.x) * kChunk;
    const uint64_t b1 = b0 + kChunk < n ? b0 + kChunk : n;
    Partial p{0.0, 0.0, 0.0};
    for (uint64_t i = b0 + threadIdx.x; i < b1; i += kThreads) {
        const double rho = double(m[i]) + 1.0;
        const double u = double(m[n + i]) / 3.0, v = double(m[2 * n + i]) / 3.0, w = double(m[3 * n + i]) / 3.0;
        p.mass += rho;
        p.ke += 0.5 * rho * (u * u + v * v + w * w);
        for (int f = 0; f < 10; f++)
            p.bad += !isfinite(m[uint64_t(f) * n + i]);
    }
    block_sum(p);
    if (threadIdx.x == 0)
        scratch[blockIdx.x] = p;
}

__global__ void __launch_bounds__(kThreads) final_sum(Partial *scratch, unsigned nparts)
{
    Partial p{0.0, 0.0, 0.0};
    for (unsigned i = threadIdx.x; i < nparts; i += kThreads) {
        p.mass += scratch[i].mass;
        p.ke += scratch[i].ke;
        p.bad += scratch[i].bad;
    }
    block_sum(p);
    if (threadIdx.x == 0)
        scratch[kMaxPartials] = p;
}

// Context identity: cuCtxGetCurrent and cuCtxGetId from the driver (by entry
// point, so that the library needs no link against libcuda).  A context id is
// unique for the life of the process, unlike the CUcontext handle value.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

bool current_context_id(unsigned long long *id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(p);
    });
    CUcontext ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx)
        return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of g_partials (the name g_partials in host code is only a
// host-side stand-in).  It is looked up with the device current, once per
// device and context: the cache entry is keyed on the context's id, so after
// the device's context is reset (cudaDeviceReset, or a host framework
// recreating the primary context, which reloads this module) the next call
// looks the address up again instead of using the old one.
Partial *scratch_for_current_device(lbm_status *st)
{
    constexpr int kMaxDevices = 64;
    struct Entry {
        unsigned long long ctx;
        Partial *addr;
    };
    static std::mutex mu;
    static Entry cache[kMaxDevices] = {};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *st = fail(LBM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    unsigned long long ctx = 0;
    const bool known = current_context_id(&ctx);
    if (known && cache[dev].addr && cache[dev].ctx == ctx) {
        *st = LBM_OK;
        return cache[dev].addr;
    }
    // set-up: look the address up in the current context (this also makes the
    // device's primary context current if the thread had none yet)
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess || !p) {
        *st = fail(LBM_ERR_CUDA, std::string("cudaGetSymbolAddress(g_partials): ") + cudaGetErrorString(e));
        return nullptr;
    }
    if (current_context_id(&ctx))
        cache[dev] = {ctx, static_cast<Partial *>(p)};
    else
        cache[dev] = {0, nullptr};  // context not identifiable: look up again on every call
    *st = LBM_OK;
    return static_cast<Partial *>(p);
}

}  // namespace

extern "C" lbm_status lbm_reduce_moments_noalloc(const float *moments, uint64_t nodes, double out[3], void *stream)
{
    if (!moments || !out)
        return fail(LBM_ERR_ARG, "lbm_reduce_moments_noalloc: null argument");
    if (nodes > kMaxNodes)
        return fail(LBM_ERR_ARG, "lbm_reduce_moments_noalloc: " + std::to_string(nodes) +
                                     " nodes exceed the fixed scratch limit of " + std::to_string(kMaxNodes) +
                                     " nodes; use lbm_reduce on a handle instead");
    out[0] = out[1] = out[2] = 0.0;
    if (nodes == 0)
        return LBM_OK;
    lbm_status st;
    Partial *scratch = scratch_for_current_device(&st);
    if (!scratch)
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned nparts = unsigned((nodes + kChunk - 1) / kChunk);
    partial_sums<<<nparts, kThreads, 0, s>>>(moments, nodes, scratch);
    final_sum<<<1, kThreads, 0, s>>>(scratch, nparts);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("lbm_reduce_moments_noalloc launch: ") + cudaGetErrorString(e));
    Partial r;
    e = cudaMemcpyAsync(&r, scratch + kMaxPartials, sizeof(r), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("lbm_reduce_moments_noalloc: ") + cudaGetErrorString(e));
    out[0] = r.mass;
    out[1] = r.ke;
    out[2] = r.bad;
    return LBM_OK;
}
