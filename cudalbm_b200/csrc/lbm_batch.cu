// lbm_batch.cu -- many independent cavities advanced by one persistent launch
// per step (lbm_batch_* of include/lbm_b200.h).
//
// Each cavity is an ordinary lbm_handle (so every per-cavity call works on
// it), moved onto the batch's stream.  The batch adds:
//   * a mesh table (lbm::BatchMesh per cavity: buffers, sizes, z-chunk,
//     relaxation constants, first work item) and two TMA descriptors per
//     cavity, both in device memory;
//   * a persistent lbm::batch_kernel sized to the GPU's resident-CTA count,
//     which claims work items from a device counter;
//   * a CUDA graph of two launches (flip 0 reads each cavity's current
//     buffer, flip 1 the other), replayed n/2 times per lbm_batch_step;
//   * an autotuner: one kernel shape for the batch, one z-chunk per size
//     class.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "lbm_b200.h"
#include "lbm_handle.hpp"
#include "lbm_step.cuh"

namespace {

lbm_status fail(lbm_status s, const std::string &m) { return lbm::record_error(s, m); }

struct BatchLauncher {
    void *fn = nullptr;
    size_t smem = 0;
    int tx = 0, ty = 0, stages = 0, npb = 0;
};

// Compiled shapes of the batched kernel: (lattice, tile x, tile y, TMA
// stages, population-plane code as in lbm::Variant).
struct BatchShape {
    int Q, tx, ty, stages, npb;
};
constexpr BatchShape kShapes[] = {{19, 32, 8, 2, 1}, {19, 16, 8, 2, 1}, {19, 32, 8, 3, 1}, {19, 32, 8, 2, 2},
                                  {19, 32, 8, 2, 4}, {19, 8, 8, 2, 1},  {27, 32, 8, 2, 1}, {27, 16, 8, 2, 1},
                                  {27, 32, 8, 2, 2}, {27, 8, 8, 2, 1}};

template <int Q, int TX, int TY, int NS, int NPB, int MINB>
BatchLauncher make_launcher(int npb_code)
{
    BatchLauncher l;
    l.fn = reinterpret_cast<void *>(&lbm::batch_kernel<Q, TX, TY, NS, NPB, MINB>);
    l.smem = lbm::SmemLayout<Q, TX, TY, NS, NPB, float>::bytes;
    l.tx = TX;
    l.ty = TY;
    l.stages = NS;
    l.npb = npb_code;
    return l;
}

bool pick_shape(int Q, int tx, int ty, int stages, int npb, BatchLauncher &out)
{
#define LBM_BATCH_SHAPE(QQ, TXX, TYY, NSS, CODE, NPB, MINB)                                   \
    if (Q == QQ && tx == TXX && ty == TYY && stages == NSS && npb == CODE) {                  \
        out = make_launcher<QQ, TXX, TYY, NSS, NPB, MINB>(CODE);                              \
        return true;                                                                          \
    }
    LBM_BATCH_SHAPE(19, 32, 8, 2, 1, 1, 3)
    LBM_BATCH_SHAPE(19, 16, 8, 2, 1, 1, 3)
    LBM_BATCH_SHAPE(19, 32, 8, 3, 1, 1, 3)
    LBM_BATCH_SHAPE(19, 32, 8, 2, 2, 2, 2)
    LBM_BATCH_SHAPE(19, 32, 8, 2, 4, 1, 4)
    LBM_BATCH_SHAPE(19, 8, 8, 2, 1, 1, 3)
    LBM_BATCH_SHAPE(27, 32, 8, 2, 1, 1, 3)
    LBM_BATCH_SHAPE(27, 16, 8, 2, 1, 1, 3)
    LBM_BATCH_SHAPE(27, 32, 8, 2, 2, 2, 2)
    LBM_BATCH_SHAPE(27, 8, 8, 2, 1, 1, 3)
#undef LBM_BATCH_SHAPE
    return false;
}

}  // namespace

struct lbm_batch {
    int device = 0, Q = 19;
    cudaStream_t stream = nullptr;
    std::vector<lbm_handle *> cav;       // creation order
    std::vector<int> zc;                 // z-planes per work item, per cavity
    std::vector<int> row_of;             // mesh-table row of each cavity
    BatchLauncher launcher;
    int grid = 0, items = 0;
    lbm::BatchMesh *d_mesh = nullptr;
    CUtensorMap *d_tmap = nullptr;
    unsigned *d_ctr = nullptr;           // [0] next item, [1] finished CTAs
    lbm::StepFault *d_err = nullptr;
    int persistent = 1;                  // 1: persistent grid; 0: one CTA per work item
    std::vector<lbm::BatchMesh> h_mesh;  // what d_mesh holds
    bool tables_valid = false;           // d_mesh/d_tmap/grid match launcher and zc
    cudaGraphExec_t exec = nullptr;      // two launches: flip 0, flip 1
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    int64_t steps = 0;
    uint64_t launches = 0, graph_launches = 0, table_bytes = 0;
};

namespace {

void drop_graph(lbm_batch *b)
{
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
}

lbm::BatchParams params_of(const lbm_batch *b)
{
    lbm::BatchParams p{};
    p.mesh = b->d_mesh;
    p.tmap = b->d_tmap;
    p.nmesh = int(b->cav.size());
    p.items = b->items;
    p.next = b->d_ctr;
    p.done = b->d_ctr + 1;
    p.fault = b->d_err;
    p.timeout_ns = 2000000000ull;
    p.persistent = b->persistent;
    return p;
}

lbm_status launch(lbm_batch *b, int flip)
{
    lbm::BatchParams p = params_of(b);
    void *args[] = {&p, &flip};
    LBM_CUDA_RETURN(cudaLaunchKernel(b->launcher.fn, dim3(b->grid), dim3(b->launcher.tx, b->launcher.ty), args,
                                     b->launcher.smem, b->stream));
    b->launches += 1;
    return LBM_OK;
}

// Mesh table, TMA descriptors and grid for the current shape and z-chunks.
// Rows are ordered by work-item size (z-chunk), then mesh size, descending,
// so that the largest items are claimed first and the tail is short.
lbm_status build_tables(lbm_batch *b)
{
    const int n = int(b->cav.size());
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        if (b->zc[a] != b->zc[c])
            return b->zc[a] > b->zc[c];
        return b->cav[a]->N > b->cav[c]->N;
    });
    lbm::EncodeTiledFn enc = lbm::encode_tiled();
    if (!enc)
        return fail(LBM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const BatchLauncher &l = b->launcher;
    std::vector<lbm::BatchMesh> mesh(n);
    std::vector<CUtensorMap> tmap(2 * size_t(n));
    b->row_of.assign(n, 0);
    int64_t items = 0;
    for (int r = 0; r < n; r++) {
        lbm_handle *h = b->cav[order[r]];
        b->row_of[order[r]] = r;
        lbm::BatchMesh &m = mesh[r];
        m.m[0] = static_cast<float *>(h->m[0]);
        m.m[1] = static_cast<float *>(h->m[1]);
        m.nx = int(h->cfg.nx);
        m.ny = int(h->cfg.ny);
        m.nz = int(h->cfg.nz);
        m.zc = std::max(1, std::min(b->zc[order[r]], m.nz));
        m.tiles_x = (m.nx + l.tx - 1) / l.tx;
        m.tiles_y = (m.ny + l.ty - 1) / l.ty;
        m.item_begin = int(items);
        m.cur = h->cur;
        m.rx = lbm::Relax{h->omega, h->t_omega, h->omega_d2, h->tau, h->cfg.u_inf};
        items += int64_t(m.tiles_x) * m.tiles_y * ((m.nz + m.zc - 1) / m.zc);
        if (items > (int64_t(1) << 30))
            return fail(LBM_ERR_ARG, "batch: too many work items");
        for (int buf = 0; buf < 2; buf++) {
            cuuint64_t dims[4] = {cuuint64_t(m.nx), cuuint64_t(m.ny), cuuint64_t(m.nz), 10};
            cuuint64_t strides[3] = {cuuint64_t(m.nx) * 4, cuuint64_t(m.nx) * m.ny * 4, cuuint64_t(h->N) * 4};
            cuuint32_t box[4] = {cuuint32_t(l.tx + 2 * lbm::Storage<float>::XPAD), cuuint32_t(l.ty + 2), 1, 10};
            cuuint32_t estr[4] = {1, 1, 1, 1};
            CUresult e = enc(&tmap[2 * r + buf], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->m[buf], dims, strides, box,
                             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (e != CUDA_SUCCESS)
                return fail(LBM_ERR_CUDA, "batch: cuTensorMapEncodeTiled failed with CUresult " + std::to_string(int(e)));
        }
    }
    b->items = int(items);
    LBM_CUDA_RETURN(cudaFuncSetAttribute(l.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(l.smem)));
    int per_sm = 0, sms = 0;
    LBM_CUDA_RETURN(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, l.fn, l.tx * l.ty, l.smem));
    LBM_CUDA_RETURN(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    if (per_sm < 1)
        return fail(LBM_ERR_CUDA, "batch: the kernel shape does not fit on one SM");
    b->grid = b->persistent ? int(std::min<int64_t>(int64_t(per_sm) * sms, items)) : int(items);
    // the previous launches read the tables: order the uploads after them
    LBM_CUDA_RETURN(cudaStreamSynchronize(b->stream));
    LBM_CUDA_RETURN(cudaMemcpy(b->d_mesh, mesh.data(), sizeof(lbm::BatchMesh) * n, cudaMemcpyHostToDevice));
    LBM_CUDA_RETURN(cudaMemcpy(b->d_tmap, tmap.data(), sizeof(CUtensorMap) * 2 * n, cudaMemcpyHostToDevice));
    b->h_mesh = mesh;
    b->tables_valid = true;
    drop_graph(b);
    return LBM_OK;
}

// Bring the tables up to date with the cavities' current buffers (a cavity
// stepped on its own, or an odd lbm_batch_step, flips its `cur`).
lbm_status refresh(lbm_batch *b)
{
    if (!b->tables_valid)
        return build_tables(b);
    bool stale = false;
    for (size_t i = 0; i < b->cav.size(); i++)
        stale |= b->h_mesh[b->row_of[i]].cur != b->cav[i]->cur;
    if (!stale)
        return LBM_OK;
    for (size_t i = 0; i < b->cav.size(); i++)
        b->h_mesh[b->row_of[i]].cur = b->cav[i]->cur;
    LBM_CUDA_RETURN(cudaStreamSynchronize(b->stream));
    LBM_CUDA_RETURN(cudaMemcpy(b->d_mesh, b->h_mesh.data(), sizeof(lbm::BatchMesh) * b->cav.size(),
                               cudaMemcpyHostToDevice));
    return LBM_OK;
}

lbm_status ensure_graph(lbm_batch *b)
{
    if (b->exec)
        return LBM_OK;
    cudaGraph_t g = nullptr;
    LBM_CUDA_RETURN(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    lbm_status s = launch(b, 0);
    if (s == LBM_OK)
        s = launch(b, 1);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    b->launches -= 2;  // captured, not launched
    if (s != LBM_OK) {
        if (g)
            cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess)
        return fail(LBM_ERR_CUDA, std::string("batch: graph capture failed: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->exec = nullptr;
        return fail(LBM_ERR_CUDA, std::string("batch: graph instantiation failed: ") + cudaGetErrorString(e));
    }
    return LBM_OK;
}

lbm_status batch_steps(lbm_batch *b, uint64_t n)
{
    lbm_status s = refresh(b);
    if (s != LBM_OK)
        return s;
    if ((s = ensure_graph(b)) != LBM_OK)
        return s;
    for (uint64_t i = 0; i + 1 < n; i += 2) {
        LBM_CUDA_RETURN(cudaGraphLaunch(b->exec, b->stream));
        b->graph_launches += 1;
        b->launches += 2;
    }
    if (n & 1) {
        if ((s = launch(b, 0)) != LBM_OK)
            return s;
        for (lbm_handle *h : b->cav)
            h->cur ^= 1;
    }
    for (lbm_handle *h : b->cav)
        h->t += int64_t(n);
    b->steps += int64_t(n);
    return LBM_OK;
}

void free_batch(lbm_batch *b)
{
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (lbm_handle *h : b->cav)
        lbm::destroy_handle(h);
    for (void *p : {static_cast<void *>(b->d_mesh), static_cast<void *>(b->d_tmap), static_cast<void *>(b->d_ctr),
                    static_cast<void *>(b->d_err)})
        if (p)
            cudaFree(p);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream)
        cudaStreamDestroy(b->stream);
    delete b;
}

// Default shape: the widest tile that divides every cavity's nx.
void default_shape(lbm_batch *b, int &tx)
{
    tx = 32;
    for (lbm_handle *h : b->cav)
        while (tx > 8 && h->cfg.nx % tx)
            tx /= 2;
}

}  // namespace

extern "C" {

lbm_status lbm_batch_create(const lbm_config *cfgs, int32_t n, lbm_batch **out)
{
    if (!cfgs || !out || n <= 0)
        return fail(LBM_ERR_ARG, "lbm_batch_create: null argument or empty batch");
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (cfgs[i].lattice != cfgs[0].lattice || cfgs[i].device != cfgs[0].device)
            return fail(LBM_ERR_ARG, "lbm_batch_create: all cavities must share the lattice and the device");
        if (cfgs[i].function_objects)
            return fail(LBM_ERR_ARG, "lbm_batch_create: batches run the plain method (no function objects)");
        if (cfgs[i].storage != LBM_STORAGE_F32)
            return fail(LBM_ERR_ARG, "lbm_batch_create: batches store moments in FP32");
    }
    lbm_batch *b = new lbm_batch();
    b->device = cfgs[0].device;
    b->Q = cfgs[0].lattice;
    auto cleanup = [&](lbm_status s) {
        std::string msg = lbm_last_error();
        free_batch(b);
        lbm::record_error(s, msg);
        return s;
    };
    for (int i = 0; i < n; i++) {
        lbm_handle *h = nullptr;
        lbm_status s = lbm_create(&cfgs[i], &h);
        if (s != LBM_OK)
            return cleanup(s);
        b->cav.push_back(h);
    }
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
        return cleanup(fail(LBM_ERR_CUDA, "lbm_batch_create: cannot create the stream"));
    // the cavities' initial fills ran on their own streams: finish them, then
    // move every cavity onto the batch stream
    for (lbm_handle *h : b->cav) {
        if (cudaStreamSynchronize(h->stream) != cudaSuccess)
            return cleanup(fail(LBM_ERR_CUDA, "lbm_batch_create: cavity set-up failed"));
        cudaStreamDestroy(h->stream);
        h->stream = b->stream;
        h->own_stream = false;
        h->batch = b;
    }
    if (cudaMalloc(&b->d_mesh, sizeof(lbm::BatchMesh) * n) != cudaSuccess ||
        cudaMalloc(&b->d_tmap, sizeof(CUtensorMap) * 2 * size_t(n)) != cudaSuccess ||
        cudaMalloc(&b->d_ctr, 2 * sizeof(unsigned)) != cudaSuccess || cudaMalloc(&b->d_err, sizeof(lbm::StepFault)) != cudaSuccess)
        return cleanup(fail(LBM_ERR_NOMEM, "lbm_batch_create: cannot allocate the batch tables"));
    b->table_bytes = sizeof(lbm::BatchMesh) * n + sizeof(CUtensorMap) * 2 * size_t(n) + 2 * sizeof(unsigned) + sizeof(lbm::StepFault);
    if (cudaMemset(b->d_ctr, 0, 2 * sizeof(unsigned)) != cudaSuccess || cudaMemset(b->d_err, 0, sizeof(lbm::StepFault)) != cudaSuccess)
        return cleanup(fail(LBM_ERR_CUDA, "lbm_batch_create: cannot clear the batch counters"));
    int tx;
    default_shape(b, tx);
    if (!pick_shape(b->Q, tx, 8, 2, 1, b->launcher))
        return cleanup(fail(LBM_ERR_ARG, "lbm_batch_create: no batched kernel for this lattice"));
    b->zc.assign(n, 16);
    lbm_status s = build_tables(b);
    if (s != LBM_OK)
        return cleanup(s);
    *out = b;
    return LBM_OK;
}

lbm_status lbm_batch_destroy(lbm_batch *b)
{
    if (b)
        free_batch(b);
    return LBM_OK;
}

lbm_status lbm_batch_cavity(lbm_batch *b, int32_t i, lbm_handle **out)
{
    if (!b || !out)
        return fail(LBM_ERR_ARG, "null argument");
    if (i < 0 || i >= int32_t(b->cav.size()))
        return fail(LBM_ERR_ARG, "lbm_batch_cavity: index out of range");
    *out = b->cav[i];
    return LBM_OK;
}

lbm_status lbm_batch_step(lbm_batch *b, uint64_t n)
{
    if (!b)
        return fail(LBM_ERR_ARG, "null batch");
    LBM_CUDA_RETURN(cudaSetDevice(b->device));
    if (n == 0)
        return LBM_OK;
    lbm_status s = refresh(b);
    if (s != LBM_OK)
        return s;
    LBM_CUDA_RETURN(cudaEventRecord(b->ev0, b->stream));
    if ((s = batch_steps(b, n)) != LBM_OK)
        return s;
    LBM_CUDA_RETURN(cudaEventRecord(b->ev1, b->stream));
    b->timed = true;
    return LBM_OK;
}

lbm_status lbm_batch_synchronize(lbm_batch *b)
{
    if (!b)
        return fail(LBM_ERR_ARG, "null batch");
    LBM_CUDA_RETURN(cudaSetDevice(b->device));
    LBM_CUDA_RETURN(cudaStreamSynchronize(b->stream));
    lbm::StepFault f{};
    LBM_CUDA_RETURN(cudaMemcpy(&f, b->d_err, sizeof(f), cudaMemcpyDeviceToHost));
    lbm_status s = lbm::check_fault(f, "a batched step kernel");
    for (size_t i = 0; i < b->cav.size() && s == LBM_OK; i++) {
        LBM_CUDA_RETURN(cudaMemcpy(&f, b->cav[i]->err, sizeof(f), cudaMemcpyDeviceToHost));
        s = lbm::check_fault(f, "a step kernel of a batch cavity");
    }
    return s;
}

lbm_status lbm_batch_autotune(lbm_batch *b, int32_t trial_steps, lbm_batch_tuning *out)
{
    if (!b)
        return fail(LBM_ERR_ARG, "null batch");
    LBM_CUDA_RETURN(cudaSetDevice(b->device));
    if (trial_steps <= 0)
        trial_steps = 10;
    trial_steps += trial_steps & 1;  // whole graph replays
    const int n = int(b->cav.size());
    LBM_CUDA_RETURN(cudaStreamSynchronize(b->stream));
    // back up every cavity's state
    std::vector<void *> backup(n, nullptr);
    std::vector<int> cur0(n);
    std::vector<int64_t> t0(n);
    auto release = [&]() {
        for (void *p : backup)
            if (p)
                cudaFree(p);
    };
    for (int i = 0; i < n; i++) {
        lbm_handle *h = b->cav[i];
        const size_t bytes = 10 * h->N * sizeof(float);
        if (cudaMalloc(&backup[i], bytes) != cudaSuccess) {
            release();
            return fail(LBM_ERR_NOMEM, "lbm_batch_autotune: no room to back up the states");
        }
        cudaMemcpyAsync(backup[i], h->m[h->cur], bytes, cudaMemcpyDeviceToDevice, b->stream);
        cur0[i] = h->cur;
        t0[i] = h->t;
    }
    const int64_t steps0 = b->steps;
    const uint64_t launches0 = b->launches, graphs0 = b->graph_launches;

    int candidates = 0;
    const int persistent0 = b->persistent;
    auto time_current = [&](double &ms_per_step) -> lbm_status {
        lbm_status s = build_tables(b);
        if (s == LBM_OK)
            s = batch_steps(b, 2);  // warm-up (and graph build)
        if (s != LBM_OK)
            return s;
        LBM_CUDA_RETURN(cudaEventRecord(b->ev0, b->stream));
        if ((s = batch_steps(b, uint64_t(trial_steps))) != LBM_OK)
            return s;
        LBM_CUDA_RETURN(cudaEventRecord(b->ev1, b->stream));
        LBM_CUDA_RETURN(cudaEventSynchronize(b->ev1));
        float ms = 0.0f;
        LBM_CUDA_RETURN(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        ms_per_step = double(ms) / trial_steps;
        candidates++;
        return LBM_OK;
    };

    lbm_status s = LBM_OK;
    BatchLauncher best_l = b->launcher;
    int best_p = persistent0;
    double best = 1e30;
    // 1. kernel shape and grid kind for the whole batch, at the current z-chunks
    for (const BatchShape &v : kShapes) {
        if (v.Q != b->Q || s != LBM_OK)
            continue;
        BatchLauncher l;
        if (!pick_shape(v.Q, v.tx, v.ty, v.stages, v.npb, l))
            continue;
        for (int pers : {1, 0}) {
            b->launcher = l;
            b->persistent = pers;
            double ms = 0.0;
            if ((s = time_current(ms)) != LBM_OK)
                break;
            if (ms < best) {
                best = ms;
                best_l = l;
                best_p = pers;
            }
        }
    }
    b->launcher = best_l;
    b->persistent = best_p;
    // 2. z-chunk per size class (distinct mesh), largest class first
    std::map<std::tuple<int64_t, int64_t, int64_t>, std::vector<int>> classes;
    for (int i = 0; i < n && s == LBM_OK; i++)
        classes[std::make_tuple(b->cav[i]->cfg.nx, b->cav[i]->cfg.ny, b->cav[i]->cfg.nz)].push_back(i);
    std::vector<std::vector<int>> order;
    for (auto &kv : classes)
        order.push_back(kv.second);
    std::sort(order.begin(), order.end(), [&](const std::vector<int> &a, const std::vector<int> &c) {
        return b->cav[a[0]]->N * a.size() > b->cav[c[0]]->N * c.size();
    });
    for (const auto &members : order) {
        if (s != LBM_OK)
            break;
        const int nz = int(b->cav[members[0]]->cfg.nz);
        int best_zc = b->zc[members[0]];
        for (int zc : {8, 16, 32, 64}) {
            if (zc > nz || zc == best_zc)
                continue;
            for (int i : members)
                b->zc[i] = zc;
            double ms = 0.0;
            if ((s = time_current(ms)) != LBM_OK)
                break;
            if (ms < best) {
                best = ms;
                best_zc = zc;
            }
        }
        for (int i : members)
            b->zc[i] = best_zc;
    }
    // restore the states and counters, then the tables of the choice
    cudaStreamSynchronize(b->stream);
    for (int i = 0; i < n; i++) {
        lbm_handle *h = b->cav[i];
        h->cur = cur0[i];
        h->t = t0[i];
        cudaMemcpyAsync(h->m[h->cur], backup[i], 10 * h->N * sizeof(float), cudaMemcpyDeviceToDevice, b->stream);
    }
    b->steps = steps0;
    b->launches = launches0;
    b->graph_launches = graphs0;
    b->timed = false;
    if (s == LBM_OK)
        s = build_tables(b);
    cudaStreamSynchronize(b->stream);
    release();
    if (s != LBM_OK)
        return s;
    if (out) {
        out->tile_x = b->launcher.tx;
        out->tile_y = b->launcher.ty;
        out->stages = b->launcher.stages;
        out->pop_buffers = b->launcher.npb;
        out->persistent = b->persistent;
        out->size_classes = int32_t(order.size());
        out->candidates = candidates;
        out->ms_per_step = best;
    }
    return LBM_OK;
}

lbm_status lbm_batch_configure(lbm_batch *b, const lbm_batch_tuning *shape)
{
    if (!b || !shape)
        return fail(LBM_ERR_ARG, "null argument");
    if (shape->persistent != 0 && shape->persistent != 1)
        return fail(LBM_ERR_ARG, "lbm_batch_configure: persistent must be 0 or 1");
    BatchLauncher l;
    if (!pick_shape(b->Q, shape->tile_x, shape->tile_y, shape->stages, shape->pop_buffers, l))
        return fail(LBM_ERR_ARG, "lbm_batch_configure: no batched kernel with that shape");
    LBM_CUDA_RETURN(cudaSetDevice(b->device));
    b->launcher = l;
    b->persistent = shape->persistent;
    return build_tables(b);
}

lbm_status lbm_batch_get_info(lbm_batch *b, lbm_batch_info *info)
{
    if (!b || !info)
        return fail(LBM_ERR_ARG, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->cavities = int32_t(b->cav.size());
    info->items = b->items;
    info->grid = b->grid;
    info->tile_x = b->launcher.tx;
    info->tile_y = b->launcher.ty;
    info->stages = b->launcher.stages;
    info->pop_buffers = b->launcher.npb;
    info->persistent = b->persistent;
    uint64_t bytes = b->table_bytes;
    for (lbm_handle *h : b->cav) {
        info->nodes += int64_t(h->N);
        bytes += h->device_bytes;
    }
    info->device_bytes = bytes;
    info->step = b->steps;
    info->kernel_launches = b->launches;
    info->graph_launches = b->graph_launches;
    if (b->timed) {
        float ms = 0.0f;
        if (cudaEventSynchronize(b->ev1) == cudaSuccess && cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess)
            info->last_step_ms = ms;
    }
    return LBM_OK;
}

}  // extern "C"
