// lbm_handle.hpp -- internal: the state behind an lbm_handle, shared by the
// translation units of the library (not installed, not part of the C ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "lbm_b200.h"
#include "lbm_step.cuh"
#include "lbm_mlp.cuh"
#include "lbm_variants.cuh"

struct lbm_batch;

struct lbm_handle {
    lbm_config cfg{};
    int Q = 19;
    size_t N = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;            // false while the handle belongs to a batch (batch stream)
    lbm_batch *batch = nullptr;        // owning batch, if any (then lbm_destroy refuses)
    void *m[2] = {nullptr, nullptr};  // moment fields in the storage format
    int storage = 0;                   // 0 FP32, 1 FP16, 2 BF16
    size_t esz = 4;                    // bytes per stored moment value
    int cur = 0;
    CUtensorMap tmap[2];
    // function objects
    float *S = nullptr, *k = nullptr;
    void *SMean = nullptr, *kMean = nullptr, *momentsMean = nullptr;
    lbm::StepFault *err = nullptr;    // device-side error record of the step kernels
    double *red = nullptr;
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    // field transfers (lbm_read_fields / lbm_write_fields): a copy stream and
    // per-half events, so that the copy of one field overlaps the conversion
    // kernel of the next (two scratch halves)
    cudaStream_t xstream = nullptr;
    cudaEvent_t xe_copied[2] = {nullptr, nullptr};
    cudaEvent_t xe_converted[2] = {nullptr, nullptr};
    // lbm_run_streamed: uploads go on xstream, downloads on dstream; one
    // monitor slot per step of the job
    cudaStream_t dstream = nullptr;
    lbm::MonitorSlot *mon_steps = nullptr;
    size_t mon_steps_cap = 0;
    float tau = 0, omega = 0, t_omega = 0, omega_d2 = 0;
    int64_t t = 0;
    lbm::Launcher launcher;
    int zc = 0;
    uint64_t device_bytes = 0;
    uint64_t launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    lbm::MonitorSlot *mon = nullptr;  // one slot, reused by every monitored step
    // learned closure (lbm_closure.cu)
    bool closure = false;
    float *dtau = nullptr;             // [N] relaxation-time correction of the current step
    lbm::MlpDevice *mlp = nullptr;     // network for the closure (host copy, passed by value)
    cudaGraphExec_t steps_graph = nullptr;  // kGraphSteps plain steps from buffer 0 (see lbm_step)
    int closure_every = 1;             // recompute dtau every this many steps
    uint64_t closure_steps = 0;        // closure steps taken since lbm_closure_set
    bool closure_fused = true;         // evaluate the network inside the step kernel (when every == 1)
    bool dtau_current = true;          // dtau[] holds the last closure step's values
    bool last_input_kept = false;      // m[cur ^ 1] is still the input of the last (fused) closure step
};

namespace lbm {

// Sets the message returned by lbm_last_error() and returns s.
lbm_status record_error(lbm_status s, const std::string &msg);

// cuTensorMapEncodeTiled from the driver (null if unavailable).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled();

// Frees a handle regardless of batch ownership (used by lbm_batch_destroy).
void destroy_handle(lbm_handle *h);

// LBM_OK, or the status and message for a device-side error record.
lbm_status check_fault(const StepFault &f, const char *who);

// Switch a handle to another compiled kernel shape (same results).
lbm_status retile(lbm_handle *h, int tx, int ty, int stages, int npb, int zc);

// One time step with the learned closure (lbm_closure.cu).
lbm_status closure_step(lbm_handle *h);

}  // namespace lbm

#define LBM_CUDA_RETURN(call)                                                                                    \
    do {                                                                                                         \
        cudaError_t e_ = (call);                                                                                 \
        if (e_ != cudaSuccess)                                                                                   \
            return lbm::record_error(e_ == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,            \
                                     std::string(#call) + ": " + cudaGetErrorString(e_) + " (" +                \
                                         std::to_string((int)e_) + ")");                                         \
    } while (0)
