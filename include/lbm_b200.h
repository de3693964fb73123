/*
 * lbm_b200.h -- C ABI of the B200 moment-representation LBM solver.
 *
 * The reference (geoenergiaUDESC/cudaLBM) compiles its hot path into each
 * executable as header-only templates and exposes no library interface; its
 * observable surface is the executables momentBasedD3Q19 / momentBasedD3Q27,
 * the case files and the .LBMBin output.  This header is the boundary that
 * replaces the reference's in-process pieces: every entry point below names
 * the reference code it stands in for.  Plain C types only; the library owns
 * all device memory; callers pass host buffers.  Every call returns an
 * lbm_status; nothing inside the library exits the process (the reference's
 * checkCudaErrors calls std::exit, src/errorHandler.cuh:88-111).
 *
 * Threading: a handle belongs to one host thread at a time and owns one CUDA
 * stream.  Different handles may be used from different threads.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_B200_ABI_VERSION 1

typedef enum lbm_status {
    LBM_OK = 0,
    LBM_ERR_ARG = 1,      /* invalid argument / size (reference: errorHandler(ERR_SIZE, ...)) */
    LBM_ERR_CUDA = 2,     /* CUDA runtime error (reference: std::exit(cudaError)) */
    LBM_ERR_NOMEM = 3,    /* device or host allocation failed */
    LBM_ERR_TIMEOUT = 4,  /* a bounded device wait gave up (kernel reported, context intact) */
    LBM_ERR_IO = 5,       /* file missing, unreadable, truncated or unwritable */
    LBM_ERR_PARSE = 6,    /* malformed case file (reference: uncaught std::runtime_error) */
    LBM_ERR_STATE = 7,    /* call not valid in the handle's current state */
    LBM_ERR_NONFINITE = 8 /* a NaN/Inf was found in the solution */
} lbm_status;

/* Function objects (reference src/functionObjects, switched on by the
 * functionObjects case file). Bit mask. */
enum {
    LBM_FO_S = 1u << 0,          /* strain-rate tensor, 6 components */
    LBM_FO_SMEAN = 1u << 1,      /* running mean of S */
    LBM_FO_K = 1u << 2,          /* k = 0.5*sqrt(u^2+v^2+w^2) of the stored (scaled) velocity */
    LBM_FO_KMEAN = 1u << 3,      /* running mean of k */
    LBM_FO_MOMENTSMEAN = 1u << 4 /* running mean of the 10 stored moments */
};

/* Field sets for lbm_read_fields / lbm_write_fields. */
typedef enum lbm_field_set {
    LBM_FIELDS_MOMENTS = 0,     /* rho-1, u, v, w, m_xx, m_xy, m_xz, m_yy, m_yz, m_zz (scaled, as stored) */
    LBM_FIELDS_S = 1,           /* S_xx, S_xy, S_xz, S_yy, S_yz, S_zz */
    LBM_FIELDS_SMEAN = 2,       /* S_xxMean ... S_zzMean */
    LBM_FIELDS_K = 3,           /* k */
    LBM_FIELDS_KMEAN = 4,       /* kMean */
    LBM_FIELDS_MOMENTSMEAN = 5  /* rhoMean ... m_zzMean */
} lbm_field_set;

/* Node order of host buffers. */
typedef enum lbm_order {
    LBM_ORDER_GLOBAL = 0, /* [field][z][y][x], x fastest */
    LBM_ORDER_TILED = 1   /* [field][reference block-tiled index]: tx + 8*(ty + 8*(tz + 8*(bx + NBX*(by + NBY*bz))))
                             (reference src/globalFunctions.cuh:208-214; the .LBMBin data order) */
} lbm_order;

/* Host value types for field transfers. */
typedef enum lbm_dtype { LBM_F32 = 0, LBM_F64 = 1 } lbm_dtype;

typedef struct lbm_config {
    int32_t lattice;          /* 19 (D3Q19) or 27 (D3Q27) */
    int32_t device;           /* CUDA device ordinal (the reference's -GPU argument, deviceList()[0]) */
    int64_t nx, ny, nz;       /* lattice size; each a multiple of 8 (reference latticeMesh.cuh:115-131) */
    float Re;                 /* Reynolds number (programControl) */
    float u_inf;              /* lid speed, U_North = {u_inf, 0, 0} (latticeMesh.cuh:183) */
    uint32_t function_objects;/* LBM_FO_* mask */
    int32_t mean_bits;        /* 32: float running means as the reference; 64: double accumulators */
    int64_t start_step;       /* absolute step index of the initial state (restart: latestTime) */
    /* kernel tiling; 0 = autotuned choice for this size class */
    int32_t tile_x, tile_y, z_chunk, stages;
    int32_t pop_buffers;      /* shared-memory population planes: 1 (two barriers per plane, 3 CTAs/SM),
                                 2 (one barrier per plane), 4 (one plane, 4 CTAs/SM; D3Q19 shapes) */
    int32_t storage;          /* LBM_STORAGE_*: how the 10 moment fields are held in device memory */
} lbm_config;

/* Moment storage formats.  Arithmetic is FP32 for all of them; the 16-bit
 * formats hold each field times a power of two (rho-1 and the second-order
 * moments x64, 3u x8 for FP16; x1 for BF16) and convert to the reference's
 * FP32 values at every host transfer. */
enum { LBM_STORAGE_F32 = 0, LBM_STORAGE_F16 = 1, LBM_STORAGE_BF16 = 2 };

typedef struct lbm_handle lbm_handle;

typedef struct lbm_info {
    int64_t step;            /* absolute step index of the next step to run */
    int64_t nodes;           /* nx*ny*nz */
    float tau, omega;        /* relaxation constants as uploaded (latticeMesh.cuh:177-201) */
    int32_t tile_x, tile_y, z_chunk, stages;
    uint64_t device_bytes;   /* device memory owned by the handle */
    double last_step_ms;     /* device time of the last lbm_step call (CUDA events) */
    uint64_t kernel_launches;/* kernels launched by this handle so far */
} lbm_info;

/* Fill *cfg with defaults (D3Q19, 64^3, Re 100, u_inf 0.05, no function objects).
 * Replaces: nothing (convenience). */
void lbm_config_default(lbm_config *cfg);

/* Allocate device state for one cavity and upload the relaxation constants.
 * Replaces host::latticeMesh (src/latticeMesh/latticeMesh.cuh:85-210), the
 * device::array allocations (momentBasedD3Q19.cu:70-79), device::halo
 * (src/blockHalo/halo.cuh:76-122) and objectRegistry allocation
 * (src/functionObjects/objectRegistry.cuh:78-87). */
lbm_status lbm_create(const lbm_config *cfg, lbm_handle **out);

/* Release everything the handle owns. */
lbm_status lbm_destroy(lbm_handle *h);

/* Initial state on the device from per-region values: region[f*7 + r] for
 * fields f in moment order and regions r = internalField, North, South, East,
 * West, Front, Back, already scaled (rho as rho-1, u*3, m_aa*4.5, m_ab*9).
 * Replaces host::array::initialConditions (src/array/hostArray.cuh:304-359)
 * and the host-side halo fill (src/blockHalo/haloFace.cuh:244-306). Function-
 * object accumulators are zeroed. */
lbm_status lbm_init_regions(lbm_handle *h, const float region[70]);

/* Upload a field set from host memory (restart from .LBMBin, hostArray.cuh:264-276).
 * `count` = number of values (nvars * nodes). */
lbm_status lbm_write_fields(lbm_handle *h, lbm_field_set set, const void *host, size_t count, lbm_dtype dtype,
                            lbm_order order);

/* Download a field set to host memory (host::toHost, src/memory/memory.cuh:157-195). */
lbm_status lbm_read_fields(lbm_handle *h, lbm_field_set set, void *host, size_t count, lbm_dtype dtype,
                           lbm_order order);

/* Advance n time steps (the momentBasedD3Q19<<<>>> launch + runTimeObjects.calculate
 * + blockHalo.swap of momentBasedD3Q19.cu:104-137, with the function objects fused
 * into the step kernel and no host synchronisation between steps).
 * Asynchronous: returns after enqueueing; errors of the launches are reported. */
lbm_status lbm_step(lbm_handle *h, uint64_t n);

/* Per-step global sums, accumulated in FP64 by the step kernel itself. */
typedef struct lbm_monitor {
    double mass;             /* sum of rho over the nodes */
    double rho_u2;           /* sum of rho*|u_stored|^2; kinetic energy = rho_u2 * 0.5 / 9 */
    uint64_t nonfinite;      /* nodes with a NaN/Inf among their 10 moments (divergence watchdog) */
} lbm_monitor;

/* lbm_step with a per-step result: step i writes its sums to out[i] (n
 * entries) by an asynchronous device-to-host copy queued after the step.
 * With page-locked `out` (lbm_host_alloc) nothing waits for the host; the
 * values are valid after lbm_synchronize.  Replaces: the reference's per-step
 * info print (momentBasedD3Q19.cu:107-110) and fieldCalculate containsNaN
 * (applications/fieldCalculate/fieldCalculate.cuh:74-110), at no extra pass. */
lbm_status lbm_step_monitored(lbm_handle *h, uint64_t n, lbm_monitor *out);

/* Kernel shape of lbm_run_streamed; 0 in a field picks its default. */
typedef struct lbm_stream_opts {
    int32_t slab;      /* planes per slab (default 16) */
    int32_t z_chunk;   /* planes per CTA inside a slab launch (default 4) */
    int32_t lead;      /* the first slab is n + lead planes high (default 2) */
} lbm_stream_opts;

/* One whole job between host buffers, with the transfers overlapped with
 * the steps: upload the 10 moment fields from `moments` (FP32, stored units,
 * [field][z][y][x]), advance n >= 1 steps, and download the results into
 * out[set] for set = LBM_FIELDS_MOMENTS ... LBM_FIELDS_MOMENTSMEAN (host
 * buffers in [field][z][y][x] order, FP32, FP64 for the running means when
 * mean_bits is 64; NULL skips a set; sets of function objects the handle
 * does not compute must be NULL).  mon[i] (NULL: none) receives step i's
 * sums as lbm_step_monitored gives them.  The function-object accumulators
 * continue from their device values, as after lbm_write_fields of the
 * moments.  The results are those of lbm_write_fields + lbm_step(n) +
 * lbm_read_fields, bit for bit (the monitor sums up to FP64 summation
 * order).
 * How: the mesh is cut into z-slabs (the first n + lead planes high, so
 * that its own last step already finishes planes, the others `slab`); slab j
 * of step s is shifted down by s planes, so that it needs only slabs j-1 and
 * j of step s-1, and all n steps of slab j run before slab j+1.  The upload
 * (a second stream, in 4-plane chunks) runs ahead of the slabs, and the
 * planes that slab j finished (n-1 planes behind its top) are downloaded (a
 * third stream) while slab j+1 runs, so the job takes about as long as the
 * larger of its two transfers instead of their sum.  A job of more than 32
 * steps runs only its first and last 16 steps this way (with the upload and
 * the download respectively) and the steps between them as whole-mesh
 * launches.
 * With 16-bit storage the moments pass through small staging blocks and the
 * storage conversion on the copy streams.  Host buffers should be
 * page-locked (lbm_host_alloc); the call returns when the results are in
 * host memory.  Not with the learned closure (LBM_ERR_STATE).  After a
 * failure the handle's moments are those of some mix of steps: write a state
 * again before stepping on.  Replaces: the reference's host-to-device copy
 * of the initial state, time loop and device-to-host copies at save steps
 * (momentBasedD3Q19.cu:70-137, src/memory/memory.cuh:157-195), which run
 * one after the other. */
lbm_status lbm_run_streamed(lbm_handle *h, const float *moments, uint64_t n, void *const out[6], lbm_monitor *mon,
                            const lbm_stream_opts *opts);

/* Wait for queued work and report device-side error flags. */
lbm_status lbm_synchronize(lbm_handle *h);

/* Global sums in double precision over all nodes: out[0] = sum(rho) (mass),
 * out[1] = sum(0.5*rho*|u|^2) with physical u = stored/3, out[2] = number of
 * non-finite values in the 10 moment fields.  Device-side reduction. */
lbm_status lbm_reduce(lbm_handle *h, double out[3]);

lbm_status lbm_get_info(lbm_handle *h, lbm_info *info);

/* Kernel variant chosen by lbm_autotune. */
typedef struct lbm_tuning {
    int32_t tile_x, tile_y;   /* x-y tile of one CTA */
    int32_t z_chunk;          /* z-planes per CTA */
    int32_t stages;           /* TMA pipeline depth (moment planes in flight) */
    int32_t pop_buffers;      /* 1: one population plane, 3 CTAs/SM; 2: two planes; 4: one plane, 4 CTAs/SM */
    double ms_per_step;       /* measured device time per step of the chosen variant */
    int32_t candidates;       /* variants timed */
    int32_t from_cache;       /* 1 if taken from the cache without timing */
    int32_t closure_fused;    /* with a learned closure: 1 if the network runs inside the step kernel */
} lbm_tuning;

/* Time every compiled kernel variant (tile shape, pipeline depth, population
 * planes) and z-chunk length on this handle's own state for `trial_steps`
 * steps each, keep the fastest, and restore the state (moments, function
 * objects and step counter) so the run continues as if nothing happened --
 * every variant computes the same bits.  Results are cached per size class
 * (lattice, mesh, function objects, mean precision) in the process, and in
 * the file named by LBM_B200_TUNE_CACHE if set.  Allocates a temporary copy
 * of the state.  Replaces: nothing in the reference, whose tiling is fixed at
 * 8^3 (src/hardwareConfig.cuh:64-95). */
lbm_status lbm_autotune(lbm_handle *h, int32_t trial_steps, lbm_tuning *out);

/* The sums of lbm_reduce over a caller-owned device array of moments
 * ([10][nodes] floats in the stored units, on the calling thread's current
 * device), for callers that must not allocate device memory: frameworks whose
 * caching allocator owns all device memory, monitors of buffers they do not
 * own, code without an lbm_handle.  It allocates nothing: its scratch (one
 * partial sum per 16384 nodes) is a fixed 1.5 MiB device array of the library,
 * present on every GPU that loads it, so at most 2^30 nodes are accepted
 * (LBM_ERR_ARG beyond).  Sums use a fixed order, so repeated calls agree bit
 * for bit.  The first call on a device (and the first after that device's
 * context has been reset) looks up the array's address; make that first call
 * before any stream capture begins.  Each call copies the three sums to host
 * memory and waits for `stream` to finish (cudaStreamSynchronize) before it
 * returns.  Calls share the array: calls that overlap on the GPU race and must
 * be serialised.  `stream` is a cudaStream_t (NULL: default stream).
 * No counterpart in the reference, which has no allocation-free entry point. */
lbm_status lbm_reduce_moments_noalloc(const float *moments, uint64_t nodes, double out[3], void *stream);

/* fieldCalculate -calculationType containsNaN / spatialMean for one saved
 * time, on the GPU `device`: `fields` is host memory holding `nfields`
 * fields of nx*ny*nz floats each, in `order` (LBM_ORDER_TILED: as stored in
 * an .LBMBin file).  Per field k: nan_count[k] = number of NaN values
 * (saturating at INT32_MAX; infinities are not NaN); mean_ref[k] = the
 * reference's spatial mean -- the float sum of the values in global node
 * order, added left to right from 0, divided by float(nodes) -- bit for bit;
 * mean[k] = the FP64 sum of the non-NaN values (fixed summation order)
 * divided by the node count.
 * Copies the fields to a temporary device buffer.  Replaces: the host loops
 * containsNaN and spatialMean of applications/fieldCalculate/
 * fieldCalculate.cuh:74-170 (with fileInput.cuh:777-820's de-interleave). */
lbm_status lbm_field_statistics(int32_t device, const float *fields, int64_t nx, int64_t ny, int64_t nz,
                                int32_t nfields, lbm_order order, int32_t *nan_count, float *mean_ref,
                                double *mean);

/* -------------------------------------------------------------- batches
 * Many independent cavities advanced together.  Every step is ONE launch of a
 * persistent kernel (as many CTAs as fit on the GPU) whose CTAs take work
 * items -- one x-y tile and z-chunk of one cavity -- from a global counter, so
 * small cavities no longer leave the GPU idle; lbm_batch_step replays a CUDA
 * graph that holds two such launches.  Each cavity computes exactly the bits
 * it computes alone.  Batches run the plain method: FP32 storage and no
 * function objects; all cavities share the lattice and the device.
 * No counterpart in the reference, which runs one cavity per process. */
typedef struct lbm_batch lbm_batch;

typedef struct lbm_batch_info {
    int32_t cavities;
    int32_t items;            /* work items per step */
    int32_t grid;             /* CTAs of the persistent launch */
    int32_t tile_x, tile_y, stages, pop_buffers;
    int32_t persistent;       /* 1: persistent grid claiming items; 0: one CTA per item */
    int64_t nodes;            /* total nodes of all cavities */
    int64_t step;             /* batch steps taken so far */
    uint64_t device_bytes;    /* device memory of the batch tables and all cavities */
    uint64_t kernel_launches; /* persistent launches so far (graph nodes included) */
    uint64_t graph_launches;  /* graph replays so far */
    double last_step_ms;      /* device time of the last lbm_batch_step call (CUDA events) */
} lbm_batch_info;

typedef struct lbm_batch_tuning {
    int32_t tile_x, tile_y, stages, pop_buffers; /* kernel shape chosen for the whole batch */
    int32_t persistent;       /* 1: as many CTAs as fit, claiming work items; 0: one CTA per item */
    int32_t size_classes;     /* distinct mesh sizes, each given its own z-chunk */
    int32_t candidates;       /* configurations timed */
    double ms_per_step;       /* measured device time per batch step of the choice */
} lbm_batch_tuning;

/* Create n cavities (cfgs[i] as for lbm_create; same lattice and device,
 * storage LBM_STORAGE_F32, no function objects) and the tables of the batched
 * kernel.  The tiling fields of the configurations are ignored (see
 * lbm_batch_autotune). */
lbm_status lbm_batch_create(const lbm_config *cfgs, int32_t n, lbm_batch **out);

/* Release the batch and all its cavities. */
lbm_status lbm_batch_destroy(lbm_batch *b);

/* Borrowed handle of cavity i (creation order), valid until lbm_batch_destroy.
 * Every lbm_* call on a handle works on it -- lbm_init_regions, field
 * transfers, lbm_reduce, even lbm_step of that cavity alone -- except
 * lbm_destroy (LBM_ERR_STATE).  The cavities share the batch's stream. */
lbm_status lbm_batch_cavity(lbm_batch *b, int32_t i, lbm_handle **out);

/* Advance every cavity n steps.  Asynchronous, like lbm_step. */
lbm_status lbm_batch_step(lbm_batch *b, uint64_t n);

/* Wait for queued work and report device-side error flags. */
lbm_status lbm_batch_synchronize(lbm_batch *b);

/* Choose the batch's kernel shape (tile, pipeline depth, population planes)
 * by timing each on the whole batch, then each size class's z-chunk, for
 * `trial_steps` steps per candidate; the cavities' states and step counters
 * are restored afterwards.  Allocates a temporary copy of the states. */
lbm_status lbm_batch_autotune(lbm_batch *b, int32_t trial_steps, lbm_batch_tuning *out);

lbm_status lbm_batch_get_info(lbm_batch *b, lbm_batch_info *info);

/* Set the kernel shape by hand: tile_x, tile_y, stages, pop_buffers and
 * persistent of *shape (the other fields are ignored).  LBM_ERR_ARG if no
 * compiled kernel has that shape. */
lbm_status lbm_batch_configure(lbm_batch *b, const lbm_batch_tuning *shape);

/* ------------------------------------------------------ learned closure
 * A per-node network predicts a correction dtau to the relaxation time of
 * an under-resolved run; no counterpart in the reference.  Network: 16
 * features -> 32 -> 32 -> 1 with GELU (tanh form).  Features of a node from its
 * stored moments m (rho-1, 3u, 3v, 3w, 4.5 m_aa, 9 m_ab): the 10 moments and
 * 3 (u_a u_b - m_ab) / (2 scale tau0) for ab = xx, xy, xz, yy, yz, zz, each
 * standardised as (f - in_mean) * in_scale.  dtau = clamp(out_scale * y,
 * dtau_lo, dtau_hi); nodes with any feature outside [in_lo, in_hi] (the range
 * seen in training) and boundary nodes keep the plain collision. */
typedef struct lbm_mlp {
    float w1[32 * 16], b1[32];      /* layer 1, [out][in] */
    float w2[32 * 32], b2[32];      /* layer 2, [out][in] */
    float w3[32], b3;               /* output */
    float in_mean[16], in_scale[16];
    float in_lo[16], in_hi[16];
    float out_scale, dtau_lo, dtau_hi;
} lbm_mlp;

typedef struct lbm_trainer lbm_trainer;

typedef struct lbm_train_options {
    int32_t steps;                  /* Adam steps */
    int32_t batch;                  /* samples per step, drawn at random */
    float lr;                       /* Adam learning rate */
    float dtau_lo, dtau_hi;         /* targets are clipped to this range (also the inference clip) */
    uint64_t seed;                  /* initial weights and batches */
} lbm_train_options;

typedef struct lbm_train_report {
    uint64_t samples, steps;
    double loss_first, loss_last;   /* mean squared error on standardised targets, first and last tenth */
    double target_rms;              /* out_scale */
} lbm_train_report;

/* Add U(-amplitude, amplitude) to the velocity (lattice units) of every
 * interior node of the current state, from a counter-based hash of `seed`. */
lbm_status lbm_perturb_velocity(lbm_handle *h, float amplitude, uint64_t seed);

/* coarse state := 2:1 box filter of the fine state (fine = 2 x coarse in
 * every direction; mean over the 8 fine nodes of every coarse node).  rho-1
 * and the velocity are averaged; each second-order moment is the mean of its
 * equilibrium part u_a u_b (so the subgrid stress mean(u_a u_b) - mean(u_a)
 * mean(u_b) is kept) plus kappa times the mean of its non-equilibrium part,
 * kappa = 2 (tau_c/tau_f) (1-omega_c)/(1-omega_f): the coarse lattice's
 * non-equilibrium stress for the same flow (twice the strain rate per step
 * at equal lattice velocity, its own tau and collision factor). */
lbm_status lbm_filter_2to1(lbm_handle *fine, lbm_handle *coarse);

/* Sample store for training, capacity in samples (16 features + 1 target). */
lbm_status lbm_trainer_create(int32_t device, uint64_t capacity, lbm_trainer **out);
lbm_status lbm_trainer_destroy(lbm_trainer *t);

/* Training pairs from one coarse step: `coarse` holds F(t) (a filtered fine
 * state) and is advanced one plain step by this call; `fine_next` is the
 * fine run two fine steps later.  For every `stride`-th interior node whose
 * post-step non-equilibrium second-order moments have an RMS (stored units)
 * above `min_neq`: the features of F(t) and the dtau for which its collision
 * gives the filtered fine state instead, to first order in dtau (the
 * estimate is a ratio with that RMS in the denominator, hence the floor).
 * *total = samples stored so far. */
lbm_status lbm_trainer_add(lbm_trainer *t, lbm_handle *coarse, lbm_handle *fine_next, uint32_t stride,
                           float min_neq, uint64_t *total);

/* Samples whose target fits one dtau per node to a window of `window`
 * consecutive coarse steps: the coarse handle holds the filtered state F(t)
 * of the fine run (whose current time is 2t); the call advances the fine run
 * by 2 x window steps and, for each j, one plain coarse step from F(t+j),
 * comparing it with F(t+j+1); per node it sums the least-squares terms of
 * every transition (residual . non-equilibrium stress, non-equilibrium
 * stress squared) and stores one sample: the features of F(t) and the dtau
 * of the summed terms.  window = 1 gives the samples of lbm_trainer_add.
 * The coarse handle is left at the last transition's coarse step.
 * Replaces: nothing in the reference (no closure). */
lbm_status lbm_trainer_add_window(lbm_trainer *t, lbm_handle *coarse, lbm_handle *fine, uint32_t window,
                                  uint32_t stride, float min_neq, uint64_t *total);

/* Copy stored samples [first, first+count) to the host (features [n][16],
 * targets [n]; either may be NULL); *total = samples stored. */
lbm_status lbm_trainer_samples(lbm_trainer *t, uint64_t first, uint64_t count, float *features, float *targets,
                               uint64_t *total);

/* Train a network on the stored samples with the GPU's forward/backward
 * kernels and Adam; fills *net (weights, normalisation, ranges, clip). */
lbm_status lbm_trainer_fit(lbm_trainer *t, const lbm_train_options *opt, lbm_mlp *net, lbm_train_report *rep);

/* Gradient of the mean squared error over samples [first, first+count) for
 * *net, from the training kernels (weights and biases of *grad filled, the
 * rest zero); *loss = the error. */
lbm_status lbm_trainer_gradient(lbm_trainer *t, const lbm_mlp *net, uint64_t first, uint64_t count, lbm_mlp *grad,
                                double *loss);

/* Raw network output y for host features [n][16]: tensor cores (FP16
 * weights and activations, FP32 accumulation) or FP32 CUDA cores. */
lbm_status lbm_mlp_infer(int32_t device, const lbm_mlp *net, const float *features, uint64_t n, float *y,
                         int32_t tensor_cores);

/* Use the network in every following lbm_step of this handle (NULL: back to
 * the plain collision).  FP32 storage, no function objects; LBM_ERR_ARG
 * unless dtau_lo <= dtau_hi and tau + dtau_lo > 0.5 (a positive viscosity
 * at every node). */
lbm_status lbm_closure_set(lbm_handle *h, const lbm_mlp *net);

/* Recompute dtau every `every` steps (default 1: every step) and reuse it in
 * between -- a lagged closure for runs where it varies slowly. */
lbm_status lbm_closure_refresh(lbm_handle *h, int32_t every);

/* The dtau field of the last closure step ([z][y][x], count = nodes).  After
 * the state has been replaced since that step (lbm_write_fields of the
 * moments, lbm_init_regions, lbm_autotune), or before any closure step, it
 * is the field the next step will use. */
lbm_status lbm_closure_dtau(lbm_handle *h, float *host, size_t count);

/* Where the network runs when it is evaluated every step: on (the default)
 * inside the step kernel -- one launch per step, no per-node dtau array in
 * HBM -- or off: a separate inference kernel writes dtau and the step kernel
 * reads it.  Both give the same bits.  Kernel shapes without a fused variant
 * (8-wide tiles) and lbm_closure_refresh intervals above 1 use the separate
 * kernels.  Replaces: nothing in the reference (no closure); the collision it
 * modifies is src/collision/secondOrder.cuh:93-105. */
lbm_status lbm_closure_fused(lbm_handle *h, int32_t on);

/* Self-test of the device-side failure path: a kernel waits with the step
 * kernels' bounded wait on an mbarrier that nothing arrives on; after
 * timeout_ns the wait gives up, records where, and the call returns
 * LBM_ERR_TIMEOUT with that record in lbm_last_error() -- the CUDA context
 * stays usable.  Replaces: nothing (the reference's waits are unbounded). */
lbm_status lbm_selftest_wait_timeout(int32_t device, uint64_t timeout_ns);

/* Page-locked host memory for fast transfers (cudaMallocHost); free with
 * lbm_host_free.  Replaces: the reference's pinned host::array variant
 * (src/array/hostArray.cuh:66-140). */
lbm_status lbm_host_alloc(size_t bytes, void **out);
lbm_status lbm_host_free(void *p);

/* ------------------------------------------------------------------ case IO */

/* A case directory as the reference solvers read it. */
typedef struct lbm_case {
    char case_name[256];
    float Re, u_inf;                 /* programControl */
    uint64_t n_time_steps, save_interval, info_interval;
    uint64_t nx, ny, nz;             /* latticeMesh */
    float Lx, Ly, Lz;
    uint32_t function_objects;       /* functionObjects -> LBM_FO_* mask */
    float region[70];                /* initialConditions, scaled as for lbm_init_regions */
    uint64_t latest_time;            /* largest t of <case_name>_<t>.LBMBin in the directory */
    int32_t has_restart;             /* 1 if such a file exists */
} lbm_case;

/* Parse the case files in `dir`.  Replaces programControl
 * (src/programControl/programControl.cuh:69-124), host::latticeMesh parsing
 * (src/latticeMesh/latticeMesh.cuh:85-131), boundaryValue/boundaryFields
 * (src/boundaryConditions/boundaryValue.cuh:147-254), initialiserSwitch
 * (src/functionObjects/functionObjects.cuh:104-107) and fileIO::latestTime
 * (src/fileIO/fileIO.cuh:222-233).  The initial conditions are read only if
 * there is no restart file, as in the reference. */
lbm_status lbm_case_read(const char *dir, lbm_case *out);

/* Write an .LBMBin file (fileIO::writeFile, src/fileIO/fileOutput.cuh:82-183):
 * `values` holds nvars*nx*ny*nz floats in [field][block-tiled node] order. */
lbm_status lbm_lbmbin_write(const char *path, uint64_t nx, uint64_t ny, uint64_t nz, int32_t nvars,
                            const char *const *names, const float *values, uint64_t time_step,
                            int32_t time_average);

/* Cut plane of a field set from the live state (fieldConvert -cutPlane,
 * applications/fieldConvert/fieldConvert.cuh:236-326, evaluated on the
 * device).  The plane is normal to `axis` (0 x, 1 y, 2 z) at `position` in
 * [0, 1] between the first and the last node plane, linearly interpolated
 * between the two bracketing node planes with weight index - floor(index)
 * (the reference uses position - floor(index), which is right only on a
 * node plane).  host_out receives count = nvars * (plane nodes) floats laid
 * out [var][b][a] with (a, b) = (y, z), (x, z) or (x, y) for axis 0, 1, 2. */
lbm_status lbm_cut_plane(lbm_handle *h, lbm_field_set set, int32_t axis, float position, float *host_out,
                         size_t count);

/* Write a VTK XML structured-grid file (fieldConvert -fileType vts,
 * src/postProcess/VTS.cuh:68-212): `values` holds nvars*nx*ny*nz floats in
 * [field][z][y][x] order; L = domain lengths (latticeMesh Lx, Ly, Lz). */
lbm_status lbm_vts_write(const char *path, uint64_t nx, uint64_t ny, uint64_t nz, const float L[3], int32_t nvars,
                         const char *const *names, const float *values);

/* Message of the last failure on this thread (empty if none). */
const char *lbm_last_error(void);

/* Human-readable name of a status code. */
const char *lbm_status_string(lbm_status s);

/* Number of nodes a field set holds per node (1, 6 or 10). */
int lbm_field_set_vars(lbm_field_set set);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
