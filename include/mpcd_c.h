/*
 * mpcd_c.h — C-ABI of the B200 SRC/MPCD time step (libmpcd_b200.so).
 *
 * Plain C: POD structs, pointers and sizes, integer status codes. No exceptions, STL or
 * torch types cross this boundary. Every entry point returns MPCD_OK (0) on success or a
 * status code; mpcd_last_error() returns the message of the calling thread's last failure.
 *
 * Conventions (identical to the reference's C++ API and file formats):
 *   - particle arrays are interleaved [x1, y1, x2, y2, ...] doubles of length 2n, in
 *     particle-id order (reference include/types.h:74-79);
 *   - cell index c = iy + Ny*ix (reference src/common_grid.cpp:18);
 *   - all RNG seeds are the reference's std::mt19937_64 seeds.
 *
 * Each function below names the reference interface it replaces (file:line, relative to
 * the reference project root).
 */
#ifndef MPCD_C_H
#define MPCD_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum mpcd_status {
    MPCD_OK = 0,
    MPCD_ERR_INVALID_ARG = 1,   /* bad size, mode or flag (reference: std::runtime_error) */
    MPCD_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    MPCD_ERR_UNSUPPORTED_BC = 3,/* a particle crossed a wall whose mode is not supported */
    MPCD_ERR_DEVICE = 4,        /* a kernel raised its device-side error flag */
    MPCD_ERR_NO_DEVICE = 5,     /* no CUDA device / extension not usable */
    MPCD_ERR_CAPACITY = 6,      /* a bounded device buffer would overflow */
    MPCD_ERR_STATE = 7          /* call order: e.g. closure without a saved reference */
};

/* ---------------------------------------------------------------- enumerations */
/* boundary modes (reference include/types.h:30-33 hold them as strings) */
enum mpcd_bc_mode {
    MPCD_BC_UNKNOWN = -1,       /* any other string: error only if a particle crosses */
    MPCD_BC_PERIODIC = 0,
    MPCD_BC_THERMALIZE = 1,
    MPCD_BC_BOUNCEBACK = 2,
    MPCD_BC_SPECULAR = 3
};
/* highMode / lowMode (reference src/zone_pass.cpp:351,357): "1+coef" or anything else */
enum mpcd_thr_mode { MPCD_THR_COEF = 0, MPCD_THR_ONE_PLUS_COEF = 1 };
/* zone layout modes (reference src/zone_pass.cpp:178,193) */
enum mpcd_layout_mode { MPCD_LAYOUT_BASE = 0, MPCD_LAYOUT_SHIFTED = 1, MPCD_LAYOUT_SINGLE_FULL = 2 };
/* numeric forms of the step */
enum mpcd_form { MPCD_FORM_PLAIN_F64 = 0 };

/* ---------------------------------------------------------------- parameters */
/* POD mirror of mpcd::Params (reference include/types.h:10-72); booleans are int32 0/1,
 * strings are the enums above. Field order follows the reference struct. */
typedef struct mpcd_params_c {
    int32_t Nx, Ny, Nc, n;
    double Lx, Ly, dt, a0;
    double alpha, kBT, g, bodyForceX;
    int32_t useThermostat, keepMeanFlow;
    int32_t boundary_left, boundary_right, boundary_bottom, boundary_top;
    double Utop, Ubottom, wallSigma;
    int32_t noSurfaceCase, redistributionEnableSurfaceTopology, redistributionWallWettingEnabled;
    int32_t useInterfaceVelocityReorientation, useIncompressibleRedistribution;
    int32_t redistribAfterCollision, useZoneRedistribution;
    int32_t zoneTileNx, zoneTileNy;
    int32_t zoneUseShiftedSecondPass, zonePassthroughMode, zoneSingleFullDomainMode;
    int32_t enableMomentumCorrectionPostRedistribution;
    double gamma, coef;
    int32_t highMode, lowMode;
    int32_t maxRedistribPasses, useLocalFluidFractionThresholds;
    double fluidFracGain, lowThrFloor, highThrFloor, lowThrBulkOverride;
    int32_t useLiquidClosure, useOptimalBetaRepair;
    double betaRepair, betaEOS, Kvirial;
    int32_t smoothPdriveAtInterzone, smoothPdriveInterzoneWidthCells;
    double smoothPdriveInterzoneBlend;
    int32_t smoothPdriveIncludeShiftedLayouts, reserved0;
} mpcd_params_c;

/* ---------------------------------------------------------------- results */
/* mpcd::WallInfo (reference include/types.h:97-111) */
typedef struct mpcd_wallinfo_c {
    int32_t nBot, nTop, nLeft, nRight;
    double dEwall, dPxBot, dPxTop, dPyBot, dPyTop, dPxLeft, dPxRight, dPyLeft, dPyRight;
} mpcd_wallinfo_c;

/* mpcd::OpenMPPassMetrics (reference include/zone_pass_openmp.h:12-27). Times are device
 * seconds; nThreadsUsed reports the number of zone blocks launched. */
typedef struct mpcd_pass_metrics_c {
    int32_t nZones, nThreadsRequested, nThreadsUsed, nParticlesMovedDense, nParticlesMovedSparse;
    int32_t reserved0;
    double corrRmsDU, corrMaxDU;
    double timeLayout, timeZoneExtract, timeSnapshot, timeAlloc, timeKernel, timePack, timeMerge;
} mpcd_pass_metrics_c;

/* mpcd::LiquidClosureMetrics (reference include/liquid_closure.h:11-27) */
typedef struct mpcd_closure_metrics_c {
    double betaRepairOpt, betaRepairApplied, betaRepairNum, betaRepairDen, betaEOSApplied;
    double meanPdriveRaw, meanPdrive, rmsRepairDU, meanAbsRepairDU, maxRepairDU;
    double rmsEOSDU, maxEOSDU, momentumDeltaX, momentumDeltaY;
    int32_t nMaskedInterzoneCells, reserved0;
} mpcd_closure_metrics_c;

/* mpcd::CellFields (reference include/types.h:81-95) as caller-owned host arrays of Nc
 * entries each; any pointer may be NULL to skip that field. */
typedef struct mpcd_cellfields_c {
    int32_t* N;
    double *Ux, *Uy, *Px, *Py, *T, *rho, *Pkin, *Pvir, *P, *rhoTarget;
} mpcd_cellfields_c;

/* Everything run_liquid_closure returns besides stateOut (reference
 * include/liquid_closure.h:29-44); caller-owned host arrays, each pointer nullable.
 * State arrays hold 2n doubles, grids Nc entries. */
typedef struct mpcd_closure_detail_c {
    double *repairedX, *repairedV;
    mpcd_cellfields_c refFields, redFields, repairedFields, outFields;
    double *pdriveRaw, *pdrive, *duRepairX, *duRepairY, *duEOSX, *duEOSY;
    int32_t* interzoneMask;
} mpcd_closure_detail_c;

/* One row of the profiled benchmark's per-step metrics (reference
 * src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:215,301-336). */
typedef struct mpcd_step_metrics_c {
    int64_t step;
    mpcd_wallinfo_c wall;
    mpcd_pass_metrics_c base, shifted;
    mpcd_closure_metrics_c closure;
    double occStd, outBand, meanKinetic, meanUx, meanUy, Qx;
    double baseOccStd, baseOutBand, shiftedOccStd, shiftedOutBand;
    double meanVelocityX, meanVelocityY;
    double timeStepTotal, timeRefBuild, timeBase, timeShifted, timeClosure, timeDiagnostics;
} mpcd_step_metrics_c;

typedef struct mpcd_ctx mpcd_ctx;

/* ---------------------------------------------------------------- library */
const char* mpcd_last_error(void);
/* 1 if a usable sm_100 device is present, else 0 (sets no error) */
int mpcd_device_available(void);
/* Parses a params.kv file (reference src/params_io.cpp:74-137; strict: every key required,
 * unknown keys ignored). Other keys are read with mpcd_read_kv_string. */
int mpcd_read_params_kv(const char* path, mpcd_params_c* out);
/* Any key of a params.kv file as a string (the reference driver reads benchmark_nSteps,
 * benchmark_metricsEvery and benchmark_dumpSteps this way:
 * src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:205-208). */
int mpcd_read_kv_string(const char* path, const char* key, char* buf, int buflen);
/* message of the last failed mpcd_read_params_kv / mpcd_read_kv_string on this thread */
const char* mpcd_io_last_error(void);

/* ---------------------------------------------------------------- context */
/* Allocates device buffers for params->n particles and params->Nc cells on `device`.
 * Validates params (reference src/zone_pass.cpp:1100-1105, src/liquid_closure.cpp:332). */
int mpcd_ctx_create(const mpcd_params_c* params, int device, mpcd_ctx** out);
/* State forms of a context. MPCD_FORM_F64, the plain form: FP64 positions and velocities,
 * results bit-exact or within 1e-12 of the reference. MPCD_FORM_F32, the precision form: per
 * particle the standard-grid cell (int32), the position inside that cell as FP32 offsets and
 * FP32 velocities (20 bytes of state instead of 32); arithmetic in FP64 registers, results
 * rounded to FP32 on every store. An FP32 context runs the whole step (mpcd_step,
 * mpcd_step_timed, mpcd_step_profile, mpcd_step_metrics, the learned closure) and state I/O in
 * FP64 particle-id order; the phase functions return MPCD_ERR_INVALID_ARG. */
enum mpcd_state_form { MPCD_FORM_F64 = 0, MPCD_FORM_F32 = 1, MPCD_FORM_FAST = 2 };
/* MPCD_FORM_FAST, the fast form (no counterpart in the reference, which has one form): the
 * FP32 precision form with the redistribution decided in parallel. Same phases and rules as
 * the plain form (stream, walls, shifted-grid SRD rotation with thermostat, base and shifted
 * zone passes, liquid closure), but every random draw comes from a hash of (step, what the
 * draw is for), so zones, cells and particles proceed independently; results are therefore
 * not the reference's trajectories but the same physics, compared statistically with the
 * plain form. State: per cell a bin of FP32 offsets inside the cell, FP32 velocities on the
 * 2^-20 grid and particle ids; cell sums are exact int64 sums, so the collision keeps every
 * SRD cell's momentum and each redistribution keeps the momentum of every cell it corrects,
 * to the last grid unit. Results do not depend on the order of particles in memory: the same
 * input gives the same output in particle-id order. Runs the whole step, state I/O and
 * metrics rows; rejects local fluid-fraction thresholds, keepMeanFlow, the single full-domain
 * zone, zone tiles above 128 cells and cells that are not squares of side a0. A cell that
 * grows beyond its bin (about 2 gamma + 8 sqrt(gamma) particles) fails the step with
 * MPCD_ERR_CAPACITY. */
int mpcd_ctx_create_form(const mpcd_params_c* params, int device, int32_t form, mpcd_ctx** out);
int mpcd_ctx_destroy(mpcd_ctx* ctx);
/* The stream every kernel of this context runs on (a cudaStream_t). */
void* mpcd_ctx_stream(mpcd_ctx* ctx);

/* Host <-> device state, particle-id order. x and v: 2n doubles each (mpcd::State.x/.v). */
int mpcd_set_state(mpcd_ctx* ctx, const double* x, const double* v, int64_t n);
int mpcd_get_state(mpcd_ctx* ctx, double* x, double* v);
/* Device-pointer variants (the same layout, already on the context's device). */
int mpcd_set_state_device(mpcd_ctx* ctx, const double* d_x, const double* d_v, int64_t n);
int mpcd_get_state_device(mpcd_ctx* ctx, double* d_x, double* d_v);

/* ---------------------------------------------------------------- phases */
/* v += (bodyForceX, g) dt; x += dt v
 * (reference src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:242-247) */
int mpcd_stream(mpcd_ctx* ctx);
/* mpcd::apply_bc_general (reference src/boundary_conditions.cpp:19-203); info nullable */
int mpcd_apply_bc(mpcd_ctx* ctx, uint64_t seed, mpcd_wallinfo_c* info);
/* mpcd::srd_cell_id_with_random_shift (reference src/srd_collision.cpp:9-45). Keeps the
 * cell ids on the device for mpcd_srd_collide; copies them to cid_out (n int32) if given. */
int mpcd_srd_shift_cells(mpcd_ctx* ctx, uint64_t seed, int32_t* cid_out);
/* mpcd::srd_collision_step (reference src/srd_collision.cpp:47-140) on the cell ids of the
 * last mpcd_srd_shift_cells call. */
int mpcd_srd_collide(mpcd_ctx* ctx, uint64_t seed);
/* the same with caller-given cell ids (n int32 in [0, Nc), host memory) */
int mpcd_srd_collide_cells(mpcd_ctx* ctx, const int32_t* cid, uint64_t seed);
/* mpcd::compute_cell_fields (reference src/common_grid.cpp:32-100) of the current state */
int mpcd_cell_fields(mpcd_ctx* ctx, double rho_target, mpcd_cellfields_c* out);
/* No counterpart in the reference: mpcd_cell_fields on a caller-owned device state, for
 * callers that must not allocate device memory (a host code that drives its own time loop
 * from a memory pool reserved up front; cudaFree would also synchronise its other streams).
 * No context is needed and nothing is allocated: the working memory is one static device
 * array of 4 * MPCD_STATIC_FIELDS_MAX_CELLS doubles (32 MiB) per device.
 *   params   grid and cell constants (Nx, Ny, Nc, Lx, Ly, Kvirial, ...); params->n is not used
 *   d_x, d_v 2n doubles each, particle-id order, on the current device
 *   d_out    DEVICE arrays of Nc entries on the current device, any pointer NULL to skip
 *   stream   a cudaStream_t (NULL: the legacy default stream); the call only enqueues work
 * Returns MPCD_ERR_CAPACITY if Nc > MPCD_STATIC_FIELDS_MAX_CELLS. The first call on a device
 * looks up the array's device address (and may load the module there): make that first call
 * before any stream capture. The address is kept for the life of the process, so a device
 * reset (cudaDeviceReset, or a reset of the primary context) after the first call is not
 * supported: the module may then be loaded at another address. Every call on a device shares
 * the array and zeroes it first; calls that overlap on the GPU race. Sums are accumulated
 * with atomics, so the fields may differ from mpcd_cell_fields in the last bits (counts are
 * exact). */
#define MPCD_STATIC_FIELDS_MAX_CELLS 1048576
int mpcd_cell_fields_static(const mpcd_params_c* params, const double* d_x, const double* d_v, int64_t n,
                            double rho_target, const mpcd_cellfields_c* d_out, void* stream);
/* Snapshot the current state as the closure's reference state ("stateRef"): its cell fields,
 * pressure drive and EOS kick. The snapshot stays until the next mpcd_save_ref (setting a new
 * state does not clear it), so stateRef and stateRed may come from separate uploads. */
int mpcd_save_ref(mpcd_ctx* ctx);
/* mpcd::run_zone_pass_openmp (reference src/zone_pass_openmp.cpp:176-182, snapshot
 * semantics of :34-172). mode: mpcd_layout_mode. metrics nullable. */
int mpcd_zone_pass(mpcd_ctx* ctx, int32_t mode, uint64_t seed_base, mpcd_pass_metrics_c* metrics);
/* mpcd::run_zone_pass (reference src/zone_pass.cpp:1096-1163): the zones one after another
 * in id order, each on the state the previous ones left, in place. One warp runs them in
 * sequence (the order is the semantics), so this is the slow pass; the validators and the
 * non-OpenMP benchmark driver of the reference use it. metrics nullable (timeKernel: device
 * seconds; nThreadsUsed: 1). */
int mpcd_zone_pass_serial(mpcd_ctx* ctx, int32_t mode, uint64_t seed_base, mpcd_pass_metrics_c* metrics);
/* mpcd::run_liquid_closure (reference src/liquid_closure.cpp:329-444) with stateRef = the
 * saved reference and stateRed = the current state; the current state becomes stateOut.
 * metrics and detail nullable. */
int mpcd_liquid_closure(mpcd_ctx* ctx, mpcd_closure_metrics_c* metrics, mpcd_closure_detail_c* detail);
/* Zone ownership map of a layout (reference src/zone_pass.cpp:1049-1063), Nc int32. */
int mpcd_zone_owner_map(mpcd_ctx* ctx, int32_t mode, int32_t* owner_out);

/* mpcd::ZoneKernelStats (reference include/zone_pass.h:24-29) */
typedef struct mpcd_zone_kernel_stats_c {
    double stats[6];  /* dense cells handled (all passes), sparse cells, moved out, moved in, corrRmsDU, corrMaxDU */
    double diag[10];  /* occStd, outBand, |dP global|, rms dPx, rms dPy, dE, NaN, 0, rms uxNow, rms uyNow */
    int32_t movedDense, movedSparse;
} mpcd_zone_kernel_stats_c;
/* mpcd::build_zone_layout (reference src/zone_pass.cpp:1049-1063 over build_layout :173-221,
 * include/zone_pass.h:58): the zones of a layout as cell rectangles. Zone id k + 1 covers
 * the cells with ix in [rects[4k], rects[4k+1]) and iy in [rects[4k+2], rects[4k+3]); zones
 * are numbered y-outer, x-inner. Host only (no device, no context). Writes *nzones; rects
 * may be NULL to query the count, else it holds 4 * cap int32. */
int mpcd_zone_layout(const mpcd_params_c* params, int32_t mode, int32_t* nzones, int32_t* rects, int32_t cap);
/* mpcd::run_zone_kernel_inplace (reference src/zone_pass.cpp:1065-1081 over run_zone_kernel
 * :669-973, include/zone_pass.h:60-64): the redistribution of one zone, the cell rectangle
 * [x0, x1) x [y0, y1), in place on the current state, with the draws of mt19937_64(seed).
 * Every cell is active (the reference's build_active_mask_vec). stats nullable. */
int mpcd_zone_kernel_inplace(mpcd_ctx* ctx, int32_t x0, int32_t x1, int32_t y0, int32_t y1, uint64_t seed,
                             mpcd_zone_kernel_stats_c* stats);
/* mpcd::build_particle_ids_in_zone (reference src/zone_pass.cpp:1083-1094,
 * include/zone_pass.h:66-68): the ids, ascending, of the particles of the current state whose
 * standard-grid cell lies in [x0, x1) x [y0, y1). *count receives their number; ids_out
 * (host, n int32) may be NULL to count only. */
int mpcd_particle_ids_in_rect(mpcd_ctx* ctx, int32_t x0, int32_t x1, int32_t y0, int32_t y1, int32_t* ids_out,
                              int64_t* count);

/* ---------------------------------------------------------------- the step */
/* Runs steps step0+1 .. step0+nsteps of the profiled benchmark loop on the device
 * (reference src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:237-279),
 * with its per-step seed schedule. If `last` is given, fills the metrics row of the last
 * step (costs extra device reductions and one synchronisation). */
int mpcd_step(mpcd_ctx* ctx, int64_t step0, int64_t nsteps, mpcd_step_metrics_c* last);
/* Independent jobs through one context, with host buffers: job j (0 <= j < njobs) loads the
 * state (x_in[j], v_in[j]), runs steps step0 + j*nsteps + 1 .. step0 + (j+1)*nsteps and stores
 * the resulting state in (x_out[j], v_out[j]), with the results of mpcd_set_state + mpcd_step
 * + mpcd_get_state per job. The upload of job j+1's input and the download of job j-1's result
 * run on two copy streams while job j steps (asynchronously when the host buffers are
 * page-locked). x_out[j] / v_out[j] may be x_in[j] / v_in[j]; no other output may alias an
 * input. Layouts as mpcd_set_state. The device status is checked after the last job: an error
 * of any job is returned then, and the outputs of that job and the jobs after it are
 * unspecified. No counterpart in the reference: its state lives in host memory. */
int mpcd_run_jobs(mpcd_ctx* ctx, int64_t njobs, const double* const* x_in, const double* const* v_in,
                  int64_t step0, int64_t nsteps, double* const* x_out, double* const* v_out);
/* Time-averaged velocity profile across the channel (no counterpart in the reference, whose
 * MATLAB tooling averages dumped states). mpcd_profile_reset clears the accumulators and, with
 * enable != 0, makes every following step of mpcd_step / mpcd_step_timed add each row's
 * momentum along x and particle count (exact int64 sums at 2^-32). mpcd_profile_read writes,
 * per row iy (Ny doubles), the accumulated momentum divided by the accumulated count, and the
 * number of steps accumulated. */
int mpcd_profile_reset(mpcd_ctx* ctx, int32_t enable);
int mpcd_profile_read(mpcd_ctx* ctx, double* ux_rows, int64_t* nsteps);
/* Device-side metrics row of the current state after a step (see mpcd_step). */
int mpcd_step_metrics(mpcd_ctx* ctx, mpcd_step_metrics_c* out);
/* mpcd_step without metrics, timed with CUDA events recorded on the context's stream
 * around the whole loop (device seconds). */
int mpcd_step_timed(mpcd_ctx* ctx, int64_t step0, int64_t nsteps, double* device_seconds);
/* Per-phase device seconds of nsteps steps (phase list in the implementation's comment:
 * stream+BC, walls, SRD index, SRD signs, collision, cell index, reference fields, zone seeds,
 * zone passes, closure cells, kick + re-sort). */
int mpcd_step_profile(mpcd_ctx* ctx, int64_t step0, int64_t nsteps, double* phase_seconds, int nphase);
/* Step replay from CUDA graphs (default on): after the first step, plain steps without a
 * metrics row are replayed from a captured graph with device-side seeds. 0 turns it off. */
int mpcd_ctx_set_graphs(mpcd_ctx* ctx, int enable);
/* Tile shape of the SRD collision (cells x threads per block: 0 = 32x128, 1 = 64x256,
 * 2 = 128x256, 3 = 256x512, 4 = 16x128, 5 = 32x256, 6 = 16x64). A context times them all on
 * its own state at its first eager collision on cell-sorted slots and keeps the fastest (the
 * autotuner). shape >= 0 sets one instead; -1 leaves it. *in_use (nullable): the shape in use,
 * -1 before the autotuner has run. Every shape gives the same results. */
#define MPCD_COLLIDE_SHAPES 7
int mpcd_ctx_collide_shape(mpcd_ctx* ctx, int32_t shape, int32_t* in_use);

/* ---------------------------------------------------------------- batched replicas */
/* Independent replicas (reference: one run of the benchmark driver per replica), each with
 * its own parameters, size, state and zone layout, advanced together: every step is issued
 * for all replicas before the next one, each on its own streams, so their kernels overlap on
 * the GPU. Members are ordinary contexts for state I/O and metrics (mpcd_batch_member). */
typedef struct mpcd_batch mpcd_batch;
int mpcd_batch_create(const mpcd_params_c* params, int count, int device, mpcd_batch** out);
int mpcd_batch_destroy(mpcd_batch* batch);
int mpcd_batch_size(mpcd_batch* batch);
mpcd_ctx* mpcd_batch_member(mpcd_batch* batch, int index);
/* steps step0+1 .. step0+nsteps for every replica; device_seconds (nullable): CUDA-event time
 * of the whole batch */
int mpcd_batch_step(mpcd_batch* batch, int64_t step0, int64_t nsteps, double* device_seconds);
/* A batch in a state form (mpcd_state_form): MPCD_FORM_F64 is mpcd_batch_create; with
 * MPCD_FORM_FAST every phase of a step is one launch for all replicas, each replica's state
 * bit-identical to that replica stepped alone (plain closure; no learned closure or profile
 * accumulation on a batch). No counterpart in the reference, which runs one channel per
 * process. */
int mpcd_batch_create_form(const mpcd_params_c* params, int count, int device, int32_t form, mpcd_batch** out);

/* ---------------------------------------------------------------- learned closure */
/* A stencil MLP standing in for the liquid closure's per-cell velocity correction
 * (reference src/liquid_closure.cpp:380-389 repair kick and :424-436 EOS kick, which the
 * reference exposes as LiquidClosureResult::duRepairX/Y, duEOSX/Y and
 * metrics.betaRepairApplied, include/liquid_closure.h:29-44). It has no counterpart in the
 * reference.
 *   features: 75 floats per cell, a 5x5 stencil (dy outer, dx inner, -2..2) of
 *             N/gamma - 1 [0..24], Ux [25..49], Uy [50..74] of the red (post-redistribution)
 *             cell fields; wrapped on periodic axes; outside a wall N term -1, U terms 0
 *   target:   2 floats, beta_applied * duRepair + duEOS of the plain closure
 *   network:  75 -> 64 -> 64 -> 2, GELU (tanh form), BF16 weights, BF16 operands of the
 *             two 64-wide layers (tcgen05 tensor cores), FP32 accumulation and output layer,
 *             kick = output * scale
 *   params:   MPCD_LEARNED_PARAMS floats: W1[64][75], b1[64], W2[64][64], b2[64], W3[2][64],
 *             b3[2], scale */
#define MPCD_LEARNED_FEATURES 75
#define MPCD_LEARNED_OUTPUTS 2
#define MPCD_LEARNED_PARAMS 9155
int mpcd_learned_param_count(void);
/* Glorot-uniform weights from seed, zero biases, scale 0 (the trainer sets it). */
int mpcd_learned_init(uint64_t seed, float* params);
/* Runs plain steps step0+1 .. step0+nsteps like mpcd_step and collects (features, target) of
 * every stride-th cell after each step's closure (offset step % stride), at most capacity
 * rows; *count = rows written. */
int mpcd_learned_samples(mpcd_ctx* ctx, int64_t step0, int64_t nsteps, int32_t stride, float* features,
                         float* targets, int64_t capacity, int64_t* count);
/* Adam training on device `device` (mini-batches of `batch` rows, shuffled per epoch from
 * seed) of the mean squared error of output - target / scale; params in/out. If params' scale
 * is not positive it is first set to the RMS of the targets. epoch_loss (nullable): the mean
 * loss of each epoch. */
int mpcd_learned_train(const float* features, const float* targets, int64_t rows, float* params, int32_t epochs,
                       int32_t batch, float lr, uint64_t seed, int device, float* epoch_loss);
/* Gradient (MPCD_LEARNED_PARAMS floats; the scale's entry 0) and loss of that error over all
 * rows, as one batch. */
int mpcd_learned_grad(const float* features, const float* targets, int64_t rows, const float* params, int device,
                      float* grad, float* loss);
/* The network's kick (output * scale) for feature rows: out has 2 floats per row. */
int mpcd_learned_predict(const float* features, int64_t rows, const float* params, int device, float* out);
/* Puts the network in the step's closure (params NULL: back to the plain closure). Each step
 * then runs the learned kick, or the plain closure when the previous step's occupancy spread
 * (occStd of the red state, as in the metrics row) exceeded occ_limit (occ_limit <= 0: never).
 * The decision is made on the device, so graph replay keeps it. */
int mpcd_learned_set(mpcd_ctx* ctx, const float* params, double occ_limit);
/* bulk_only (default 1): cells whose 5x5 stencil crosses a wall get no learned kick (the
 * network's inputs there are partly wall padding); 0: every cell gets the network's kick. */
int mpcd_learned_options(mpcd_ctx* ctx, int32_t bulk_only);
/* Steps run with each closure since mpcd_learned_set, and the mode of the next step
 * (1 learned, 0 plain). */
int mpcd_learned_stats(mpcd_ctx* ctx, int64_t* plain_steps, int64_t* learned_steps, int32_t* next_mode);

/* Page-locked host memory (for staging states); NULL on failure. */
void* mpcd_host_alloc(size_t bytes);
void mpcd_host_free(void* p);
/* Number of kernels this context has launched so far. */
int64_t mpcd_launch_count(mpcd_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* MPCD_C_H */
