// libmpcd_b200.so: the C-ABI of include/mpcd_c.h over the sm_100a kernels.
//
// The state lives on the device in "slots": x and v as double2, plus the particle id of each
// slot. Slots are re-sorted by (cell, particle id) at the end of every step (inside the
// closure kick), so per-cell work reads contiguous memory; every API that exchanges particle
// arrays with the host uses particle-id order, as the reference does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <utility>
#include <vector>

#include "mpcd_c.h"

#include "bc.cuh"
#include "cells.cuh"
#include "closure.cuh"
#include "common.cuh"
#include "fast.cuh"
#include "fast_batch.cuh"
#include "learned.cuh"
#include "sort.cuh"
#include "zone.cuh"

using namespace mpcd_dev;

namespace {

thread_local std::string g_err;

int set_err(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess) return set_err(MPCD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kThreads = 256;
inline int blocks_for(int64_t n, int t = kThreads) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

struct CellIndex {
    int* count = nullptr;      // Nc
    uint64_t* start = nullptr; // Nc + 1: exclusive scan of (count, count >= 2) packed in a u64
    int* pos = nullptr;        // n
    int* slots = nullptr;      // n
};

struct Layout {
    int nZones = 0;
    int maxArea = 0, maxTX = 0, maxTY = 0;
    int4* rects = nullptr;
    int* owner = nullptr;
    std::vector<int4> hrects;
    std::vector<int> howner;
};

// Phase boundaries recorded on the context's stream (profiling runs only).
constexpr int kProfMarks = 24;
struct Prof {
    cudaEvent_t ev[kProfMarks];
    int label[kProfMarks];  // phase label of the interval ending at this mark
    int n;
};

}  // namespace

struct mpcd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    mpcd_params_c pc{};
    DevParams P{};
    int n = 0, Nc = 0;
    // state: the plain form keeps xb, vb; the FP32 precision form (f32) keeps offb, cellb, v32b
    bool f32 = false;
    double2* xb[2] = {nullptr, nullptr};
    double2* vb[2] = {nullptr, nullptr};
    float2* offb[2] = {nullptr, nullptr};
    int* cellb[2] = {nullptr, nullptr};
    float2* v32b[2] = {nullptr, nullptr};
    int* pidb[2] = {nullptr, nullptr};
    int xv = 0, pp = 0;
    // Position buffers are addressed as [k ^ xflip] for view index k: the zone passes update
    // positions in place and velocities out of place, so each pass flips xv and xflip together
    // (the positions stay in their buffer); a whole step leaves xflip as it found it.
    int xflip = 0;
    int* cidStd = nullptr;
    int* cidSrd = nullptr;
    uint64_t* sortKeys = nullptr;  // n: (particle id, slot) keys of the index being built
    // The step's first standard-grid index is built on the walls stream, beside the SRD index
    // and the collision (it needs the streamed cell ids only), with its own keys; the main
    // stream joins it at its first use (ensure_std_index).
    uint64_t* sortKeysSide = nullptr;  // n
    cudaEvent_t stdIdxDone = nullptr;
    bool stdIdxPending = false;
    int rankCells = 1;             // cells per block of k_cell_rank
    bool cidStdValid = false;
    bool srdCellsValid = false;
    CellIndex idxStd, idxSrd;
    bool idxStdValid = false;
    uint64_t* blockSums = nullptr;
    uint64_t* blockSumsWalls = nullptr;  // the walls' scan runs beside the index scans
    int blockSumsCap = 0;
    // walls
    BcWork W{};
    int nwords = 0;
    int bcBlocks = 0;
    double* wallOut = nullptr;  // 9 doubles
    // collision: rotation-sign streams, double-buffered; step s+1's stream is generated on a
    // side stream while step s's zone passes run
    uint8_t* signs = nullptr;       // synchronous use (phase API)
    uint8_t* signsBuf[2] = {nullptr, nullptr};
    int64_t signsStep[2] = {-1, -1};
    cudaStream_t side = nullptr;
    // thermal-wall velocities of a step (they need the post-BC positions only) run on their
    // own stream, beside the SRD index build, and join before the collision
    cudaStream_t walls = nullptr;
    cudaEvent_t bcDone = nullptr, wallsDone = nullptr;
    bool wallsPending = false;
    // CUDA-graph replay of the plain step: the step number and its seeds live on the device
    // (step_begin, in k_srd_shift); one graph per entry parity of the ping-pong buffers
    bool graphMode = false;            // true while a step is being captured
    bool useGraphs = true;
    long long* dStep = nullptr;        // device: number of the last step begun
    uint64_t* stepSeeds = nullptr;     // device: kStepSeeds
    cudaEvent_t sideDone = nullptr;    // the captured step joins its sign prefetch
    cudaGraphExec_t gexec[8] = {};  // by (xv, pp, xflip) at step entry
    int64_t gkernels[8] = {};
    struct HostFlags {
        int xv, pp, xflip;
        bool cidStdValid, srdCellsValid, idxStdValid, refValid;
    } gpost[8];
    cudaEvent_t signsReady[2] = {nullptr, nullptr};
    cudaEvent_t collDone = nullptr;
    // mpcd_run_jobs: double-buffered device staging of job inputs and results (x then v,
    // 2n double2 each) and the streams that copy them to and from the host
    double2* jobIn[2] = {nullptr, nullptr};
    double2* jobOut[2] = {nullptr, nullptr};
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t upDone[2] = {nullptr, nullptr}, inFree[2] = {nullptr, nullptr};
    cudaEvent_t outReady[2] = {nullptr, nullptr}, downDone[2] = {nullptr, nullptr};
    // zones
    Layout lay[3];  // base, shifted, single_full
    uint64_t* seeds = nullptr;
    int2* zoneMoved = nullptr;
    double2* zoneCorr = nullptr;
    int* overflow = nullptr;
    int* nOverflow = nullptr;
    int* ovDone = nullptr;       // overflow blocks finished (the last computes the pass metrics)
    // serial pass (allocated on first use): pass-input lists + live-list area, per-cell
    // current list start and count, the area's top, per-cell corrections of a zone
    int* slotsLive = nullptr;
    int* liveCnt = nullptr;
    int* liveStart = nullptr;
    int* liveTop = nullptr;
    double2* duScratch = nullptr;
    int64_t liveCap = 0;
    // fast form (MPCD_FORM_FAST): per-cell bins (ping-pong), the running step, wall hits, the
    // reference sums of the step-start state, the red momenta, the pending closure kick, the
    // moved counts, and the two zone layouts with the zone kernel's working-set sizes
    bool fast = false;
    FastParams F{};
    FastBins fb{};      // the standard-cell bins (the zone passes update them in place)
    int* fcnt2 = nullptr;  // the second count array (the zone passes' counts ping-pong)
    longlong2* fmid = nullptr;  // per cell the base pass's output momentum
    FastBins sb{};  // the stream's destination bins (swapped with fb after the stream)
    int* fspill = nullptr;   // collision tiles left to the spill kernel, and their count
    int* fnSpill = nullptr;
    int fcTY = 16, fcTilesY = 0, fcTiles = 0, fcPcap = 0;  // collision tiles: rows, tile rows, tiles, capacity
    bool fcTuned = false;  // the collision's tile rows chosen by timing (fast_tune_collide)
    size_t fcSmem = 0;
    FastStep* fstep = nullptr;
    FastWall* fwall = nullptr;
    longlong4* fref = nullptr;
    longlong2* fred = nullptr;
    int2* fkick = nullptr;
    bool fkickPending = false;
    int* fmoved = nullptr;  // base dense, base sparse, shifted dense, shifted sparse, zones out of records
    int4* frects[2] = {nullptr, nullptr};
    int fnz[2] = {0, 0};
    int zSyncWarps = 0;  // zones per block of the phase-synchronous zone pass (0: one per block)
    int fzMaxCells = 0, fzWinCap = 0, fzNsmCap = 0, fzRecCap = 0, fzWarps = 8;
    bool fzTuned = false;  // zones per block of the decision kernel chosen by timing (fast_tune_zone)
    size_t fzSmem = 0;
    // zone decisions handed to the apply kernel: per cell summary and removal masks, per zone records
    unsigned long long* fzMeta = nullptr;
    uint4* fzRm = nullptr;
    int* fzRecPid = nullptr;
    float2* fzRecOff = nullptr;
    int2* fzRecQ = nullptr;
    // launch order of the decision kernel (zones of similar cost together, heaviest first in
    // each window): per zone its cost, the order
    bool fzOrderOn = true;
    int* fzCost = nullptr;
    int* fzOrder = nullptr;
    // velocity profile accumulation (mpcd_profile_*): per row, momentum (int64 at 2^-32) and count
    bool profOn = false;
    unsigned long long* profP = nullptr;
    unsigned long long* profN = nullptr;
    int64_t profSteps = 0;
    // single-zone API (allocated on first use): the zone's rectangle, its kernel-side
    // diagnostics (8 doubles) and the global sums around it (32 doubles)
    int4* zkRect = nullptr;
    double* zkDiag = nullptr;
    double* zkOut = nullptr;
    // learned closure (mpcd_learned_set): parameters, the per-step mode flag (1 learned,
    // 0 plain) decided on the device from the previous step's occupancy spread, step counts
    // per mode, the spread sums, the predicted kick, and the red fields the stencil reads
    bool learnedOn = false;
    bool sampling = false;     // red fields wanted (dataset collection)
    double learnedLimit = 0.0;
    int learnedBulkOnly = 1;   // no learned kick in cells whose stencil crosses a wall
    int tcGrid = 0;            // CTAs of the tensor-core inference kernel
    float* lparams = nullptr;
    int* lmode = nullptr;
    long long* lcount = nullptr;
    double* lsums = nullptr;
    double* duLX = nullptr;
    double* duLY = nullptr;
    unsigned long long* duLSum = nullptr;  // sum over cells of N du (x, y), int64 at 2^-32; particles kicked
    float4* redFeat = nullptr;  // per cell of the red state: (N/gamma - 1, Ux, Uy, 0)
    ZoneArgs zA{};             // the zone pass in progress (zone_pass_prep .. zone_pass_finish)
    int zMode = 0;
    int* zoneCost = nullptr;   // per zone: cost bucket
    int* zoneHist = nullptr;   // kCostBuckets
    int* zoneOrder = nullptr;  // launch order, heaviest first
    char* ovMem = nullptr;
    size_t ovPerBlock = 0;
    int ovBlocks = 2;
    int zMaxCells = 0, zWinCap = 0, zArenaCap = 0, zNsmCap = 0;
    int collideShape = -1;     // index into kCollideShape; -1: autotune at the next eager collision
                               // that finds the slots in (cell, id) order
    bool slotsSorted = false;  // slots in (cell, id) order: false after a state upload until a step
    int collideTiles[kCollideShapes] = {};
    size_t zSmem = 0;
    int ovMaxCells = 0, ovWinCap = 0, ovArenaCap = 0, ovNsmCap = 0;
    double* passOut = nullptr;  // 4 doubles
    // closure
    int* mask = nullptr;
    int nMasked = 0;
    double *refN = nullptr, *refPx = nullptr, *refPy = nullptr, *refUx = nullptr, *refUy = nullptr, *refT = nullptr,
           *refRho = nullptr, *refPkin = nullptr, *refPvir = nullptr, *refP = nullptr;
    int* refNi = nullptr;
    bool refValid = false;
    double *pdRaw = nullptr, *pdrive = nullptr, *eosX = nullptr, *eosY = nullptr, *duRX = nullptr, *duRY = nullptr;
    double* cols = nullptr;     // Nc * kKickCols
    double* partial = nullptr;  // reduction partials
    int partialCap = 0;
    double* red = nullptr;      // small results: [0..1] num,den  [2..] others
    double* fieldTmp = nullptr; // 11 * Nc scratch for field outputs
    int* fieldTmpN = nullptr;
    double2* vrep = nullptr;
    int* cellOf = nullptr;      // n: cell of each cell-index position (flat kick)
    // status
    DevStatus* st = nullptr;
    DevStatus* hst = nullptr;
    double* hred = nullptr;
    // metrics
    mpcd_step_metrics_c last{};
    int64_t launches = 0;
    cudaEvent_t ev[8];
};

namespace {

const char* dev_error_text(int code) {
    switch (code) {
        case kErrUnsupportedBcLeft: return "Unsupported boundary_left mode";
        case kErrUnsupportedBcRight: return "Unsupported boundary_right mode";
        case kErrUnsupportedBcBottom: return "Unsupported boundary_bottom mode";
        case kErrUnsupportedBcTop: return "Unsupported boundary_top mode";
        case kErrZoneCapacity: return "zone working set exceeded its capacity";
        case kErrTableRange: return "minimal step outside the +-2 cell tables";
        case kErrBcLateSweep: return "a particle crossed a wall again after the first boundary sweep (displacement larger than the box): not supported on the device path";
        case kErrEventCapacity: return "more thermal wall hits than the event buffer holds";
        case kErrCellId: return "cell id outside [0, Nc)";
        case kErrTargetIsSource: return "a dense cell targeted itself (periodic axis shorter than 3 cells)";
        case kErrRngCapacity: return "collision sign stream shorter than the number of cells with >= 2 particles";
        case kErrTensorWait: return "a tensor-core MMA of the learned closure did not complete within the wait limit; "
                                    "the step's learned kicks are not trusted (results of every CTA of that launch)";
        case kErrBinCapacity: return "fast form: a cell holds more particles than its bin (capacity K)";
        case kErrRecordCapacity: return "fast form: a zone's moves outgrew its record area";
        case kErrLearnedRange: return "learned closure: a cell's kick N du exceeds the bound of its exact int64 sum (2^8 per cell)";
        default: return "device error";
    }
}

// synchronise and turn a raised device flag into a status code
void mark(mpcd_ctx* c, Prof* p, int label) {
    if (!p || p->n >= kProfMarks) return;
    p->label[p->n] = label;
    cudaEventRecord(p->ev[p->n++], c->stream);
}

// The state views of ping-pong buffer k, and a launch site written once for both forms:
// WITH_VIEW(k, ...) runs its body with S, the view of buffer k; WITH_VIEWS(k, k2, ...) also
// binds T, the view of buffer k2.
inline View64 view64(const mpcd_ctx* c, int k) { return View64{c->xb[k ^ c->xflip], c->vb[k]}; }
inline View32 view32(const mpcd_ctx* c, int k) {
    return View32{c->offb[k ^ c->xflip], c->cellb[k ^ c->xflip], c->v32b[k]};
}
// positions of the current state, and the other position buffer (free as scratch)
inline double2* cur_x(const mpcd_ctx* c) { return c->xb[c->xv ^ c->xflip]; }
inline double2* spare_x(const mpcd_ctx* c) { return c->xb[c->xv ^ c->xflip ^ 1]; }
#define WITH_VIEW(k, ...)                          \
    do {                                           \
        if (c->f32) {                              \
            const View32 S = view32(c, (k));       \
            __VA_ARGS__;                           \
        } else {                                   \
            const View64 S = view64(c, (k));       \
            __VA_ARGS__;                           \
        }                                          \
    } while (0)
#define WITH_VIEWS(k, k2, ...)                                        \
    do {                                                              \
        if (c->f32) {                                                 \
            const View32 S = view32(c, (k)), T = view32(c, (k2));     \
            __VA_ARGS__;                                              \
        } else {                                                      \
            const View64 S = view64(c, (k)), T = view64(c, (k2));     \
            __VA_ARGS__;                                              \
        }                                                             \
    } while (0)

// A kernel's dynamic shared-memory limit belongs to the function (per device) and so to every
// context of the process: raise it to what one context needs, never below another's need.
bool raise_smem(const void* fn, size_t need, int device) {
    if (need <= 48 * 1024) return true;
    static std::mutex m;
    static std::map<std::pair<const void*, int>, size_t> done;
    std::lock_guard<std::mutex> g(m);
    size_t& cur = done[{fn, device}];
    if (need <= cur) return true;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cur = need;
    return true;
}

int check_device(mpcd_ctx* c) {
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->side) CUDA_TRY(cudaStreamSynchronize(c->side));
    if (c->walls) CUDA_TRY(cudaStreamSynchronize(c->walls));
    CUDA_TRY(cudaMemcpy(c->hst, c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost));
    if (c->hst->code != 0) {
        const int code = c->hst->code;
        const int detail = c->hst->detail;
        cudaMemset(c->st, 0, sizeof(DevStatus));
        const int rc = (code >= kErrUnsupportedBcLeft && code <= kErrUnsupportedBcTop) ? MPCD_ERR_UNSUPPORTED_BC
                       : (code == kErrZoneCapacity || code == kErrEventCapacity || code == kErrRngCapacity ||
                          code == kErrBinCapacity || code == kErrRecordCapacity) ? MPCD_ERR_CAPACITY
                       : (code == kErrCellId) ? MPCD_ERR_INVALID_ARG
                                              : MPCD_ERR_DEVICE;
        return set_err(rc, std::string(dev_error_text(code)) + " (detail " + std::to_string(detail) + ")");
    }
    return MPCD_OK;
}

template <typename T>
int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    CUDA_TRY(cudaMalloc((void**)p, count * sizeof(T)));
    return MPCD_OK;
}

// ---------------------------------------------------------------- layouts (host, static)
std::vector<int> start_indices(int N, int tile, int off) {
    std::vector<int> s{0};
    for (int v = off; v < N; v += tile)
        if (v > 0 && v < N) s.push_back(v);
    return s;
}

// reference src/zone_pass.cpp:173-221
void build_layout(const mpcd_params_c& p, int mode, Layout& L) {
    L.hrects.clear();
    L.howner.assign((size_t)p.Nc, 0);
    if (mode == MPCD_LAYOUT_SINGLE_FULL) {
        L.hrects.push_back(make_int4(0, p.Nx, 0, p.Ny));
        std::fill(L.howner.begin(), L.howner.end(), 1);
    } else {
        const int offx = (mode == MPCD_LAYOUT_SHIFTED) ? p.zoneTileNx / 2 : 0;
        const int offy = (mode == MPCD_LAYOUT_SHIFTED) ? p.zoneTileNy / 2 : 0;
        const auto xs = start_indices(p.Nx, p.zoneTileNx, offx);
        const auto ys = start_indices(p.Ny, p.zoneTileNy, offy);
        int id = 0;
        for (int y : ys)
            for (int x : xs) {
                const int xe = std::min(x + p.zoneTileNx, p.Nx), ye = std::min(y + p.zoneTileNy, p.Ny);
                L.hrects.push_back(make_int4(x, xe, y, ye));
                ++id;
                for (int ix = x; ix < xe; ++ix)
                    for (int iy = y; iy < ye; ++iy) L.howner[(size_t)iy + (size_t)p.Ny * ix] = id;
            }
    }
    L.nZones = (int)L.hrects.size();
    L.maxArea = L.maxTX = L.maxTY = 0;
    for (const auto& r : L.hrects) {
        L.maxTX = std::max(L.maxTX, r.y - r.x);
        L.maxTY = std::max(L.maxTY, r.w - r.z);
        L.maxArea = std::max(L.maxArea, (r.y - r.x) * (r.w - r.z));
    }
}

bool periodic_x(const mpcd_params_c& p) { return p.boundary_left == MPCD_BC_PERIODIC && p.boundary_right == MPCD_BC_PERIODIC; }
bool periodic_y(const mpcd_params_c& p) { return p.boundary_bottom == MPCD_BC_PERIODIC && p.boundary_top == MPCD_BC_PERIODIC; }

// build_interzone_mask (reference src/liquid_closure.cpp:143-213), static per run
std::vector<int> interzone_mask(const mpcd_params_c& p, const Layout& base, const Layout& shifted) {
    std::vector<int> mask((size_t)p.Nc, 0);
    if (!p.smoothPdriveAtInterzone || !p.useZoneRedistribution || p.zonePassthroughMode || p.zoneSingleFullDomainMode) return mask;
    const bool px = periodic_x(p), py = periodic_y(p);
    auto boundary = [&](const std::vector<int>& own) {
        std::vector<int> b((size_t)p.Nc, 0);
        for (int ix = 0; ix < p.Nx; ++ix)
            for (int iy = 0; iy < p.Ny; ++iy) {
                const int c = iy + p.Ny * ix;
                const int right = (ix + 1 < p.Nx) ? iy + p.Ny * (ix + 1) : (px ? iy : -1);
                const int up = (iy + 1 < p.Ny) ? (iy + 1) + p.Ny * ix : (py ? p.Ny * ix : -1);
                b[(size_t)c] = (right >= 0 && own[(size_t)right] != own[(size_t)c]) || (up >= 0 && own[(size_t)up] != own[(size_t)c]);
            }
        return b;
    };
    auto dilate = [&](const std::vector<int>& in) {
        const int w = p.smoothPdriveInterzoneWidthCells;
        if (w <= 0) return in;
        std::vector<int> out((size_t)p.Nc, 0);
        for (int ix = 0; ix < p.Nx; ++ix)
            for (int iy = 0; iy < p.Ny; ++iy) {
                bool on = false;
                for (int dx = -w; dx <= w && !on; ++dx)
                    for (int dy = -w; dy <= w; ++dy) {
                        int jx = ix + dx, jy = iy + dy;
                        if (px) jx = ((jx % p.Nx) + p.Nx) % p.Nx;
                        else if (jx < 0 || jx >= p.Nx) continue;
                        if (py) jy = ((jy % p.Ny) + p.Ny) % p.Ny;
                        else if (jy < 0 || jy >= p.Ny) continue;
                        if (in[(size_t)jy + (size_t)p.Ny * jx]) { on = true; break; }
                    }
                out[(size_t)iy + (size_t)p.Ny * ix] = on;
            }
        return out;
    };
    mask = dilate(boundary(base.howner));
    if (p.smoothPdriveIncludeShiftedLayouts) {
        const auto s = dilate(boundary(shifted.howner));
        for (size_t c = 0; c < mask.size(); ++c) mask[c] = (mask[c] || s[c]) ? 1 : 0;
    }
    return mask;
}

int validate(const mpcd_params_c& p) {
    if (p.Nx < 1 || p.Ny < 1 || p.n < 0) return set_err(MPCD_ERR_INVALID_ARG, "Nx, Ny must be >= 1 and n >= 0");
    if ((int64_t)p.Nx * p.Ny != p.Nc) return set_err(MPCD_ERR_INVALID_ARG, "Nc must equal Nx*Ny");
    if ((int64_t)p.Nc >= (1LL << 31) || (int64_t)p.n * 2 >= (1LL << 31)) return set_err(MPCD_ERR_INVALID_ARG, "problem too large for 32-bit indices");
    if (!(p.Lx > 0.0) || !(p.Ly > 0.0) || !(p.a0 > 0.0)) return set_err(MPCD_ERR_INVALID_ARG, "Lx, Ly, a0 must be > 0");
    if (p.zoneTileNx < 1 || p.zoneTileNy < 1) return set_err(MPCD_ERR_INVALID_ARG, "zone tiles must be >= 1");
    if (p.maxRedistribPasses < 0) return set_err(MPCD_ERR_INVALID_ARG, "maxRedistribPasses must be >= 0");
    return MPCD_OK;
}

// Host-side derived constants; libm values where the reference calls libm.
DevParams make_dev_params(const mpcd_params_c& p) {
    DevParams d{};
    d.Nx = p.Nx; d.Ny = p.Ny; d.Nc = p.Nc; d.n = p.n;
    d.Lx = p.Lx; d.Ly = p.Ly; d.dt = p.dt; d.a0 = p.a0;
    d.dx = p.Lx / (double)p.Nx;
    d.dy = p.Ly / (double)p.Ny;
    d.Vc = d.dx * d.dy;
    d.invDx = 1.0 / d.dx;
    d.invDy = 1.0 / d.dy;
    d.invA0 = 1.0 / d.a0;
    d.invLx = 1.0 / d.Lx;
    d.invLy = 1.0 / d.Ly;
    d.alpha = p.alpha; d.kBT = p.kBT; d.g = p.g; d.bodyForceX = p.bodyForceX;
    d.useThermostat = p.useThermostat; d.keepMeanFlow = p.keepMeanFlow;
    d.bc[0] = p.boundary_left; d.bc[1] = p.boundary_right; d.bc[2] = p.boundary_bottom; d.bc[3] = p.boundary_top;
    d.perx = periodic_x(p); d.pery = periodic_y(p);
    d.Utop = p.Utop; d.Ubottom = p.Ubottom; d.wallSigma = p.wallSigma;
    d.tileNx = p.zoneTileNx; d.tileNy = p.zoneTileNy;
    d.momCorr = p.enableMomentumCorrectionPostRedistribution;
    d.maxPasses = p.maxRedistribPasses;
    d.useLFF = p.useLocalFluidFractionThresholds;
    d.gamma = p.gamma; d.coef = p.coef;
    // occupancy_thresholds (reference src/zone_pass.cpp:347-366)
    d.highThr = (p.highMode == MPCD_THR_ONE_PLUS_COEF) ? p.gamma * (1.0 + p.coef) : p.gamma + p.gamma * p.coef;
    d.lowThrBulk = (p.lowMode == MPCD_THR_ONE_PLUS_COEF) ? p.gamma / (1.0 + p.coef) : p.gamma - p.gamma * p.coef;
    if (std::isfinite(p.lowThrBulkOverride)) d.lowThrBulk = p.lowThrBulkOverride;
    d.lowFrac = 1.0 / (1.0 + p.coef);
    d.highFrac = 1.0 + p.coef;
    d.fluidFracGain = p.fluidFracGain; d.lowThrFloor = p.lowThrFloor; d.highThrFloor = p.highThrFloor;
    d.lowThrBulkInt = (int)std::ceil(d.lowThrBulk);
    d.useLiquidClosure = p.useLiquidClosure; d.useOptimalBetaRepair = p.useOptimalBetaRepair;
    d.smoothWidth = p.smoothPdriveInterzoneWidthCells;
    d.betaRepair = p.betaRepair; d.betaEOS = p.betaEOS; d.Kvirial = p.Kvirial;
    d.smoothBlend = p.smoothPdriveInterzoneBlend;
    d.rhoTarget = p.gamma / ((p.Lx / (double)p.Nx) * (p.Ly / (double)p.Ny));
    // the largest FP32 offset strictly below a cell width (FP32 form positions)
    auto below = [](double w) {
        float f = (float)w;
        while ((double)f >= w) f = std::nextafter(f, 0.0f);
        return f;
    };
    d.offMaxX = below(d.dx);
    d.offMaxY = below(d.dy);
    // rotation constants (reference src/srd_collision.cpp:93-94 evaluates cos/sin of theta)
    const double th[3] = {0.0, p.alpha * 1.0, p.alpha * -1.0};
    for (int k = 0; k < 3; ++k) {
        d.rotCos[k] = std::cos(th[k]);
        d.rotSin[k] = std::sin(th[k]);
    }
    // angular bins and step lengths of small integer steps (reference src/zone_pass.cpp:451-459)
    for (int b = -2; b <= 2; ++b)
        for (int a = -2; a <= 2; ++a) {
            const double ang = std::atan2((double)b, (double)a);
            int ib = (int)std::floor((ang + M_PI) / (2.0 * M_PI / 8.0));
            ib = ((ib % 8) + 8) % 8;
            d.atanBin[(a + 2) + 5 * (b + 2)] = ib;
            d.hypotTab[(a + 2) + 5 * (b + 2)] = std::hypot((double)a, (double)b);
        }
    return d;
}

// ---------------------------------------------------------------- index sort
int scan_u64(mpcd_ctx* c, const uint64_t* in, int64_t n, uint64_t* out, cudaStream_t s = nullptr,
             uint64_t* sums = nullptr) {
    if (!s) s = c->stream;
    if (!sums) sums = c->blockSums;
    if (n <= kSmallScan) {
        k_scan_small<<<1, kScanThreads, 0, s>>>(in, (int)n, out); ++c->launches;
        CUDA_TRY(cudaGetLastError());
        return MPCD_OK;
    }
    const int nb = (int)std::max<int64_t>(1, (n + kScanTile - 1) / kScanTile);
    if (nb > c->blockSumsCap) return set_err(MPCD_ERR_CAPACITY, "scan block buffer too small");
    k_scan_reduce<<<nb, kScanThreads, 0, s>>>(in, n, sums); ++c->launches;
    k_scan_blocks<<<1, kScanThreads, 0, s>>>(sums, nb); ++c->launches;
    k_scan_apply<<<nb, kScanThreads, 0, s>>>(in, n, sums, out); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// I.count is all zero between builds (set at creation, cleared again by the scan's read).
// s, keys, sums: the stream and scratch buffers (default: the context's stream, sortKeys and
// blockSums).
int build_index(mpcd_ctx* c, const int* cid, CellIndex& I, Prof* pf = nullptr, int label = -1,
                cudaStream_t s = nullptr, uint64_t* keys = nullptr, uint64_t* sums = nullptr) {
    if (!s) s = c->stream;
    if (!keys) keys = c->sortKeys;
    if (!sums) sums = c->blockSums;
    if (c->n > 0) {
        k_histogram<<<blocks_for(c->n, kThreads * kIndexItems), kThreads, 0, s>>>(cid, c->n, I.count, I.pos);
        ++c->launches;
    }
    if (c->Nc <= kSmallScan) {
        k_scan_counts_small<<<1, kScanThreads, 0, s>>>(I.count, c->Nc, I.start); ++c->launches;
    } else {
        const int nb = (c->Nc + kScanTile - 1) / kScanTile;
        if (nb > c->blockSumsCap) return set_err(MPCD_ERR_CAPACITY, "scan block buffer too small");
        k_count_scan_reduce<<<nb, kScanThreads, 0, s>>>(I.count, c->Nc, sums); ++c->launches;
        k_scan_blocks<<<1, kScanThreads, 0, s>>>(sums, nb); ++c->launches;
        k_count_scan_apply<<<nb, kScanThreads, 0, s>>>(I.count, c->Nc, sums, I.start); ++c->launches;
    }
    if (c->n > 0) {
        k_scatter_keys<<<blocks_for(c->n, kThreads * kIndexItems), kThreads, 0, s>>>(
            cid, I.pos, c->pidb[c->pp], c->n, I.start, keys); ++c->launches;
        k_cell_rank<<<blocks_for(c->Nc, c->rankCells), kRankThreads, 0, s>>>(I.start, c->Nc, c->rankCells, keys,
                                                                            I.slots); ++c->launches;
    }
    CUDA_TRY(cudaGetLastError());
    mark(c, pf, label);
    return MPCD_OK;
}

__global__ void k_set_step(long long* step, long long value) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step = value;
}

// the wall bitmaps and counters of a boundary sweep, cleared in one launch
__global__ void k_walls_clear(BcWork W, int nwords) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nwords) {
        W.bitsX[i] = 0u;
        W.bitsY[i] = 0u;
    }
    if (i < 4) W.ints[i] = 0;
    if (i == 0) *W.nEvents = 0;
}

// the particle state of slots [0, n) from S to T, in one launch
template <class V>
__global__ void k_copy_state(V S, V T, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        T.copy_pos(i, S, i);
        T.set_vel(i, S.vel(i));
    }
}

// the velocities of slots [0, n) from S to T
template <class V>
__global__ void k_copy_vel(V S, V T, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) T.set_vel(i, S.vel(i));
}

template <class V>
__global__ void k_std_cells(DevParams P, V S, int* __restrict__ cid) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < P.n) cid[s] = S.std_cell(s, P);
}

int ensure_std_index(mpcd_ctx* c, Prof* pf = nullptr) {
    if (c->stdIdxPending) {  // built on the walls stream
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->stdIdxDone, 0));
        c->stdIdxPending = false;
    }
    if (c->idxStdValid) return MPCD_OK;
    if (!c->cidStdValid) {
        WITH_VIEW(c->xv, k_std_cells<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, S, c->cidStd));
        ++c->launches;
        c->cidStdValid = true;
    }
    const int rc = build_index(c, c->cidStd, c->idxStd, pf, 5);
    if (!rc) c->idxStdValid = true;
    return rc;
}

void invalidate_positions(mpcd_ctx* c) {
    c->cidStdValid = false;
    c->idxStdValid = false;
    c->srdCellsValid = false;
}

// ---------------------------------------------------------------- host <-> device in id order
__global__ void k_gather_by_pid(const double2* __restrict__ x, const double2* __restrict__ v, const int* __restrict__ pid,
                                int n, double2* __restrict__ xo, double2* __restrict__ vo) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = pid[s];
    if (xo) xo[p] = x[s];
    if (vo) vo[p] = v[s];
}

// FP32 form, state I/O: positions and velocities in particle-id order, widened to FP64
__global__ void k_f32_by_pid(DevParams P, View32 S, const int* __restrict__ pid, int n, double2* __restrict__ xo,
                             double2* __restrict__ vo) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = pid[s];
    if (xo) xo[p] = S.pos(s, P);
    if (vo) vo[p] = S.vel(s);
}

// FP32 form, state I/O: FP64 positions and velocities (slot s = particle id s) into the view
__global__ void k_f32_from(DevParams P, const double2* __restrict__ x, const double2* __restrict__ v, int n, View32 S) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double2 X = x[s];
    S.set_pos(s, X, cell_of(X.x, X.y, P), P);
    S.set_vel(s, v[s]);
}

__global__ void k_int_by_pid(const int* __restrict__ a, const int* __restrict__ pid, int n, int* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[pid[s]] = a[s];
}

__global__ void k_int_to_slots(const int* __restrict__ byPid, const int* __restrict__ pid, int n, int Nc,
                               int* __restrict__ out, DevStatus* st) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int c = byPid[pid[s]];
    if (c < 0 || c >= Nc) raise_error(st, kErrCellId, pid[s]);
    out[s] = (c < 0) ? 0 : ((c >= Nc) ? Nc - 1 : c);
}

__global__ void k_stream_only(DevParams P, double2* __restrict__ x, double2* __restrict__ v) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n) return;
    double2 xs = x[s], vs = v[s];
    vs.x = __dadd_rn(vs.x, __dmul_rn(P.bodyForceX, P.dt));
    vs.y = __dadd_rn(vs.y, __dmul_rn(P.g, P.dt));
    xs.x = __dadd_rn(xs.x, __dmul_rn(P.dt, vs.x));
    xs.y = __dadd_rn(xs.y, __dmul_rn(P.dt, vs.y));
    x[s] = xs;
    v[s] = vs;
}

__global__ void k_srd_cells(DevParams P, const double2* __restrict__ x, const double* __restrict__ shift, int* __restrict__ cid) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < P.n) cid[s] = srd_cell(x[s].x, x[s].y, shift[0], shift[1], P);
}

template <class V>
__global__ void k_sub_mean(V S, int n, const double* __restrict__ sums) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double mx = __ddiv_rn(sums[1], (double)n), my = __ddiv_rn(sums[2], (double)n);
    const double2 w = S.vel(s);
    S.set_vel(s, make_double2(__dsub_rn(w.x, mx), __dsub_rn(w.y, my)));
}

int reduce_cols(mpcd_ctx* c, const double* cols, int64_t rows, int K, unsigned maxMask, double* out) {
    const int rowsPerBlock = 8192;
    const int nb = (int)std::max<int64_t>(1, (rows + rowsPerBlock - 1) / rowsPerBlock);
    if ((int64_t)nb * K > c->partialCap) return set_err(MPCD_ERR_CAPACITY, "reduction buffer too small");
    k_reduce_partial<<<nb, kRedThreads, 0, c->stream>>>(cols, rows, K, maxMask, rowsPerBlock, c->partial); ++c->launches;
    k_reduce_final<<<1, kRedThreads, 0, c->stream>>>(c->partial, nb, K, maxMask, out); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// ---------------------------------------------------------------- phases
// overlap: the wall-velocity kernels go to c->walls and run_collide joins them before the
// collision (the step's path); otherwise everything stays on the context's stream
int run_bc(mpcd_ctx* c, bool doStream, uint64_t seed, int* cidStd, int* cidSrd, bool wantInfo, Prof* pf = nullptr,
           bool overlap = false) {
    BcWork& W = c->W;
    k_walls_clear<<<blocks_for(c->nwords), kThreads, 0, c->stream>>>(W, c->nwords); ++c->launches;
    if (wantInfo)
        WITH_VIEW(c->xv, k_stream_bc<true><<<c->bcBlocks, kThreads, 0, c->stream>>>(c->P, doStream ? 1 : 0, S, c->pidb[c->pp],
                                                                                   cidStd, cidSrd, W, c->st));
    else
        WITH_VIEW(c->xv, k_stream_bc<false><<<c->bcBlocks, kThreads, 0, c->stream>>>(c->P, doStream ? 1 : 0, S, c->pidb[c->pp],
                                                                                    cidStd, cidSrd, W, c->st));
    ++c->launches;
    mark(c, pf, 0);
    cudaStream_t ws = c->stream;
    uint64_t* sums = c->blockSums;
    if (overlap && c->walls) {
        CUDA_TRY(cudaEventRecord(c->bcDone, c->stream));
        CUDA_TRY(cudaStreamWaitEvent(c->walls, c->bcDone, 0));
        ws = c->walls;
        sums = c->blockSumsWalls;
    }
    k_word_counts<<<blocks_for(c->nwords), kThreads, 0, ws>>>(W.bitsX, W.bitsY, c->nwords, W.wordCount); ++c->launches;
    int rc = scan_u64(c, W.wordCount, c->nwords, W.wordPrefix, ws, sums);
    if (rc) return rc;
    k_wall_normals<<<1, kNormThreads, 0, ws>>>(seed, W.wordPrefix + c->nwords, W.normalCap, W.normals, c->st,
                                               c->graphMode ? c->stepSeeds : nullptr); ++c->launches;
    WITH_VIEW(c->xv, k_wall_apply<<<blocks_for(W.eventCap), kThreads, 0, ws>>>(c->P, S, W, c->st)); ++c->launches;
    if (wantInfo)
        k_wall_reduce<<<1, 32, 0, ws>>>(W.blockPartial, c->bcBlocks, W.contrib, W.wordPrefix + c->nwords, W.normalCap, c->wallOut); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    if (ws != c->stream) {
        CUDA_TRY(cudaEventRecord(c->wallsDone, ws));
        c->wallsPending = true;
    }
    mark(c, pf, 1);
    return MPCD_OK;
}

// the collision with tile shape k on ping-pong buffer `buf`
static int launch_collide(mpcd_ctx* c, int k, int buf, const uint8_t* signs, const uint64_t* gs, cudaStream_t s) {
    const int tile = c->collideTiles[k];
    const size_t smem = (size_t)tile * (sizeof(double2) + sizeof(int));
#define MPCD_COLLIDE(K)                                                                                      \
    case K:                                                                                                  \
        WITH_VIEW(buf, (k_srd_collide<std::remove_const_t<decltype(S)>, kCollideShape[K].cells, kCollideShape[K].threads>          \
                        <<<blocks_for(c->Nc, kCollideShape[K].cells), kCollideShape[K].threads, smem, s>>>(  \
                            c->P, c->idxSrd.start, c->idxSrd.slots, signs, c->Nc, S, c->st, gs, c->signsBuf[1], \
                            tile)));                                                                         \
        break;
    switch (k) {
        MPCD_COLLIDE(0)
        MPCD_COLLIDE(1)
        MPCD_COLLIDE(2)
        MPCD_COLLIDE(3)
        MPCD_COLLIDE(4)
        MPCD_COLLIDE(5)
        MPCD_COLLIDE(6)
        default: return set_err(MPCD_ERR_INVALID_ARG, "collision tile shape out of range");
    }
#undef MPCD_COLLIDE
    ++c->launches;
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// Autotuner of the collision tile shape: on a scratch copy of the velocities (the spare
// ping-pong buffer) every candidate runs once to warm up, then the candidates run in turn for
// three rounds, and the shape with the fastest single run is kept for the context. Running the
// rounds in turn keeps clock ramps at the start of a run from favouring the later candidates.
static int tune_collide(mpcd_ctx* c, const uint8_t* signs) {
    const int spare = c->xv ^ 1;
    if (c->n > 0) {
        WITH_VIEWS(c->xv, spare, k_copy_state<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, T, c->n));
        ++c->launches;
    }
    constexpr int kRounds = 3;
    cudaEvent_t ev[kRounds * kCollideShapes + 1];
    for (auto& e : ev) e = nullptr;
    int rc = MPCD_OK;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "tuning events");
    for (int k = 0; k < kCollideShapes && !rc; ++k) rc = launch_collide(c, k, spare, signs, nullptr, c->stream);
    if (!rc && cudaEventRecord(ev[0], c->stream) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "tuning event");
    for (int i = 0; i < kRounds * kCollideShapes && !rc; ++i) {
        rc = launch_collide(c, i % kCollideShapes, spare, signs, nullptr, c->stream);
        if (!rc && cudaEventRecord(ev[i + 1], c->stream) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "tuning event");
    }
    float best[kCollideShapes];
    for (float& b : best) b = 1e30f;
    if (!rc && cudaEventSynchronize(ev[kRounds * kCollideShapes]) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "tuning");
    for (int i = 0; i < kRounds * kCollideShapes && !rc; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "tuning time");
        best[i % kCollideShapes] = std::min(best[i % kCollideShapes], ms);
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (rc) return rc;
    int pick = 0;
    for (int k = 1; k < kCollideShapes; ++k)
        if (best[k] < best[pick]) pick = k;
    c->collideShape = pick;
    return check_device(c);
}

// step < 0: phase API (sign stream generated here, synchronously); otherwise the stream of
// that step from the double buffer (generated ahead on the side stream when possible)
int run_collide(mpcd_ctx* c, uint64_t seed, Prof* pf = nullptr, int64_t step = -1) {
    int rc = build_index(c, c->cidSrd, c->idxSrd, pf, 2);
    if (rc) return rc;
    const uint8_t* signs = c->signs;
    const uint64_t* gs = c->graphMode ? c->stepSeeds : nullptr;
    if (c->graphMode) {
        signs = c->signsBuf[0];  // or signsBuf[1]: k_srd_collide picks by the step's parity
    } else if (step < 0) {
        k_srd_signs<<<1, kSignThreads, 0, c->stream>>>(seed, c->Nc, c->signs, nullptr, nullptr); ++c->launches;
    } else {
        const int b = (int)(step & 1);
        if (c->signsStep[b] != step) {
            k_srd_signs<<<1, kSignThreads, 0, c->stream>>>(seed, c->Nc, c->signsBuf[b], nullptr, nullptr); ++c->launches;
            c->signsStep[b] = step;
        } else {
            CUDA_TRY(cudaStreamWaitEvent(c->stream, c->signsReady[b], 0));
        }
        signs = c->signsBuf[b];
    }
    mark(c, pf, 3);
    if (c->wallsPending) {  // the collision reads the wall-updated velocities
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->wallsDone, 0));
        c->wallsPending = false;
    }
    // Tuned only on cell-sorted slots: an uploaded state is in particle-id order, whose scattered
    // gathers favour other tile shapes than the sorted layout every later step has.
    if (c->collideShape < 0 && !c->graphMode && c->slotsSorted) {
        rc = tune_collide(c, signs);
        if (rc) return rc;
    }
    rc = launch_collide(c, c->collideShape < 0 ? 1 : c->collideShape, c->xv, signs, gs, c->stream);
    if (rc) return rc;
    if (c->P.keepMeanFlow) {
        WITH_VIEW(c->xv, k_particle_cols<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, c->n, c->cols)); ++c->launches;
        rc = reduce_cols(c, c->cols, c->n, 3, 0u, c->red + 8);
        if (rc) return rc;
        WITH_VIEW(c->xv, k_sub_mean<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, c->n, c->red + 8)); ++c->launches;
    }
    CUDA_TRY(cudaGetLastError());
    mark(c, pf, 4);
    if (c->graphMode) {
        // the next step's sign stream on the side stream; the captured step joins it at its end
        CUDA_TRY(cudaEventRecord(c->collDone, c->stream));
        CUDA_TRY(cudaStreamWaitEvent(c->side, c->collDone, 0));
        k_srd_signs<<<1, kSignThreads, 0, c->side>>>(0, c->Nc, c->signsBuf[0], gs, c->signsBuf[1]); ++c->launches;
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaEventRecord(c->sideDone, c->side));
    } else if (step >= 0) {
        // generate the next step's sign stream on the side stream, after this collision
        // (which is the last reader of the buffer it overwrites' previous contents)
        const int b = (int)((step + 1) & 1);
        CUDA_TRY(cudaEventRecord(c->collDone, c->stream));
        CUDA_TRY(cudaStreamWaitEvent(c->side, c->collDone, 0));
        const uint64_t next = 433494437ULL + 10007ULL * (uint64_t)(step + 1);
        k_srd_signs<<<1, kSignThreads, 0, c->side>>>(next, c->Nc, c->signsBuf[b], nullptr, nullptr); ++c->launches;
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaEventRecord(c->signsReady[b], c->side));
        c->signsStep[b] = step + 1;
    }
    return MPCD_OK;
}

// reference fields of the current state + pdrive + EOS kick (depend on the reference only);
// inStep: called from the step, where a learned step (device mode flag) skips them
int run_save_ref(mpcd_ctx* c, Prof* pf = nullptr, bool inStep = false) {
    int rc = ensure_std_index(c, pf);
    if (rc) return rc;
    FieldsOut o{};
    o.N = c->refNi; o.Ux = c->refUx; o.Uy = c->refUy; o.Px = c->refPx; o.Py = c->refPy; o.T = c->refT;
    o.rho = c->refRho; o.Pkin = c->refPkin; o.Pvir = c->refPvir; o.P = c->refP;
    const int* skip = (inStep && c->learnedOn) ? c->lmode : nullptr;  // learned steps need no reference
    WITH_VIEW(c->xv, k_cell_fields<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->idxStd.start, c->idxStd.slots, S,
                                                                                  c->P.rhoTarget, o, skip));
    ++c->launches;
    k_pdrive<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->refPkin, c->refPvir, c->pdRaw, skip); ++c->launches;
    k_pdrive_blend<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->pdRaw, c->mask, c->nMasked > 0, c->pdrive, skip);
    ++c->launches;
    k_eos<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->pdrive, c->eosX, c->eosY, skip); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    mark(c, pf, 6);
    c->refValid = true;
    return MPCD_OK;
}

// The snapshot pass in three parts, so that a batch can run the middle one for all its
// replicas in one launch: prep (index, seeds, output copies, launch order; fills c->zA),
// the zone kernel, and finish (overflow zones, metrics, state flags).
int zone_pass_prep(mpcd_ctx* c, int mode, uint64_t seedBase, Prof* pf = nullptr) {
    if (!c->cidStdValid) {
        WITH_VIEW(c->xv, k_std_cells<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, S, c->cidStd)); ++c->launches;
        c->cidStdValid = true;
    }
    int rc = ensure_std_index(c, pf);
    if (rc) return rc;
    // the seed of the shifted pass (seedBase + 4099) also when the single full-domain zone runs it
    const bool shiftedPass = mode == MPCD_LAYOUT_SHIFTED;
    if (mode != MPCD_LAYOUT_SHIFTED && mode != MPCD_LAYOUT_SINGLE_FULL) mode = MPCD_LAYOUT_BASE;
    if (c->pc.zoneSingleFullDomainMode) mode = MPCD_LAYOUT_SINGLE_FULL;
    Layout& L = c->lay[mode];
    k_zone_seeds<<<(L.nZones + kSeedZonesPerBlock - 1) / kSeedZonesPerBlock, kSeedZonesPerBlock * 2, 0, c->stream>>>(
        seedBase, L.nZones, c->seeds, c->graphMode ? c->stepSeeds : nullptr, shiftedPass ? kSeedShifted : kSeedBase);
    ++c->launches;
    mark(c, pf, 7);
    // velocities out of place (output starts as a copy of the input; zones write what they
    // change), positions in place (the zone kernel never reads them)
    const int xi = c->xv, xo = c->xv ^ 1;
    if (c->n > 0) {
        WITH_VIEWS(xi, xo, k_copy_vel<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, T, c->n));
        ++c->launches;
    }
    ZoneArgs A{};
    A.P = c->P;
    A.rects = L.rects;
    A.owner = L.owner;
    A.start = c->idxStd.start;
    A.slots = c->idxStd.slots;
    A.vin = c->vb[xi];
    A.xout = cur_x(c);
    A.vout = c->vb[xo];
    A.f32 = c->f32 ? 1 : 0;
    A.in32 = view32(c, xi);
    A.out32 = View32{c->offb[xi ^ c->xflip], c->cellb[xi ^ c->xflip], c->v32b[xo]};
    A.cid = c->cidStd;
    A.seeds = c->seeds;
    A.nZones = L.nZones;
    A.maxCells = c->zMaxCells;
    A.winCap = c->zWinCap;
    A.arenaCap = c->zArenaCap;
    A.nsmCap = c->zNsmCap;
    A.overflow = c->overflow;
    A.nOverflow = c->nOverflow;
    A.zoneMoved = c->zoneMoved;
    A.zoneCorr = c->zoneCorr;
    A.st = c->st;
    // heaviest zones first (by estimated dense-phase work) in the base pass; the shifted pass
    // runs after the base pass has evened the counts, its zones cost about the same, and the
    // two ordering kernels would cost more than the tail they save
    if (mode == MPCD_LAYOUT_SHIFTED) {
        A.order = nullptr;
    } else {
        k_zone_cost<<<blocks_for(L.nZones), kThreads, 0, c->stream>>>(c->P, L.rects, c->idxStd.start, L.nZones,
                                                                       c->zoneCost, c->zoneHist); ++c->launches;
        k_zone_order<<<1, 1024, 0, c->stream>>>(c->zoneCost, c->zoneHist, L.nZones, c->zoneOrder); ++c->launches;
        A.order = c->zoneOrder;
    }
    CUDA_TRY(cudaGetLastError());
    c->zA = A;
    c->zMode = mode;
    return MPCD_OK;
}

int zone_pass_kernel(mpcd_ctx* c) {
    const ZoneArgs& A = c->zA;
    const int W = c->zSyncWarps;
    const int per = (int)c->zSmem;
    const int blocks = W > 0 ? (A.nZones + W - 1) / W : 0;
#define MPCD_ZONE_SYNC(F, K) k_zone_pass_sync<F, K><<<blocks, 32 * K, (size_t)K * per, c->stream>>>(A, per)
    if (W == 16) {
        if (c->f32) MPCD_ZONE_SYNC(true, 16); else MPCD_ZONE_SYNC(false, 16);
    } else if (W == 8) {
        if (c->f32) MPCD_ZONE_SYNC(true, 8); else MPCD_ZONE_SYNC(false, 8);
    } else if (W == 4) {
        if (c->f32) MPCD_ZONE_SYNC(true, 4); else MPCD_ZONE_SYNC(false, 4);
    } else if (c->f32) {
        k_zone_pass<true><<<A.nZones, 32, c->zSmem, c->stream>>>(A);
    } else {
        k_zone_pass<false><<<A.nZones, 32, c->zSmem, c->stream>>>(A);
    }
#undef MPCD_ZONE_SYNC
    ++c->launches;
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// the overflow kernel's job for the pass in progress (its arguments with the global-memory
// working set's capacities); the pass metrics (a serial sum over the zones) only if wanted:
// the phase API and the metrics step of mpcd_step report them, plain steps do not
OverflowJob overflow_job(const mpcd_ctx* c, bool metrics) {
    OverflowJob J{};
    J.A = c->zA;
    J.A.order = nullptr;
    J.A.maxCells = c->ovMaxCells;
    J.A.winCap = c->ovWinCap;
    J.A.arenaCap = c->ovArenaCap;
    J.A.nsmCap = c->ovNsmCap;
    J.gmem = c->ovMem;
    J.perBlock = c->ovPerBlock;
    J.blocksDone = c->ovDone;
    J.metricsOut = metrics ? c->passOut + (c->zMode == MPCD_LAYOUT_SHIFTED ? 4 : 0) : nullptr;
    return J;
}

// host-side state after a pass: velocities in the other buffer, positions in place
void zone_pass_flip(mpcd_ctx* c) {
    c->xv ^= 1;
    c->xflip ^= 1;
    c->idxStdValid = false;  // cid was updated for moved particles; positions changed
    c->srdCellsValid = false;
}

int zone_pass_finish(mpcd_ctx* c, Prof* pf = nullptr, bool metrics = true) {
    const OverflowJob J = overflow_job(c, metrics);
    if (c->f32)
        k_zone_overflow<true><<<c->ovBlocks, 32, 0, c->stream>>>(J.A, J.gmem, J.perBlock, J.blocksDone, J.metricsOut);
    else
        k_zone_overflow<false><<<c->ovBlocks, 32, 0, c->stream>>>(J.A, J.gmem, J.perBlock, J.blocksDone, J.metricsOut);
    ++c->launches;
    CUDA_TRY(cudaGetLastError());
    mark(c, pf, 8);
    zone_pass_flip(c);
    return MPCD_OK;
}

int run_zone_pass(mpcd_ctx* c, int mode, uint64_t seedBase, Prof* pf = nullptr) {
    int rc = zone_pass_prep(c, mode, seedBase, pf);
    if (!rc) rc = zone_pass_kernel(c);
    if (!rc) rc = zone_pass_finish(c, pf);
    return rc;
}

__global__ void k_live_init(const uint64_t* __restrict__ start, int Nc, int* __restrict__ cnt, int* __restrict__ st,
                            int* __restrict__ top, int n) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < Nc) {
        const int a = (int)(uint32_t)start[c];
        st[c] = a;
        cnt[c] = (int)(uint32_t)start[c + 1] - a;
    }
    if (c == 0) *top = n;
}

// The serial zone kernel over nZones rectangles (device), in place on the current state; zone
// k draws from mt19937_64(seedBase + 104729 (k + 1)) (src/zone_pass_openmp.cpp:78 and the
// serial pass). Pass metrics go to metricsOut (4 doubles); zoneDiag (nullable) receives the
// single-zone diagnostics of ZoneArgs::zoneDiag.
static int launch_zone_serial(mpcd_ctx* c, const int4* rects, const int* owner, int nZones, uint64_t seedBase,
                              double* zoneDiag, double* metricsOut) {
    if (!c->cidStdValid) {
        k_std_cells<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, view64(c, c->xv), c->cidStd); ++c->launches;
        c->cidStdValid = true;
    }
    int rc = ensure_std_index(c);
    if (rc) return rc;
    if (!c->slotsLive) {
        // every zone appends at most the particles of its cells; overlapping layouts revisit
        // some cells, so twice the particles (plus slack) bounds the live-list area
        c->liveCap = 2LL * c->n + 1024;
        if (c->n + c->liveCap >= (1LL << 31)) return set_err(MPCD_ERR_CAPACITY, "serial pass: too many particles");
        CUDA_TRY(cudaMalloc(&c->slotsLive, sizeof(int) * (size_t)(c->n + c->liveCap)));
        CUDA_TRY(cudaMalloc(&c->liveCnt, sizeof(int) * (size_t)c->Nc));
        CUDA_TRY(cudaMalloc(&c->liveStart, sizeof(int) * (size_t)c->Nc));
        CUDA_TRY(cudaMalloc(&c->liveTop, sizeof(int)));
        CUDA_TRY(cudaMalloc(&c->duScratch, sizeof(double2) * (size_t)std::max(std::max(c->zMaxCells, c->ovMaxCells), 1)));
    }
    k_zone_seeds<<<(nZones + kSeedZonesPerBlock - 1) / kSeedZonesPerBlock, kSeedZonesPerBlock * 2, 0, c->stream>>>(
        seedBase, nZones, c->seeds, nullptr, kSeedBase); ++c->launches;
    if (c->n > 0)
        CUDA_TRY(cudaMemcpyAsync(c->slotsLive, c->idxStd.slots, sizeof(int) * (size_t)c->n, cudaMemcpyDeviceToDevice, c->stream));
    k_live_init<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->idxStd.start, c->Nc, c->liveCnt, c->liveStart, c->liveTop,
                                                               c->n); ++c->launches;
    ZoneArgs A{};
    A.P = c->P;
    A.rects = rects;
    A.owner = owner;
    A.start = c->idxStd.start;
    A.slots = c->slotsLive;
    A.vin = c->vb[c->xv];
    A.xout = cur_x(c);
    A.vout = c->vb[c->xv];
    A.cid = c->cidStd;
    A.seeds = c->seeds;
    A.nZones = nZones;
    A.maxCells = c->zMaxCells;
    A.winCap = c->zWinCap;
    A.arenaCap = c->zArenaCap;
    A.nsmCap = c->zNsmCap;
    A.overflow = c->overflow;
    A.nOverflow = c->nOverflow;
    A.zoneMoved = c->zoneMoved;
    A.zoneCorr = c->zoneCorr;
    A.order = nullptr;
    A.st = c->st;
    A.serial = 1;
    A.slotsW = c->slotsLive;
    A.liveCnt = c->liveCnt;
    A.liveStart = c->liveStart;
    A.liveTop = c->liveTop;
    A.liveEnd = (int)(c->n + c->liveCap);
    A.pid = c->pidb[c->pp];
    A.duScratch = c->duScratch;
    A.zoneDiag = zoneDiag;
    ZoneArgs B = A;
    B.maxCells = c->ovMaxCells;
    B.winCap = c->ovWinCap;
    B.arenaCap = c->ovArenaCap;
    B.nsmCap = c->ovNsmCap;
    k_zone_serial<<<1, 32, c->zSmem, c->stream>>>(A, B, c->ovMem); ++c->launches;
    k_zone_metrics<<<1, 256, 0, c->stream>>>(c->zoneMoved, c->zoneCorr, nZones, metricsOut, c->nOverflow); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    c->idxStdValid = false;  // positions and velocities changed in place
    c->cidStdValid = false;
    c->srdCellsValid = false;
    return MPCD_OK;
}

// run_zone_pass (src/zone_pass.cpp:1096-1163) on the current state, in place
int run_zone_pass_serial(mpcd_ctx* c, int mode, uint64_t seedBase) {
    if (mode != MPCD_LAYOUT_SHIFTED && mode != MPCD_LAYOUT_SINGLE_FULL) mode = MPCD_LAYOUT_BASE;
    if (c->pc.zoneSingleFullDomainMode) mode = MPCD_LAYOUT_SINGLE_FULL;
    const Layout& L = c->lay[mode];
    return launch_zone_serial(c, L.rects, L.owner, L.nZones, seedBase, nullptr,
                              c->passOut + (mode == MPCD_LAYOUT_SHIFTED ? 4 : 0));
}

// closure on the current (red) state; permute: write particles in (cell, id) order into the
// other buffers (next step's layout), as the step does; vrep: repaired velocities wanted.
// In the step, with a network set (mpcd_learned_set), the device mode flag picks the learned
// or the plain kick per step.
int run_closure(mpcd_ctx* c, bool permute, bool wantRep, bool wantStats, Prof* pf = nullptr) {
    if (!c->refValid) return set_err(MPCD_ERR_STATE, "liquid closure needs a saved reference state (mpcd_save_ref)");
    int rc = ensure_std_index(c, pf);
    if (rc) return rc;
    const bool learned = permute && c->learnedOn;
    RedFields rf{};
    if (learned || c->sampling) {  // the stencil features read the red fields
        rf.feat = c->redFeat;
    }
    // the step's fast path; learned steps always take it (their closure has no diagnostics)
    const bool flat = permute && (learned || (!wantRep && !wantStats));
    WITH_VIEW(c->xv, k_closure_cells<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(
                         c->P, c->idxStd.start, c->idxStd.slots, S, c->refPx, c->refPy, c->refUx, c->refUy, rf, c->duRX,
                         c->duRY, c->cols, flat ? c->cellOf : nullptr));
    ++c->launches;
    rc = reduce_cols(c, c->cols, c->Nc, 2, 0u, c->red);
    if (rc) return rc;
    mark(c, pf, 9);
    const int nx = c->xv, np = c->pp;
    if (learned) {
        CUDA_TRY(cudaMemsetAsync(c->duLSum, 0, 3 * sizeof(unsigned long long), c->stream));
        k_mlp_tc<false><<<c->tcGrid, kTcThreads, kTcSmem, c->stream>>>(c->P, c->redFeat, nullptr, 0,
                                                                        c->lparams, c->duLX, c->duLY, nullptr, c->lmode,
                                                                        c->duLSum, c->learnedBulkOnly, c->st);
        ++c->launches;
    }
    if (flat) {
        WITH_VIEWS(nx, nx ^ 1, k_kick_flat<<<blocks_for(c->n, kThreads * kKickItems), kThreads, 0, c->stream>>>(
                                   c->P, c->n, c->cellOf, c->idxStd.slots, c->red, c->duRX, c->duRY, c->eosX, c->eosY, S,
                                   c->pidb[np], T, c->pidb[np ^ 1], learned ? c->lmode : nullptr, c->duLX, c->duLY,
                                   reinterpret_cast<const long long*>(c->duLSum)));
        ++c->launches;
    } else {
        WITH_VIEWS(nx, nx ^ 1, k_kick<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(
                                   c->P, c->idxStd.start, c->idxStd.slots, c->red, c->duRX, c->duRY, c->eosX, c->eosY, S,
                                   c->pidb[np], permute ? 1 : 0, T, permute ? c->pidb[np ^ 1] : nullptr,
                                   wantRep ? c->vrep : nullptr, wantStats ? c->cols : nullptr));
        ++c->launches;
    }
    CUDA_TRY(cudaGetLastError());
    if (learned) {
        // the next step's mode, from this step's occupancy spread (the red counts)
        k_count_cols<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->idxStd.start, c->Nc, c->P.highThr, c->P.lowThrBulk,
                                                                    c->cols); ++c->launches;
        rc = reduce_cols(c, c->cols, c->Nc, 3, 0u, c->lsums);
        if (rc) return rc;
        k_learned_decide<<<1, 1, 0, c->stream>>>(c->lsums, c->Nc, c->pc.gamma, c->learnedLimit, c->lmode, c->lcount);
        ++c->launches;
        if (wantStats) CUDA_TRY(cudaMemsetAsync(c->red + 2, 0, sizeof(double) * kKickCols, c->stream));
    } else if (wantStats) {
        // sum, max, sum, sum, max, sum, sum, sum, sum
        rc = reduce_cols(c, c->cols, c->Nc, kKickCols, (1u << 1) | (1u << 4), c->red + 2);
        if (rc) return rc;
    }
    if (permute) {
        c->xv ^= 1;
        c->pp ^= 1;
        c->slotsSorted = true;
        k_iota<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->idxStd.slots, c->n); ++c->launches;
        CUDA_TRY(cudaGetLastError());
        mark(c, pf, 10);
        // the standard index stays valid (same cells, identity slots); per-slot cell ids and
        // SRD cells refer to the old layout
        c->cidStdValid = false;
        c->srdCellsValid = false;
    }
    return MPCD_OK;
}

#include "fast_host.inc"

}  // namespace

// ====================================================================== C-ABI
extern "C" {

const char* mpcd_last_error(void) { return g_err.c_str(); }

int mpcd_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, 0) != cudaSuccess) return 0;
    return pr.major >= 10 ? 1 : 0;
}

int mpcd_ctx_destroy(mpcd_ctx* c) {
    if (!c) return MPCD_OK;
    cudaSetDevice(c->device);
    fast_free(c);
    if (c->profP) cudaFree(c->profP);
    if (c->profN) cudaFree(c->profN);
    void* ptrs[] = {c->xb[0], c->xb[1], c->vb[0], c->vb[1], c->offb[0], c->offb[1], c->cellb[0], c->cellb[1],
                    c->v32b[0], c->v32b[1], c->pidb[0], c->pidb[1], c->cidStd, c->cidSrd, c->sortKeys, c->sortKeysSide,
                    c->idxStd.count, c->idxStd.start, c->idxStd.pos, c->idxStd.slots,
                    c->idxSrd.count, c->idxSrd.start, c->idxSrd.pos, c->idxSrd.slots,
                    c->blockSums, c->blockSumsWalls, c->W.bitsX, c->W.bitsY, c->W.wordCount, c->W.wordPrefix, c->W.events,
                    c->W.nEvents, c->W.normals, c->W.contrib, c->W.blockPartial, c->W.ints, c->W.srdShift,
                    c->wallOut, c->signs, c->seeds, c->zoneMoved, c->zoneCorr, c->overflow, c->nOverflow, c->ovDone,
                    c->zoneCost, c->zoneHist, c->zoneOrder, c->dStep, c->stepSeeds,
                    c->slotsLive, c->liveCnt, c->liveStart, c->liveTop, c->duScratch, c->zkRect, c->zkDiag, c->zkOut,
                    c->lparams, c->lmode, c->lcount, c->lsums, c->duLX, c->duLY, c->duLSum, c->redFeat,
                    c->ovMem, c->passOut, c->mask, c->refPx, c->refPy, c->refUx, c->refUy, c->refT, c->refRho,
                    c->refPkin, c->refPvir, c->refP, c->refNi, c->pdRaw, c->pdrive, c->eosX, c->eosY, c->duRX,
                    c->duRY, c->cols, c->partial, c->red, c->fieldTmp, c->fieldTmpN, c->vrep, c->cellOf, c->st};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int k = 0; k < 3; ++k) {
        if (c->lay[k].rects) cudaFree(c->lay[k].rects);
        if (c->lay[k].owner) cudaFree(c->lay[k].owner);
    }
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->side) cudaStreamSynchronize(c->side);
    if (c->walls) cudaStreamSynchronize(c->walls);
    for (cudaStream_t q : {c->up, c->down})
        if (q) cudaStreamSynchronize(q);
    for (cudaEvent_t e : {c->signsReady[0], c->signsReady[1], c->collDone, c->bcDone, c->wallsDone, c->sideDone, c->stdIdxDone,
                          c->upDone[0], c->upDone[1], c->inFree[0], c->inFree[1], c->outReady[0], c->outReady[1],
                          c->downDone[0], c->downDone[1]})
        if (e) cudaEventDestroy(e);
    for (double2* b : {c->jobIn[0], c->jobIn[1], c->jobOut[0], c->jobOut[1]})
        if (b) cudaFree(b);
    for (cudaStream_t q : {c->up, c->down})
        if (q) cudaStreamDestroy(q);
    for (auto& g : c->gexec)
        if (g) cudaGraphExecDestroy(g);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->walls) cudaStreamDestroy(c->walls);
    if (c->signsBuf[0]) cudaFree(c->signsBuf[0]);
    if (c->signsBuf[1]) cudaFree(c->signsBuf[1]);
    if (c->hst) cudaFreeHost(c->hst);
    if (c->hred) cudaFreeHost(c->hred);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return MPCD_OK;
}

int mpcd_ctx_create(const mpcd_params_c* params, int device, mpcd_ctx** out) {
    return mpcd_ctx_create_form(params, device, MPCD_FORM_F64, out);
}

int mpcd_ctx_create_form(const mpcd_params_c* params, int device, int32_t form, mpcd_ctx** out) {
    if (form != MPCD_FORM_F64 && form != MPCD_FORM_F32 && form != MPCD_FORM_FAST)
        return set_err(MPCD_ERR_INVALID_ARG, "unknown state form");
    if (!params || !out) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    int rc = validate(*params);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(MPCD_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return set_err(MPCD_ERR_INVALID_ARG, "device index out of range");
    mpcd_ctx* c = new mpcd_ctx();
    std::memset(c->ev, 0, sizeof(c->ev));
    c->device = device;
    c->pc = *params;
    c->P = make_dev_params(*params);
    c->n = params->n;
    c->Nc = params->Nc;
    auto fail = [&](int code) {
        mpcd_ctx_destroy(c);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "stream"));
    const int n = c->n, Nc = c->Nc;
    if (form == MPCD_FORM_FAST) {
        rc = fast_create(c, *params, device);
        if (rc) return fail(rc);
        *out = c;
        return MPCD_OK;
    }
#define ALLOC(p, cnt) \
    if ((rc = dalloc(&(p), (cnt)))) return fail(rc)
    c->f32 = form == MPCD_FORM_F32;
    for (int k = 0; k < 2; ++k) {
        if (c->f32) {
            ALLOC(c->offb[k], (size_t)n);
            ALLOC(c->cellb[k], (size_t)n);
            ALLOC(c->v32b[k], (size_t)n);
        } else {
            ALLOC(c->xb[k], (size_t)n);
            ALLOC(c->vb[k], (size_t)n);
        }
        ALLOC(c->pidb[k], (size_t)n);
    }
    ALLOC(c->cidStd, (size_t)n);
    ALLOC(c->cidSrd, (size_t)n);
    ALLOC(c->sortKeys, (size_t)n);
    ALLOC(c->sortKeysSide, (size_t)n);
    c->rankCells = rank_cells_per_block(n, Nc);
    for (CellIndex* I : {&c->idxStd, &c->idxSrd}) {
        ALLOC(I->count, (size_t)Nc);
        if (cudaMemset(I->count, 0, sizeof(int) * (size_t)std::max(Nc, 1)) != cudaSuccess)
            return fail(set_err(MPCD_ERR_CUDA, "index counts"));
        ALLOC(I->start, (size_t)Nc + 1);
        ALLOC(I->pos, (size_t)n);
        ALLOC(I->slots, (size_t)n);
    }
    c->nwords = (n + 31) / 32 + 1;
    c->blockSumsCap = (int)std::max<int64_t>(1, ((int64_t)std::max(Nc, c->nwords) + kScanTile - 1) / kScanTile) + 1;
    ALLOC(c->blockSums, (size_t)c->blockSumsCap);
    ALLOC(c->blockSumsWalls, (size_t)c->blockSumsCap);
    c->bcBlocks = blocks_for(n);
    BcWork& W = c->W;
    ALLOC(W.bitsX, (size_t)c->nwords);
    ALLOC(W.bitsY, (size_t)c->nwords);
    ALLOC(W.wordCount, (size_t)c->nwords);
    ALLOC(W.wordPrefix, (size_t)c->nwords + 1);
    W.eventCap = std::max(4096, std::min(n, std::max(65536, n / 8)));
    W.normalCap = 2 * W.eventCap;
    ALLOC(W.events, (size_t)W.eventCap);
    ALLOC(W.nEvents, 1);
    ALLOC(W.normals, 2 * (size_t)W.normalCap);
    ALLOC(W.contrib, (size_t)kWallDoubles * W.normalCap);
    ALLOC(W.blockPartial, (size_t)kWallDoubles * c->bcBlocks);
    ALLOC(W.ints, 4);
    ALLOC(W.srdShift, 2);
    ALLOC(c->wallOut, kWallDoubles);
    ALLOC(c->signs, (size_t)Nc);
    ALLOC(c->signsBuf[0], (size_t)Nc);
    ALLOC(c->signsBuf[1], (size_t)Nc);
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->signsReady[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->signsReady[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->collDone, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->walls, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->bcDone, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->wallsDone, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->stdIdxDone, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->sideDone, cudaEventDisableTiming) != cudaSuccess)
        return fail(set_err(MPCD_ERR_CUDA, "side stream"));
    ALLOC(c->dStep, 1);
    ALLOC(c->stepSeeds, (size_t)kStepSeeds);
    // zone layouts
    build_layout(*params, MPCD_LAYOUT_BASE, c->lay[0]);
    build_layout(*params, MPCD_LAYOUT_SHIFTED, c->lay[1]);
    build_layout(*params, MPCD_LAYOUT_SINGLE_FULL, c->lay[2]);
    int maxZones = 0, maxArea = 0, maxTX = 0, maxTY = 0;
    for (int k = 0; k < 3; ++k) {
        Layout& L = c->lay[k];
        ALLOC(L.rects, L.hrects.size());
        ALLOC(L.owner, (size_t)Nc);
        if (cudaMemcpy(L.rects, L.hrects.data(), L.hrects.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.owner, L.howner.data(), (size_t)Nc * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(set_err(MPCD_ERR_CUDA, "layout upload"));
        maxZones = std::max(maxZones, L.nZones);
        maxArea = std::max(maxArea, L.maxArea);
        maxTX = std::max(maxTX, L.maxTX);
        maxTY = std::max(maxTY, L.maxTY);
    }
    ALLOC(c->seeds, (size_t)maxZones * kMtN);
    ALLOC(c->zoneMoved, (size_t)maxZones);
    ALLOC(c->zoneCorr, (size_t)maxZones);
    ALLOC(c->overflow, (size_t)maxZones);
    ALLOC(c->zoneCost, (size_t)maxZones);
    ALLOC(c->zoneHist, (size_t)kCostBuckets);
    if (cudaMemset(c->zoneHist, 0, sizeof(int) * kCostBuckets) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "zone histogram"));
    ALLOC(c->zoneOrder, (size_t)maxZones);
    ALLOC(c->nOverflow, 1);
    ALLOC(c->ovDone, 1);
    if (cudaMemset(c->ovDone, 0, sizeof(int)) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "overflow block counter"));
    if (cudaMemset(c->nOverflow, 0, sizeof(int)) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "overflow counter"));
    ALLOC(c->passOut, 8);
    // collision tiles: room for 1.5x the mean particles per cell plus 8, per cell of a block
    {
        const double ppc = (double)n / (double)std::max(Nc, 1);
        bool ok = true;
#define MPCD_COLLIDE_ATTR(K)                                                                                          \
    {                                                                                                                 \
        const int cells = kCollideShape[K].cells;                                                                     \
        c->collideTiles[K] = std::max(256, std::min(8192, (int)(cells * (1.5 * ppc + 8.0))));                         \
        const size_t sm = (size_t)c->collideTiles[K] * (sizeof(double2) + sizeof(int));                               \
        ok = ok &&                                                                                                    \
             raise_smem((const void*)k_srd_collide<View64, kCollideShape[K].cells, kCollideShape[K].threads>, sm,      \
                        device) &&                                                                                    \
             raise_smem((const void*)k_srd_collide<View32, kCollideShape[K].cells, kCollideShape[K].threads>, sm,      \
                        device);                                                                                      \
    }
        MPCD_COLLIDE_ATTR(0)
        MPCD_COLLIDE_ATTR(1)
        MPCD_COLLIDE_ATTR(2)
        MPCD_COLLIDE_ATTR(3)
        MPCD_COLLIDE_ATTR(4)
        MPCD_COLLIDE_ATTR(5)
        MPCD_COLLIDE_ATTR(6)
#undef MPCD_COLLIDE_ATTR
        if (!ok) return fail(set_err(MPCD_ERR_CUDA, "collision shared memory attribute"));
    }
    // fast path: tiles of the base/shifted layouts in shared memory
    {
        const Layout& B = c->lay[0];
        const Layout& S = c->lay[1];
        const int area = std::max(B.maxArea, S.maxArea);
        const int tx = std::max(B.maxTX, S.maxTX), ty = std::max(B.maxTY, S.maxTY);
        c->zMaxCells = std::max(1, area);
        c->zWinCap = (tx + 4) * (ty + 4);
        c->zNsmCap = (tx + 2) * (ty + 2);
        const double g = std::max(1.0, params->gamma);
        // arena for the lists a zone materialises (receivers, donors): ~0.8 of the zone's
        // particles covers typical passes; a zone that runs out is re-run on the overflow path
        c->zArenaCap = ((int)std::ceil(0.8 * g * area) + 128 + 31) / 32 * 32;
        c->zSmem = ZoneMem<uint16_t>::bytes(c->zMaxCells, c->zWinCap, c->zArenaCap, c->zNsmCap);
        if (c->zSmem > 200 * 1024 || c->zArenaCap > 65535 || c->zMaxCells > 65535) {
            // too large for the shared-memory path (or its 16-bit offsets): every zone takes
            // the overflow path
            c->zMaxCells = 0;
            c->zSmem = ZoneMem<uint16_t>::bytes(0, 0, 0, 0);
        }
        if (!raise_smem((const void*)k_zone_pass<false>, c->zSmem, device) ||
            !raise_smem((const void*)k_zone_pass<true>, c->zSmem, device) ||
            !raise_smem((const void*)k_zone_serial, c->zSmem, device))
            return fail(set_err(MPCD_ERR_CUDA, "zone shared memory attribute"));
        // the phase-synchronous kernel: the most warps per block (16, 8 or 4) whose working
        // sets fit in 200 KB; MPCD_ZONE_SYNC_WARPS picks another (0: one zone per block)
        c->zSyncWarps = 0;
        if (c->zMaxCells > 0)
            for (int W : {16, 8, 4})
                if ((size_t)W * c->zSmem <= 200 * 1024) {
                    c->zSyncWarps = W;
                    break;
                }
        if (const char* e = std::getenv("MPCD_ZONE_SYNC_WARPS")) {
            const int v = std::atoi(e);
            if ((v == 0 || v == 4 || v == 8 || v == 16) && (size_t)v * c->zSmem <= 200 * 1024) c->zSyncWarps = v;
        }
        bool okSync = true;
#define MPCD_ZONE_SYNC_ATTR(K)                                                                         \
        if (c->zSyncWarps == K)                                                                        \
            okSync = raise_smem((const void*)k_zone_pass_sync<false, K>, (size_t)K * c->zSmem, device) && \
                     raise_smem((const void*)k_zone_pass_sync<true, K>, (size_t)K * c->zSmem, device);
        MPCD_ZONE_SYNC_ATTR(4)
        MPCD_ZONE_SYNC_ATTR(8)
        MPCD_ZONE_SYNC_ATTR(16)
#undef MPCD_ZONE_SYNC_ATTR
        if (!okSync) return fail(set_err(MPCD_ERR_CUDA, "zone shared memory attribute"));
        c->ovMaxCells = maxArea;
        c->ovWinCap = (maxTX + 4) * (maxTY + 4);
        c->ovNsmCap = (maxTX + 2) * (maxTY + 2);
        // every materialised list fits in (particles of the zone + 4 per cell) entries after
        // compaction; bound the zone's particles by all particles
        c->ovArenaCap = (int)std::min<int64_t>((int64_t)n + 4LL * maxArea + 4096, (1LL << 31) - 1);
        c->ovPerBlock = (ZoneMem<int>::bytes(c->ovMaxCells, c->ovWinCap, c->ovArenaCap, c->ovNsmCap) + 255) / 256 * 256;
        ALLOC(c->ovMem, c->ovPerBlock * (size_t)c->ovBlocks);
    }
    // closure
    const auto mask = interzone_mask(*params, c->lay[params->zoneSingleFullDomainMode ? 2 : 0],
                                     c->lay[params->zoneSingleFullDomainMode ? 2 : 1]);
    c->nMasked = 0;
    for (int m : mask) c->nMasked += (m == 1);
    ALLOC(c->mask, (size_t)Nc);
    if (cudaMemcpy(c->mask, mask.data(), (size_t)Nc * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_err(MPCD_ERR_CUDA, "mask upload"));
    for (double** p : {&c->refPx, &c->refPy, &c->refUx, &c->refUy, &c->refT, &c->refRho, &c->refPkin, &c->refPvir,
                       &c->refP, &c->pdRaw, &c->pdrive, &c->eosX, &c->eosY, &c->duRX, &c->duRY})
        ALLOC(*p, (size_t)Nc);
    ALLOC(c->refNi, (size_t)Nc);
    ALLOC(c->cols, (size_t)std::max<int64_t>((int64_t)Nc * kKickCols, 3LL * n));
    c->partialCap = (int)(((int64_t)std::max(Nc, n) + 8191) / 8192 + 1) * kRedMaxCols;
    ALLOC(c->partial, (size_t)c->partialCap);
    ALLOC(c->red, 32);
    ALLOC(c->fieldTmp, 11 * (size_t)Nc);
    ALLOC(c->fieldTmpN, (size_t)Nc);
    ALLOC(c->vrep, (size_t)n);
    ALLOC(c->cellOf, (size_t)n);
    ALLOC(c->st, 1);
#undef ALLOC
    if (cudaMemset(c->st, 0, sizeof(DevStatus)) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "memset"));
    if (cudaMallocHost((void**)&c->hst, sizeof(DevStatus)) != cudaSuccess ||
        cudaMallocHost((void**)&c->hred, 32 * sizeof(double)) != cudaSuccess)
        return fail(set_err(MPCD_ERR_CUDA, "pinned host"));
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(set_err(MPCD_ERR_CUDA, "event"));
    *out = c;
    return MPCD_OK;
}

void* mpcd_ctx_stream(mpcd_ctx* c) { return c ? (void*)c->stream : nullptr; }

static int set_state_impl(mpcd_ctx* c, const double* x, const double* v, int64_t n, cudaMemcpyKind kind) {
    if (!c || !x || !v) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (n != c->n) return set_err(MPCD_ERR_INVALID_ARG, "state size does not match params.n");
    CUDA_TRY(cudaSetDevice(c->device));
    if (c->fast) return fast_set_state(c, x, v, kind);
    c->xv = 0;
    c->pp = 0;
    c->xflip = 0;
    c->slotsSorted = false;
    if (n > 0 && c->f32) {
        // staged through FP64 scratch, then split into cell, FP32 offset and FP32 velocity
        double2 *tx = nullptr, *tv = nullptr;
        int rc = dalloc(&tx, (size_t)n);
        if (!rc) rc = dalloc(&tv, (size_t)n);
        if (!rc && (cudaMemcpyAsync(tx, x, sizeof(double2) * (size_t)n, kind, c->stream) != cudaSuccess ||
                    cudaMemcpyAsync(tv, v, sizeof(double2) * (size_t)n, kind, c->stream) != cudaSuccess))
            rc = set_err(MPCD_ERR_CUDA, "state upload");
        if (!rc) {
            k_f32_from<<<blocks_for(n), kThreads, 0, c->stream>>>(c->P, tx, tv, (int)n, view32(c, 0)); ++c->launches;
            k_iota<<<blocks_for(n), kThreads, 0, c->stream>>>(c->pidb[0], (int)n); ++c->launches;
            if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "state conversion");
        }
        cudaFree(tx);
        cudaFree(tv);
        if (rc) return rc;
    } else if (n > 0) {
        CUDA_TRY(cudaMemcpyAsync(c->xb[0], x, sizeof(double2) * (size_t)n, kind, c->stream));
        CUDA_TRY(cudaMemcpyAsync(c->vb[0], v, sizeof(double2) * (size_t)n, kind, c->stream));
        k_iota<<<blocks_for(n), kThreads, 0, c->stream>>>(c->pidb[0], (int)n); ++c->launches;
        CUDA_TRY(cudaGetLastError());
    }
    invalidate_positions(c);
    return check_device(c);
}

int mpcd_set_state(mpcd_ctx* c, const double* x, const double* v, int64_t n) {
    return set_state_impl(c, x, v, n, cudaMemcpyHostToDevice);
}
int mpcd_set_state_device(mpcd_ctx* c, const double* x, const double* v, int64_t n) {
    return set_state_impl(c, x, v, n, cudaMemcpyDeviceToDevice);
}

static int get_state_impl(mpcd_ctx* c, double* x, double* v, bool toHost) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    CUDA_TRY(cudaSetDevice(c->device));
    if (c->fast) return fast_get_state(c, x, v, toHost);
    if (c->n == 0) return MPCD_OK;
    const cudaMemcpyKind k = toHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (c->f32) {
        double2 *tx = nullptr, *tv = nullptr;
        int rc = dalloc(&tx, (size_t)c->n);
        if (!rc) rc = dalloc(&tv, (size_t)c->n);
        if (!rc) {
            k_f32_by_pid<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, view32(c, c->xv), c->pidb[c->pp], c->n, tx, tv);
            ++c->launches;
            if ((x && cudaMemcpyAsync(x, tx, sizeof(double2) * (size_t)c->n, k, c->stream) != cudaSuccess) ||
                (v && cudaMemcpyAsync(v, tv, sizeof(double2) * (size_t)c->n, k, c->stream) != cudaSuccess) ||
                cudaStreamSynchronize(c->stream) != cudaSuccess)
                rc = set_err(MPCD_ERR_CUDA, "state download");
        }
        cudaFree(tx);
        cudaFree(tv);
        if (rc) return rc;
        return check_device(c);
    }
    double2* tx = spare_x(c);
    double2* tv = c->vb[c->xv ^ 1];
    k_gather_by_pid<<<blocks_for(c->n), kThreads, 0, c->stream>>>(cur_x(c), c->vb[c->xv], c->pidb[c->pp], c->n, tx, tv); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    if (x) CUDA_TRY(cudaMemcpyAsync(x, tx, sizeof(double2) * (size_t)c->n, k, c->stream));
    if (v) CUDA_TRY(cudaMemcpyAsync(v, tv, sizeof(double2) * (size_t)c->n, k, c->stream));
    return check_device(c);
}

int mpcd_get_state(mpcd_ctx* c, double* x, double* v) { return get_state_impl(c, x, v, true); }
int mpcd_get_state_device(mpcd_ctx* c, double* x, double* v) { return get_state_impl(c, x, v, false); }

int mpcd_stream(mpcd_ctx* c) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    CUDA_TRY(cudaSetDevice(c->device));
    k_stream_only<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, cur_x(c), c->vb[c->xv]); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    invalidate_positions(c);
    return check_device(c);
}

int mpcd_apply_bc(mpcd_ctx* c, uint64_t seed, mpcd_wallinfo_c* info) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = run_bc(c, false, seed, nullptr, nullptr, info != nullptr);
    if (rc) return rc;
    invalidate_positions(c);
    rc = check_device(c);
    if (rc) return rc;
    if (info) {
        int ints[4];
        double d[kWallDoubles];
        CUDA_TRY(cudaMemcpy(ints, c->W.ints, sizeof ints, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(d, c->wallOut, sizeof d, cudaMemcpyDeviceToHost));
        info->nBot = ints[0]; info->nTop = ints[1]; info->nLeft = ints[2]; info->nRight = ints[3];
        info->dEwall = d[0]; info->dPxBot = d[1]; info->dPxTop = d[2]; info->dPyBot = d[3]; info->dPyTop = d[4];
        info->dPxLeft = d[5]; info->dPxRight = d[6]; info->dPyLeft = d[7]; info->dPyRight = d[8];
    }
    return MPCD_OK;
}

int mpcd_srd_shift_cells(mpcd_ctx* c, uint64_t seed, int32_t* cid_out) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    CUDA_TRY(cudaSetDevice(c->device));
    k_srd_shift<<<1, 1, 0, c->stream>>>(c->P, seed, c->W.srdShift, nullptr); ++c->launches;
    k_srd_cells<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, cur_x(c), c->W.srdShift, c->cidSrd); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    c->srdCellsValid = true;
    if (cid_out && c->n > 0) {
        int* tmp = c->idxSrd.pos;  // scratch: particle-id order
        k_int_by_pid<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->cidSrd, c->pidb[c->pp], c->n, tmp); ++c->launches;
        CUDA_TRY(cudaMemcpyAsync(cid_out, tmp, sizeof(int) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    }
    return check_device(c);
}

int mpcd_srd_collide(mpcd_ctx* c, uint64_t seed) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    if (!c->srdCellsValid) return set_err(MPCD_ERR_STATE, "no SRD cell ids: call mpcd_srd_shift_cells first");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = run_collide(c, seed);
    if (rc) return rc;
    return check_device(c);
}

int mpcd_srd_collide_cells(mpcd_ctx* c, const int32_t* cid, uint64_t seed) {
    if (!c || !cid) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    CUDA_TRY(cudaSetDevice(c->device));
    if (c->n > 0) {
        int* tmp = c->idxSrd.pos;
        CUDA_TRY(cudaMemcpyAsync(tmp, cid, sizeof(int) * (size_t)c->n, cudaMemcpyHostToDevice, c->stream));
        k_int_to_slots<<<blocks_for(c->n), kThreads, 0, c->stream>>>(tmp, c->pidb[c->pp], c->n, c->Nc, c->cidSrd, c->st); ++c->launches;
        CUDA_TRY(cudaGetLastError());
        int rc = check_device(c);
        if (rc) return rc;
    }
    c->srdCellsValid = true;
    return mpcd_srd_collide(c, seed);
}

static int fields_to_host(mpcd_ctx* c, const FieldsOut& o, mpcd_cellfields_c* out) {
    const size_t nc = (size_t)c->Nc;
    if (out->N) CUDA_TRY(cudaMemcpyAsync(out->N, o.N, nc * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    const double* src[10] = {o.Ux, o.Uy, o.Px, o.Py, o.T, o.rho, o.Pkin, o.Pvir, o.P, o.rhoTarget};
    double* dst[10] = {out->Ux, out->Uy, out->Px, out->Py, out->T, out->rho, out->Pkin, out->Pvir, out->P, out->rhoTarget};
    for (int k = 0; k < 10; ++k)
        if (dst[k]) CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], nc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return MPCD_OK;
}

static FieldsOut tmp_fields(mpcd_ctx* c) {
    FieldsOut o{};
    double* b = c->fieldTmp;
    const size_t nc = (size_t)c->Nc;
    o.N = c->fieldTmpN;
    o.Ux = b; o.Uy = b + nc; o.Px = b + 2 * nc; o.Py = b + 3 * nc; o.T = b + 4 * nc; o.rho = b + 5 * nc;
    o.Pkin = b + 6 * nc; o.Pvir = b + 7 * nc; o.P = b + 8 * nc; o.rhoTarget = b + 9 * nc;
    return o;
}

int mpcd_cell_fields(mpcd_ctx* c, double rho_target, mpcd_cellfields_c* out) {
    if (!c || !out) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = ensure_std_index(c);
    if (rc) return rc;
    const FieldsOut o = tmp_fields(c);
    k_cell_fields<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->idxStd.start, c->idxStd.slots, view64(c, c->xv), rho_target, o); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    rc = fields_to_host(c, o, out);
    if (rc) return rc;
    return check_device(c);
}

int mpcd_save_ref(mpcd_ctx* c) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = run_save_ref(c);
    if (rc) return rc;
    return check_device(c);
}

static int pass_metrics_to_host(mpcd_ctx* c, int mode, mpcd_pass_metrics_c* m) {
    double d[4];
    CUDA_TRY(cudaMemcpy(d, c->passOut + (mode == MPCD_LAYOUT_SHIFTED ? 4 : 0), sizeof d, cudaMemcpyDeviceToHost));
    std::memset(m, 0, sizeof *m);
    const Layout& L = c->lay[c->pc.zoneSingleFullDomainMode ? 2 : mode];
    m->nZones = L.nZones;
    m->nThreadsRequested = 1;
    m->nThreadsUsed = L.nZones;
    m->nParticlesMovedDense = (int)d[0];
    m->nParticlesMovedSparse = (int)d[1];
    m->corrRmsDU = d[2];
    m->corrMaxDU = d[3];
    return MPCD_OK;
}

int mpcd_zone_pass(mpcd_ctx* c, int32_t mode, uint64_t seed_base, mpcd_pass_metrics_c* metrics) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    if (!c->pc.useIncompressibleRedistribution || !c->pc.useZoneRedistribution)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl requires useIncompressibleRedistribution=true and useZoneRedistribution=true");
    if (c->pc.redistributionEnableSurfaceTopology || c->pc.redistributionWallWettingEnabled || c->pc.useInterfaceVelocityReorientation)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl is restricted to no surface / no wetting / no reorientation");
    CUDA_TRY(cudaSetDevice(c->device));
    if (mode < 0 || mode > 2) mode = MPCD_LAYOUT_BASE;
    CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
    int rc = run_zone_pass(c, mode, seed_base);
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
    rc = check_device(c);
    if (rc) return rc;
    if (metrics) {
        rc = pass_metrics_to_host(c, mode, metrics);
        if (rc) return rc;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
        metrics->timeKernel = ms * 1e-3;
    }
    return MPCD_OK;
}

int mpcd_zone_owner_map(mpcd_ctx* c, int32_t mode, int32_t* owner_out) {
    if (!c || !owner_out) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (mode < 0 || mode > 2) mode = MPCD_LAYOUT_BASE;
    if (c->pc.zoneSingleFullDomainMode) mode = MPCD_LAYOUT_SINGLE_FULL;
    std::memcpy(owner_out, c->lay[mode].howner.data(), sizeof(int32_t) * (size_t)c->Nc);
    return MPCD_OK;
}

static void closure_metrics_from(mpcd_ctx* c, const double* r, mpcd_closure_metrics_c* m) {
    // r: [0] num [1] den [2..10] kick columns
    std::memset(m, 0, sizeof *m);
    const double num = r[0], den = r[1];
    double opt = 0.0;
    if (std::isfinite(num) && std::isfinite(den) && den > 0.0) opt = std::max(num / den, 0.0);
    m->betaRepairNum = num;
    m->betaRepairDen = den;
    m->betaRepairOpt = opt;
    if (!c->pc.useOptimalBetaRepair || !std::isfinite(opt) || !std::isfinite(den) || den < 1e-20)
        m->betaRepairApplied = c->pc.betaRepair;
    else
        m->betaRepairApplied = std::clamp(opt, 0.0, 2.0);
    m->betaEOSApplied = c->pc.betaEOS;
    const double nn = (double)std::max(c->n, 1);
    m->rmsRepairDU = (c->n > 0) ? std::sqrt(r[2] / nn) : 0.0;
    m->maxRepairDU = (c->n > 0) ? r[3] : 0.0;
    m->meanAbsRepairDU = r[4] / (double)std::max(c->Nc, 1);
    m->rmsEOSDU = (c->n > 0) ? std::sqrt(r[5] / nn) : 0.0;
    m->maxEOSDU = (c->n > 0) ? r[6] : 0.0;
    m->momentumDeltaX = r[9] - r[7];
    m->momentumDeltaY = r[10] - r[8];
    m->nMaskedInterzoneCells = c->nMasked;
}

int mpcd_zone_pass_serial(mpcd_ctx* c, int32_t mode, uint64_t seed_base, mpcd_pass_metrics_c* metrics) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    if (!c->pc.useIncompressibleRedistribution || !c->pc.useZoneRedistribution)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass requires useIncompressibleRedistribution=true and useZoneRedistribution=true");
    if (c->pc.redistributionEnableSurfaceTopology || c->pc.redistributionWallWettingEnabled || c->pc.useInterfaceVelocityReorientation)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass is restricted to no surface / no wetting / no reorientation");
    CUDA_TRY(cudaSetDevice(c->device));
    if (mode < 0 || mode > 2) mode = MPCD_LAYOUT_BASE;
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    CUDA_TRY(cudaEventRecord(a, c->stream));
    int rc = run_zone_pass_serial(c, mode, seed_base);
    CUDA_TRY(cudaEventRecord(b, c->stream));
    if (rc == MPCD_OK) rc = check_device(c);
    float ms = 0.f;
    if (rc == MPCD_OK) cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (metrics) {
        rc = pass_metrics_to_host(c, mode, metrics);
        if (rc) return rc;
        metrics->nThreadsUsed = 1;
        metrics->timeKernel = ms * 1e-3;
    }
    return MPCD_OK;
}

// ---------------------------------------------------------------- single zones
// (reference include/zone_pass.h:60-72: build_zone_layout, run_zone_kernel_inplace,
// build_particle_ids_in_zone)

int mpcd_zone_layout(const mpcd_params_c* params, int32_t mode, int32_t* nzones, int32_t* rects, int32_t cap) {
    if (!params || !nzones) return set_err(MPCD_ERR_INVALID_ARG, "mpcd_zone_layout: null argument");
    if (params->Nx <= 0 || params->Ny <= 0 || params->zoneTileNx <= 0 || params->zoneTileNy <= 0)
        return set_err(MPCD_ERR_INVALID_ARG, "mpcd_zone_layout: grid and tile sizes must be positive");
    if (mode != MPCD_LAYOUT_SHIFTED && mode != MPCD_LAYOUT_SINGLE_FULL) mode = MPCD_LAYOUT_BASE;
    if (params->zoneSingleFullDomainMode) mode = MPCD_LAYOUT_SINGLE_FULL;
    mpcd_params_c p = *params;
    p.Nc = p.Nx * p.Ny;
    Layout L;
    build_layout(p, mode, L);
    *nzones = L.nZones;
    if (rects) {
        if (cap < L.nZones) return set_err(MPCD_ERR_CAPACITY, "mpcd_zone_layout: rects holds fewer than nzones zones");
        for (int z = 0; z < L.nZones; ++z) {
            rects[4 * z] = L.hrects[z].x;
            rects[4 * z + 1] = L.hrects[z].y;
            rects[4 * z + 2] = L.hrects[z].z;
            rects[4 * z + 3] = L.hrects[z].w;
        }
    }
    return MPCD_OK;
}

}  // extern "C"

namespace mpcd_dev {
// per cell of a cell index: count, count^2, out-of-band flag (bulk thresholds), non-empty flag
__global__ void k_zone_count_cols(const uint64_t* __restrict__ start, int Nc, double highThr, double lowThr,
                                  double* __restrict__ cols) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nc) return;
    const double n = (double)((uint32_t)start[c + 1] - (uint32_t)start[c]);
    cols[4 * (size_t)c] = n;
    cols[4 * (size_t)c + 1] = __dmul_rn(n, n);
    cols[4 * (size_t)c + 2] = ((n > highThr) || (n > 0.0 && n < lowThr)) ? 1.0 : 0.0;
    cols[4 * (size_t)c + 3] = (n > 0.0) ? 1.0 : 0.0;
}

// flag[pid] = 1 for the particles whose standard-grid cell lies in R = (x0, x1, y0, y1)
__global__ void k_rect_flags(const int* __restrict__ cid, const int* __restrict__ pid, int n, int Ny, int4 R,
                             uint8_t* __restrict__ flag) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int c = cid[s];
    const int ix = c / Ny, iy = c - ix * Ny;
    flag[pid[s]] = (ix >= R.x && ix < R.y && iy >= R.z && iy < R.w) ? 1 : 0;
}

// per chunk of `chunk` consecutive ids: the number of flagged ids
__global__ void k_rect_chunk_counts(const uint8_t* __restrict__ flag, int n, int chunk, uint64_t* __restrict__ counts) {
    __shared__ int sh[kThreads];
    const int64_t a = (int64_t)blockIdx.x * chunk, b = min((int64_t)n, a + chunk);
    int k = 0;
    for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) k += flag[i];
    sh[threadIdx.x] = k;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[blockIdx.x] = (uint64_t)sh[0];
}

// per chunk: its flagged ids, ascending, from the chunk's offset on
__global__ void k_rect_chunk_write(const uint8_t* __restrict__ flag, int n, int chunk, const uint64_t* __restrict__ offs,
                                   int* __restrict__ ids) {
    __shared__ int warpTot[kThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int64_t a = (int64_t)blockIdx.x * chunk, b = min((int64_t)n, a + chunk);
    int64_t base = (int64_t)offs[blockIdx.x];
    for (int64_t i0 = a; i0 < b; i0 += blockDim.x) {
        const int64_t i = i0 + t;
        const bool f = i < b && flag[i];
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) warpTot[w] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            if (k < w) before += warpTot[k];
            total += warpTot[k];
        }
        if (f) ids[base + before + __popc(m & ((1u << lane) - 1u))] = (int)i;
        base += total;
        __syncthreads();
    }
}
}  // namespace mpcd_dev

extern "C" {

static int check_rect(const mpcd_ctx* c, int32_t x0, int32_t x1, int32_t y0, int32_t y1) {
    if (x0 < 0 || y0 < 0 || x1 > c->pc.Nx || y1 > c->pc.Ny || x0 >= x1 || y0 >= y1)
        return set_err(MPCD_ERR_INVALID_ARG, "zone rectangle outside the grid or empty");
    return MPCD_OK;
}

int mpcd_particle_ids_in_rect(mpcd_ctx* c, int32_t x0, int32_t x1, int32_t y0, int32_t y1, int32_t* ids_out,
                              int64_t* count) {
    if (!c || !count) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    int rc = check_rect(c, x0, x1, y0, y1);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(c->device));
    *count = 0;
    if (c->n == 0) return MPCD_OK;
    if (!c->cidStdValid) {
        k_std_cells<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, view64(c, c->xv), c->cidStd); ++c->launches;
        c->cidStdValid = true;
    }
    // scratch in sortKeys (8n bytes): n flag bytes, then the chunk counts and their scan
    const int chunk = (int)std::max<int64_t>(4096, ((int64_t)c->n + kSmallScan - 1) / kSmallScan);
    const int nChunks = (int)(((int64_t)c->n + chunk - 1) / chunk);
    uint8_t* flag = reinterpret_cast<uint8_t*>(c->sortKeys);
    uint64_t* counts = c->sortKeys + ((size_t)c->n + 7) / 8;
    uint64_t* offs = counts + nChunks;
    if ((size_t)(((size_t)c->n + 7) / 8 + 2 * (size_t)nChunks + 1) > (size_t)c->n)
        return set_err(MPCD_ERR_CAPACITY, "particle ids: scratch too small");
    k_rect_flags<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->cidStd, c->pidb[c->pp], c->n, c->pc.Ny,
                                                               make_int4(x0, x1, y0, y1), flag); ++c->launches;
    k_rect_chunk_counts<<<nChunks, kThreads, 0, c->stream>>>(flag, c->n, chunk, counts); ++c->launches;
    rc = scan_u64(c, counts, nChunks, offs);
    if (rc) return rc;
    uint64_t total = 0;
    CUDA_TRY(cudaMemcpyAsync(&total, offs + nChunks, sizeof total, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    *count = (int64_t)total;
    if (ids_out && total > 0) {
        int* dIds = c->cidSrd;  // n ints, free outside the SRD phase
        k_rect_chunk_write<<<nChunks, kThreads, 0, c->stream>>>(flag, c->n, chunk, offs, dIds); ++c->launches;
        CUDA_TRY(cudaMemcpyAsync(ids_out, dIds, sizeof(int32_t) * (size_t)total, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        c->srdCellsValid = false;
    }
    return check_device(c);
}

int mpcd_zone_kernel_inplace(mpcd_ctx* c, int32_t x0, int32_t x1, int32_t y0, int32_t y1, uint64_t seed,
                             mpcd_zone_kernel_stats_c* out) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    if (c->pc.redistributionEnableSurfaceTopology || c->pc.redistributionWallWettingEnabled || c->pc.useInterfaceVelocityReorientation)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_kernel is restricted to no surface / no wetting / no reorientation");
    int rc = check_rect(c, x0, x1, y0, y1);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(c->device));
    if (!c->zkRect) {
        CUDA_TRY(cudaMalloc(&c->zkRect, sizeof(int4)));
        CUDA_TRY(cudaMalloc(&c->zkDiag, 8 * sizeof(double)));
        CUDA_TRY(cudaMalloc(&c->zkOut, 32 * sizeof(double)));
    }
    const int4 R = make_int4(x0, x1, y0, y1);
    CUDA_TRY(cudaMemcpyAsync(c->zkRect, &R, sizeof R, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemsetAsync(c->zkOut, 0, 32 * sizeof(double), c->stream));
    // global kinetic energy and momentum before (zk[0..2]: E, Px, Py)
    if (c->n > 0) {
        WITH_VIEW(c->xv, k_particle_cols<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, c->n, c->cols)); ++c->launches;
        rc = reduce_cols(c, c->cols, c->n, 3, 0u, c->zkOut);
        if (rc) return rc;
    }
    // the zone: seed = seedBase + 104729 (0 + 1) in the serial kernel's schedule
    rc = launch_zone_serial(c, c->zkRect, c->lay[MPCD_LAYOUT_BASE].owner, 1, seed - 104729ULL, c->zkDiag, c->zkOut + 8);
    if (rc) return rc;
    // after: counts (zk[12..15]) and global sums (zk[3..5])
    k_std_cells<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, view64(c, c->xv), c->cidStd); ++c->launches;
    c->cidStdValid = true;
    rc = ensure_std_index(c);
    if (rc) return rc;
    k_zone_count_cols<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->idxStd.start, c->Nc, c->P.highThr, c->P.lowThrBulk,
                                                                      c->cols); ++c->launches;
    rc = reduce_cols(c, c->cols, c->Nc, 4, 0u, c->zkOut + 12);
    if (rc) return rc;
    if (c->n > 0) {
        WITH_VIEW(c->xv, k_particle_cols<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, c->n, c->cols)); ++c->launches;
        rc = reduce_cols(c, c->cols, c->n, 3, 0u, c->zkOut + 3);
        if (rc) return rc;
    }
    CUDA_TRY(cudaGetLastError());
    rc = check_device(c);
    if (rc) return rc;
    if (!out) return MPCD_OK;
    double zk[32], dg[8];
    int2 moved;
    double2 corr;
    CUDA_TRY(cudaMemcpy(zk, c->zkOut, sizeof zk, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(dg, c->zkDiag, sizeof dg, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&moved, c->zoneMoved, sizeof moved, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&corr, c->zoneCorr, sizeof corr, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    // stats (src/zone_pass.cpp:764-767,855-858,911-922)
    out->stats[0] = dg[6];
    out->stats[1] = dg[7];
    out->stats[2] = out->stats[3] = (double)moved.x + (double)moved.y;
    out->stats[4] = corr.x;
    out->stats[5] = corr.y;
    out->movedDense = moved.x;
    out->movedSparse = moved.y;
    // diag (src/zone_pass.cpp:924-970); every cell is active (build_active_mask_vec)
    const double Nc = (double)std::max(1, c->Nc);
    const double mean = zk[12] / Nc;
    double var = zk[13] / Nc - mean * mean;
    if (var < 0.0) var = 0.0;
    out->diag[0] = std::sqrt(var) / std::max(c->pc.gamma, 1e-30);
    out->diag[1] = zk[14] / Nc;
    const double dPx = zk[4] - zk[1], dPy = zk[5] - zk[2];
    out->diag[2] = std::sqrt(dPx * dPx + dPy * dPy);
    out->diag[3] = dg[3] > 0.0 ? std::sqrt(dg[2] / dg[3]) : 0.0;
    out->diag[4] = dg[5] > 0.0 ? std::sqrt(dg[4] / dg[5]) : 0.0;
    out->diag[5] = zk[3] - zk[0];
    out->diag[6] = std::numeric_limits<double>::quiet_NaN();
    out->diag[7] = 0.0;
    const double nVel = zk[15];
    out->diag[8] = nVel > 0.0 ? std::sqrt(dg[0] / nVel) : 0.0;
    out->diag[9] = nVel > 0.0 ? std::sqrt(dg[1] / nVel) : 0.0;
    return MPCD_OK;
}

int mpcd_liquid_closure(mpcd_ctx* c, mpcd_closure_metrics_c* metrics, mpcd_closure_detail_c* detail) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (c->f32 || c->fast) return set_err(MPCD_ERR_INVALID_ARG, "the FP32 precision and fast forms run the whole step only (mpcd_step*, state I/O, metrics)");
    if (!c->pc.useLiquidClosure) return set_err(MPCD_ERR_INVALID_ARG, "run_liquid_closure requires useLiquidClosure=true");
    CUDA_TRY(cudaSetDevice(c->device));
    const bool wantRep = detail && (detail->repairedV || detail->repairedX || detail->repairedFields.N ||
                                    detail->repairedFields.Px || detail->repairedFields.Ux || detail->repairedFields.T);
    int rc;
    if (detail) {  // fields of the red state, before the kicks
        if (!c->refValid) return set_err(MPCD_ERR_STATE, "liquid closure needs a saved reference state (mpcd_save_ref)");
        rc = ensure_std_index(c);
        if (rc) return rc;
        const FieldsOut o = tmp_fields(c);
        k_cell_fields<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->idxStd.start, c->idxStd.slots, view64(c, c->xv), c->P.rhoTarget, o); ++c->launches;
        rc = fields_to_host(c, o, &detail->redFields);
        if (rc) return rc;
        CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    rc = run_closure(c, false, wantRep, true);
    if (rc) return rc;
    // pdrive sums for the means
    rc = reduce_cols(c, c->pdRaw, c->Nc, 1, 0u, c->red + 16);
    if (rc) return rc;
    rc = reduce_cols(c, c->pdrive, c->Nc, 1, 0u, c->red + 17);
    if (rc) return rc;
    rc = check_device(c);
    if (rc) return rc;
    double r[18];
    CUDA_TRY(cudaMemcpy(r, c->red, sizeof r, cudaMemcpyDeviceToHost));
    mpcd_closure_metrics_c m;
    closure_metrics_from(c, r, &m);
    m.meanPdriveRaw = (c->Nc > 0) ? r[16] / (double)c->Nc : 0.0;
    m.meanPdrive = (c->Nc > 0) ? r[17] / (double)c->Nc : 0.0;
    if (metrics) *metrics = m;
    if (detail) {
        const size_t nc = (size_t)c->Nc;
        FieldsOut ref{};
        ref.N = c->refNi; ref.Ux = c->refUx; ref.Uy = c->refUy; ref.Px = c->refPx; ref.Py = c->refPy; ref.T = c->refT;
        ref.rho = c->refRho; ref.Pkin = c->refPkin; ref.Pvir = c->refPvir; ref.P = c->refP; ref.rhoTarget = nullptr;
        mpcd_cellfields_c rf = detail->refFields;
        if (rf.rhoTarget) {
            std::vector<double> t(nc, c->P.rhoTarget);
            std::memcpy(rf.rhoTarget, t.data(), nc * sizeof(double));
            rf.rhoTarget = nullptr;
        }
        rc = fields_to_host(c, ref, &rf);
        if (rc) return rc;
        const double* src[6] = {c->pdRaw, c->pdrive, c->duRX, c->duRY, c->eosX, c->eosY};
        double* dst[6] = {detail->pdriveRaw, detail->pdrive, detail->duRepairX, detail->duRepairY, detail->duEOSX, detail->duEOSY};
        for (int k = 0; k < 6; ++k)
            if (dst[k]) CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], nc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (detail->interzoneMask) CUDA_TRY(cudaMemcpyAsync(detail->interzoneMask, c->mask, nc * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        const FieldsOut o = tmp_fields(c);
        if (wantRep) {
            // repaired state: positions unchanged, velocities = vrep
            if (detail->repairedX || detail->repairedV) {
                k_gather_by_pid<<<blocks_for(c->n), kThreads, 0, c->stream>>>(cur_x(c), c->vrep, c->pidb[c->pp], c->n,
                                                                              spare_x(c), c->vb[c->xv ^ 1]); ++c->launches;
                if (detail->repairedX) CUDA_TRY(cudaMemcpyAsync(detail->repairedX, spare_x(c), sizeof(double2) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
                if (detail->repairedV) CUDA_TRY(cudaMemcpyAsync(detail->repairedV, c->vb[c->xv ^ 1], sizeof(double2) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
                CUDA_TRY(cudaStreamSynchronize(c->stream));
            }
            k_cell_fields<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->idxStd.start, c->idxStd.slots, View64{nullptr, c->vrep}, c->P.rhoTarget, o); ++c->launches;
            rc = fields_to_host(c, o, &detail->repairedFields);
            if (rc) return rc;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
        }
        k_cell_fields<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->idxStd.start, c->idxStd.slots, view64(c, c->xv), c->P.rhoTarget, o); ++c->launches;
        rc = fields_to_host(c, o, &detail->outFields);
        if (rc) return rc;
        rc = check_device(c);
        if (rc) return rc;
    }
    return MPCD_OK;
}


// ---------------------------------------------------------------- the step
static int count_metrics(mpcd_ctx* c, double* dst /* device: 3 doubles */) {
    k_count_cols<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->idxStd.start, c->Nc, c->P.highThr, c->P.lowThrBulk, c->cols); ++c->launches;
    CUDA_TRY(cudaGetLastError());
    return reduce_cols(c, c->cols, c->Nc, 3, 0u, dst);
}

// One iteration of the profiled benchmark loop (reference
// src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:241-279) with its seeds.
// The step in three parts around its two zone kernels: head (stream, walls, collision,
// reference fields, base-pass prep), mid (base-pass finish, shifted-pass prep), tail
// (shifted-pass finish, closure and re-sort). step_once runs them with each replica's own
// zone kernels; a batch runs the zone kernels of all its replicas in one launch.
// step_mid and step_tail begin with the finish of a zone pass; their _b parts are the rest, so
// that a batch can run the finish and the following index build for all replicas at once.
static int step_head(mpcd_ctx* c, int64_t step, bool metrics, Prof* pf) {
    const uint64_t s = (uint64_t)step;
    if (metrics) CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
    mark(c, pf, -1);
    k_srd_shift<<<1, 1, 0, c->stream>>>(c->P, 130363ULL + 10007ULL * s, c->W.srdShift,
                                        c->graphMode ? c->stepSeeds : nullptr, c->graphMode ? c->dStep : nullptr,
                                        c->stepSeeds); ++c->launches;
    const bool overlap = pf == nullptr && c->walls;
    int rc = run_bc(c, true, 104729ULL + 10007ULL * s, c->cidStd, c->cidSrd, metrics, pf, overlap);
    if (rc) return rc;
    c->cidStdValid = true;
    c->srdCellsValid = true;
    c->idxStdValid = false;
    if (overlap) {
        // the standard-grid index on the walls stream, after the wall kernels (whose end the
        // collision waits for), beside the SRD index and the collision on the main stream
        rc = build_index(c, c->cidStd, c->idxStd, nullptr, -1, c->walls, c->sortKeysSide, c->blockSumsWalls);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(c->stdIdxDone, c->walls));
        c->stdIdxPending = true;
        c->idxStdValid = true;
    }
    rc = run_collide(c, 433494437ULL + 10007ULL * s, pf, step);
    if (rc) return rc;
    rc = run_save_ref(c, pf, true);
    if (rc) return rc;
    if (metrics) CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
    return zone_pass_prep(c, MPCD_LAYOUT_BASE, 88172645463325252ULL + 10007ULL * s, pf);
}

static int step_mid_b(mpcd_ctx* c, int64_t step, bool metrics, Prof* pf) {
    const uint64_t s = (uint64_t)step;
    int rc = MPCD_OK;
    if (metrics) {
        CUDA_TRY(cudaEventRecord(c->ev[2], c->stream));
        rc = ensure_std_index(c);
        if (rc) return rc;
        rc = count_metrics(c, c->red + 20);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(c->ev[3], c->stream));
    }
    return zone_pass_prep(c, MPCD_LAYOUT_SHIFTED, 88172645463325252ULL + 4099ULL + 10007ULL * s, pf);
}

static int step_mid(mpcd_ctx* c, int64_t step, bool metrics, Prof* pf) {
    const int rc = zone_pass_finish(c, pf, metrics);
    return rc ? rc : step_mid_b(c, step, metrics, pf);
}

static int step_tail_b(mpcd_ctx* c, bool metrics, Prof* pf) {
    int rc = MPCD_OK;
    if (metrics) {
        CUDA_TRY(cudaEventRecord(c->ev[4], c->stream));
        rc = ensure_std_index(c);
        if (rc) return rc;
        rc = count_metrics(c, c->red + 23);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(c->ev[5], c->stream));
    }
    rc = run_closure(c, true, false, metrics, pf);
    if (rc) return rc;
    if (metrics) {
        CUDA_TRY(cudaEventRecord(c->ev[6], c->stream));
        rc = reduce_cols(c, c->pdRaw, c->Nc, 1, 0u, c->red + 16);
        if (rc) return rc;
        rc = reduce_cols(c, c->pdrive, c->Nc, 1, 0u, c->red + 17);
        if (rc) return rc;
        WITH_VIEW(c->xv, k_particle_cols<<<blocks_for(c->n), kThreads, 0, c->stream>>>(S, c->n, c->cols)); ++c->launches;
        rc = reduce_cols(c, c->cols, c->n, 3, 0u, c->red + 26);
        if (rc) return rc;
        FieldsOut o{};
        o.Ux = c->fieldTmp;
        o.Uy = c->fieldTmp + c->Nc;
        WITH_VIEW(c->xv, k_cell_fields<<<blocks_for(c->Nc), kThreads, 0, c->stream>>>(c->P, c->idxStd.start, c->idxStd.slots,
                                                                                      S, c->P.rhoTarget, o));
        ++c->launches;
        rc = reduce_cols(c, c->fieldTmp, c->Nc, 1, 0u, c->red + 29);
        if (rc) return rc;
        rc = reduce_cols(c, c->fieldTmp + c->Nc, c->Nc, 1, 0u, c->red + 30);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(c->ev[7], c->stream));
    }
    if (c->graphMode) CUDA_TRY(cudaStreamWaitEvent(c->stream, c->sideDone, 0));  // join the sign prefetch
    return MPCD_OK;
}

static int step_tail(mpcd_ctx* c, bool metrics, Prof* pf) {
    const int rc = zone_pass_finish(c, pf, metrics);
    return rc ? rc : step_tail_b(c, metrics, pf);
}

static int step_once(mpcd_ctx* c, int64_t step, bool metrics, Prof* pf = nullptr) {
    int rc = step_head(c, step, metrics, pf);
    if (!rc) rc = zone_pass_kernel(c);
    if (!rc) rc = step_mid(c, step, metrics, pf);
    if (!rc) rc = zone_pass_kernel(c);
    if (!rc) rc = step_tail(c, metrics, pf);
    return rc;
}

// A step replayed from a CUDA graph. The graph of each entry parity of the ping-pong
// buffers is captured from step_once on first use; the step number and seeds come from the
// device (step_begin, run by the step's k_srd_shift, increments *dStep), so one graph serves every step. Needs the step's
// sign stream prefetched by the step before (signsStep), like the eager path's fast case.
static int graph_step(mpcd_ctx* c, int64_t step) {
    const int key = (c->xv * 2 + c->pp) * 2 + c->xflip;
    if (!c->gexec[key]) {
        const int64_t l0 = c->launches;
        CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->graphMode = true;
        const int rc = step_once(c, step, false);
        c->graphMode = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (rc != MPCD_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != MPCD_OK ? rc : set_err(MPCD_ERR_CUDA, std::string("step capture: ") + cudaGetErrorString(e));
        }
        const cudaError_t ei = cudaGraphInstantiate(&c->gexec[key], g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            c->gexec[key] = nullptr;
            cudaGetLastError();
            return set_err(MPCD_ERR_CUDA, std::string("step graph instantiate: ") + cudaGetErrorString(ei));
        }
        c->gkernels[key] = c->launches - l0;
        c->launches = l0;
        c->gpost[key] = {c->xv, c->pp, c->xflip, c->cidStdValid, c->srdCellsValid, c->idxStdValid, c->refValid};
    } else {
        const auto& f = c->gpost[key];  // host-side state after the step, as step_once leaves it
        c->xv = f.xv;
        c->pp = f.pp;
        c->xflip = f.xflip;
        c->slotsSorted = true;
        c->cidStdValid = f.cidStdValid;
        c->srdCellsValid = f.srdCellsValid;
        c->idxStdValid = f.idxStdValid;
        c->refValid = f.refValid;
    }
    // the sign stream of this step may come from an eager step's prefetch on the side stream
    CUDA_TRY(cudaStreamWaitEvent(c->stream, c->signsReady[step & 1], 0));
    k_set_step<<<1, 1, 0, c->stream>>>(c->dStep, (long long)(step - 1)); ++c->launches;
    CUDA_TRY(cudaGraphLaunch(c->gexec[key], c->stream));
    c->launches += c->gkernels[key];
    c->signsStep[(step + 1) & 1] = step + 1;
    return MPCD_OK;
}

// steps step0+1 .. step0+nsteps; the metrics step (if any), steps whose sign stream was
// not prefetched and steps before the collision tile shape is tuned run eagerly, the others
// from graphs
static int profile_accumulate(mpcd_ctx* c) {
    if (!c->profOn) return MPCD_OK;
    WITH_VIEW(c->xv, k_profile_slots<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, S, c->n, c->profP, c->profN));
    ++c->launches;
    ++c->profSteps;
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

static int run_steps(mpcd_ctx* c, int64_t step0, int64_t nsteps, bool metricsLast) {
    for (int64_t k = 1; k <= nsteps; ++k) {
        const int64_t s = step0 + k;
        const bool m = metricsLast && k == nsteps;
        int rc;
        if (c->useGraphs && !m && c->signsStep[s & 1] == s && c->collideShape >= 0)
            rc = graph_step(c, s);
        else
            rc = step_once(c, s, m);
        if (!rc) rc = profile_accumulate(c);
        if (rc) return rc;
    }
    return MPCD_OK;
}

static void occ_from(const mpcd_ctx* c, const double* r, double* occ, double* ob) {
    const double N = (double)std::max(1, c->Nc);
    const double mean = r[0] / N;
    double var = r[1] / N - mean * mean;
    if (var < 0.0) var = 0.0;
    *occ = std::sqrt(var) / std::max(c->pc.gamma, 1e-12);
    *ob = r[2] / N;
}

int mpcd_step(mpcd_ctx* c, int64_t step0, int64_t nsteps, mpcd_step_metrics_c* last) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (nsteps < 0) return set_err(MPCD_ERR_INVALID_ARG, "nsteps must be >= 0");
    if (!c->pc.useIncompressibleRedistribution || !c->pc.useZoneRedistribution || !c->pc.useLiquidClosure)
        return set_err(MPCD_ERR_INVALID_ARG, "the benchmark step needs useIncompressibleRedistribution, useZoneRedistribution and useLiquidClosure");
    if (c->pc.redistributionEnableSurfaceTopology || c->pc.redistributionWallWettingEnabled || c->pc.useInterfaceVelocityReorientation)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl is restricted to no surface / no wetting / no reorientation");
    CUDA_TRY(cudaSetDevice(c->device));
    if (c->fast) {
        int rc = fast_steps(c, step0, nsteps, nullptr);
        if (!rc) rc = check_device(c);
        if (!rc && last && nsteps > 0) {
            rc = fast_metrics(c, last, step0 + nsteps);
            if (!rc) c->last = *last;
        }
        return rc;
    }
    {
        const int rc = run_steps(c, step0, nsteps, last != nullptr);
        if (rc) return rc;
    }
    int rc = check_device(c);
    if (rc) return rc;
    if (last && nsteps > 0) {
        mpcd_step_metrics_c& M = *last;
        std::memset(&M, 0, sizeof M);
        M.step = step0 + nsteps;
        double r[32];
        int ints[4];
        double wd[kWallDoubles];
        CUDA_TRY(cudaMemcpy(r, c->red, sizeof r, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(ints, c->W.ints, sizeof ints, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(wd, c->wallOut, sizeof wd, cudaMemcpyDeviceToHost));
        M.wall.nBot = ints[0]; M.wall.nTop = ints[1]; M.wall.nLeft = ints[2]; M.wall.nRight = ints[3];
        M.wall.dEwall = wd[0]; M.wall.dPxBot = wd[1]; M.wall.dPxTop = wd[2]; M.wall.dPyBot = wd[3]; M.wall.dPyTop = wd[4];
        M.wall.dPxLeft = wd[5]; M.wall.dPxRight = wd[6]; M.wall.dPyLeft = wd[7]; M.wall.dPyRight = wd[8];
        rc = pass_metrics_to_host(c, MPCD_LAYOUT_BASE, &M.base);
        if (rc) return rc;
        rc = pass_metrics_to_host(c, MPCD_LAYOUT_SHIFTED, &M.shifted);
        if (rc) return rc;
        closure_metrics_from(c, r, &M.closure);
        M.closure.meanPdriveRaw = r[16] / (double)std::max(1, c->Nc);
        M.closure.meanPdrive = r[17] / (double)std::max(1, c->Nc);
        occ_from(c, r + 20, &M.baseOccStd, &M.baseOutBand);
        occ_from(c, r + 23, &M.shiftedOccStd, &M.shiftedOutBand);
        M.occStd = M.shiftedOccStd;
        M.outBand = M.shiftedOutBand;
        const double nn = (double)std::max(c->n, 1);
        M.meanKinetic = r[26] / nn;
        M.meanVelocityX = r[27] / nn;
        M.meanVelocityY = r[28] / nn;
        M.meanUx = r[29] / (double)std::max(1, c->Nc);
        M.meanUy = r[30] / (double)std::max(1, c->Nc);
        M.Qx = M.meanUx * c->pc.Ly;
        float t[7];
        for (int k = 0; k < 7; ++k) cudaEventElapsedTime(&t[k], c->ev[k], c->ev[k + 1]);
        M.timeRefBuild = t[0] * 1e-3;
        M.timeBase = t[1] * 1e-3;
        M.timeShifted = t[3] * 1e-3;
        M.timeClosure = t[5] * 1e-3;
        M.timeDiagnostics = (t[2] + t[4] + t[6]) * 1e-3;
        M.timeStepTotal = M.timeRefBuild + M.timeBase + M.timeShifted + M.timeClosure + M.timeDiagnostics;
        M.base.timeKernel = M.timeBase;
        M.shifted.timeKernel = M.timeShifted;
        c->last = M;
    }
    return MPCD_OK;
}

// the state from device buffers (x, v: n double2 each, particle-id order), enqueued on the
// context's stream without a host synchronisation
static int load_state_async(mpcd_ctx* c, const double2* x, const double2* v) {
    c->xv = 0;
    c->pp = 0;
    c->xflip = 0;
    c->slotsSorted = false;
    if (c->n > 0) {
        if (c->f32) {
            k_f32_from<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, x, v, c->n, view32(c, 0)); ++c->launches;
        } else {
            CUDA_TRY(cudaMemcpyAsync(c->xb[0], x, sizeof(double2) * (size_t)c->n, cudaMemcpyDeviceToDevice, c->stream));
            CUDA_TRY(cudaMemcpyAsync(c->vb[0], v, sizeof(double2) * (size_t)c->n, cudaMemcpyDeviceToDevice, c->stream));
        }
        k_iota<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->pidb[0], c->n); ++c->launches;
    }
    invalidate_positions(c);
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// the state into device buffers in particle-id order, enqueued on the context's stream
static int store_state_async(mpcd_ctx* c, double2* x, double2* v) {
    if (c->n == 0) return MPCD_OK;
    if (c->f32) {
        k_f32_by_pid<<<blocks_for(c->n), kThreads, 0, c->stream>>>(c->P, view32(c, c->xv), c->pidb[c->pp], c->n, x, v);
    } else {
        k_gather_by_pid<<<blocks_for(c->n), kThreads, 0, c->stream>>>(cur_x(c), c->vb[c->xv], c->pidb[c->pp], c->n, x, v);
    }
    ++c->launches;
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

static int ensure_job_buffers(mpcd_ctx* c) {
    if (c->up) return MPCD_OK;
    for (int b = 0; b < 2; ++b) {
        int rc = dalloc(&c->jobIn[b], 2 * (size_t)c->n);
        if (!rc) rc = dalloc(&c->jobOut[b], 2 * (size_t)c->n);
        if (rc) return rc;
        for (cudaEvent_t* e : {&c->upDone[b], &c->inFree[b], &c->outReady[b], &c->downDone[b]})
            CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&c->down, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->up, cudaStreamNonBlocking));
    return MPCD_OK;
}

int mpcd_run_jobs(mpcd_ctx* c, int64_t njobs, const double* const* x_in, const double* const* v_in, int64_t step0,
                  int64_t nsteps, double* const* x_out, double* const* v_out) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (njobs < 0 || nsteps < 0) return set_err(MPCD_ERR_INVALID_ARG, "njobs and nsteps must be >= 0");
    if (njobs == 0) return MPCD_OK;
    if (!x_in || !v_in || !x_out || !v_out) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    for (int64_t j = 0; j < njobs; ++j)
        if (!x_in[j] || !v_in[j] || !x_out[j] || !v_out[j]) return set_err(MPCD_ERR_INVALID_ARG, "null job buffer");
    if (nsteps > 0 &&
        (!c->pc.useIncompressibleRedistribution || !c->pc.useZoneRedistribution || !c->pc.useLiquidClosure))
        return set_err(MPCD_ERR_INVALID_ARG, "the benchmark step needs useIncompressibleRedistribution, useZoneRedistribution and useLiquidClosure");
    if (nsteps > 0 && (c->pc.redistributionEnableSurfaceTopology || c->pc.redistributionWallWettingEnabled ||
                       c->pc.useInterfaceVelocityReorientation))
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl is restricted to no surface / no wetting / no reorientation");
    CUDA_TRY(cudaSetDevice(c->device));
    int rc = ensure_job_buffers(c);
    if (rc) return rc;
    const size_t bytes = sizeof(double2) * (size_t)c->n;
    // job j's input into jobIn[j & 1], once the load of job j-2 has read that buffer
    auto upload = [&](int64_t j) -> int {
        const int b = (int)(j & 1);
        CUDA_TRY(cudaStreamWaitEvent(c->up, c->inFree[b], 0));
        CUDA_TRY(cudaMemcpyAsync(c->jobIn[b], x_in[j], bytes, cudaMemcpyHostToDevice, c->up));
        CUDA_TRY(cudaMemcpyAsync(c->jobIn[b] + c->n, v_in[j], bytes, cudaMemcpyHostToDevice, c->up));
        CUDA_TRY(cudaEventRecord(c->upDone[b], c->up));
        return MPCD_OK;
    };
    // events not yet recorded count as complete in waits
    for (int64_t j = 0; j < njobs && !rc; ++j) {
        const int b = (int)(j & 1);
        if (j == 0) rc = upload(0);
        if (rc) break;
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->upDone[b], 0));
        rc = load_state_async(c, c->jobIn[b], c->jobIn[b] + c->n);
        if (rc) break;
        CUDA_TRY(cudaEventRecord(c->inFree[b], c->stream));
        if (j + 1 < njobs) rc = upload(j + 1);  // overlaps this job's steps
        if (!rc) rc = run_steps(c, step0 + j * nsteps, nsteps, false);
        if (rc) break;
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->downDone[b], 0));  // job j-2's result has left
        rc = store_state_async(c, c->jobOut[b], c->jobOut[b] + c->n);
        if (rc) break;
        CUDA_TRY(cudaEventRecord(c->outReady[b], c->stream));
        CUDA_TRY(cudaStreamWaitEvent(c->down, c->outReady[b], 0));
        CUDA_TRY(cudaMemcpyAsync(x_out[j], c->jobOut[b], bytes, cudaMemcpyDeviceToHost, c->down));
        CUDA_TRY(cudaMemcpyAsync(v_out[j], c->jobOut[b] + c->n, bytes, cudaMemcpyDeviceToHost, c->down));
        CUDA_TRY(cudaEventRecord(c->downDone[b], c->down));
        // no host synchronisation per job: a status read would queue behind this job's
        // download on the copy engine; the device status is checked once at the end
    }
    const cudaError_t e1 = cudaStreamSynchronize(c->up), e2 = cudaStreamSynchronize(c->down);
    if (rc) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess) return set_err(MPCD_ERR_CUDA, "job copies");
    return check_device(c);
}

int mpcd_step_metrics(mpcd_ctx* c, mpcd_step_metrics_c* out) {
    if (!c || !out) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    *out = c->last;
    return MPCD_OK;
}

int mpcd_profile_reset(mpcd_ctx* c, int32_t enable) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    CUDA_TRY(cudaSetDevice(c->device));
    const int Ny = c->pc.Ny;
    if (!c->profP) {
        CUDA_TRY(cudaMalloc(&c->profP, sizeof(unsigned long long) * (size_t)Ny));
        CUDA_TRY(cudaMalloc(&c->profN, sizeof(unsigned long long) * (size_t)Ny));
    }
    CUDA_TRY(cudaMemsetAsync(c->profP, 0, sizeof(unsigned long long) * (size_t)Ny, c->stream));
    CUDA_TRY(cudaMemsetAsync(c->profN, 0, sizeof(unsigned long long) * (size_t)Ny, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->profOn = enable != 0;
    c->profSteps = 0;
    return MPCD_OK;
}

int mpcd_profile_read(mpcd_ctx* c, double* ux_rows, int64_t* nsteps) {
    if (!c || !ux_rows) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (!c->profP) return set_err(MPCD_ERR_INVALID_ARG, "profile accumulation was never reset");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const int Ny = c->pc.Ny;
    std::vector<unsigned long long> P((size_t)Ny), N((size_t)Ny);
    CUDA_TRY(cudaMemcpy(P.data(), c->profP, sizeof(unsigned long long) * (size_t)Ny, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(N.data(), c->profN, sizeof(unsigned long long) * (size_t)Ny, cudaMemcpyDeviceToHost));
    for (int iy = 0; iy < Ny; ++iy)
        ux_rows[iy] = N[(size_t)iy] ? (double)(long long)P[(size_t)iy] * 0x1p-32 / (double)N[(size_t)iy] : 0.0;
    if (nsteps) *nsteps = c->profSteps;
    return MPCD_OK;
}


int mpcd_step_timed(mpcd_ctx* c, int64_t step0, int64_t nsteps, double* device_seconds) {
    if (!c || !device_seconds) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaEventRecord(a, c->stream));
    int rc = MPCD_OK;
    if (c->fast) {
        // the device step counter is set before the timed region
        const long long s0 = (long long)step0;
        CUDA_TRY(cudaMemcpy(&c->fstep->step, &s0, sizeof s0, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaEventRecord(a, c->stream));
        for (int64_t k = 0; k < nsteps && rc == MPCD_OK; ++k) rc = fast_step(c, nullptr);
    } else {
        rc = run_steps(c, step0, nsteps, false);
    }
    CUDA_TRY(cudaEventRecord(b, c->stream));
    CUDA_TRY(cudaEventSynchronize(b));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    *device_seconds = ms * 1e-3;
    return check_device(c);
}

int64_t mpcd_launch_count(mpcd_ctx* c) { return c ? c->launches : 0; }


// Per-phase device time over nsteps steps (events at phase boundaries on the context's
// stream; one synchronisation per step). phase_seconds[k] accumulates phase k:
// 0 stream+BC, 1 thermal walls, 2 SRD cell index, 3 SRD sign stream, 4 collision,
// 5 standard cell index (3 per step), 6 reference fields + pdrive + EOS kick,
// 7 zone seeds (2), 8 zone passes (2), 9 closure cells + beta reduction, 10 kick + re-sort.
int mpcd_step_profile(mpcd_ctx* c, int64_t step0, int64_t nsteps, double* phase_seconds, int nphase) {
    if (!c || !phase_seconds) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    for (int k = 0; k < nphase; ++k) phase_seconds[k] = 0.0;
    Prof pf;
    for (auto& e : pf.ev) CUDA_TRY(cudaEventCreate(&e));
    int rc = MPCD_OK;
    if (c->fast) {
        const long long s0 = (long long)step0;
        CUDA_TRY(cudaMemcpy(&c->fstep->step, &s0, sizeof s0, cudaMemcpyHostToDevice));
    }
    for (int64_t k = 1; k <= nsteps && rc == MPCD_OK; ++k) {
        pf.n = 0;
        rc = c->fast ? fast_step(c, &pf) : step_once(c, step0 + k, false, &pf);
        if (rc) break;
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (int i = 1; i < pf.n; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, pf.ev[i - 1], pf.ev[i]);
            const int lab = pf.label[i];
            if (lab >= 0 && lab < nphase) phase_seconds[lab] += ms * 1e-3;
        }
    }
    for (auto& e : pf.ev) cudaEventDestroy(e);
    if (rc) return rc;
    return check_device(c);
}


// Page-locked host memory for callers that stage states (the end-to-end benchmark).
void* mpcd_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_err(MPCD_ERR_CUDA, "cudaMallocHost failed");
        return nullptr;
    }
    return p;
}
void mpcd_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// mpcd_cell_fields_static: compute_cell_fields (reference src/common_grid.cpp:32-100) of a
// caller-owned device state, without a context and without allocating device memory.
//
// It serves callers that must not allocate: a host code that embeds the MPCD state in its own
// time loop, has reserved the device memory it may use up front (its own pool sized to the
// GPU), and needs the cell fields between steps. Creating a context would allocate; and
// cudaFree synchronises the whole device, which would stall the caller's other streams.
//
// Its only working memory is the file-scope array below: per cell, the particle count, the two
// momentum sums and the sum of squared peculiar speeds. The array is shared by every call on
// a device, so calls whose work overlaps on the GPU (two streams, two host threads) race on it
// and must be serialised by the caller.
namespace mpcd_dev {

constexpr int kStaticMaxDevices = 64;

// 4 doubles per cell: [count | sum vx | sum vy | sum |v - u|^2], each block Nc long.
__global__ void k_static_accumulate(DevParams P, const double* __restrict__ x, const double* __restrict__ v,
                                    int n, double* __restrict__ acc) {
    const size_t nc = (size_t)P.Nc;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = cell_of(x[2 * (size_t)i], x[2 * (size_t)i + 1], P);
        atomicAdd(acc + c, 1.0);
        atomicAdd(acc + nc + c, v[2 * (size_t)i]);
        atomicAdd(acc + 2 * nc + c, v[2 * (size_t)i + 1]);
    }
}

__global__ void k_static_peculiar(DevParams P, const double* __restrict__ x, const double* __restrict__ v,
                                  int n, double* __restrict__ acc) {
    const size_t nc = (size_t)P.Nc;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = cell_of(x[2 * (size_t)i], x[2 * (size_t)i + 1], P);
        const double m = acc[c];
        if (m < 2.0) continue;  // a cell of one particle has no thermal degrees of freedom
        const double ux = __ddiv_rn(acc[nc + c], m), uy = __ddiv_rn(acc[2 * nc + c], m);
        const double ax = __dsub_rn(v[2 * (size_t)i], ux), ay = __dsub_rn(v[2 * (size_t)i + 1], uy);
        atomicAdd(acc + 3 * nc + c, __dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)));
    }
}

// The per-cell formulas of k_cell_fields, from the accumulated sums.
__global__ void k_static_finish(DevParams Pm, const double* __restrict__ acc, double rhoTarget, FieldsOut o) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Pm.Nc) return;
    const size_t nc = (size_t)Pm.Nc;
    const int m = (int)acc[c];
    const double px = acc[nc + c], py = acc[2 * nc + c];
    double ux = 0.0, uy = 0.0;
    if (m > 0) {
        ux = __ddiv_rn(px, (double)m);
        uy = __ddiv_rn(py, (double)m);
    }
    const double rho = __ddiv_rn((double)m, Pm.Vc);
    double T = 0.0, pk = 0.0;
    const int dof = 2 * max(m - 1, 0);
    if (dof > 0) {
        T = __ddiv_rn(acc[3 * nc + c], (double)dof);
        pk = __dmul_rn(rho, T);
    }
    const double pv = __dmul_rn(Pm.Kvirial, __dsub_rn(rho, rhoTarget));
    if (o.N) o.N[c] = m;
    if (o.Ux) o.Ux[c] = ux;
    if (o.Uy) o.Uy[c] = uy;
    if (o.Px) o.Px[c] = px;
    if (o.Py) o.Py[c] = py;
    if (o.T) o.T[c] = T;
    if (o.rho) o.rho[c] = rho;
    if (o.Pkin) o.Pkin[c] = pk;
    if (o.Pvir) o.Pvir[c] = pv;
    if (o.P) o.P[c] = __dadd_rn(pk, pv);
    if (o.rhoTarget) o.rhoTarget[c] = rhoTarget;
}

}  // namespace mpcd_dev

// The scratch of mpcd_cell_fields_static: 4 * MPCD_STATIC_FIELDS_MAX_CELLS doubles (32 MiB),
// part of the module's static device memory on every device the library is loaded on.
static __device__ __align__(256) double g_static_fields_scratch[4 * (size_t)MPCD_STATIC_FIELDS_MAX_CELLS];

namespace {

std::mutex g_static_mu;
double* g_static_ptr[mpcd_dev::kStaticMaxDevices] = {};

// Set-up, once per device, with that device current: the device address of the scratch array.
// This is the first call's extra work (it may also load the module onto the device).
int static_scratch(int dev, double** out) {
    if (dev < 0 || dev >= mpcd_dev::kStaticMaxDevices)
        return set_err(MPCD_ERR_INVALID_ARG, "mpcd_cell_fields_static: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_fields_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_err(MPCD_ERR_CUDA, std::string("mpcd_cell_fields_static: cudaGetSymbolAddress failed: ") +
                                              cudaGetErrorString(e));
        }
        g_static_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_static_ptr[dev];
    return MPCD_OK;
}

}  // namespace

extern "C" int mpcd_cell_fields_static(const mpcd_params_c* params, const double* d_x, const double* d_v, int64_t n,
                                       double rho_target, const mpcd_cellfields_c* d_out, void* stream) {
    if (!params || !d_out || (n > 0 && (!d_x || !d_v)))
        return set_err(MPCD_ERR_INVALID_ARG, "mpcd_cell_fields_static: null argument");
    int rc = validate(*params);
    if (rc) return rc;
    if (n < 0 || 2 * n >= (1LL << 31)) return set_err(MPCD_ERR_INVALID_ARG, "mpcd_cell_fields_static: n out of range");
    if (params->Nc > MPCD_STATIC_FIELDS_MAX_CELLS)
        return set_err(MPCD_ERR_CAPACITY, "mpcd_cell_fields_static: Nc = " + std::to_string(params->Nc) +
                                              " exceeds the static scratch maximum of " +
                                              std::to_string(MPCD_STATIC_FIELDS_MAX_CELLS) + " cells");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    double* acc = nullptr;
    rc = static_scratch(dev, &acc);
    if (rc) return rc;
    const DevParams P = make_dev_params(*params);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t nc = (size_t)params->Nc;
    // everything the kernels accumulate into starts at zero
    CUDA_TRY(cudaMemsetAsync(acc, 0, 4 * nc * sizeof(double), s));
    const bool wantT = d_out->T || d_out->Pkin || d_out->P;
    if (n > 0) {
        const int grid = (int)std::min<int64_t>(blocks_for(n), 148 * 16);
        k_static_accumulate<<<grid, kThreads, 0, s>>>(P, d_x, d_v, (int)n, acc);
        CUDA_TRY(cudaGetLastError());
        if (wantT) {
            k_static_peculiar<<<grid, kThreads, 0, s>>>(P, d_x, d_v, (int)n, acc);
            CUDA_TRY(cudaGetLastError());
        }
    }
    FieldsOut o{};
    o.N = d_out->N;
    o.Ux = d_out->Ux; o.Uy = d_out->Uy; o.Px = d_out->Px; o.Py = d_out->Py; o.T = d_out->T;
    o.rho = d_out->rho; o.Pkin = d_out->Pkin; o.Pvir = d_out->Pvir; o.P = d_out->P; o.rhoTarget = d_out->rhoTarget;
    k_static_finish<<<blocks_for(params->Nc), kThreads, 0, s>>>(P, acc, rho_target, o);
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// ---------------------------------------------------------------------------------------------
// Batched replicas: independent contexts (own parameters, sizes, states and zone layouts) that
// advance together. Each step is issued for every replica before the next step, each replica
// on its own streams and from its own step graph, so their kernels run side by side on the GPU.
struct FastBatch;
struct mpcd_batch {
    int device = 0;
    FastBatch* fast = nullptr;  // fast-form replicas: one launch per phase (fast_batch.inc)
    std::vector<mpcd_ctx*> members;
    cudaStream_t stream = nullptr;  // timing and the fork/join of the members' streams
    cudaEvent_t start = nullptr, stop = nullptr, fork = nullptr;
    std::vector<cudaEvent_t> done;
    // the zone kernels of all replicas as one launch per pass: arguments and zone-count prefix
    // sums per (buffer parity, pass), staged in page-locked memory (constant per slot, so a
    // captured copy replays correctly) and copied to the device before the launch
    ZoneArgs* hArgs = nullptr;
    int* hOffs = nullptr;
    ZoneArgs* dArgs = nullptr;
    int* dOffs = nullptr;
    size_t zSmem = 0;
    OverflowJob* hOv = nullptr;  // the overflow kernels' jobs, staged the same way
    OverflowJob* dOv = nullptr;
    int ovBlocks = 0;            // overflow blocks per replica (the same for all)
    // whole batched steps replayed from CUDA graphs, one per buffer parity of the replicas
    bool useGraphs = true;
    cudaGraphExec_t gexec[8] = {};  // by (xv, pp, xflip) of the replicas at step entry
    std::vector<mpcd_ctx::HostFlags> gpost[8];
    std::vector<int64_t> gkernels[8];
    long long** dStepPtrs = nullptr;  // each replica's device step counter
    // the replicas' standard-grid index builds after a zone pass as one launch per kernel
    // (batch_index): job tables per particle-id buffer parity, block prefix sums
    bool indexBatched = false;  // every replica has Nc <= kSmallScan
    IndexJob* dJobs[2] = {};
    int* dOffsHist = nullptr;   // count + 1: blocks of the histogram and the scatter
    int* dOffsRank = nullptr;   // count + 1: blocks of the rank sort
    int histBlocks = 0, rankBlocks = 0;
};

#include "fast_batch.inc"

__global__ void k_set_steps(long long** steps, int n, long long value) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) *steps[i] = value;
}

// the zone kernels of pass `pass` (0 base, 1 shifted) of every replica in one launch; each
// replica's zone_pass_prep has filled its zA
static int batch_zone_kernel(mpcd_batch* b, int pass) {
    const int n = (int)b->members.size();
    const int slot = (b->members[0]->xv & 1) * 2 + pass;
    ZoneArgs* h = b->hArgs + (size_t)slot * n;
    int* ho = b->hOffs + (size_t)slot * (n + 1);
    ho[0] = 0;
    for (int r = 0; r < n; ++r) {
        h[r] = b->members[r]->zA;
        ho[r + 1] = ho[r] + h[r].nZones;
    }
    ZoneArgs* d = b->dArgs + (size_t)slot * n;
    int* dof = b->dOffs + (size_t)slot * (n + 1);
    CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(ZoneArgs) * n, cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaMemcpyAsync(dof, ho, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, b->stream));
    if (ho[n] > 0) {
        k_zone_pass_batch<false><<<ho[n], 32, b->zSmem, b->stream>>>(d, dof, n);
        ++b->members[0]->launches;
    }
    CUDA_TRY(cudaGetLastError());
    return MPCD_OK;
}

// f(c) on every replica, each on its own stream, forked from and joined back into the batch
// stream by events
template <class F>
static int batch_each(mpcd_batch* b, F f) {
    CUDA_TRY(cudaEventRecord(b->fork, b->stream));
    for (size_t r = 0; r < b->members.size(); ++r) {
        mpcd_ctx* c = b->members[r];
        CUDA_TRY(cudaStreamWaitEvent(c->stream, b->fork, 0));
        const int rc = f(c);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(b->done[r], c->stream));
        CUDA_TRY(cudaStreamWaitEvent(b->stream, b->done[r], 0));
    }
    return MPCD_OK;
}

// the standard-grid cell index of every replica, built by one launch per kernel on the batch
// stream (the replicas share one particle-id buffer parity)
static int batch_index(mpcd_batch* b) {
    const int n = (int)b->members.size();
    const IndexJob* jobs = b->dJobs[b->members[0]->pp];
    mpcd_ctx* c0 = b->members[0];
    if (b->histBlocks > 0) {
        k_histogram_batch<<<b->histBlocks, kThreads, 0, b->stream>>>(jobs, b->dOffsHist, n); ++c0->launches;
    }
    k_scan_counts_small_batch<<<n, kScanThreads, 0, b->stream>>>(jobs); ++c0->launches;
    if (b->histBlocks > 0) {
        k_scatter_keys_batch<<<b->histBlocks, kThreads, 0, b->stream>>>(jobs, b->dOffsHist, n); ++c0->launches;
    }
    k_cell_rank_batch<<<b->rankBlocks, kRankThreads, 0, b->stream>>>(jobs, b->dOffsRank, n); ++c0->launches;
    CUDA_TRY(cudaGetLastError());
    for (mpcd_ctx* c : b->members) c->idxStdValid = true;
    return MPCD_OK;
}

// the overflow kernels of pass `pass` of every replica in one launch on the batch stream (after
// the batched zone kernel), then each replica's host-side flip; staged like the zone arguments
static int batch_zone_finish(mpcd_batch* b, int pass) {
    const int n = (int)b->members.size();
    const int slot = (b->members[0]->xv & 1) * 2 + pass;
    OverflowJob* h = b->hOv + (size_t)slot * n;
    for (int r = 0; r < n; ++r) h[r] = overflow_job(b->members[r], false);
    OverflowJob* d = b->dOv + (size_t)slot * n;
    CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(OverflowJob) * n, cudaMemcpyHostToDevice, b->stream));
    k_zone_overflow_batch<<<n * b->ovBlocks, 32, 0, b->stream>>>(d, b->ovBlocks);
    ++b->members[0]->launches;
    CUDA_TRY(cudaGetLastError());
    for (mpcd_ctx* c : b->members) zone_pass_flip(c);
    return MPCD_OK;
}

// one batched step: each replica's parts on its own streams, forked from and joined into the
// batch stream. Where the replicas are joined anyway (around the zone kernels), the batch
// stream also runs the overflow kernels of all replicas as one launch and, when every replica
// is small enough for the one-block scan and all share a particle-id buffer parity, the
// standard-grid index builds that follow each pass.
static int batch_step_body(mpcd_batch* b, int64_t step) {
    bool idx = b->indexBatched;
    for (mpcd_ctx* c : b->members) idx = idx && c->pp == b->members[0]->pp;
    int rc = batch_each(b, [&](mpcd_ctx* c) { return step_head(c, step, false, nullptr); });
    if (!rc) rc = batch_zone_kernel(b, 0);
    if (!rc) rc = batch_zone_finish(b, 0);
    if (!rc && idx) rc = batch_index(b);
    if (!rc) rc = batch_each(b, [&](mpcd_ctx* c) { return step_mid_b(c, step, false, nullptr); });
    if (!rc) rc = batch_zone_kernel(b, 1);
    if (!rc) rc = batch_zone_finish(b, 1);
    if (!rc && idx) rc = batch_index(b);
    if (!rc) rc = batch_each(b, [&](mpcd_ctx* c) { return step_tail_b(c, false, nullptr); });
    return rc;
}

// a batched step replayed from the graph of the replicas' buffer parity (captured on first
// use); every replica's sign stream must have been prefetched by the step before
static int batch_graph_step(mpcd_batch* b, int64_t step) {
    const int n = (int)b->members.size();
    mpcd_ctx* c0 = b->members[0];
    const int key = (c0->xv * 2 + c0->pp) * 2 + c0->xflip;
    if (!b->gexec[key]) {
        std::vector<int64_t> l0(n);
        for (int r = 0; r < n; ++r) l0[r] = b->members[r]->launches;
        CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        for (mpcd_ctx* c : b->members) c->graphMode = true;
        const int rc = batch_step_body(b, step);
        for (mpcd_ctx* c : b->members) c->graphMode = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc != MPCD_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != MPCD_OK ? rc : set_err(MPCD_ERR_CUDA, std::string("batch step capture: ") + cudaGetErrorString(e));
        }
        const cudaError_t ei = cudaGraphInstantiate(&b->gexec[key], g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            b->gexec[key] = nullptr;
            cudaGetLastError();
            return set_err(MPCD_ERR_CUDA, std::string("batch step graph instantiate: ") + cudaGetErrorString(ei));
        }
        b->gpost[key].resize(n);
        b->gkernels[key].resize(n);
        for (int r = 0; r < n; ++r) {
            mpcd_ctx* c = b->members[r];
            b->gkernels[key][r] = c->launches - l0[r];
            c->launches = l0[r];
            b->gpost[key][r] = {c->xv, c->pp, c->xflip, c->cidStdValid, c->srdCellsValid, c->idxStdValid, c->refValid};
        }
    }
    for (int r = 0; r < n; ++r) {
        mpcd_ctx* c = b->members[r];
        const mpcd_ctx::HostFlags& f = b->gpost[key][r];
        c->xv = f.xv;
        c->pp = f.pp;
        c->xflip = f.xflip;
        c->slotsSorted = true;
        c->cidStdValid = f.cidStdValid;
        c->srdCellsValid = f.srdCellsValid;
        c->idxStdValid = f.idxStdValid;
        c->refValid = f.refValid;
        CUDA_TRY(cudaStreamWaitEvent(b->stream, c->signsReady[step & 1], 0));
    }
    k_set_steps<<<(n + 255) / 256, 256, 0, b->stream>>>(b->dStepPtrs, n, (long long)(step - 1));
    CUDA_TRY(cudaGraphLaunch(b->gexec[key], b->stream));
    for (int r = 0; r < n; ++r) {
        mpcd_ctx* c = b->members[r];
        c->launches += b->gkernels[key][r];
        c->signsStep[(step + 1) & 1] = step + 1;
    }
    return MPCD_OK;
}

extern "C" {

int mpcd_ctx_collide_shape(mpcd_ctx* c, int32_t shape, int32_t* in_use) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    if (shape < -1 || shape >= kCollideShapes) return set_err(MPCD_ERR_INVALID_ARG, "collision tile shape out of range");
    if (shape >= 0) {
        CUDA_TRY(cudaSetDevice(c->device));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (auto& g : c->gexec)  // captured steps hold the previous shape
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        c->collideShape = shape;
    }
    if (in_use) *in_use = c->collideShape;
    return MPCD_OK;
}

int mpcd_ctx_set_graphs(mpcd_ctx* c, int enable) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    c->useGraphs = enable != 0;
    return MPCD_OK;
}

int mpcd_batch_destroy(mpcd_batch* b) {
    if (!b) return MPCD_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    fast_batch_free(b->fast);
    for (auto& g : b->gexec)
        if (g) cudaGraphExecDestroy(g);
    if (b->hArgs) cudaFreeHost(b->hArgs);
    if (b->hOffs) cudaFreeHost(b->hOffs);
    if (b->dArgs) cudaFree(b->dArgs);
    if (b->dOffs) cudaFree(b->dOffs);
    if (b->hOv) cudaFreeHost(b->hOv);
    if (b->dOv) cudaFree(b->dOv);
    if (b->dStepPtrs) cudaFree(b->dStepPtrs);
    for (IndexJob* j : b->dJobs)
        if (j) cudaFree(j);
    if (b->dOffsHist) cudaFree(b->dOffsHist);
    if (b->dOffsRank) cudaFree(b->dOffsRank);
    if (b->fork) cudaEventDestroy(b->fork);
    for (mpcd_ctx* c : b->members) mpcd_ctx_destroy(c);
    for (cudaEvent_t e : b->done)
        if (e) cudaEventDestroy(e);
    if (b->start) cudaEventDestroy(b->start);
    if (b->stop) cudaEventDestroy(b->stop);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MPCD_OK;
}

int mpcd_batch_create(const mpcd_params_c* params, int count, int device, mpcd_batch** out) {
    if (!params || !out || count < 1) return set_err(MPCD_ERR_INVALID_ARG, "null argument or empty batch");
    *out = nullptr;
    mpcd_batch* b = new mpcd_batch();
    b->device = device;
    for (int i = 0; i < count; ++i) {
        mpcd_ctx* c = nullptr;
        const int rc = mpcd_ctx_create(params + i, device, &c);
        if (rc) {
            const std::string msg = "replica " + std::to_string(i) + ": " + g_err;
            mpcd_batch_destroy(b);
            return set_err(rc, msg);
        }
        b->members.push_back(c);
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->start) != cudaSuccess || cudaEventCreate(&b->stop) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        mpcd_batch_destroy(b);
        return set_err(MPCD_ERR_CUDA, "batch stream");
    }
    {
        // staging of the batched zone kernels (4 slots: buffer parity x pass), the shared
        // memory of the largest working set plus the arguments, the step counters
        const size_t nslots = 4;
        std::vector<long long*> steps((size_t)count);
        for (int r = 0; r < count; ++r) {
            b->zSmem = std::max(b->zSmem, b->members[r]->zSmem + (size_t)kZoneArgsSmem);
            steps[(size_t)r] = b->members[r]->dStep;
        }
        b->ovBlocks = b->members[0]->ovBlocks;
        for (mpcd_ctx* c : b->members)
            if (c->ovBlocks != b->ovBlocks) {
                mpcd_batch_destroy(b);
                return set_err(MPCD_ERR_INVALID_ARG, "replicas with different overflow block counts");
            }
        if (cudaMallocHost((void**)&b->hArgs, sizeof(ZoneArgs) * count * nslots) != cudaSuccess ||
            cudaMallocHost((void**)&b->hOffs, sizeof(int) * (count + 1) * nslots) != cudaSuccess ||
            cudaMalloc((void**)&b->dArgs, sizeof(ZoneArgs) * count * nslots) != cudaSuccess ||
            cudaMalloc((void**)&b->dOffs, sizeof(int) * (count + 1) * nslots) != cudaSuccess ||
            cudaMallocHost((void**)&b->hOv, sizeof(OverflowJob) * count * nslots) != cudaSuccess ||
            cudaMalloc((void**)&b->dOv, sizeof(OverflowJob) * count * nslots) != cudaSuccess ||
            cudaMalloc((void**)&b->dStepPtrs, sizeof(long long*) * count) != cudaSuccess ||
            cudaMemcpy(b->dStepPtrs, steps.data(), sizeof(long long*) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
            !raise_smem((const void*)k_zone_pass_batch<false>, b->zSmem, device)) {
            cudaGetLastError();
            mpcd_batch_destroy(b);
            return set_err(MPCD_ERR_CUDA, "batch zone-pass staging");
        }
    }
    b->done.assign((size_t)count, nullptr);
    for (auto& e : b->done)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            mpcd_batch_destroy(b);
            return set_err(MPCD_ERR_CUDA, "batch events");
        }
    {
        // job tables of the batched index builds (the buffers they name never move)
        b->indexBatched = true;
        std::vector<int> oh(1, 0), orank(1, 0);
        for (mpcd_ctx* c : b->members) {
            b->indexBatched = b->indexBatched && c->Nc <= kSmallScan;
            oh.push_back(oh.back() + (c->n > 0 ? blocks_for(c->n, kThreads * kIndexItems) : 0));
            orank.push_back(orank.back() + blocks_for(c->Nc, c->rankCells));
        }
        b->histBlocks = oh.back();
        b->rankBlocks = orank.back();
        bool ok = cudaMalloc((void**)&b->dOffsHist, sizeof(int) * oh.size()) == cudaSuccess &&
                  cudaMalloc((void**)&b->dOffsRank, sizeof(int) * orank.size()) == cudaSuccess &&
                  cudaMemcpy(b->dOffsHist, oh.data(), sizeof(int) * oh.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(b->dOffsRank, orank.data(), sizeof(int) * orank.size(), cudaMemcpyHostToDevice) == cudaSuccess;
        for (int q = 0; q < 2 && ok; ++q) {
            std::vector<IndexJob> jobs;
            for (mpcd_ctx* c : b->members) {
                CellIndex& I = c->idxStd;
                jobs.push_back(IndexJob{c->cidStd, I.count, I.pos, I.start, I.slots, c->pidb[q], c->sortKeys, c->n,
                                        c->Nc, c->rankCells});
            }
            ok = cudaMalloc((void**)&b->dJobs[q], sizeof(IndexJob) * jobs.size()) == cudaSuccess &&
                 cudaMemcpy(b->dJobs[q], jobs.data(), sizeof(IndexJob) * jobs.size(), cudaMemcpyHostToDevice) ==
                     cudaSuccess;
        }
        if (!ok) {
            cudaGetLastError();
            mpcd_batch_destroy(b);
            return set_err(MPCD_ERR_CUDA, "batch index tables");
        }
    }
    *out = b;
    return MPCD_OK;
}

int mpcd_batch_create_form(const mpcd_params_c* params, int count, int device, int32_t form, mpcd_batch** out) {
    if (form == MPCD_FORM_F64) return mpcd_batch_create(params, count, device, out);
    if (form != MPCD_FORM_FAST) return set_err(MPCD_ERR_INVALID_ARG, "batched replicas: the F64 and fast forms");
    if (!params || !out || count < 1) return set_err(MPCD_ERR_INVALID_ARG, "null argument or empty batch");
    *out = nullptr;
    mpcd_batch* b = new mpcd_batch();
    b->device = device;
    for (int i = 0; i < count; ++i) {
        mpcd_ctx* c = nullptr;
        const int rc = mpcd_ctx_create_form(params + i, device, MPCD_FORM_FAST, &c);
        if (rc) {
            const std::string msg = "replica " + std::to_string(i) + ": " + g_err;
            mpcd_batch_destroy(b);
            return set_err(rc, msg);
        }
        b->members.push_back(c);
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->start) != cudaSuccess || cudaEventCreate(&b->stop) != cudaSuccess) {
        cudaGetLastError();
        mpcd_batch_destroy(b);
        return set_err(MPCD_ERR_CUDA, "batch stream");
    }
    const int rc = fast_batch_init(b);
    if (rc) {
        const std::string msg = g_err;
        mpcd_batch_destroy(b);
        return set_err(rc, msg);
    }
    *out = b;
    return MPCD_OK;
}

int mpcd_batch_size(mpcd_batch* b) { return b ? (int)b->members.size() : 0; }

mpcd_ctx* mpcd_batch_member(mpcd_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->members.size()) return nullptr;
    return b->members[(size_t)i];
}

int mpcd_batch_step(mpcd_batch* b, int64_t step0, int64_t nsteps, double* device_seconds) {
    if (!b) return set_err(MPCD_ERR_INVALID_ARG, "null batch");
    if (nsteps < 0) return set_err(MPCD_ERR_INVALID_ARG, "nsteps must be >= 0");
    if (b->fast) return fast_batch_step(b, step0, nsteps, device_seconds);
    for (mpcd_ctx* c : b->members)
        if (!c->pc.useIncompressibleRedistribution || !c->pc.useZoneRedistribution || !c->pc.useLiquidClosure)
            return set_err(MPCD_ERR_INVALID_ARG, "the benchmark step needs useIncompressibleRedistribution, useZoneRedistribution and useLiquidClosure");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaEventRecord(b->start, b->stream));
    for (mpcd_ctx* c : b->members) CUDA_TRY(cudaStreamWaitEvent(c->stream, b->start, 0));
    for (int64_t k = 1; k <= nsteps; ++k) {
        const int64_t s = step0 + k;
        // the graph needs every replica's sign stream prefetched, one common buffer parity and
        // every replica's collision tile shape tuned
        bool graph = b->useGraphs;
        for (mpcd_ctx* c : b->members)
            graph = graph && c->useGraphs && c->signsStep[s & 1] == s && c->xv == b->members[0]->xv &&
                    c->pp == b->members[0]->pp && c->xflip == b->members[0]->xflip && c->collideShape >= 0;
        const int rc = graph ? batch_graph_step(b, s) : batch_step_body(b, s);
        if (rc) return rc;
    }
    for (size_t i = 0; i < b->members.size(); ++i) {
        mpcd_ctx* c = b->members[i];
        CUDA_TRY(cudaEventRecord(b->done[i], c->stream));
        CUDA_TRY(cudaStreamWaitEvent(b->stream, b->done[i], 0));
        if (c->side) CUDA_TRY(cudaStreamWaitEvent(b->stream, c->signsReady[(step0 + nsteps + 1) & 1], 0));
    }
    CUDA_TRY(cudaEventRecord(b->stop, b->stream));
    CUDA_TRY(cudaEventSynchronize(b->stop));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, b->start, b->stop));
    if (device_seconds) *device_seconds = ms * 1e-3;
    for (mpcd_ctx* c : b->members) {
        const int rc = check_device(c);
        if (rc) return rc;
    }
    return MPCD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- learned closure
static void drop_graphs(mpcd_ctx* c) {
    for (auto& g : c->gexec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// the tensor-core kernels' shared memory opt-in and their persistent grid: tiles of 128 rows,
// at most 4 CTAs per SM
static int tc_setup(int device, int rows, int* grid) {
    CUDA_TRY(cudaFuncSetAttribute(k_mlp_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    CUDA_TRY(cudaFuncSetAttribute(k_mlp_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int tiles = (rows + kTcRows - 1) / kTcRows;
    *grid = std::max(1, std::min(tiles, 4 * sms));
    return MPCD_OK;
}

// the tensor-core training kernel: its shared memory, and the SMs (one CTA each at most)
static int tg_setup(int device, int* sms) {
    CUDA_TRY(cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTgSmem));
    CUDA_TRY(cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, device));
    return MPCD_OK;
}
static unsigned tg_grid(int rows, int sms) { return (unsigned)std::max(1, std::min((rows + 127) / 128, sms)); }

static int ensure_learned_buffers(mpcd_ctx* c) {
    if (c->lparams) return MPCD_OK;
    int rc = tc_setup(c->device, c->Nc, &c->tcGrid);
    if (rc) return rc;
    if ((rc = dalloc(&c->lparams, kParams)) || (rc = dalloc(&c->lmode, 1)) || (rc = dalloc(&c->lcount, 2)) ||
        (rc = dalloc(&c->lsums, 3)) || (rc = dalloc(&c->duLX, (size_t)c->Nc)) || (rc = dalloc(&c->duLY, (size_t)c->Nc)) ||
        (rc = dalloc(&c->redFeat, (size_t)c->Nc)) || (rc = dalloc(&c->duLSum, 3)))
        return rc;
    return MPCD_OK;
}

static int step_flags_ok(const mpcd_ctx* c) {
    if (!c->pc.useIncompressibleRedistribution || !c->pc.useZoneRedistribution || !c->pc.useLiquidClosure)
        return set_err(MPCD_ERR_INVALID_ARG, "the benchmark step needs useIncompressibleRedistribution, useZoneRedistribution and useLiquidClosure");
    if (c->pc.redistributionEnableSurfaceTopology || c->pc.redistributionWallWettingEnabled || c->pc.useInterfaceVelocityReorientation)
        return set_err(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl is restricted to no surface / no wetting / no reorientation");
    return MPCD_OK;
}

// Context-free device work of the trainer: a device, a stream and its buffers, freed on exit.
struct LearnedDev {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> bufs;
    template <typename T>
    int alloc(T** p, size_t count) {
        const int rc = dalloc(p, count);
        if (rc == MPCD_OK) bufs.push_back((void*)*p);
        return rc;
    }
    int open(int dev) {
        device = dev;
        CUDA_TRY(cudaSetDevice(dev));
        CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        return MPCD_OK;
    }
    ~LearnedDev() {
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : bufs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

// synchronises the learned-closure stream and reports its device status
static int learned_status(LearnedDev& D, DevStatus* dS) {
    DevStatus hs{};
    CUDA_TRY(cudaMemcpyAsync(&hs, dS, sizeof hs, cudaMemcpyDeviceToHost, D.stream));
    CUDA_TRY(cudaStreamSynchronize(D.stream));
    if (hs.code) return set_err(MPCD_ERR_DEVICE, std::string(dev_error_text(hs.code)) + " (detail " + std::to_string(hs.detail) + ")");
    return MPCD_OK;
}

static int learned_rows_ok(const float* X, const float* Y, int64_t rows, const float* params) {
    if (!X || !params || rows < 1 || rows > (int64_t)INT32_MAX / kFeat)
        return set_err(MPCD_ERR_INVALID_ARG, "null argument or rows out of range");
    (void)Y;
    return MPCD_OK;
}

extern "C" {

static_assert(kParams == MPCD_LEARNED_PARAMS && kFeat == MPCD_LEARNED_FEATURES && kOut == MPCD_LEARNED_OUTPUTS,
              "C-ABI network layout");

int mpcd_learned_param_count(void) { return kParams; }

int mpcd_learned_init(uint64_t seed, float* params) {
    if (!params) return set_err(MPCD_ERR_INVALID_ARG, "null params");
    uint64_t st = seed;
    auto next = [&st]() {  // splitmix64
        uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    auto fill = [&](int off, int fanOut, int fanIn) {  // Glorot uniform
        const double b = std::sqrt(6.0 / (double)(fanIn + fanOut));
        for (int i = 0; i < fanOut * fanIn; ++i) {
            const double u = (double)(next() >> 11) * 0x1.0p-53;
            params[off + i] = (float)((2.0 * u - 1.0) * b);
        }
    };
    for (int i = 0; i < kParams; ++i) params[i] = 0.0f;
    fill(kOffW1, kHid, kFeat);
    fill(kOffW2, kHid, kHid);
    fill(kOffW3, kOut, kHid);
    return MPCD_OK;  // biases 0; the output scale 0 = set by the trainer
}

int mpcd_learned_set(mpcd_ctx* c, const float* params, double occ_limit) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    drop_graphs(c);  // captured steps hold the previous closure
    if (!params) {
        c->learnedOn = false;
        return MPCD_OK;
    }
    if (!(params[kOffScale] > 0.0f)) return set_err(MPCD_ERR_INVALID_ARG, "the network's output scale is not set (train it first)");
    int rc = ensure_learned_buffers(c);
    if (rc) return rc;
    const int one = 1;
    CUDA_TRY(cudaMemcpy(c->lparams, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(c->lmode, &one, sizeof one, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(c->lcount, 0, sizeof(long long) * 2));
    c->learnedLimit = occ_limit;
    c->learnedOn = true;
    return MPCD_OK;
}

int mpcd_learned_options(mpcd_ctx* c, int32_t bulk_only) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->learnedBulkOnly = bulk_only != 0;
    return MPCD_OK;
}

int mpcd_learned_stats(mpcd_ctx* c, int64_t* plain_steps, int64_t* learned_steps, int32_t* next_mode) {
    if (!c) return set_err(MPCD_ERR_INVALID_ARG, "null context");
    long long n[2] = {0, 0};
    int mode = 0;
    if (c->lcount) {
        CUDA_TRY(cudaSetDevice(c->device));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        CUDA_TRY(cudaMemcpy(n, c->lcount, sizeof n, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(&mode, c->lmode, sizeof mode, cudaMemcpyDeviceToHost));
    }
    if (plain_steps) *plain_steps = n[0];
    if (learned_steps) *learned_steps = n[1];
    if (next_mode) *next_mode = c->learnedOn ? mode : 0;
    return MPCD_OK;
}

int mpcd_learned_samples(mpcd_ctx* c, int64_t step0, int64_t nsteps, int32_t stride, float* features, float* targets,
                         int64_t capacity, int64_t* count) {
    if (!c || !features || !targets || !count) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (nsteps < 0 || stride < 1 || capacity < 0) return set_err(MPCD_ERR_INVALID_ARG, "nsteps, stride or capacity out of range");
    if (c->learnedOn) return set_err(MPCD_ERR_STATE, "samples come from the plain closure: unset the network first");
    int rc = step_flags_ok(c);
    if (rc) return rc;
    *count = 0;
    CUDA_TRY(cudaSetDevice(c->device));
    rc = ensure_learned_buffers(c);
    if (rc) return rc;
    const int perStep = (c->Nc + stride - 1) / stride;
    const int64_t total = std::min<int64_t>(capacity, (int64_t)perStep * nsteps);
    float *dX = nullptr, *dY = nullptr;
    if ((rc = dalloc(&dX, (size_t)std::max<int64_t>(total, 1) * kFeat))) return rc;
    if ((rc = dalloc(&dY, (size_t)std::max<int64_t>(total, 1) * kOut))) {
        cudaFree(dX);
        return rc;
    }
    int64_t got = 0;
    if (c->fast) {
        rc = fast_samples(c, step0, nsteps, stride, dX, dY, total, &got);
        nsteps = 0;  // the loop below is the slot forms'
    }
    c->sampling = !c->fast;
    for (int64_t k = 1; k <= nsteps && rc == MPCD_OK; ++k) {
        const int64_t s = step0 + k;
        rc = step_once(c, s, false);
        if (rc || got >= total) continue;
        const int offset = (int)(s % stride);
        int cnt = (c->Nc - offset + stride - 1) / stride;
        cnt = (int)std::min<int64_t>(cnt, total - got);
        if (cnt <= 0) continue;
        k_learned_samples<<<blocks_for(cnt), kThreads, 0, c->stream>>>(c->P, c->redFeat, c->duRX, c->duRY,
                                                                       c->eosX, c->eosY, c->red, stride, offset, cnt,
                                                                       dX + got * kFeat, dY + got * kOut);
        ++c->launches;
        if (cudaGetLastError() != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "k_learned_samples launch");
        got += cnt;
    }
    c->sampling = false;
    drop_graphs(c);  // graphs captured while sampling write the red fields; recapture without
    if (rc == MPCD_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = set_err(MPCD_ERR_CUDA, "samples");
    if (rc == MPCD_OK && got > 0) {
        if (cudaMemcpy(features, dX, sizeof(float) * kFeat * got, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(targets, dY, sizeof(float) * kOut * got, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = set_err(MPCD_ERR_CUDA, "samples copy");
    }
    cudaFree(dX);
    cudaFree(dY);
    if (rc) return rc;
    *count = got;
    return check_device(c);
}

int mpcd_learned_predict(const float* features, int64_t rows, const float* params, int device, float* out) {
    int rc = learned_rows_ok(features, nullptr, rows, params);
    if (rc) return rc;
    if (!out) return set_err(MPCD_ERR_INVALID_ARG, "null output");
    LearnedDev D;
    float *dX, *dP, *dO;
    DevStatus* dS;
    int grid = 0;
    if ((rc = D.open(device)) || (rc = D.alloc(&dX, (size_t)rows * kFeat)) || (rc = D.alloc(&dP, kParams)) ||
        (rc = D.alloc(&dO, (size_t)rows * kOut)) || (rc = D.alloc(&dS, 1)) || (rc = tc_setup(device, (int)rows, &grid)))
        return rc;
    CUDA_TRY(cudaMemcpyAsync(dX, features, sizeof(float) * kFeat * rows, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemcpyAsync(dP, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemsetAsync(dS, 0, sizeof(DevStatus), D.stream));
    DevParams P{};
    k_mlp_tc<true><<<grid, kTcThreads, kTcSmem, D.stream>>>(P, nullptr, dX, (int)rows, dP, nullptr,
                                                            nullptr, dO, nullptr, nullptr, 0, dS);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, dO, sizeof(float) * kOut * rows, cudaMemcpyDeviceToHost, D.stream));
    DevStatus hs{};
    CUDA_TRY(cudaMemcpyAsync(&hs, dS, sizeof hs, cudaMemcpyDeviceToHost, D.stream));
    CUDA_TRY(cudaStreamSynchronize(D.stream));
    if (hs.code) return set_err(MPCD_ERR_DEVICE, std::string(dev_error_text(hs.code)) + " (detail " + std::to_string(hs.detail) + ")");
    return MPCD_OK;
}

int mpcd_learned_grad(const float* features, const float* targets, int64_t rows, const float* params, int device,
                      float* grad, float* loss) {
    int rc = learned_rows_ok(features, targets, rows, params);
    if (rc) return rc;
    if (!targets || !grad || !loss) return set_err(MPCD_ERR_INVALID_ARG, "null argument");
    if (!(params[kOffScale] > 0.0f)) return set_err(MPCD_ERR_INVALID_ARG, "the network's output scale is not set");
    LearnedDev D;
    float *dX, *dY, *dP, *dG, *dL;
    int* dI;
    DevStatus* dS;
    int sms = 0;
    if ((rc = D.open(device)) || (rc = D.alloc(&dX, (size_t)rows * kFeat)) || (rc = D.alloc(&dY, (size_t)rows * kOut)) ||
        (rc = D.alloc(&dP, kParams)) || (rc = D.alloc(&dG, kParams)) || (rc = D.alloc(&dL, 1)) ||
        (rc = D.alloc(&dI, (size_t)rows)) || (rc = D.alloc(&dS, 1)) || (rc = tg_setup(device, &sms)))
        return rc;
    std::vector<int> idx((size_t)rows);
    for (int64_t i = 0; i < rows; ++i) idx[(size_t)i] = (int)i;
    CUDA_TRY(cudaMemcpyAsync(dX, features, sizeof(float) * kFeat * rows, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemcpyAsync(dY, targets, sizeof(float) * kOut * rows, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemcpyAsync(dP, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemcpyAsync(dI, idx.data(), sizeof(int) * rows, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemsetAsync(dG, 0, sizeof(float) * kParams, D.stream));
    CUDA_TRY(cudaMemsetAsync(dL, 0, sizeof(float), D.stream));
    CUDA_TRY(cudaMemsetAsync(dS, 0, sizeof(DevStatus), D.stream));
    k_mlp_grad_tc<<<tg_grid((int)rows, sms), 128, kTgSmem, D.stream>>>(dX, dY, dI, (int)rows, (int)rows,
                                                                       1.0f / params[kOffScale], dP, dG, dL, dS);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(grad, dG, sizeof(float) * kParams, cudaMemcpyDeviceToHost, D.stream));
    CUDA_TRY(cudaMemcpyAsync(loss, dL, sizeof(float), cudaMemcpyDeviceToHost, D.stream));
    return learned_status(D, dS);
}

int mpcd_learned_train(const float* features, const float* targets, int64_t rows, float* params, int32_t epochs,
                       int32_t batch, float lr, uint64_t seed, int device, float* epoch_loss) {
    int rc = learned_rows_ok(features, targets, rows, params);
    if (rc) return rc;
    if (!targets) return set_err(MPCD_ERR_INVALID_ARG, "null targets");
    if (epochs < 0 || batch < 1 || !(lr > 0.0f)) return set_err(MPCD_ERR_INVALID_ARG, "epochs, batch or lr out of range");
    if (!(params[kOffScale] > 0.0f)) {  // the output scale: RMS of the targets
        double ss = 0.0;
        for (int64_t i = 0; i < rows * kOut; ++i) ss += (double)targets[i] * (double)targets[i];
        const double rms = std::sqrt(ss / (double)(rows * kOut));
        params[kOffScale] = (float)(rms > 0.0 ? rms : 1.0);
    }
    LearnedDev D;
    float *dX, *dY, *dP, *dG, *dM, *dV, *dL;
    int* dI;
    DevStatus* dS;
    int sms = 0;
    const int64_t nb = (rows + batch - 1) / batch;
    if ((rc = D.open(device)) || (rc = D.alloc(&dX, (size_t)rows * kFeat)) || (rc = D.alloc(&dY, (size_t)rows * kOut)) ||
        (rc = D.alloc(&dP, kParams)) || (rc = D.alloc(&dG, kParams)) || (rc = D.alloc(&dM, kParams)) ||
        (rc = D.alloc(&dV, kParams)) || (rc = D.alloc(&dL, (size_t)nb)) || (rc = D.alloc(&dI, (size_t)rows)) ||
        (rc = D.alloc(&dS, 1)) || (rc = tg_setup(device, &sms)))
        return rc;
    CUDA_TRY(cudaMemsetAsync(dS, 0, sizeof(DevStatus), D.stream));
    CUDA_TRY(cudaMemcpyAsync(dX, features, sizeof(float) * kFeat * rows, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemcpyAsync(dY, targets, sizeof(float) * kOut * rows, cudaMemcpyHostToDevice, D.stream));
    CUDA_TRY(cudaMemcpyAsync(dP, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, D.stream));
    for (float* b : {dG, dM, dV}) CUDA_TRY(cudaMemsetAsync(b, 0, sizeof(float) * kParams, D.stream));
    const float yinv = 1.0f / params[kOffScale];
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<int> idx((size_t)rows);
    std::vector<float> lossB((size_t)nb);
    std::mt19937_64 rng(seed);
    int64_t t = 0;
    for (int e = 0; e < epochs; ++e) {
        for (int64_t i = 0; i < rows; ++i) idx[(size_t)i] = (int)i;
        for (int64_t i = rows - 1; i > 0; --i) std::swap(idx[(size_t)i], idx[(size_t)(rng() % (uint64_t)(i + 1))]);
        CUDA_TRY(cudaStreamSynchronize(D.stream));  // idx is re-filled on the host
        CUDA_TRY(cudaMemcpyAsync(dI, idx.data(), sizeof(int) * rows, cudaMemcpyHostToDevice, D.stream));
        CUDA_TRY(cudaMemsetAsync(dL, 0, sizeof(float) * nb, D.stream));
        for (int64_t b = 0; b < nb; ++b) {
            const int64_t r0 = b * batch;
            const int n = (int)std::min<int64_t>(batch, rows - r0);
            ++t;
            k_mlp_grad_tc<<<tg_grid(n, sms), 128, kTgSmem, D.stream>>>(dX, dY, dI + r0, n, n, yinv, dP, dG, dL + b, dS);
            k_adam<<<(kTrained + 255) / 256, 256, 0, D.stream>>>(dP, dG, dM, dV, kTrained, lr, b1, b2, eps,
                                                                 1.0f - (float)std::pow((double)b1, (double)t),
                                                                 1.0f - (float)std::pow((double)b2, (double)t));
        }
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(lossB.data(), dL, sizeof(float) * nb, cudaMemcpyDeviceToHost, D.stream));
        if ((rc = learned_status(D, dS))) return rc;
        if (epoch_loss) {
            double sum = 0.0;
            for (int64_t b = 0; b < nb; ++b) sum += (double)lossB[(size_t)b] * (double)std::min<int64_t>(batch, rows - b * batch);
            epoch_loss[e] = (float)(sum / (double)rows);
        }
    }
    CUDA_TRY(cudaMemcpyAsync(params, dP, sizeof(float) * kTrained, cudaMemcpyDeviceToHost, D.stream));
    CUDA_TRY(cudaStreamSynchronize(D.stream));
    return MPCD_OK;
}

}  // extern "C"
