// mpcd_b200.hpp — the reference's C++ API (namespace mpcd) over the C-ABI of libmpcd_b200.so.
//
// Header-only C++17. A program written against the reference's headers (include/types.h,
// boundary_conditions.h, common_grid.h, srd_collision.h, zone_pass_openmp.h, liquid_closure.h,
// params_io.h, state_io.h, dump_io.h) compiles against this header instead (the same-named
// headers under include/compat/ include it) and links libmpcd_b200.so in place of the
// reference's sources. Types keep the reference's names, members and defaults; functions keep
// its signatures, in-place/by-value ownership and std::runtime_error messages.
//
// Every physics call runs on the GPU: the shim uploads the caller's vectors to a device
// context, runs the phase there and downloads the result. A context is cached per thread
// and reused while the parameters stay the same. For long runs, mpcd::b200::Session keeps
// the state resident on the device across steps instead (the fast path).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mpcd_c.h"

namespace mpcd {

// ------------------------------------------------------------------------- types
// reference include/types.h:10-72
struct Params {
    int Nx;
    int Ny;
    int Nc;
    int n;
    double Lx;
    double Ly;
    double dt;
    double a0;
    double alpha;
    double kBT;
    double g;
    double bodyForceX;
    bool useThermostat;
    bool keepMeanFlow;
    std::string boundary_left;
    std::string boundary_right;
    std::string boundary_bottom;
    std::string boundary_top;
    double Utop;
    double Ubottom;
    double wallSigma;
    bool noSurfaceCase;
    bool redistributionEnableSurfaceTopology;
    bool redistributionWallWettingEnabled;
    bool useInterfaceVelocityReorientation;
    bool useIncompressibleRedistribution;
    bool redistribAfterCollision;
    bool useZoneRedistribution;
    int zoneTileNx;
    int zoneTileNy;
    bool zoneUseShiftedSecondPass;
    bool zonePassthroughMode;
    bool zoneSingleFullDomainMode;
    bool enableMomentumCorrectionPostRedistribution;
    double gamma;
    double coef;
    std::string highMode;
    std::string lowMode;
    int maxRedistribPasses;
    bool useLocalFluidFractionThresholds;
    double fluidFracGain;
    double lowThrFloor;
    double highThrFloor;
    double lowThrBulkOverride;
    bool useLiquidClosure;
    bool useOptimalBetaRepair;
    double betaRepair;
    double betaEOS;
    double Kvirial;
    bool smoothPdriveAtInterzone;
    int smoothPdriveInterzoneWidthCells;
    double smoothPdriveInterzoneBlend;
    bool smoothPdriveIncludeShiftedLayouts;
};

// reference include/types.h:74-79: x and v interleaved [x1, y1, x2, y2, ...]
struct State {
    std::vector<double> x;
    std::vector<double> v;
    std::vector<std::uint8_t> type;
    std::vector<double> r0;
};

// reference include/types.h:81-95
struct CellFields {
    int Nx;
    int Ny;
    std::vector<std::int32_t> N;
    std::vector<double> Ux;
    std::vector<double> Uy;
    std::vector<double> Px;
    std::vector<double> Py;
    std::vector<double> T;
    std::vector<double> rho;
    std::vector<double> Pkin;
    std::vector<double> Pvir;
    std::vector<double> P;
    std::vector<double> rhoTarget;
};

// reference include/types.h:97-111
struct WallInfo {
    int nBot = 0;
    int nTop = 0;
    int nLeft = 0;
    int nRight = 0;
    double dEwall = 0.0;
    double dPxBot = 0.0;
    double dPxTop = 0.0;
    double dPyBot = 0.0;
    double dPyTop = 0.0;
    double dPxLeft = 0.0;
    double dPxRight = 0.0;
    double dPyLeft = 0.0;
    double dPyRight = 0.0;
};

// reference include/types.h:113-123
struct RunOutStep {
    std::string inputTag;
    std::string outputTag;
    double pBotInst = 0.0;
    double pTopInst = 0.0;
    double pMeanInst = 0.0;
    std::array<double, 6> redistribStats{};
    std::array<double, 10> redistDiag{};
    std::string layoutMode;
    int nZonesExecuted = 0;
};

// reference include/zone_pass.h:12-30: one zone of a layout and the layout
struct ZoneDescriptor {
    int id = 0;
    std::vector<int> cellIds;
    std::vector<char> maskVec;
};

struct ZoneLayout {
    std::string mode;
    std::vector<ZoneDescriptor> zones;
    std::vector<std::int32_t> ownerMap;  // Nc entries, c = iy + Ny * ix
};

// reference include/zone_pass.h:24-29: what run_zone_kernel_inplace reports
struct ZoneKernelStats {
    std::array<double, 6> stats{};
    std::array<double, 10> diag{};
    int movedDense = 0;
    int movedSparse = 0;
};

// reference include/zone_pass.h: the serial pass's result
struct ZonePassMetrics {
    double occStdBefore = 0.0;
    double occStdAfter = 0.0;
    double outBandBefore = 0.0;
    double outBandAfter = 0.0;
    int nDenseBefore = 0;
    int nDenseAfter = 0;
    int nSparseBefore = 0;
    int nSparseAfter = 0;
    int nEmptyActiveBefore = 0;
    int nEmptyActiveAfter = 0;
    int nParticlesMovedDense = 0;
    int nParticlesMovedSparse = 0;
    int nZonesExecuted = 0;
    double corrRmsDU = 0.0;
    double corrMaxDU = 0.0;
    double momentumDeltaX = 0.0;
    double momentumDeltaY = 0.0;
    std::string layoutMode;
};

struct ZonePassResult {
    State stateOut;
    CellFields beforeFields;
    CellFields afterFields;
    ZonePassMetrics metrics;
    std::vector<std::int32_t> zoneOwnerMap;
};

// reference include/zone_pass_openmp.h:12-33. Times are device seconds of the pass.
struct OpenMPPassMetrics {
    int nZones = 0;
    int nThreadsRequested = 1;
    int nThreadsUsed = 1;
    int nParticlesMovedDense = 0;
    int nParticlesMovedSparse = 0;
    double corrRmsDU = 0.0;
    double corrMaxDU = 0.0;
    double timeLayout = 0.0;
    double timeZoneExtract = 0.0;
    double timeSnapshot = 0.0;
    double timeAlloc = 0.0;
    double timeKernel = 0.0;
    double timePack = 0.0;
    double timeMerge = 0.0;
};

struct OpenMPPassResult {
    State stateOut;
    std::vector<std::int32_t> zoneOwnerMap;
    OpenMPPassMetrics metrics;
};

// reference include/liquid_closure.h:11-44
struct LiquidClosureMetrics {
    double betaRepairOpt = 0.0;
    double betaRepairApplied = 0.0;
    double betaRepairNum = 0.0;
    double betaRepairDen = 0.0;
    double betaEOSApplied = 0.0;
    double meanPdriveRaw = 0.0;
    double meanPdrive = 0.0;
    double rmsRepairDU = 0.0;
    double meanAbsRepairDU = 0.0;
    double maxRepairDU = 0.0;
    double rmsEOSDU = 0.0;
    double maxEOSDU = 0.0;
    double momentumDeltaX = 0.0;
    double momentumDeltaY = 0.0;
    int nMaskedInterzoneCells = 0;
};

struct LiquidClosureResult {
    State stateOut;
    State stateRepaired;
    CellFields refFields;
    CellFields redFields;
    CellFields repairedFields;
    CellFields outFields;
    std::vector<double> pdriveRaw;
    std::vector<double> pdrive;
    std::vector<double> duRepairX;
    std::vector<double> duRepairY;
    std::vector<double> duEOSX;
    std::vector<double> duEOSY;
    std::vector<std::int32_t> interzoneMask;
    LiquidClosureMetrics metrics;
};

// ------------------------------------------------------------------------- C-ABI glue
namespace b200 {

inline void check(int rc) {
    if (rc != MPCD_OK) throw std::runtime_error(mpcd_last_error());
}

inline int bc_mode(const std::string& s) {
    if (s == "periodic") return MPCD_BC_PERIODIC;
    if (s == "thermalize") return MPCD_BC_THERMALIZE;
    if (s == "bounceback") return MPCD_BC_BOUNCEBACK;
    if (s == "specular") return MPCD_BC_SPECULAR;
    return MPCD_BC_UNKNOWN;
}

inline mpcd_params_c to_c(const Params& p) {
    mpcd_params_c c;
    std::memset(&c, 0, sizeof c);
    c.Nx = p.Nx; c.Ny = p.Ny; c.Nc = p.Nc; c.n = p.n;
    c.Lx = p.Lx; c.Ly = p.Ly; c.dt = p.dt; c.a0 = p.a0;
    c.alpha = p.alpha; c.kBT = p.kBT; c.g = p.g; c.bodyForceX = p.bodyForceX;
    c.useThermostat = p.useThermostat; c.keepMeanFlow = p.keepMeanFlow;
    c.boundary_left = bc_mode(p.boundary_left);
    c.boundary_right = bc_mode(p.boundary_right);
    c.boundary_bottom = bc_mode(p.boundary_bottom);
    c.boundary_top = bc_mode(p.boundary_top);
    c.Utop = p.Utop; c.Ubottom = p.Ubottom; c.wallSigma = p.wallSigma;
    c.noSurfaceCase = p.noSurfaceCase;
    c.redistributionEnableSurfaceTopology = p.redistributionEnableSurfaceTopology;
    c.redistributionWallWettingEnabled = p.redistributionWallWettingEnabled;
    c.useInterfaceVelocityReorientation = p.useInterfaceVelocityReorientation;
    c.useIncompressibleRedistribution = p.useIncompressibleRedistribution;
    c.redistribAfterCollision = p.redistribAfterCollision;
    c.useZoneRedistribution = p.useZoneRedistribution;
    c.zoneTileNx = p.zoneTileNx; c.zoneTileNy = p.zoneTileNy;
    c.zoneUseShiftedSecondPass = p.zoneUseShiftedSecondPass;
    c.zonePassthroughMode = p.zonePassthroughMode;
    c.zoneSingleFullDomainMode = p.zoneSingleFullDomainMode;
    c.enableMomentumCorrectionPostRedistribution = p.enableMomentumCorrectionPostRedistribution;
    c.gamma = p.gamma; c.coef = p.coef;
    c.highMode = (p.highMode == "1+coef") ? MPCD_THR_ONE_PLUS_COEF : MPCD_THR_COEF;
    c.lowMode = (p.lowMode == "1+coef") ? MPCD_THR_ONE_PLUS_COEF : MPCD_THR_COEF;
    c.maxRedistribPasses = p.maxRedistribPasses;
    c.useLocalFluidFractionThresholds = p.useLocalFluidFractionThresholds;
    c.fluidFracGain = p.fluidFracGain; c.lowThrFloor = p.lowThrFloor; c.highThrFloor = p.highThrFloor;
    c.lowThrBulkOverride = p.lowThrBulkOverride;
    c.useLiquidClosure = p.useLiquidClosure; c.useOptimalBetaRepair = p.useOptimalBetaRepair;
    c.betaRepair = p.betaRepair; c.betaEOS = p.betaEOS; c.Kvirial = p.Kvirial;
    c.smoothPdriveAtInterzone = p.smoothPdriveAtInterzone;
    c.smoothPdriveInterzoneWidthCells = p.smoothPdriveInterzoneWidthCells;
    c.smoothPdriveInterzoneBlend = p.smoothPdriveInterzoneBlend;
    c.smoothPdriveIncludeShiftedLayouts = p.smoothPdriveIncludeShiftedLayouts;
    return c;
}

// The CUDA device the shim's contexts live on (default 0).
inline int& device() {
    static int d = 0;
    return d;
}

// A device context for one parameter set (RAII over mpcd_ctx).
class Context {
public:
    explicit Context(const Params& p, int dev) : pc_(to_c(p)), dev_(dev) { check(mpcd_ctx_create(&pc_, dev, &h_)); }
    ~Context() {
        if (h_) mpcd_ctx_destroy(h_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    mpcd_ctx* get() const { return h_; }
    bool matches(const mpcd_params_c& pc, int dev) const { return dev == dev_ && std::memcmp(&pc, &pc_, sizeof pc) == 0; }

private:
    mpcd_params_c pc_;
    int dev_;
    mpcd_ctx* h_ = nullptr;
};

// The calling thread's context for these parameters; re-created when they change.
inline mpcd_ctx* context_for(const Params& p) {
    thread_local std::unique_ptr<Context> cached;
    const mpcd_params_c pc = to_c(p);
    if (!cached || !cached->matches(pc, device())) {
        cached.reset();
        cached.reset(new Context(p, device()));
    }
    return cached->get();
}

// Rethrows a wall-mode failure with the reference's message, which names the mode string.
inline void check_bc(int rc, const Params& p) {
    if (rc == MPCD_ERR_UNSUPPORTED_BC) {
        const std::string m = mpcd_last_error();
        const char* sides[4] = {"left", "right", "bottom", "top"};
        const std::string* modes[4] = {&p.boundary_left, &p.boundary_right, &p.boundary_bottom, &p.boundary_top};
        for (int k = 0; k < 4; ++k)
            if (m.find(std::string("boundary_") + sides[k]) != std::string::npos)
                throw std::runtime_error(std::string("Unsupported boundary_") + sides[k] + " mode: " + *modes[k]);
    }
    check(rc);
}

inline void upload(mpcd_ctx* c, const std::vector<double>& x, const std::vector<double>& v, int n) {
    check(mpcd_set_state(c, x.data(), v.data(), n));
}

inline CellFields make_fields(const Params& p) {
    CellFields G;
    G.Nx = p.Nx;
    G.Ny = p.Ny;
    const std::size_t nc = static_cast<std::size_t>(p.Nc);
    G.N.assign(nc, 0);
    for (auto* f : {&G.Ux, &G.Uy, &G.Px, &G.Py, &G.T, &G.rho, &G.Pkin, &G.Pvir, &G.P, &G.rhoTarget}) f->assign(nc, 0.0);
    return G;
}

inline mpcd_cellfields_c view(CellFields& G) {
    mpcd_cellfields_c c;
    c.N = G.N.data();
    c.Ux = G.Ux.data(); c.Uy = G.Uy.data(); c.Px = G.Px.data(); c.Py = G.Py.data(); c.T = G.T.data();
    c.rho = G.rho.data(); c.Pkin = G.Pkin.data(); c.Pvir = G.Pvir.data(); c.P = G.P.data();
    c.rhoTarget = G.rhoTarget.data();
    return c;
}

// Device-resident stepping: the state stays on the GPU across steps (the benchmark loop of
// src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:237-279).
class Session {
public:
    Session(const Params& p, const State& s, int dev = device()) : p_(p), ctx_(p, dev) {
        if (s.x.size() != 2u * (std::size_t)p.n || s.v.size() != 2u * (std::size_t)p.n)
            throw std::runtime_error("Session: unexpected state size");
        upload(ctx_.get(), s.x, s.v, p.n);
    }
    // steps step0+1 .. step0+nsteps; fills *last with the metrics row of the last step if given
    void step(std::int64_t step0, std::int64_t nsteps, mpcd_step_metrics_c* last = nullptr) {
        check_bc(mpcd_step(ctx_.get(), step0, nsteps, last), p_);
    }
    void get(State& s) {
        s.x.resize(2u * (std::size_t)p_.n);
        s.v.resize(2u * (std::size_t)p_.n);
        check(mpcd_get_state(ctx_.get(), s.x.data(), s.v.data()));
    }
    CellFields fields(double rhoTarget) {
        CellFields G = make_fields(p_);
        mpcd_cellfields_c c = view(G);
        check(mpcd_cell_fields(ctx_.get(), rhoTarget, &c));
        return G;
    }
    mpcd_ctx* handle() const { return ctx_.get(); }

private:
    Params p_;
    Context ctx_;
};

}  // namespace b200

// ------------------------------------------------------------------------- grid helpers
// reference src/common_grid.cpp:9-19
inline int cell_id_from_position(double x, double y, const Params& params) {
    const double dx = params.Lx / static_cast<double>(params.Nx);
    const double dy = params.Ly / static_cast<double>(params.Ny);
    int ix = static_cast<int>(std::floor(x / dx));
    int iy = static_cast<int>(std::floor(y / dy));
    ix = ix < 0 ? 0 : (ix >= params.Nx ? params.Nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= params.Ny ? params.Ny - 1 : iy);
    return iy + params.Ny * ix;
}

// reference src/common_grid.cpp:21-30
inline std::vector<int> build_cell_ids(const std::vector<double>& x, const Params& params) {
    if (x.size() != static_cast<std::size_t>(2 * params.n)) throw std::runtime_error("build_cell_ids: unexpected x size");
    std::vector<int> cid(static_cast<std::size_t>(params.n));
    for (int i = 0; i < params.n; ++i) cid[(std::size_t)i] = cell_id_from_position(x[2 * (std::size_t)i], x[2 * (std::size_t)i + 1], params);
    return cid;
}

// reference src/boundary_conditions.cpp:9-17
inline bool is_periodic_pair(const Params& params, const std::string& axis_name) {
    if (axis_name == "x") return params.boundary_left == "periodic" && params.boundary_right == "periodic";
    if (axis_name == "y") return params.boundary_bottom == "periodic" && params.boundary_top == "periodic";
    throw std::runtime_error("Unknown axis in is_periodic_pair: " + axis_name);
}

// ------------------------------------------------------------------------- physics (GPU)
// reference src/boundary_conditions.cpp:19-203
inline void apply_bc_general(std::vector<double>& x, std::vector<double>& v, const Params& params, WallInfo& info,
                             std::uint64_t rng_seed) {
    mpcd_ctx* c = b200::context_for(params);
    b200::upload(c, x, v, params.n);
    mpcd_wallinfo_c w;
    b200::check_bc(mpcd_apply_bc(c, rng_seed, &w), params);
    b200::check(mpcd_get_state(c, x.data(), v.data()));
    info.nBot = w.nBot; info.nTop = w.nTop; info.nLeft = w.nLeft; info.nRight = w.nRight;
    info.dEwall = w.dEwall;
    info.dPxBot = w.dPxBot; info.dPxTop = w.dPxTop; info.dPyBot = w.dPyBot; info.dPyTop = w.dPyTop;
    info.dPxLeft = w.dPxLeft; info.dPxRight = w.dPxRight; info.dPyLeft = w.dPyLeft; info.dPyRight = w.dPyRight;
}

// reference src/srd_collision.cpp:9-45
inline std::vector<int> srd_cell_id_with_random_shift(const std::vector<double>& x, const Params& params,
                                                      std::uint64_t rng_seed) {
    mpcd_ctx* c = b200::context_for(params);
    b200::upload(c, x, x, params.n);  // the cells depend on positions only
    std::vector<int> cid(static_cast<std::size_t>(params.n));
    b200::check(mpcd_srd_shift_cells(c, rng_seed, cid.data()));
    return cid;
}

// reference src/srd_collision.cpp:47-140
inline void srd_collision_step(std::vector<double>& v, const std::vector<int>& cid, const Params& params,
                               std::uint64_t rng_seed) {
    if (cid.size() != static_cast<std::size_t>(params.n)) throw std::runtime_error("srd_collision_step: unexpected cid size");
    mpcd_ctx* c = b200::context_for(params);
    b200::upload(c, v, v, params.n);  // the collision reads velocities and the given cells only
    b200::check(mpcd_srd_collide_cells(c, cid.data(), rng_seed));
    b200::check(mpcd_get_state(c, nullptr, v.data()));
}

// reference src/common_grid.cpp:32-100
inline CellFields compute_cell_fields(const std::vector<double>& x, const std::vector<double>& v, const Params& params,
                                      double rhoTargetScalar) {
    if (x.size() != static_cast<std::size_t>(2 * params.n) || v.size() != static_cast<std::size_t>(2 * params.n))
        throw std::runtime_error("compute_cell_fields: unexpected state size");
    mpcd_ctx* c = b200::context_for(params);
    b200::upload(c, x, v, params.n);
    CellFields G = b200::make_fields(params);
    mpcd_cellfields_c view = b200::view(G);
    b200::check(mpcd_cell_fields(c, rhoTargetScalar, &view));
    return G;
}

// reference src/zone_pass_openmp.cpp:176-202 (all four entry points share the snapshot
// semantics of :34-172; the GPU runs every zone of the pass at once)
inline OpenMPPassResult run_zone_pass_openmp(const State& stateIn, const Params& params, const std::string& layoutMode,
                                             std::uint64_t rngSeedBase, int nThreadsRequested) {
    mpcd_ctx* c = b200::context_for(params);
    if (stateIn.x.size() != 2u * (std::size_t)params.n || stateIn.v.size() != 2u * (std::size_t)params.n)
        throw std::runtime_error("run_zone_pass_openmp: unexpected state size");
    const int mode = (layoutMode == "shifted") ? MPCD_LAYOUT_SHIFTED : MPCD_LAYOUT_BASE;
    OpenMPPassResult out;
    out.stateOut = stateIn;
    b200::upload(c, stateIn.x, stateIn.v, params.n);
    mpcd_pass_metrics_c m;
    b200::check(mpcd_zone_pass(c, mode, rngSeedBase, &m));
    b200::check(mpcd_get_state(c, out.stateOut.x.data(), out.stateOut.v.data()));
    out.zoneOwnerMap.assign(static_cast<std::size_t>(params.Nc), 0);
    b200::check(mpcd_zone_owner_map(c, params.zoneSingleFullDomainMode ? MPCD_LAYOUT_SINGLE_FULL : mode, out.zoneOwnerMap.data()));
    OpenMPPassMetrics& M = out.metrics;
    M.nZones = m.nZones;
    M.nThreadsRequested = nThreadsRequested;
    M.nThreadsUsed = m.nThreadsUsed;
    M.nParticlesMovedDense = m.nParticlesMovedDense;
    M.nParticlesMovedSparse = m.nParticlesMovedSparse;
    M.corrRmsDU = m.corrRmsDU;
    M.corrMaxDU = m.corrMaxDU;
    M.timeLayout = m.timeLayout; M.timeZoneExtract = m.timeZoneExtract; M.timeSnapshot = m.timeSnapshot;
    M.timeAlloc = m.timeAlloc; M.timeKernel = m.timeKernel; M.timePack = m.timePack; M.timeMerge = m.timeMerge;
    return out;
}
inline OpenMPPassResult run_zone_pass_openmp_base(const State& stateIn, const Params& params, std::uint64_t rngSeedBase,
                                                  int nThreadsRequested) {
    return run_zone_pass_openmp(stateIn, params, "base", rngSeedBase, nThreadsRequested);
}
inline OpenMPPassResult run_zone_pass_sync_serial(const State& stateIn, const Params& params, const std::string& layoutMode,
                                                  std::uint64_t rngSeedBase) {
    return run_zone_pass_openmp(stateIn, params, layoutMode, rngSeedBase, 1);
}
inline OpenMPPassResult run_zone_pass_sync_serial_base(const State& stateIn, const Params& params, std::uint64_t rngSeedBase) {
    return run_zone_pass_openmp(stateIn, params, "base", rngSeedBase, 1);
}

namespace b200 {
// Occupancy diagnostics of a count field (reference src/zone_pass.cpp:975-1047). The
// threshold maps of those functions only matter for empty cells, which can be neither dense
// nor sparse, so the bulk thresholds decide every cell.
struct CountStats {
    double occStd, outBand;
    int nDense, nSparse, nEmpty;
};
inline CountStats count_stats(const std::vector<std::int32_t>& N, const Params& p) {
    const double highThr = (p.highMode == "1+coef") ? p.gamma * (1.0 + p.coef) : p.gamma + p.gamma * p.coef;
    double lowThr = (p.lowMode == "1+coef") ? p.gamma / (1.0 + p.coef) : p.gamma - p.gamma * p.coef;
    if (std::isfinite(p.lowThrBulkOverride)) lowThr = p.lowThrBulkOverride;
    CountStats s{0.0, 0.0, 0, 0, 0};
    if (N.empty()) return s;
    double sum = 0.0;
    for (std::int32_t n : N) sum += static_cast<double>(n);
    const double mean = sum / static_cast<double>(N.size());
    double acc = 0.0;
    int nOut = 0;
    for (std::int32_t n : N) {
        const double d = static_cast<double>(n) - mean;
        acc += d * d;
        const bool dense = static_cast<double>(n) > highThr;
        const bool sparse = n > 0 && static_cast<double>(n) < lowThr;
        s.nDense += dense;
        s.nSparse += sparse;
        s.nEmpty += (n == 0);
        nOut += (dense || sparse);
    }
    s.occStd = std::sqrt(acc / static_cast<double>(N.size())) / std::max(p.gamma, 1e-30);
    s.outBand = static_cast<double>(nOut) / static_cast<double>(N.size());
    return s;
}
inline std::pair<double, double> total_momentum(const std::vector<double>& v, int n) {
    double px = 0.0, py = 0.0;
    for (int i = 0; i < n; ++i) {
        px += v[2 * (std::size_t)i];
        py += v[2 * (std::size_t)i + 1];
    }
    return {px, py};
}
}  // namespace b200

// reference src/zone_pass.cpp:1096-1163: the zones one after another, in place
inline ZonePassResult run_zone_pass(const State& stateIn, const Params& params, const std::string& layoutMode,
                                    std::uint64_t rngSeedBase) {
    mpcd_ctx* c = b200::context_for(params);
    if (stateIn.x.size() != 2u * (std::size_t)params.n || stateIn.v.size() != 2u * (std::size_t)params.n)
        throw std::runtime_error("run_zone_pass: unexpected state size");
    const int mode = (layoutMode == "shifted") ? MPCD_LAYOUT_SHIFTED : MPCD_LAYOUT_BASE;
    const double rhoTarget = params.gamma / ((params.Lx / (double)params.Nx) * (params.Ly / (double)params.Ny));
    ZonePassResult out;
    out.stateOut = stateIn;
    b200::upload(c, stateIn.x, stateIn.v, params.n);
    out.beforeFields = b200::make_fields(params);
    mpcd_cellfields_c bv = b200::view(out.beforeFields);
    b200::check(mpcd_cell_fields(c, rhoTarget, &bv));
    mpcd_pass_metrics_c m;
    b200::check(mpcd_zone_pass_serial(c, mode, rngSeedBase, &m));
    b200::check(mpcd_get_state(c, out.stateOut.x.data(), out.stateOut.v.data()));
    out.afterFields = b200::make_fields(params);
    mpcd_cellfields_c av = b200::view(out.afterFields);
    b200::check(mpcd_cell_fields(c, rhoTarget, &av));
    out.zoneOwnerMap.assign(static_cast<std::size_t>(params.Nc), 0);
    b200::check(mpcd_zone_owner_map(c, params.zoneSingleFullDomainMode ? MPCD_LAYOUT_SINGLE_FULL : mode, out.zoneOwnerMap.data()));
    ZonePassMetrics& M = out.metrics;
    M.layoutMode = layoutMode;
    M.nZonesExecuted = m.nZones;
    const auto b = b200::count_stats(out.beforeFields.N, params), a = b200::count_stats(out.afterFields.N, params);
    M.occStdBefore = b.occStd; M.occStdAfter = a.occStd;
    M.outBandBefore = b.outBand; M.outBandAfter = a.outBand;
    M.nDenseBefore = b.nDense; M.nDenseAfter = a.nDense;
    M.nSparseBefore = b.nSparse; M.nSparseAfter = a.nSparse;
    M.nEmptyActiveBefore = b.nEmpty; M.nEmptyActiveAfter = a.nEmpty;
    M.nParticlesMovedDense = m.nParticlesMovedDense;
    M.nParticlesMovedSparse = m.nParticlesMovedSparse;
    M.corrRmsDU = m.corrRmsDU;
    M.corrMaxDU = m.corrMaxDU;
    const auto p0 = b200::total_momentum(stateIn.v, params.n), p1 = b200::total_momentum(out.stateOut.v, params.n);
    M.momentumDeltaX = p1.first - p0.first;
    M.momentumDeltaY = p1.second - p0.second;
    return out;
}

// reference src/zone_pass.cpp:1049-1063 (build_layout :173-221): the zones as cell lists in
// ix-outer, iy-inner order, each with its Nc-cell mask, and the ownership map
inline ZoneLayout build_zone_layout(const Params& params, const std::string& mode) {
    const mpcd_params_c pc = b200::to_c(params);
    const int m = (mode == "single_full") ? MPCD_LAYOUT_SINGLE_FULL : (mode == "shifted") ? MPCD_LAYOUT_SHIFTED : MPCD_LAYOUT_BASE;
    std::int32_t nz = 0;
    b200::check(mpcd_zone_layout(&pc, m, &nz, nullptr, 0));
    std::vector<std::int32_t> r(4u * (std::size_t)nz);
    b200::check(mpcd_zone_layout(&pc, m, &nz, r.data(), nz));
    ZoneLayout L;
    L.mode = mode;
    L.ownerMap.assign(static_cast<std::size_t>(params.Nc), 0);
    L.zones.reserve(static_cast<std::size_t>(nz));
    for (int z = 0; z < nz; ++z) {
        ZoneDescriptor d;
        d.id = z + 1;
        d.maskVec.assign(static_cast<std::size_t>(params.Nc), 0);
        for (int ix = r[4 * z]; ix < r[4 * z + 1]; ++ix)
            for (int iy = r[4 * z + 2]; iy < r[4 * z + 3]; ++iy) {
                const int c = iy + params.Ny * ix;
                d.cellIds.push_back(c);
                d.maskVec[static_cast<std::size_t>(c)] = 1;
                L.ownerMap[static_cast<std::size_t>(c)] = d.id;
            }
        L.zones.push_back(std::move(d));
    }
    return L;
}

namespace b200 {
// The cell rectangle [x0, x1) x [y0, y1) a zone covers. The GPU kernels run rectangular zones,
// which is what every layout of build_zone_layout holds; any other cell set is rejected.
inline std::array<int, 4> zone_rect(const ZoneDescriptor& zone, const Params& p) {
    if (zone.cellIds.empty()) throw std::runtime_error("zone has no cells");
    int x0 = p.Nx, x1 = -1, y0 = p.Ny, y1 = -1;
    for (int c : zone.cellIds) {
        if (c < 0 || c >= p.Nc) throw std::runtime_error("zone cell id out of range");
        const int ix = c / p.Ny, iy = c - ix * p.Ny;
        x0 = std::min(x0, ix); x1 = std::max(x1, ix + 1);
        y0 = std::min(y0, iy); y1 = std::max(y1, iy + 1);
    }
    const std::size_t area = (std::size_t)(x1 - x0) * (std::size_t)(y1 - y0);
    std::size_t inMask = 0;
    if (zone.maskVec.size() == static_cast<std::size_t>(p.Nc))
        for (int ix = x0; ix < x1; ++ix)
            for (int iy = y0; iy < y1; ++iy) inMask += zone.maskVec[(std::size_t)iy + (std::size_t)p.Ny * ix] ? 1u : 0u;
    if (zone.cellIds.size() != area || inMask != area)
        throw std::runtime_error("zone is not a rectangle of cells: the GPU zone kernel runs the rectangular zones of build_zone_layout");
    return {x0, x1, y0, y1};
}
}  // namespace b200

// reference src/zone_pass.cpp:1065-1081: one zone's redistribution, in place, on the GPU
inline ZoneKernelStats run_zone_kernel_inplace(std::vector<double>& x, std::vector<double>& v, const Params& params,
                                               const ZoneDescriptor& zone, std::uint64_t rngSeed) {
    if (x.size() != 2u * (std::size_t)params.n || v.size() != 2u * (std::size_t)params.n)
        throw std::runtime_error("run_zone_kernel_inplace: unexpected state size");
    const auto r = b200::zone_rect(zone, params);
    mpcd_ctx* c = b200::context_for(params);
    b200::upload(c, x, v, params.n);
    mpcd_zone_kernel_stats_c s;
    b200::check(mpcd_zone_kernel_inplace(c, r[0], r[1], r[2], r[3], rngSeed, &s));
    b200::check(mpcd_get_state(c, x.data(), v.data()));
    ZoneKernelStats out;
    std::copy(s.stats, s.stats + 6, out.stats.begin());
    std::copy(s.diag, s.diag + 10, out.diag.begin());
    out.movedDense = s.movedDense;
    out.movedSparse = s.movedSparse;
    return out;
}

// reference src/zone_pass.cpp:1083-1094: ids (ascending) of the particles whose cell is in the zone
inline std::vector<int> build_particle_ids_in_zone(const std::vector<double>& x, const Params& params,
                                                   const ZoneDescriptor& zone) {
    if (x.size() != 2u * (std::size_t)params.n) throw std::runtime_error("build_particle_ids_in_zone: unexpected state size");
    const auto r = b200::zone_rect(zone, params);
    mpcd_ctx* c = b200::context_for(params);
    const std::vector<double> v(x.size(), 0.0);
    b200::upload(c, x, v, params.n);
    std::vector<int> ids(static_cast<std::size_t>(params.n));
    std::int64_t count = 0;
    static_assert(sizeof(int) == sizeof(std::int32_t), "int32 ids");
    b200::check(mpcd_particle_ids_in_rect(c, r[0], r[1], r[2], r[3], reinterpret_cast<std::int32_t*>(ids.data()), &count));
    ids.resize(static_cast<std::size_t>(count));
    return ids;
}

// reference src/liquid_closure.cpp:329-444
inline LiquidClosureResult run_liquid_closure(const State& stateRef, const State& stateRed, const Params& params) {
    if (!params.useLiquidClosure) throw std::runtime_error("run_liquid_closure requires useLiquidClosure=true");
    if (stateRef.x.size() != stateRed.x.size() || stateRef.v.size() != stateRed.v.size())
        throw std::runtime_error("run_liquid_closure requires ref/red states with matching sizes");
    mpcd_ctx* c = b200::context_for(params);
    b200::upload(c, stateRef.x, stateRef.v, params.n);
    b200::check(mpcd_save_ref(c));
    b200::upload(c, stateRed.x, stateRed.v, params.n);
    LiquidClosureResult R;
    const std::size_t nc = static_cast<std::size_t>(params.Nc);
    R.stateOut = stateRed;
    R.stateRepaired = stateRed;
    R.refFields = b200::make_fields(params);
    R.redFields = b200::make_fields(params);
    R.repairedFields = b200::make_fields(params);
    R.outFields = b200::make_fields(params);
    for (auto* g : {&R.pdriveRaw, &R.pdrive, &R.duRepairX, &R.duRepairY, &R.duEOSX, &R.duEOSY}) g->assign(nc, 0.0);
    R.interzoneMask.assign(nc, 0);
    mpcd_closure_detail_c d;
    d.repairedX = R.stateRepaired.x.data();
    d.repairedV = R.stateRepaired.v.data();
    d.refFields = b200::view(R.refFields);
    d.redFields = b200::view(R.redFields);
    d.repairedFields = b200::view(R.repairedFields);
    d.outFields = b200::view(R.outFields);
    d.pdriveRaw = R.pdriveRaw.data(); d.pdrive = R.pdrive.data();
    d.duRepairX = R.duRepairX.data(); d.duRepairY = R.duRepairY.data();
    d.duEOSX = R.duEOSX.data(); d.duEOSY = R.duEOSY.data();
    d.interzoneMask = R.interzoneMask.data();
    mpcd_closure_metrics_c m;
    b200::check(mpcd_liquid_closure(c, &m, &d));
    b200::check(mpcd_get_state(c, R.stateOut.x.data(), R.stateOut.v.data()));
    LiquidClosureMetrics& M = R.metrics;
    M.betaRepairOpt = m.betaRepairOpt; M.betaRepairApplied = m.betaRepairApplied;
    M.betaRepairNum = m.betaRepairNum; M.betaRepairDen = m.betaRepairDen; M.betaEOSApplied = m.betaEOSApplied;
    M.meanPdriveRaw = m.meanPdriveRaw; M.meanPdrive = m.meanPdrive;
    M.rmsRepairDU = m.rmsRepairDU; M.meanAbsRepairDU = m.meanAbsRepairDU; M.maxRepairDU = m.maxRepairDU;
    M.rmsEOSDU = m.rmsEOSDU; M.maxEOSDU = m.maxEOSDU;
    M.momentumDeltaX = m.momentumDeltaX; M.momentumDeltaY = m.momentumDeltaY;
    M.nMaskedInterzoneCells = m.nMaskedInterzoneCells;
    return R;
}

// ------------------------------------------------------------------------- files
// reference src/params_io.cpp:74-137 (every key required; booleans "true"/"false"/"1"/"0")
inline Params read_params_kv(const std::string& filepath) {
    mpcd_params_c c;
    if (mpcd_read_params_kv(filepath.c_str(), &c) != MPCD_OK) throw std::runtime_error(mpcd_io_last_error());
    auto str = [&](const char* key) {
        char buf[256];
        if (mpcd_read_kv_string(filepath.c_str(), key, buf, (int)sizeof buf) != MPCD_OK)
            throw std::runtime_error(mpcd_io_last_error());
        return std::string(buf);
    };
    Params p;
    p.Nx = c.Nx; p.Ny = c.Ny; p.Nc = c.Nc; p.n = c.n;
    p.Lx = c.Lx; p.Ly = c.Ly; p.dt = c.dt; p.a0 = c.a0;
    p.alpha = c.alpha; p.kBT = c.kBT; p.g = c.g; p.bodyForceX = c.bodyForceX;
    p.useThermostat = c.useThermostat; p.keepMeanFlow = c.keepMeanFlow;
    p.boundary_left = str("boundary_left");
    p.boundary_right = str("boundary_right");
    p.boundary_bottom = str("boundary_bottom");
    p.boundary_top = str("boundary_top");
    p.Utop = c.Utop; p.Ubottom = c.Ubottom; p.wallSigma = c.wallSigma;
    p.noSurfaceCase = c.noSurfaceCase;
    p.redistributionEnableSurfaceTopology = c.redistributionEnableSurfaceTopology;
    p.redistributionWallWettingEnabled = c.redistributionWallWettingEnabled;
    p.useInterfaceVelocityReorientation = c.useInterfaceVelocityReorientation;
    p.useIncompressibleRedistribution = c.useIncompressibleRedistribution;
    p.redistribAfterCollision = c.redistribAfterCollision;
    p.useZoneRedistribution = c.useZoneRedistribution;
    p.zoneTileNx = c.zoneTileNx; p.zoneTileNy = c.zoneTileNy;
    p.zoneUseShiftedSecondPass = c.zoneUseShiftedSecondPass;
    p.zonePassthroughMode = c.zonePassthroughMode;
    p.zoneSingleFullDomainMode = c.zoneSingleFullDomainMode;
    p.enableMomentumCorrectionPostRedistribution = c.enableMomentumCorrectionPostRedistribution;
    p.gamma = c.gamma; p.coef = c.coef;
    p.highMode = str("highMode");
    p.lowMode = str("lowMode");
    p.maxRedistribPasses = c.maxRedistribPasses;
    p.useLocalFluidFractionThresholds = c.useLocalFluidFractionThresholds;
    p.fluidFracGain = c.fluidFracGain; p.lowThrFloor = c.lowThrFloor; p.highThrFloor = c.highThrFloor;
    p.lowThrBulkOverride = c.lowThrBulkOverride;
    p.useLiquidClosure = c.useLiquidClosure; p.useOptimalBetaRepair = c.useOptimalBetaRepair;
    p.betaRepair = c.betaRepair; p.betaEOS = c.betaEOS; p.Kvirial = c.Kvirial;
    p.smoothPdriveAtInterzone = c.smoothPdriveAtInterzone;
    p.smoothPdriveInterzoneWidthCells = c.smoothPdriveInterzoneWidthCells;
    p.smoothPdriveInterzoneBlend = c.smoothPdriveInterzoneBlend;
    p.smoothPdriveIncludeShiftedLayouts = c.smoothPdriveIncludeShiftedLayouts;
    return p;
}

namespace b200 {
template <typename T>
std::vector<T> read_raw(const std::string& path, std::size_t count) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot open binary file: " + path);
    std::vector<T> out(count);
    in.read(reinterpret_cast<char*>(out.data()), static_cast<std::streamsize>(count * sizeof(T)));
    if (!in) throw std::runtime_error("Cannot read expected payload from: " + path);
    return out;
}
template <typename T>
void write_raw(const std::string& path, const std::vector<T>& data) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw std::runtime_error("Cannot open binary file for writing: " + path);
    out.write(reinterpret_cast<const char*>(data.data()), static_cast<std::streamsize>(data.size() * sizeof(T)));
    if (!out) throw std::runtime_error("Cannot write payload to: " + path);
}
template <typename T>
void write_grid(const std::string& path, int Nx, int Ny, const std::vector<T>& data, const char* what) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw std::runtime_error(std::string("Cannot open ") + what + " grid file for writing: " + path);
    const std::int32_t hdr[2] = {Nx, Ny};
    out.write(reinterpret_cast<const char*>(hdr), sizeof hdr);
    out.write(reinterpret_cast<const char*>(data.data()), static_cast<std::streamsize>(data.size() * sizeof(T)));
    if (!out) throw std::runtime_error(std::string("Failed while writing ") + what + " grid payload");
}
}  // namespace b200

// reference src/state_io.cpp: raw little-endian arrays, x/v/r0 of 2n doubles, type of n bytes
inline State read_state(const std::string& x_path, const std::string& v_path, const std::string& type_path,
                        const std::string& r0_path, bool has_type, bool has_r0, int n_expected) {
    State s;
    const std::size_t n2 = 2u * static_cast<std::size_t>(n_expected);
    s.x = b200::read_raw<double>(x_path, n2);
    s.v = b200::read_raw<double>(v_path, n2);
    if (has_type) s.type = b200::read_raw<std::uint8_t>(type_path, static_cast<std::size_t>(n_expected));
    if (has_r0) s.r0 = b200::read_raw<double>(r0_path, n2);
    return s;
}
inline void write_xy_interleaved(const std::string& filepath, const std::vector<double>& data, int n_expected) {
    if (data.size() != 2u * static_cast<std::size_t>(n_expected))
        throw std::runtime_error("Interleaved XY buffer has unexpected size for write: " + filepath);
    b200::write_raw(filepath, data);
}
inline void write_u8(const std::string& filepath, const std::vector<std::uint8_t>& data, int n_expected) {
    if (data.size() != static_cast<std::size_t>(n_expected)) throw std::runtime_error("u8 buffer has unexpected size for write: " + filepath);
    b200::write_raw(filepath, data);
}

// reference src/dump_io.cpp: int32 Nx, Ny, then N and the ten double fields in struct order
inline void write_cell_fields_bin(const std::string& filepath, const CellFields& G) {
    std::ofstream out(filepath, std::ios::binary);
    if (!out) throw std::runtime_error("Cannot open cell field file for writing: " + filepath);
    const std::int32_t hdr[2] = {G.Nx, G.Ny};
    out.write(reinterpret_cast<const char*>(hdr), sizeof hdr);
    auto put = [&](const auto& v) {
        out.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(v[0])));
        if (!out) throw std::runtime_error("Failed while writing cell field payload");
    };
    put(G.N);
    for (const auto* f : {&G.Ux, &G.Uy, &G.Px, &G.Py, &G.T, &G.rho, &G.Pkin, &G.Pvir, &G.P, &G.rhoTarget}) put(*f);
}

// reference src/params_io.cpp:139-151
inline void write_runout_kv(const std::string& filepath, const RunOutStep& runout) {
    std::ofstream fout(filepath);
    if (!fout) throw std::runtime_error("Cannot open runout file for writing: " + filepath);
    fout << "inputTag=" << runout.inputTag << '\n';
    fout << "outputTag=" << runout.outputTag << '\n';
    fout << "pBotInst=" << runout.pBotInst << '\n';
    fout << "pTopInst=" << runout.pTopInst << '\n';
    fout << "pMeanInst=" << runout.pMeanInst << '\n';
    fout << "layoutMode=" << runout.layoutMode << '\n';
    fout << "nZonesExecuted=" << runout.nZonesExecuted << '\n';
}

// reference src/zone_pass.cpp:1165-1181 (same layout as write_i32_grid_bin_lc)
inline void write_i32_grid_bin(const std::string& filepath, int Nx, int Ny, const std::vector<std::int32_t>& data) {
    if (data.size() != static_cast<std::size_t>(Nx) * static_cast<std::size_t>(Ny))
        throw std::runtime_error("write_i32_grid_bin: unexpected data size");
    b200::write_grid(filepath, Nx, Ny, data, "i32");
}

// reference src/liquid_closure.cpp:446-480
inline void write_f64_grid_bin(const std::string& filepath, int Nx, int Ny, const std::vector<double>& data) {
    if (data.size() != static_cast<std::size_t>(Nx) * static_cast<std::size_t>(Ny))
        throw std::runtime_error("write_f64_grid_bin: unexpected data size");
    b200::write_grid(filepath, Nx, Ny, data, "f64");
}
inline void write_i32_grid_bin_lc(const std::string& filepath, int Nx, int Ny, const std::vector<std::int32_t>& data) {
    if (data.size() != static_cast<std::size_t>(Nx) * static_cast<std::size_t>(Ny))
        throw std::runtime_error("write_i32_grid_bin_lc: unexpected data size");
    b200::write_grid(filepath, Nx, Ny, data, "i32");
}

}  // namespace mpcd
