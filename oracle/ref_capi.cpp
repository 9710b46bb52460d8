// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// extern "C" wrapper around the UNMODIFIED reference sources (compiled from the reference
// project's src/*.cpp by oracle/Makefile into oracle/_ref/libmpcdref.so). It lets the
// tests call the reference's own functions on the same inputs as the oracle and the GPU
// path, through the POD types of include/mpcd_c.h.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "boundary_conditions.h"
#include "common_grid.h"
#include "liquid_closure.h"
#include "srd_collision.h"
#include "types.h"
#include "zone_pass.h"
#include "zone_pass_openmp.h"

#include "mpcd_c.h"

namespace {

thread_local std::string g_err;

const char* bc_name(int m) {
    switch (m) {
        case MPCD_BC_PERIODIC: return "periodic";
        case MPCD_BC_THERMALIZE: return "thermalize";
        case MPCD_BC_BOUNCEBACK: return "bounceback";
        case MPCD_BC_SPECULAR: return "specular";
        default: return "unknown";
    }
}

mpcd::Params to_params(const mpcd_params_c* c) {
    mpcd::Params p{};
    p.Nx = c->Nx; p.Ny = c->Ny; p.Nc = c->Nc; p.n = c->n;
    p.Lx = c->Lx; p.Ly = c->Ly; p.dt = c->dt; p.a0 = c->a0;
    p.alpha = c->alpha; p.kBT = c->kBT; p.g = c->g; p.bodyForceX = c->bodyForceX;
    p.useThermostat = c->useThermostat != 0; p.keepMeanFlow = c->keepMeanFlow != 0;
    p.boundary_left = bc_name(c->boundary_left);
    p.boundary_right = bc_name(c->boundary_right);
    p.boundary_bottom = bc_name(c->boundary_bottom);
    p.boundary_top = bc_name(c->boundary_top);
    p.Utop = c->Utop; p.Ubottom = c->Ubottom; p.wallSigma = c->wallSigma;
    p.noSurfaceCase = c->noSurfaceCase != 0;
    p.redistributionEnableSurfaceTopology = c->redistributionEnableSurfaceTopology != 0;
    p.redistributionWallWettingEnabled = c->redistributionWallWettingEnabled != 0;
    p.useInterfaceVelocityReorientation = c->useInterfaceVelocityReorientation != 0;
    p.useIncompressibleRedistribution = c->useIncompressibleRedistribution != 0;
    p.redistribAfterCollision = c->redistribAfterCollision != 0;
    p.useZoneRedistribution = c->useZoneRedistribution != 0;
    p.zoneTileNx = c->zoneTileNx; p.zoneTileNy = c->zoneTileNy;
    p.zoneUseShiftedSecondPass = c->zoneUseShiftedSecondPass != 0;
    p.zonePassthroughMode = c->zonePassthroughMode != 0;
    p.zoneSingleFullDomainMode = c->zoneSingleFullDomainMode != 0;
    p.enableMomentumCorrectionPostRedistribution = c->enableMomentumCorrectionPostRedistribution != 0;
    p.gamma = c->gamma; p.coef = c->coef;
    p.highMode = (c->highMode == MPCD_THR_ONE_PLUS_COEF) ? "1+coef" : "coef";
    p.lowMode = (c->lowMode == MPCD_THR_ONE_PLUS_COEF) ? "1+coef" : "coef";
    p.maxRedistribPasses = c->maxRedistribPasses;
    p.useLocalFluidFractionThresholds = c->useLocalFluidFractionThresholds != 0;
    p.fluidFracGain = c->fluidFracGain; p.lowThrFloor = c->lowThrFloor;
    p.highThrFloor = c->highThrFloor; p.lowThrBulkOverride = c->lowThrBulkOverride;
    p.useLiquidClosure = c->useLiquidClosure != 0;
    p.useOptimalBetaRepair = c->useOptimalBetaRepair != 0;
    p.betaRepair = c->betaRepair; p.betaEOS = c->betaEOS; p.Kvirial = c->Kvirial;
    p.smoothPdriveAtInterzone = c->smoothPdriveAtInterzone != 0;
    p.smoothPdriveInterzoneWidthCells = c->smoothPdriveInterzoneWidthCells;
    p.smoothPdriveInterzoneBlend = c->smoothPdriveInterzoneBlend;
    p.smoothPdriveIncludeShiftedLayouts = c->smoothPdriveIncludeShiftedLayouts != 0;
    return p;
}

const char* layout_name(int mode) {
    if (mode == MPCD_LAYOUT_SHIFTED) return "shifted";
    if (mode == MPCD_LAYOUT_SINGLE_FULL) return "single_full";
    return "base";
}

mpcd::State make_state(const mpcd::Params& p, const double* x, const double* v) {
    mpcd::State s;
    s.x.assign(x, x + 2 * static_cast<std::size_t>(p.n));
    s.v.assign(v, v + 2 * static_cast<std::size_t>(p.n));
    return s;
}

void copy_fields(const mpcd::CellFields& G, mpcd_cellfields_c* out) {
    if (!out) return;
    const std::size_t nc = G.N.size();
    if (out->N) std::memcpy(out->N, G.N.data(), nc * sizeof(int32_t));
    const std::vector<double>* src[10] = {&G.Ux, &G.Uy, &G.Px, &G.Py, &G.T, &G.rho, &G.Pkin, &G.Pvir, &G.P, &G.rhoTarget};
    double* dst[10] = {out->Ux, out->Uy, out->Px, out->Py, out->T, out->rho, out->Pkin, out->Pvir, out->P, out->rhoTarget};
    for (int k = 0; k < 10; ++k)
        if (dst[k]) std::memcpy(dst[k], src[k]->data(), nc * sizeof(double));
}

void copy_vec(const std::vector<double>& a, double* out) {
    if (out) std::memcpy(out, a.data(), a.size() * sizeof(double));
}

void fill_closure_metrics(const mpcd::LiquidClosureMetrics& m, mpcd_closure_metrics_c* o) {
    if (!o) return;
    o->betaRepairOpt = m.betaRepairOpt; o->betaRepairApplied = m.betaRepairApplied;
    o->betaRepairNum = m.betaRepairNum; o->betaRepairDen = m.betaRepairDen;
    o->betaEOSApplied = m.betaEOSApplied; o->meanPdriveRaw = m.meanPdriveRaw;
    o->meanPdrive = m.meanPdrive; o->rmsRepairDU = m.rmsRepairDU;
    o->meanAbsRepairDU = m.meanAbsRepairDU; o->maxRepairDU = m.maxRepairDU;
    o->rmsEOSDU = m.rmsEOSDU; o->maxEOSDU = m.maxEOSDU;
    o->momentumDeltaX = m.momentumDeltaX; o->momentumDeltaY = m.momentumDeltaY;
    o->nMaskedInterzoneCells = m.nMaskedInterzoneCells;
}

void fill_pass_metrics(const mpcd::OpenMPPassMetrics& m, mpcd_pass_metrics_c* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->nZones = m.nZones; o->nThreadsRequested = m.nThreadsRequested; o->nThreadsUsed = m.nThreadsUsed;
    o->nParticlesMovedDense = m.nParticlesMovedDense; o->nParticlesMovedSparse = m.nParticlesMovedSparse;
    o->corrRmsDU = m.corrRmsDU; o->corrMaxDU = m.corrMaxDU;
    o->timeLayout = m.timeLayout; o->timeZoneExtract = m.timeZoneExtract; o->timeSnapshot = m.timeSnapshot;
    o->timeAlloc = m.timeAlloc; o->timeKernel = m.timeKernel; o->timePack = m.timePack; o->timeMerge = m.timeMerge;
}

// driver diagnostics (reference main_..._shifted_profiled.cpp:105-155), restated verbatim in
// meaning because the driver keeps them in an anonymous namespace
double mean_field(const std::vector<double>& f) {
    if (f.empty()) return 0.0;
    double s = 0.0;
    for (double x : f) s += x;
    return s / static_cast<double>(f.size());
}

void occstd_outband(const mpcd::CellFields& G, const mpcd::Params& params, double* occ, double* out) {
    const double gamma = params.gamma, coef = params.coef;
    double highThr = (params.highMode == "1+coef") ? gamma * (1.0 + coef) : gamma + gamma * coef;
    double lowThr = (params.lowMode == "1+coef") ? gamma / (1.0 + coef) : gamma - gamma * coef;
    if (std::isfinite(params.lowThrBulkOverride)) lowThr = params.lowThrBulkOverride;
    int outBandCount = 0, activeCount = 0;
    std::vector<double> Nact;
    for (double n : G.N) {
        Nact.push_back(n);
        ++activeCount;
        if ((n > highThr) || (n > 0.0 && n < lowThr)) ++outBandCount;
    }
    double mean = 0.0;
    for (double n : Nact) mean += n;
    mean /= std::max(1, activeCount);
    double var = 0.0;
    for (double n : Nact) { double d = n - mean; var += d * d; }
    var /= std::max(1, activeCount);
    *occ = std::sqrt(var) / std::max(gamma, 1e-12);
    *out = static_cast<double>(outBandCount) / std::max(1, activeCount);
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

#define REF_TRY try {
#define REF_CATCH } catch (const std::exception& e) { g_err = e.what(); return 1; }

int ref_stream(const mpcd_params_c* pc, double* x, double* v) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    for (int i = 0; i < p.n; ++i) {
        v[2 * i] += p.bodyForceX * p.dt;
        v[2 * i + 1] += p.g * p.dt;
        x[2 * i] += p.dt * v[2 * i];
        x[2 * i + 1] += p.dt * v[2 * i + 1];
    }
    return 0;
    REF_CATCH
}

int ref_apply_bc(const mpcd_params_c* pc, double* x, double* v, uint64_t seed, mpcd_wallinfo_c* info) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    mpcd::State s = make_state(p, x, v);
    mpcd::WallInfo w;
    mpcd::apply_bc_general(s.x, s.v, p, w, seed);
    std::memcpy(x, s.x.data(), s.x.size() * sizeof(double));
    std::memcpy(v, s.v.data(), s.v.size() * sizeof(double));
    if (info) {
        info->nBot = w.nBot; info->nTop = w.nTop; info->nLeft = w.nLeft; info->nRight = w.nRight;
        info->dEwall = w.dEwall; info->dPxBot = w.dPxBot; info->dPxTop = w.dPxTop;
        info->dPyBot = w.dPyBot; info->dPyTop = w.dPyTop; info->dPxLeft = w.dPxLeft;
        info->dPxRight = w.dPxRight; info->dPyLeft = w.dPyLeft; info->dPyRight = w.dPyRight;
    }
    return 0;
    REF_CATCH
}

int ref_srd_shift_cells(const mpcd_params_c* pc, const double* x, uint64_t seed, int32_t* cid) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    std::vector<double> xv(x, x + 2 * static_cast<std::size_t>(p.n));
    const auto c = mpcd::srd_cell_id_with_random_shift(xv, p, seed);
    for (int i = 0; i < p.n; ++i) cid[i] = c[static_cast<std::size_t>(i)];
    return 0;
    REF_CATCH
}

int ref_srd_collide(const mpcd_params_c* pc, double* v, const int32_t* cid, uint64_t seed) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    std::vector<double> vv(v, v + 2 * static_cast<std::size_t>(p.n));
    std::vector<int> c(cid, cid + p.n);
    mpcd::srd_collision_step(vv, c, p, seed);
    std::memcpy(v, vv.data(), vv.size() * sizeof(double));
    return 0;
    REF_CATCH
}

int ref_cell_fields(const mpcd_params_c* pc, const double* x, const double* v, double rho_target,
                    mpcd_cellfields_c* out) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    mpcd::State s = make_state(p, x, v);
    copy_fields(mpcd::compute_cell_fields(s.x, s.v, p, rho_target), out);
    return 0;
    REF_CATCH
}

int ref_zone_owner_map(const mpcd_params_c* pc, int32_t mode, int32_t* owner) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    const auto L = mpcd::build_zone_layout(p, layout_name(mode));
    std::memcpy(owner, L.ownerMap.data(), L.ownerMap.size() * sizeof(int32_t));
    return static_cast<int>(L.zones.size()) > 0 ? 0 : 0;
    REF_CATCH
}

// nthreads > 0: run_zone_pass_openmp; nthreads == 0: run_zone_pass_sync_serial.
int ref_zone_pass(const mpcd_params_c* pc, const double* xin, const double* vin, double* xout, double* vout,
                  int32_t mode, uint64_t seed_base, int32_t nthreads, mpcd_pass_metrics_c* m) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    mpcd::State s = make_state(p, xin, vin);
    const auto r = (nthreads > 0) ? mpcd::run_zone_pass_openmp(s, p, layout_name(mode), seed_base, nthreads)
                                  : mpcd::run_zone_pass_sync_serial(s, p, layout_name(mode), seed_base);
    std::memcpy(xout, r.stateOut.x.data(), r.stateOut.x.size() * sizeof(double));
    std::memcpy(vout, r.stateOut.v.data(), r.stateOut.v.size() * sizeof(double));
    fill_pass_metrics(r.metrics, m);
    return 0;
    REF_CATCH
}

// mpcd::run_zone_pass (src/zone_pass.cpp:1096-1163): zones one after another, in place
int ref_zone_pass_serial(const mpcd_params_c* pc, const double* xin, const double* vin, double* xout, double* vout,
                         int32_t mode, uint64_t seed_base, mpcd_pass_metrics_c* m) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    mpcd::State s = make_state(p, xin, vin);
    const auto r = mpcd::run_zone_pass(s, p, layout_name(mode), seed_base);
    std::memcpy(xout, r.stateOut.x.data(), r.stateOut.x.size() * sizeof(double));
    std::memcpy(vout, r.stateOut.v.data(), r.stateOut.v.size() * sizeof(double));
    if (m) {
        std::memset(m, 0, sizeof *m);
        m->nZones = r.metrics.nZonesExecuted;
        m->nThreadsRequested = 1;
        m->nThreadsUsed = 1;
        m->nParticlesMovedDense = r.metrics.nParticlesMovedDense;
        m->nParticlesMovedSparse = r.metrics.nParticlesMovedSparse;
        m->corrRmsDU = r.metrics.corrRmsDU;
        m->corrMaxDU = r.metrics.corrMaxDU;
    }
    return 0;
    REF_CATCH
}

int ref_liquid_closure(const mpcd_params_c* pc, const double* refx, const double* refv, const double* redx,
                       const double* redv, double* outx, double* outv, mpcd_closure_metrics_c* m,
                       mpcd_closure_detail_c* d) {
    REF_TRY
    const mpcd::Params p = to_params(pc);
    const mpcd::State ref = make_state(p, refx, refv);
    const mpcd::State red = make_state(p, redx, redv);
    const auto r = mpcd::run_liquid_closure(ref, red, p);
    copy_vec(r.stateOut.x, outx);
    copy_vec(r.stateOut.v, outv);
    fill_closure_metrics(r.metrics, m);
    if (d) {
        copy_vec(r.stateRepaired.x, d->repairedX);
        copy_vec(r.stateRepaired.v, d->repairedV);
        copy_fields(r.refFields, &d->refFields);
        copy_fields(r.redFields, &d->redFields);
        copy_fields(r.repairedFields, &d->repairedFields);
        copy_fields(r.outFields, &d->outFields);
        copy_vec(r.pdriveRaw, d->pdriveRaw);
        copy_vec(r.pdrive, d->pdrive);
        copy_vec(r.duRepairX, d->duRepairX);
        copy_vec(r.duRepairY, d->duRepairY);
        copy_vec(r.duEOSX, d->duEOSX);
        copy_vec(r.duEOSY, d->duEOSY);
        if (d->interzoneMask)
            std::memcpy(d->interzoneMask, r.interzoneMask.data(), r.interzoneMask.size() * sizeof(int32_t));
    }
    return 0;
    REF_CATCH
}

// One iteration of the profiled benchmark loop body (reference
// main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:241-279 and its metrics row
// :288-336), calling the reference library functions in the same order with the same seeds.
int ref_step(const mpcd_params_c* pc, double* x, double* v, int64_t step, int32_t nthreads,
             mpcd_step_metrics_c* m) {
    REF_TRY
    const mpcd::Params params = to_params(pc);
    mpcd::State stateRef = make_state(params, x, v);
    const std::uint64_t s = static_cast<std::uint64_t>(step);
    for (int i = 0; i < params.n; ++i) {
        stateRef.v[2 * i] += params.bodyForceX * params.dt;
        stateRef.v[2 * i + 1] += params.g * params.dt;
        stateRef.x[2 * i] += params.dt * stateRef.v[2 * i];
        stateRef.x[2 * i + 1] += params.dt * stateRef.v[2 * i + 1];
    }
    mpcd::WallInfo wallInfo;
    mpcd::apply_bc_general(stateRef.x, stateRef.v, params, wallInfo, 104729ULL + 10007ULL * s);
    const auto cid = mpcd::srd_cell_id_with_random_shift(stateRef.x, params, 130363ULL + 10007ULL * s);
    mpcd::srd_collision_step(stateRef.v, cid, params, 433494437ULL + 10007ULL * s);
    const auto baseResult = mpcd::run_zone_pass_openmp(stateRef, params, "base", 88172645463325252ULL + 10007ULL * s, nthreads);
    const auto shiftedResult = mpcd::run_zone_pass_openmp(baseResult.stateOut, params, "shifted",
                                                          88172645463325252ULL + 4099ULL + 10007ULL * s, nthreads);
    const auto closureResult = mpcd::run_liquid_closure(stateRef, shiftedResult.stateOut, params);
    std::memcpy(x, closureResult.stateOut.x.data(), closureResult.stateOut.x.size() * sizeof(double));
    std::memcpy(v, closureResult.stateOut.v.data(), closureResult.stateOut.v.size() * sizeof(double));
    if (m) {
        std::memset(m, 0, sizeof(*m));
        m->step = step;
        m->wall.nBot = wallInfo.nBot; m->wall.nTop = wallInfo.nTop; m->wall.nLeft = wallInfo.nLeft;
        m->wall.nRight = wallInfo.nRight; m->wall.dEwall = wallInfo.dEwall;
        m->wall.dPxBot = wallInfo.dPxBot; m->wall.dPxTop = wallInfo.dPxTop;
        m->wall.dPyBot = wallInfo.dPyBot; m->wall.dPyTop = wallInfo.dPyTop;
        fill_pass_metrics(baseResult.metrics, &m->base);
        fill_pass_metrics(shiftedResult.metrics, &m->shifted);
        fill_closure_metrics(closureResult.metrics, &m->closure);
        const double dx = params.Lx / params.Nx, dy = params.Ly / params.Ny;
        const double rhoTarget = params.gamma / (dx * dy);
        const auto baseFields = mpcd::compute_cell_fields(baseResult.stateOut.x, baseResult.stateOut.v, params, rhoTarget);
        const auto shiftedFields = mpcd::compute_cell_fields(shiftedResult.stateOut.x, shiftedResult.stateOut.v, params, rhoTarget);
        occstd_outband(baseFields, params, &m->baseOccStd, &m->baseOutBand);
        occstd_outband(shiftedFields, params, &m->shiftedOccStd, &m->shiftedOutBand);
        m->occStd = m->shiftedOccStd;
        m->outBand = m->shiftedOutBand;
        const auto& st = closureResult.stateOut;
        double ke = 0.0, mx = 0.0, my = 0.0;
        for (int i = 0; i < params.n; ++i) ke += 0.5 * (st.v[2 * i] * st.v[2 * i] + st.v[2 * i + 1] * st.v[2 * i + 1]);
        for (int i = 0; i < params.n; ++i) mx += st.v[2 * i];
        for (int i = 0; i < params.n; ++i) my += st.v[2 * i + 1];
        const double nn = static_cast<double>(std::max(params.n, 1));
        m->meanKinetic = ke / nn;
        m->meanVelocityX = mx / nn;
        m->meanVelocityY = my / nn;
        m->meanUx = mean_field(closureResult.outFields.Ux);
        m->meanUy = mean_field(closureResult.outFields.Uy);
        m->Qx = m->meanUx * params.Ly;
    }
    return 0;
    REF_CATCH
}

}  // extern "C"
