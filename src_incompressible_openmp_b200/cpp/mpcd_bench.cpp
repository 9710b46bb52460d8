// mpcd_bench: the profiled Poiseuille benchmark driver on the GPU, with the reference driver's
// command line and outputs (src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:
// 187-423):
//
//   mpcd_bench params.kv state_x.bin state_v.bin state_type.bin state_r0.bin out_prefix has_type has_r0 nthreads
//
// writes <out_prefix>_metrics.csv (same columns), <out_prefix>_runout.kv (same keys) and the
// snapshots of benchmark_dumpSteps (<out_prefix>_stepNNNN_{x,v,type,r0,cellfields}.bin).
//
// Resume: with the optional key benchmark_startStep = k, the input state is taken as the state
// after step k (e.g. the step-k snapshot of an earlier run) and the run continues with steps
// k+1 .. benchmark_nSteps, with the seeds, metrics rows and snapshot names of those steps.
//
// Unlike the reference driver, the state stays on the device for the whole run
// (mpcd::b200::Session): the host only sees the metrics rows and the dumps. nthreads is
// recorded but does not change the computation. Timing columns: timeStepTotal and the phase
// columns of a metrics row are device seconds of that step (CUDA events); the loop totals in
// the runout file are host wall seconds, and the per-phase totals split them by the device
// phase fractions measured on the metrics steps.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "mpcd_b200.hpp"

namespace {

using Clock = std::chrono::steady_clock;
double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

std::string kv_string(const std::string& path, const char* key) {
    char buf[4096];
    if (mpcd_read_kv_string(path.c_str(), key, buf, (int)sizeof buf) != MPCD_OK)
        throw std::runtime_error(std::string("Missing benchmark key: ") + key);
    return buf;
}

std::string kv_optional(const std::string& path, const char* key, const char* dflt) {
    char buf[4096];
    if (mpcd_read_kv_string(path.c_str(), key, buf, (int)sizeof buf) != MPCD_OK) return dflt;
    return buf;
}

std::vector<int> parse_steps(const std::string& s) {
    std::vector<int> out;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        const auto b = tok.find_first_not_of(" \t\r\n");
        if (b == std::string::npos) continue;
        const auto e = tok.find_last_not_of(" \t\r\n");
        out.push_back(std::stoi(tok.substr(b, e - b + 1)));
    }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    return out;
}

void dump(const std::string& prefix0, int step, const mpcd::State& s, const mpcd::CellFields& G, int n, bool has_type,
          bool has_r0) {
    std::ostringstream oss;
    oss << prefix0 << "_step" << std::setw(4) << std::setfill('0') << step;
    const std::string p = oss.str();
    mpcd::write_xy_interleaved(p + "_x.bin", s.x, n);
    mpcd::write_xy_interleaved(p + "_v.bin", s.v, n);
    if (has_type) mpcd::write_u8(p + "_type.bin", s.type, n);
    if (has_r0) mpcd::write_xy_interleaved(p + "_r0.bin", s.r0, n);
    mpcd::write_cell_fields_bin(p + "_cellfields.bin", G);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 10) {
        std::cerr << "Usage: " << argv[0]
                  << " params.kv state_x.bin state_v.bin state_type.bin state_r0.bin out_prefix has_type has_r0 nthreads\n";
        return 2;
    }
    const std::string params_path = argv[1], x_path = argv[2], v_path = argv[3], type_path = argv[4], r0_path = argv[5];
    const std::string out_prefix = argv[6];
    const bool has_type = std::string(argv[7]) == "1";
    const bool has_r0 = std::string(argv[8]) == "1";
    const int nthreads = std::max(1, std::stoi(argv[9]));
    try {
        const mpcd::Params params = mpcd::read_params_kv(params_path);
        const int nSteps = std::stoi(kv_string(params_path, "benchmark_nSteps"));
        const int metricsEvery = std::stoi(kv_string(params_path, "benchmark_metricsEvery"));
        const std::string dumpCsv = kv_string(params_path, "benchmark_dumpSteps");
        const int startStep = std::stoi(kv_optional(params_path, "benchmark_startStep", "0"));
        if (startStep < 0 || startStep > nSteps) throw std::runtime_error("benchmark_startStep out of range");
        const std::vector<int> dumpSteps = parse_steps(dumpCsv);
        auto isDump = [&](int s) { return std::binary_search(dumpSteps.begin(), dumpSteps.end(), s); };
        auto isMetrics = [&](int s) { return metricsEvery > 0 && (s % metricsEvery == 0 || s == nSteps); };

        mpcd::State state = mpcd::read_state(x_path, v_path, type_path, r0_path, has_type, has_r0, params.n);
        const double rhoTarget = params.gamma / ((params.Lx / params.Nx) * (params.Ly / params.Ny));

        std::ofstream metrics(out_prefix + "_metrics.csv");
        if (!metrics) throw std::runtime_error("Cannot open metrics CSV for writing");
        metrics << "step,occStd,outBand,meanKinetic,meanUx,meanUy,Qx,baseOccStd,baseOutBand,shiftedOccStd,shiftedOutBand,"
                   "meanPdrive,meanPdriveRaw,meanVelocityX,meanVelocityY,particlesMovedDense,particlesMovedSparse,"
                   "betaRepairOpt,betaRepairApplied,betaRepairNum,betaRepairDen,rmsRepairDU,maxRepairDU,meanAbsRepairDU,"
                   "nMaskedInterzoneCells,momentumDeltaX,momentumDeltaY,nThreadsUsedBase,nThreadsUsedShifted,"
                   "timeStepTotal,timeRefBuild,timeBase,timeShifted,timeClosure,timeDiagnostics,timeDump\n";
        std::ofstream manifest(out_prefix + "_runout.kv");
        if (!manifest) throw std::runtime_error("Cannot open benchmark runout file");
        manifest << "inputTag=" << x_path << "\n";
        manifest << "outputTag=" << out_prefix << "\n";
        manifest << "benchmark_nSteps=" << nSteps << "\n";
        manifest << "benchmark_metricsEvery=" << metricsEvery << "\n";
        manifest << "benchmark_dumpSteps=" << dumpCsv << "\n";
        manifest << "nThreadsRequested=" << nthreads << "\n";

        const auto tAll0 = Clock::now();
        mpcd::b200::Session S(params, state);
        double tLoop = 0.0, tDumps = 0.0;
        double devTotal = 0.0, devRef = 0.0, devBase = 0.0, devShift = 0.0, devClos = 0.0, devDiag = 0.0;
        if (startStep == 0 && isDump(0)) {
            const auto t0 = Clock::now();
            dump(out_prefix, 0, state, S.fields(rhoTarget), params.n, has_type, has_r0);
            tDumps += seconds(t0, Clock::now());
        }
        mpcd_step_metrics_c m{};
        int step = startStep;
        while (step < nSteps) {
            int stop = step + 1;
            while (stop < nSteps && !isMetrics(stop) && !isDump(stop)) ++stop;
            const bool want = isMetrics(stop) || stop == nSteps;
            const auto t0 = Clock::now();
            S.step(step, stop - step, want ? &m : nullptr);
            tLoop += seconds(t0, Clock::now());
            step = stop;
            if (want) {
                devTotal += m.timeStepTotal; devRef += m.timeRefBuild; devBase += m.timeBase;
                devShift += m.timeShifted; devClos += m.timeClosure; devDiag += m.timeDiagnostics;
            }
            if (isMetrics(step)) {
                metrics << step << ',' << m.occStd << ',' << m.outBand << ',' << m.meanKinetic << ',' << m.meanUx << ','
                        << m.meanUy << ',' << m.Qx << ',' << m.baseOccStd << ',' << m.baseOutBand << ','
                        << m.shiftedOccStd << ',' << m.shiftedOutBand << ',' << m.closure.meanPdrive << ','
                        << m.closure.meanPdriveRaw << ',' << m.meanVelocityX << ',' << m.meanVelocityY << ','
                        << (m.base.nParticlesMovedDense + m.shifted.nParticlesMovedDense) << ','
                        << (m.base.nParticlesMovedSparse + m.shifted.nParticlesMovedSparse) << ','
                        << m.closure.betaRepairOpt << ',' << m.closure.betaRepairApplied << ','
                        << m.closure.betaRepairNum << ',' << m.closure.betaRepairDen << ',' << m.closure.rmsRepairDU << ','
                        << m.closure.maxRepairDU << ',' << m.closure.meanAbsRepairDU << ','
                        << m.closure.nMaskedInterzoneCells << ',' << m.closure.momentumDeltaX << ','
                        << m.closure.momentumDeltaY << ',' << m.base.nThreadsUsed << ',' << m.shifted.nThreadsUsed << ','
                        << m.timeStepTotal << ',' << m.timeRefBuild << ',' << m.timeBase << ',' << m.timeShifted << ','
                        << m.timeClosure << ',' << m.timeDiagnostics << ',' << 0.0 << '\n';
            }
            if (isDump(step)) {
                const auto td = Clock::now();
                S.get(state);
                dump(out_prefix, step, state, S.fields(rhoTarget), params.n, has_type, has_r0);
                tDumps += seconds(td, Clock::now());
            }
            if (step == nSteps) {
                manifest << "finalOccStd=" << m.shiftedOccStd << "\n";
                manifest << "finalOutBand=" << m.shiftedOutBand << "\n";
                manifest << "finalMeanKinetic=" << m.meanKinetic << "\n";
                manifest << "finalMeanVelocityX=" << m.meanVelocityX << "\n";
                manifest << "finalMeanVelocityY=" << m.meanVelocityY << "\n";
                manifest << "finalQx=" << m.Qx << "\n";
                manifest << "totalParticlesMovedDense=" << (m.base.nParticlesMovedDense + m.shifted.nParticlesMovedDense) << "\n";
                manifest << "totalParticlesMovedSparse=" << (m.base.nParticlesMovedSparse + m.shifted.nParticlesMovedSparse) << "\n";
                manifest << "finalBetaRepairOpt=" << m.closure.betaRepairOpt << "\n";
                manifest << "finalBetaRepairApplied=" << m.closure.betaRepairApplied << "\n";
                manifest << "finalBetaRepairNum=" << m.closure.betaRepairNum << "\n";
                manifest << "finalBetaRepairDen=" << m.closure.betaRepairDen << "\n";
                manifest << "finalRmsRepairDU=" << m.closure.rmsRepairDU << "\n";
                manifest << "finalMaxRepairDU=" << m.closure.maxRepairDU << "\n";
                manifest << "finalMeanAbsRepairDU=" << m.closure.meanAbsRepairDU << "\n";
                manifest << "finalMomentumDeltaX=" << m.closure.momentumDeltaX << "\n";
                manifest << "finalMomentumDeltaY=" << m.closure.momentumDeltaY << "\n";
                manifest << "nThreadsUsedBase=" << m.base.nThreadsUsed << "\n";
                manifest << "nThreadsUsedShifted=" << m.shifted.nThreadsUsed << "\n";
            }
        }
        const double totalWall = seconds(tAll0, Clock::now());
        auto frac = [&](double part) { return devTotal > 0.0 ? part / devTotal : 0.0; };
        const double loop = tLoop + tDumps;
        manifest << "timeTotalWall=" << totalWall << "\n";
        manifest << "timeLoopTotal=" << loop << "\n";
        manifest << "timeRefBuild=" << frac(devRef) * tLoop << "\n";
        manifest << "timeBase=" << frac(devBase) * tLoop << "\n";
        manifest << "timeShifted=" << frac(devShift) * tLoop << "\n";
        manifest << "timeClosure=" << frac(devClos) * tLoop << "\n";
        manifest << "timeDiagnostics=" << frac(devDiag) * tLoop << "\n";
        manifest << "timeDumps=" << tDumps << "\n";
        manifest << "timePerStepMean=" << (loop / std::max(1, nSteps)) << "\n";
        manifest << "fracRefBuild=" << (loop > 0 ? frac(devRef) * tLoop / loop : 0.0) << "\n";
        manifest << "fracBase=" << (loop > 0 ? frac(devBase) * tLoop / loop : 0.0) << "\n";
        manifest << "fracShifted=" << (loop > 0 ? frac(devShift) * tLoop / loop : 0.0) << "\n";
        manifest << "fracClosure=" << (loop > 0 ? frac(devClos) * tLoop / loop : 0.0) << "\n";
        manifest << "fracDiagnostics=" << (loop > 0 ? frac(devDiag) * tLoop / loop : 0.0) << "\n";
        manifest << "fracDumps=" << (loop > 0 ? tDumps / loop : 0.0) << "\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "Fatal error: " << e.what() << '\n';
        return 1;
    }
}
