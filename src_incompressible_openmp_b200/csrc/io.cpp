// params.kv reader for the C-ABI (reference src/params_io.cpp:21-137): '#' comments, trimmed
// key=value lines, every key required, unknown keys ignored, integers through std::stoi,
// doubles through std::stod, booleans "true"/"1"/"false"/"0". Boundary and threshold modes
// become the enums of include/mpcd_c.h.
#include <cctype>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "mpcd_c.h"

namespace {

thread_local std::string g_io_err;

std::string trim(const std::string& s) {
    std::size_t b = 0;
    while (b < s.size() && std::isspace(static_cast<unsigned char>(s[b]))) ++b;
    std::size_t e = s.size();
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) --e;
    return s.substr(b, e - b);
}

std::unordered_map<std::string, std::string> read_kv(const std::string& path) {
    std::ifstream fin(path);
    if (!fin) throw std::runtime_error("Cannot open params file: " + path);
    std::unordered_map<std::string, std::string> kv;
    std::string line;
    while (std::getline(fin, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        const auto pos = line.find('=');
        if (pos == std::string::npos) throw std::runtime_error("Invalid key=value line in params file: " + line);
        kv[trim(line.substr(0, pos))] = trim(line.substr(pos + 1));
    }
    return kv;
}

const std::string& req(const std::unordered_map<std::string, std::string>& kv, const std::string& key) {
    auto it = kv.find(key);
    if (it == kv.end()) throw std::runtime_error("Missing required params key: " + key);
    return it->second;
}

int req_int(const std::unordered_map<std::string, std::string>& kv, const char* k) { return std::stoi(req(kv, k)); }
double req_dbl(const std::unordered_map<std::string, std::string>& kv, const char* k) { return std::stod(req(kv, k)); }
int req_bool(const std::unordered_map<std::string, std::string>& kv, const char* k) {
    const std::string& s = req(kv, k);
    if (s == "true" || s == "1") return 1;
    if (s == "false" || s == "0") return 0;
    throw std::runtime_error("Invalid boolean value: " + s);
}
int bc_mode(const std::string& s) {
    if (s == "periodic") return MPCD_BC_PERIODIC;
    if (s == "thermalize") return MPCD_BC_THERMALIZE;
    if (s == "bounceback") return MPCD_BC_BOUNCEBACK;
    if (s == "specular") return MPCD_BC_SPECULAR;
    return MPCD_BC_UNKNOWN;
}

}  // namespace

extern "C" {

const char* mpcd_io_last_error(void) { return g_io_err.c_str(); }

int mpcd_read_params_kv(const char* path, mpcd_params_c* p) {
    if (!path || !p) return MPCD_ERR_INVALID_ARG;
    try {
        const auto kv = read_kv(path);
        mpcd_params_c o;
        std::memset(&o, 0, sizeof o);
        o.Nx = req_int(kv, "Nx"); o.Ny = req_int(kv, "Ny"); o.Nc = req_int(kv, "Nc"); o.n = req_int(kv, "n");
        o.Lx = req_dbl(kv, "Lx"); o.Ly = req_dbl(kv, "Ly"); o.dt = req_dbl(kv, "dt"); o.a0 = req_dbl(kv, "a0");
        o.alpha = req_dbl(kv, "alpha"); o.kBT = req_dbl(kv, "kBT"); o.g = req_dbl(kv, "g");
        o.bodyForceX = req_dbl(kv, "bodyForceX");
        o.useThermostat = req_bool(kv, "useThermostat"); o.keepMeanFlow = req_bool(kv, "keepMeanFlow");
        o.boundary_left = bc_mode(req(kv, "boundary_left"));
        o.boundary_right = bc_mode(req(kv, "boundary_right"));
        o.boundary_bottom = bc_mode(req(kv, "boundary_bottom"));
        o.boundary_top = bc_mode(req(kv, "boundary_top"));
        o.Utop = req_dbl(kv, "Utop"); o.Ubottom = req_dbl(kv, "Ubottom"); o.wallSigma = req_dbl(kv, "wallSigma");
        o.noSurfaceCase = req_bool(kv, "noSurfaceCase");
        o.redistributionEnableSurfaceTopology = req_bool(kv, "redistributionEnableSurfaceTopology");
        o.redistributionWallWettingEnabled = req_bool(kv, "redistributionWallWettingEnabled");
        o.useInterfaceVelocityReorientation = req_bool(kv, "useInterfaceVelocityReorientation");
        o.useIncompressibleRedistribution = req_bool(kv, "useIncompressibleRedistribution");
        o.redistribAfterCollision = req_bool(kv, "redistribAfterCollision");
        o.useZoneRedistribution = req_bool(kv, "useZoneRedistribution");
        o.zoneTileNx = req_int(kv, "zoneTileNx"); o.zoneTileNy = req_int(kv, "zoneTileNy");
        o.zoneUseShiftedSecondPass = req_bool(kv, "zoneUseShiftedSecondPass");
        o.zonePassthroughMode = req_bool(kv, "zonePassthroughMode");
        o.zoneSingleFullDomainMode = req_bool(kv, "zoneSingleFullDomainMode");
        o.enableMomentumCorrectionPostRedistribution = req_bool(kv, "enableMomentumCorrectionPostRedistribution");
        o.gamma = req_dbl(kv, "gamma"); o.coef = req_dbl(kv, "coef");
        o.highMode = (req(kv, "highMode") == "1+coef") ? MPCD_THR_ONE_PLUS_COEF : MPCD_THR_COEF;
        o.lowMode = (req(kv, "lowMode") == "1+coef") ? MPCD_THR_ONE_PLUS_COEF : MPCD_THR_COEF;
        o.maxRedistribPasses = req_int(kv, "maxRedistribPasses");
        o.useLocalFluidFractionThresholds = req_bool(kv, "useLocalFluidFractionThresholds");
        o.fluidFracGain = req_dbl(kv, "fluidFracGain"); o.lowThrFloor = req_dbl(kv, "lowThrFloor");
        o.highThrFloor = req_dbl(kv, "highThrFloor"); o.lowThrBulkOverride = req_dbl(kv, "lowThrBulkOverride");
        o.useLiquidClosure = req_bool(kv, "useLiquidClosure");
        o.useOptimalBetaRepair = req_bool(kv, "useOptimalBetaRepair");
        o.betaRepair = req_dbl(kv, "betaRepair"); o.betaEOS = req_dbl(kv, "betaEOS"); o.Kvirial = req_dbl(kv, "Kvirial");
        o.smoothPdriveAtInterzone = req_bool(kv, "smoothPdriveAtInterzone");
        o.smoothPdriveInterzoneWidthCells = req_int(kv, "smoothPdriveInterzoneWidthCells");
        o.smoothPdriveInterzoneBlend = req_dbl(kv, "smoothPdriveInterzoneBlend");
        o.smoothPdriveIncludeShiftedLayouts = req_bool(kv, "smoothPdriveIncludeShiftedLayouts");
        *p = o;
        return MPCD_OK;
    } catch (const std::exception& e) {
        g_io_err = e.what();
        return MPCD_ERR_INVALID_ARG;
    }
}

// Any key of a params.kv file as a string (the benchmark keys benchmark_nSteps,
// benchmark_metricsEvery and benchmark_dumpSteps are read this way by the reference driver).
int mpcd_read_kv_string(const char* path, const char* key, char* buf, int buflen) {
    if (!path || !key || !buf || buflen <= 0) return MPCD_ERR_INVALID_ARG;
    try {
        const auto kv = read_kv(path);
        const std::string& v = req(kv, key);
        if ((int)v.size() + 1 > buflen) {
            g_io_err = "buffer too small";
            return MPCD_ERR_INVALID_ARG;
        }
        std::memcpy(buf, v.c_str(), v.size() + 1);
        return MPCD_OK;
    } catch (const std::exception& e) {
        g_io_err = e.what();
        return MPCD_ERR_INVALID_ARG;
    }
}

}  // extern "C"
