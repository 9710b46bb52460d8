// TEST/BASELINE INFRASTRUCTURE ONLY — times the UNMODIFIED reference on a bounded sample.
//
// The reference's zone pass costs O(zones x particles) per step: each zone rebuilds cell ids
// for the whole domain and copies the whole state (src/zone_pass_openmp.cpp:63-96), and each
// layout allocates one Nc-sized mask per zone (src/zone_pass.cpp:208). At 2048x512 cells that
// is ~10^3 s per step, so this harness runs one full step of everything except the zone
// passes, and for each pass runs a sample of zones through exactly the per-zone body of
// run_zone_pass_snapshot_impl (extract ids, snapshot copy, run_zone_kernel_inplace, pack)
// in an OpenMP parallel loop with the same schedule, then scales the sampled wall time to
// all zones. All physics calls are the reference's own library functions.
//
// usage: ref_sampled params.kv x.bin v.bin nthreads zones_per_thread step
// prints one JSON object with the measured and extrapolated times.
#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#include "boundary_conditions.h"
#include "common_grid.h"
#include "liquid_closure.h"
#include "params_io.h"
#include "srd_collision.h"
#include "state_io.h"
#include "types.h"
#include "zone_pass.h"

using namespace mpcd;
using Clock = std::chrono::steady_clock;

static double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// Zone rectangles of a layout, in id order (same construction as build_layout).
static std::vector<std::array<int, 4>> rects(const Params& p, bool shifted) {
    auto starts = [](int N, int tile, int off) {
        std::vector<int> s{0};
        for (int v = off; v < N; v += tile)
            if (v > 0 && v < N) s.push_back(v);
        return s;
    };
    const auto xs = starts(p.Nx, p.zoneTileNx, shifted ? p.zoneTileNx / 2 : 0);
    const auto ys = starts(p.Ny, p.zoneTileNy, shifted ? p.zoneTileNy / 2 : 0);
    std::vector<std::array<int, 4>> r;
    for (int y : ys)
        for (int x : xs) r.push_back({x, std::min(x + p.zoneTileNx, p.Nx), y, std::min(y + p.zoneTileNy, p.Ny)});
    return r;
}

struct PassTime {
    double layoutPerZone = 0, wallSample = 0, mergePerParticle = 0;
    int nZones = 0, nSample = 0;
    double extrapolated = 0;
    State out;  // the input with the sampled zones' results merged in
};

static PassTime sampled_pass(const State& in, const Params& p, bool shifted, std::uint64_t seedBase, int T, int k) {
    PassTime t;
    const auto R = rects(p, shifted);
    t.nZones = static_cast<int>(R.size());
    const int S = std::min(t.nZones, T * k);
    t.nSample = S;
    // layout: one ZoneDescriptor with an Nc mask per zone, as build_layout does
    std::vector<int> pick(S);
    for (int j = 0; j < S; ++j) pick[j] = static_cast<int>((static_cast<long long>(j) * t.nZones) / S);
    auto t0 = Clock::now();
    std::vector<ZoneDescriptor> Z(S);
    for (int j = 0; j < S; ++j) {
        const auto& q = R[pick[j]];
        Z[j].id = pick[j] + 1;
        Z[j].maskVec.assign(static_cast<std::size_t>(p.Nc), 0);
        for (int ix = q[0]; ix < q[1]; ++ix)
            for (int iy = q[2]; iy < q[3]; ++iy) {
                const int c = iy + p.Ny * ix;
                Z[j].cellIds.push_back(c);
                Z[j].maskVec[c] = 1;
            }
    }
    t.layoutPerZone = secs(t0, Clock::now()) / std::max(1, S);
    std::vector<std::vector<int>> ids(S);
    std::vector<std::vector<double>> xp(S), vp(S);
    omp_set_dynamic(0);
    omp_set_num_threads(T);
    t0 = Clock::now();
#pragma omp parallel for schedule(static)
    for (int j = 0; j < S; ++j) {
        ids[j] = build_particle_ids_in_zone(in.x, p, Z[j]);
        std::vector<double> xl = in.x, vl = in.v;
        run_zone_kernel_inplace(xl, vl, p, Z[j], seedBase + 104729ULL * static_cast<std::uint64_t>(pick[j] + 1));
        xp[j].resize(2 * ids[j].size());
        vp[j].resize(2 * ids[j].size());
        for (std::size_t q = 0; q < ids[j].size(); ++q) {
            const int pid = ids[j][q];
            xp[j][2 * q] = xl[2 * pid]; xp[j][2 * q + 1] = xl[2 * pid + 1];
            vp[j][2 * q] = vl[2 * pid]; vp[j][2 * q + 1] = vl[2 * pid + 1];
        }
    }
    t.wallSample = secs(t0, Clock::now());
    t.out = in;
    State& out = t.out;
    t0 = Clock::now();
    std::size_t merged = 0;
    for (int j = 0; j < S; ++j)
        for (std::size_t q = 0; q < ids[j].size(); ++q) {
            const int pid = ids[j][q];
            out.x[2 * pid] = xp[j][2 * q]; out.x[2 * pid + 1] = xp[j][2 * q + 1];
            out.v[2 * pid] = vp[j][2 * q]; out.v[2 * pid + 1] = vp[j][2 * q + 1];
            ++merged;
        }
    t.mergePerParticle = secs(t0, Clock::now()) / std::max<std::size_t>(1, merged);
    // static schedule: each thread runs ceil(nZones/T) zones; the sample ran ceil(S/T)
    const double perThreadFull = std::ceil(static_cast<double>(t.nZones) / T);
    const double perThreadSample = std::ceil(static_cast<double>(S) / T);
    t.extrapolated = t.layoutPerZone * t.nZones + t.wallSample * (perThreadFull / perThreadSample) +
                     t.mergePerParticle * static_cast<double>(p.n);
    return t;
}

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s params.kv x.bin v.bin nthreads zones_per_thread step\n", argv[0]);
        return 2;
    }
    try {
        const Params params = read_params_kv(argv[1]);
        State state = read_state(argv[2], argv[3], "", "", false, false, params.n);
        const int T = std::max(1, std::stoi(argv[4]));
        const int k = std::max(1, std::stoi(argv[5]));
        const std::uint64_t step = static_cast<std::uint64_t>(std::stoll(argv[6]));
        // the step of src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:237-279:
        // stateRef is the streamed, wall-treated and collided state; the base pass reads it, the
        // shifted pass the base pass's output, and the closure gets (stateRef, shifted output)
        auto t0 = Clock::now();
        State cur = state;
        for (int i = 0; i < params.n; ++i) {
            cur.v[2 * i] += params.bodyForceX * params.dt;
            cur.v[2 * i + 1] += params.g * params.dt;
            cur.x[2 * i] += params.dt * cur.v[2 * i];
            cur.x[2 * i + 1] += params.dt * cur.v[2 * i + 1];
        }
        WallInfo w;
        apply_bc_general(cur.x, cur.v, params, w, 104729ULL + 10007ULL * step);
        const auto cid = srd_cell_id_with_random_shift(cur.x, params, 130363ULL + 10007ULL * step);
        srd_collision_step(cur.v, cid, params, 433494437ULL + 10007ULL * step);
        const double tRef = secs(t0, Clock::now());
        const PassTime b = sampled_pass(cur, params, false, 88172645463325252ULL + 10007ULL * step, T, k);
        const PassTime s = sampled_pass(b.out, params, true, 88172645463325252ULL + 4099ULL + 10007ULL * step, T, k);
        t0 = Clock::now();
        const auto cl = run_liquid_closure(cur, s.out, params);
        const double tClosure = secs(t0, Clock::now());
        const double tStep = tRef + b.extrapolated + s.extrapolated + tClosure;
        std::printf("{\"n\": %d, \"Nc\": %d, \"threads\": %d, \"t_refbuild\": %.6f, \"t_closure\": %.6f, "
                    "\"base_zones\": %d, \"base_sampled\": %d, \"base_wall_sampled\": %.6f, \"base_extrapolated\": %.6f, "
                    "\"shifted_zones\": %d, \"shifted_sampled\": %d, \"shifted_wall_sampled\": %.6f, \"shifted_extrapolated\": %.6f, "
                    "\"t_step_extrapolated\": %.6f, \"moved_check\": %d}\n",
                    params.n, params.Nc, T, tRef, tClosure, b.nZones, b.nSample, b.wallSample, b.extrapolated, s.nZones,
                    s.nSample, s.wallSample, s.extrapolated, tStep, cl.metrics.nMaskedInterzoneCells);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "Fatal error: %s\n", e.what());
        return 1;
    }
}
