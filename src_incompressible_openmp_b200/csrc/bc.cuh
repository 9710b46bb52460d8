// Streaming, wall boundary conditions and the thermal-wall Gaussian draws.
//
// Reference: stream + body force (src/main_benchmark_poiseuille_openmp_profiled_shifted_
// profiled.cpp:242-247) and apply_bc_general (src/boundary_conditions.cpp:19-203).
//
// apply_bc_general makes four sweeps over all particles; a thermalising wall draws two
// N(0,1) deviates per hit from ONE normal_distribution object and ONE mt19937_64 for the
// whole call, in (sweep, particle id, side) order. Every thermal hit consumes exactly one
// polar-method pair, so hit e (in that order) uses pair e. Positions never depend on
// velocities, so each particle's four sweeps can be replayed independently:
//   k_stream_bc      streams, replays positions, finishes velocities of particles without
//                    thermal hits, marks thermal hits in per-particle-id bitmaps (sweep 0)
//   k_wall_normals   one block generates the polar pairs in order (MT19937-64 + log_cr)
//   k_wall_apply     replays each thermal particle with its pairs, ranked by the bitmaps
#pragma once

#include "common.cuh"

namespace mpcd_dev {

constexpr int kWallDoubles = 9;  // dEwall, dPxBot, dPxTop, dPyBot, dPyTop, dPxLeft, dPxRight, dPyLeft, dPyRight

struct WallEvent {
    int slot;
    int pid;
    double x, y, vx, vy;  // streamed, pre-BC state
};

struct BcWork {
    // bitmaps of particles with a thermal x (left/right) or y (bottom/top) hit in sweep 0
    uint32_t* bitsX;
    uint32_t* bitsY;
    uint64_t* wordCount;    // popc(bitsX[w]) + popc(bitsY[w]); scanned into wordPrefix
    uint64_t* wordPrefix;   // nwords + 1
    WallEvent* events;
    int* nEvents;           // appended thermal particles
    int eventCap;
    double* normals;        // 2 per pair
    int normalCap;          // pairs
    double* contrib;        // kWallDoubles per pair slot (deterministic WallInfo)
    double* blockPartial;   // kWallDoubles per k_stream_bc block
    int* ints;              // nBot, nTop, nLeft, nRight
    double* srdShift;       // sx, sy of the step
};

// One particle through the four sweeps. kDry: thermal hits leave velocities undefined and
// only count; otherwise pair (firstPair + k) serves the particle's k-th thermal hit.
// Returns false on an unsupported mode (error code in *err).
template <bool kDry, bool kInfo = true>
__device__ __forceinline__ bool bc_replay(double& x, double& y, double& vx, double& vy, const DevParams& P,
                                          const double* __restrict__ normals, int firstPair, int pairCap, int& thermX0,
                                          int& thermY0, int& late, double* acc, int* nhit, int* err) {
    const double Lx = P.Lx, Ly = P.Ly, sig = P.wallSigma;
    int k = 0;  // thermal hits so far
    // pair index of the k-th hit, kept inside the buffer (an overflow has raised an error)
#define PAIR(k) (2 * min(firstPair + (k), pairCap - 1))
    for (int sweep = 0; sweep < 4; ++sweep) {
        if (x < 0.0) {
            const double ox = vx, oy = vy;
            const int m = P.bc[0];
            if (m == 0) {
                x = __dadd_rn(x, Lx);
            } else if (m >= 1 && m <= 3) {
                x = -x;
                if (m == 1) {
                    if (sweep == 0) ++thermX0; else late = 1;
                    if (!kDry) {
                        vx = fabs(__dmul_rn(sig, normals[PAIR(k)]));
                        vy = __dmul_rn(sig, normals[PAIR(k) + 1]);
                    }
                    ++k;
                } else if (m == 2) {
                    vx = fabs(vx);
                    vy = -vy;
                } else {
                    vx = fabs(vx);
                }
                if (kInfo) {
                    const double dvx = __dsub_rn(vx, ox), dvy = __dsub_rn(vy, oy);
                    nhit[2] += 1;
                    acc[0] = __dadd_rn(acc[0], __dmul_rn(0.5, __dsub_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)),
                                                                      __dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)))));
                    acc[5] = __dadd_rn(acc[5], fabs(dvx));
                    acc[7] = __dadd_rn(acc[7], dvy);
                }
            } else {
                *err = kErrUnsupportedBcLeft;
                return false;
            }
        }
        if (x > Lx) {
            const double ox = vx, oy = vy;
            const int m = P.bc[1];
            if (m == 0) {
                x = __dsub_rn(x, Lx);
            } else if (m >= 1 && m <= 3) {
                x = __dsub_rn(__dmul_rn(2.0, Lx), x);
                if (m == 1) {
                    if (sweep == 0) ++thermX0; else late = 1;
                    if (!kDry) {
                        vx = -fabs(__dmul_rn(sig, normals[PAIR(k)]));
                        vy = __dmul_rn(sig, normals[PAIR(k) + 1]);
                    }
                    ++k;
                } else if (m == 2) {
                    vx = -fabs(vx);
                    vy = -vy;
                } else {
                    vx = -fabs(vx);
                }
                if (kInfo) {
                    const double dvx = __dsub_rn(vx, ox), dvy = __dsub_rn(vy, oy);
                    nhit[3] += 1;
                    acc[0] = __dadd_rn(acc[0], __dmul_rn(0.5, __dsub_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)),
                                                                      __dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)))));
                    acc[6] = __dadd_rn(acc[6], fabs(dvx));
                    acc[8] = __dadd_rn(acc[8], dvy);
                }
            } else {
                *err = kErrUnsupportedBcRight;
                return false;
            }
        }
        if (y < 0.0) {
            const double ox = vx, oy = vy;
            const int m = P.bc[2];
            if (m == 0) {
                y = __dadd_rn(y, Ly);
            } else if (m >= 1 && m <= 3) {
                y = -y;
                if (m == 1) {
                    if (sweep == 0) ++thermY0; else late = 1;
                    if (!kDry) {
                        vx = __dadd_rn(P.Ubottom, __dmul_rn(sig, normals[PAIR(k)]));
                        vy = fabs(__dmul_rn(sig, normals[PAIR(k) + 1]));
                    }
                    ++k;
                } else if (m == 2) {
                    vx = __dsub_rn(__dmul_rn(2.0, P.Ubottom), vx);
                    vy = fabs(vy);
                } else {
                    vy = fabs(vy);
                }
                if (kInfo) {
                    const double dvx = __dsub_rn(vx, ox), dvy = __dsub_rn(vy, oy);
                    nhit[0] += 1;
                    acc[0] = __dadd_rn(acc[0], __dmul_rn(0.5, __dsub_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)),
                                                                      __dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)))));
                    acc[1] = __dadd_rn(acc[1], dvx);
                    acc[3] = __dadd_rn(acc[3], fabs(dvy));
                }
            } else {
                *err = kErrUnsupportedBcBottom;
                return false;
            }
        }
        if (y > Ly) {
            const double ox = vx, oy = vy;
            const int m = P.bc[3];
            if (m == 0) {
                y = __dsub_rn(y, Ly);
            } else if (m >= 1 && m <= 3) {
                y = __dsub_rn(__dmul_rn(2.0, Ly), y);
                if (m == 1) {
                    if (sweep == 0) ++thermY0; else late = 1;
                    if (!kDry) {
                        vx = __dadd_rn(P.Utop, __dmul_rn(sig, normals[PAIR(k)]));
                        vy = -fabs(__dmul_rn(sig, normals[PAIR(k) + 1]));
                    }
                    ++k;
                } else if (m == 2) {
                    vx = __dsub_rn(__dmul_rn(2.0, P.Utop), vx);
                    vy = -fabs(vy);
                } else {
                    vy = -fabs(vy);
                }
                if (kInfo) {
                    const double dvx = __dsub_rn(vx, ox), dvy = __dsub_rn(vy, oy);
                    nhit[1] += 1;
                    acc[0] = __dadd_rn(acc[0], __dmul_rn(0.5, __dsub_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)),
                                                                      __dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)))));
                    acc[2] = __dadd_rn(acc[2], dvx);
                    acc[4] = __dadd_rn(acc[4], fabs(dvy));
                }
            } else {
                *err = kErrUnsupportedBcTop;
                return false;
            }
        }
    }
#undef PAIR
    // final wrap / clamp (src/boundary_conditions.cpp:178-202)
    if (P.perx) {
        x = __dsub_rn(x, __dmul_rn(floor_div(x, Lx, P.invLx), Lx));
    } else {
        if (x < 0.0) x = 0.0;
        if (x > Lx) x = Lx;
    }
    if (P.pery) {
        y = __dsub_rn(y, __dmul_rn(floor_div(y, Ly, P.invLy), Ly));
    } else {
        if (y < 0.0) y = 0.0;
        if (y > Ly) y = Ly;
    }
    return true;
}

// SRD cell of a position on the shifted grid (src/srd_collision.cpp:18-43)
__device__ __forceinline__ int srd_cell(double x, double y, double sx, double sy, const DevParams& P) {
    double xs = __dadd_rn(x, sx), ys = __dadd_rn(y, sy);
    if (P.perx) {
        xs = __dsub_rn(xs, __dmul_rn(floor_div(xs, P.Lx, P.invLx), P.Lx));
    } else {
        if (xs < 0.0) xs = 0.0;
        if (xs >= P.Lx) xs = nextafter(P.Lx, 0.0);
    }
    if (P.pery) {
        ys = __dsub_rn(ys, __dmul_rn(floor_div(ys, P.Ly, P.invLy), P.Ly));
    } else {
        if (ys < 0.0) ys = 0.0;
        if (ys >= P.Ly) ys = nextafter(P.Ly, 0.0);
    }
    int ix = (int)floor_div(xs, P.a0, P.invA0), iy = (int)floor_div(ys, P.a0, P.invA0);
    if (ix < 0) ix = 0;
    if (ix >= P.Nx) ix = P.Nx - 1;
    if (iy < 0) iy = 0;
    if (iy >= P.Ny) iy = P.Ny - 1;
    return iy + P.Ny * ix;
}

// The two shift draws U(-a0/2, a0/2) of srd_cell_id_with_random_shift: outputs 0 and 1 of
// mt19937_64(seed), which need seeded words 0, 1, 2, 156, 157 only. One thread.
// stepCounter (graph replay): first begin the step on the device (step_begin), then draw its
// shift from the device seed table
__global__ void k_srd_shift(DevParams P, uint64_t seed, double* out, const uint64_t* seedDev,
                            long long* stepCounter = nullptr, uint64_t* stepSeeds = nullptr) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (stepCounter) step_begin(stepCounter, stepSeeds);
    if (seedDev) seed = seedDev[kSeedSrdShift];
    uint64_t w[kMtM + 2];
    w[0] = seed;
    for (int i = 1; i < kMtM + 2; ++i) w[i] = mt_seed_next(w[i - 1], i);
    const uint64_t o0 = mt_temper(w[kMtM] ^ mt_mix(w[0], w[1]));
    const uint64_t o1 = mt_temper(w[kMtM + 1] ^ mt_mix(w[1], w[2]));
    const double a = __dmul_rn(-0.5, P.a0), b = __dmul_rn(0.5, P.a0);
    out[0] = __dadd_rn(__dmul_rn(canon(o0), __dsub_rn(b, a)), a);
    out[1] = __dadd_rn(__dmul_rn(canon(o1), __dsub_rn(b, a)), a);
}

// Streams (optional), replays the sweeps, and computes the cell ids the next phases need.
// S: slot-ordered state. cidStd: cell on the standard grid; cidSrd (optional): SRD cell.
template <bool kInfo, class V>
__global__ void k_stream_bc(DevParams P, int doStream, V S, const int* __restrict__ pid, int* __restrict__ cidStd,
                            int* __restrict__ cidSrd, BcWork W, DevStatus* st) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kWallDoubles];
    for (int k = 0; k < kWallDoubles; ++k) acc[k] = 0.0;
    int nhit[4] = {0, 0, 0, 0};
    if (s < P.n) {
        double2 xs = S.pos(s, P), vs = S.vel(s);
        if (doStream) {
            vs.x = __dadd_rn(vs.x, __dmul_rn(P.bodyForceX, P.dt));
            vs.y = __dadd_rn(vs.y, __dmul_rn(P.g, P.dt));
            xs.x = __dadd_rn(xs.x, __dmul_rn(P.dt, vs.x));
            xs.y = __dadd_rn(xs.y, __dmul_rn(P.dt, vs.y));
        }
        const double2 x0 = xs, v0 = vs;
        int tx = 0, ty = 0, late = 0, err = 0;
        double a2[kWallDoubles];
        int h2[4] = {0, 0, 0, 0};
        for (int k = 0; k < kWallDoubles; ++k) a2[k] = 0.0;
        const bool ok = bc_replay<true, kInfo>(xs.x, xs.y, vs.x, vs.y, P, nullptr, 0, 1, tx, ty, late, a2, h2, &err);
        if (!ok) {
            raise_error(st, err, s);
        } else if (tx + ty == 0 && !late) {
            S.set_vel(s, vs);
            for (int k = 0; k < kWallDoubles; ++k) acc[k] = a2[k];
            for (int k = 0; k < 4; ++k) nhit[k] = h2[k];
        } else {
            if (late || tx > 1 || ty > 1) raise_error(st, kErrBcLateSweep, pid[s]);
            const int p = pid[s];
            if (tx) atomicOr(&W.bitsX[p >> 5], 1u << (p & 31));
            if (ty) atomicOr(&W.bitsY[p >> 5], 1u << (p & 31));
            const int e = atomicAdd(W.nEvents, 1);
            if (e < W.eventCap) {
                WallEvent ev;
                ev.slot = s;
                ev.pid = p;
                ev.x = x0.x;
                ev.y = x0.y;
                ev.vx = v0.x;
                ev.vy = v0.y;
                W.events[e] = ev;
            } else {
                raise_error(st, kErrEventCapacity, e);
            }
        }
        const int cs = cell_of(xs.x, xs.y, P);
        S.set_pos(s, xs, cs, P);
        if (cidStd) cidStd[s] = cs;
        if (cidSrd) cidSrd[s] = srd_cell(xs.x, xs.y, W.srdShift[0], W.srdShift[1], P);
    }
    if (!kInfo) return;
    // block partial WallInfo of particles finished here (fixed reduction order)
    __shared__ double sh[kWallDoubles][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < kWallDoubles; ++k) {
        double a = acc[k];
        for (int o = 16; o > 0; o >>= 1) a = __dadd_rn(a, __shfl_down_sync(0xffffffffu, a, o));
        if (lane == 0) sh[k][wid] = a;
    }
    for (int k = 0; k < 4; ++k) {
        int c = nhit[k];
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0 && c) atomicAdd(&W.ints[k], c);
    }
    __syncthreads();
    if (threadIdx.x < kWallDoubles) {
        double a = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a = __dadd_rn(a, sh[threadIdx.x][w]);
        W.blockPartial[blockIdx.x * kWallDoubles + threadIdx.x] = a;
    }
}

__global__ void k_word_counts(const uint32_t* __restrict__ bx, const uint32_t* __restrict__ by, int nwords,
                              uint64_t* __restrict__ cnt) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nwords) cnt[w] = (uint64_t)(__popc(bx[w]) + __popc(by[w]));
}

// One block of 320 threads generates pairs 0 .. nPairs-1 of normal_distribution(0,1) on
// mt19937_64(seed): attempt a uses draws 2a, 2a+1; accepted attempts become pairs in
// order; pair p = (y*mult, x*mult) = (first deviate, cached second deviate).
constexpr int kNormThreads = 320;
__global__ void __launch_bounds__(kNormThreads) k_wall_normals(uint64_t seed, const uint64_t* __restrict__ totalPairs,
                                                             int cap, double* __restrict__ normals, DevStatus* st,
                                                             const uint64_t* seedDev) {
    if (seedDev) seed = seedDev[kSeedBc];
    __shared__ uint64_t mt[kMtN];
    __shared__ uint64_t scanSh[32];
    const int t = threadIdx.x;
    const int need = (int)*totalPairs;
    if (need > cap) {
        if (t == 0) raise_error(st, kErrEventCapacity, need);
        return;
    }
    if (need == 0) return;
    if (t == 0) {
        uint64_t w = seed;
        mt[0] = w;
        for (int i = 1; i < kMtN; ++i) {
            w = mt_seed_next(w, i);
            mt[i] = w;
        }
    }
    __syncthreads();
    int produced = 0;
    while (produced < need) {
        // in-place twist, reads before writes in each half
        uint64_t nv = 0;
        if (t < kMtN - kMtM) nv = mt[t + kMtM] ^ mt_mix(mt[t], mt[t + 1]);
        __syncthreads();
        if (t < kMtN - kMtM) mt[t] = nv;
        __syncthreads();
        if (t >= kMtN - kMtM && t < kMtN) {
            const uint64_t nxt = (t + 1 < kMtN) ? mt[t + 1] : mt[0];
            nv = mt[t - (kMtN - kMtM)] ^ mt_mix(mt[t], nxt);
        }
        __syncthreads();
        if (t >= kMtN - kMtM && t < kMtN) mt[t] = nv;
        __syncthreads();
        // 156 attempts per block of 312 draws
        double xa = 0.0, ya = 0.0, r2 = 0.0;
        int acc = 0;
        if (t < kMtN / 2) {
            xa = __dsub_rn(__dmul_rn(2.0, canon(mt_temper(mt[2 * t]))), 1.0);
            ya = __dsub_rn(__dmul_rn(2.0, canon(mt_temper(mt[2 * t + 1]))), 1.0);
            r2 = __dadd_rn(__dmul_rn(xa, xa), __dmul_rn(ya, ya));
            acc = !(r2 > 1.0 || r2 == 0.0);
        }
        uint64_t tot;
        const int rank = (int)block_exclusive_scan((uint64_t)acc, scanSh, &tot);
        const int p = produced + rank;
        if (acc && p < need) {
            const double mult = sqrt(__ddiv_rn(__dmul_rn(-2.0, mpcd_dd::log_cr(r2)), r2));
            normals[2 * p] = __dmul_rn(ya, mult);
            normals[2 * p + 1] = __dmul_rn(xa, mult);
        }
        produced += (int)tot;
        __syncthreads();
    }
}

// Thermal particles: replay with their pairs; write the final velocity and the WallInfo
// contribution at the slot of their first pair.
template <class V>
__global__ void k_wall_apply(DevParams P, V S, BcWork W, DevStatus* st) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = min(*W.nEvents, W.eventCap);
    if (e >= ne) return;
    const WallEvent ev = W.events[e];
    const int p = ev.pid, w = p >> 5;
    const uint32_t below = (1u << (p & 31)) - 1u;
    const int first = (int)W.wordPrefix[w] + __popc(W.bitsX[w] & below) + __popc(W.bitsY[w] & below);
    if (first + 2 > W.normalCap) {  // pairs were not generated (capacity error already raised)
        raise_error(st, kErrEventCapacity, first);
        return;
    }
    double x = ev.x, y = ev.y, vx = ev.vx, vy = ev.vy;
    double acc[kWallDoubles];
    for (int k = 0; k < kWallDoubles; ++k) acc[k] = 0.0;
    int nhit[4] = {0, 0, 0, 0}, tx = 0, ty = 0, late = 0, err = 0;
    if (!bc_replay<false>(x, y, vx, vy, P, W.normals, first, W.normalCap, tx, ty, late, acc, nhit, &err)) {
        raise_error(st, err, ev.slot);
        return;
    }
    S.set_vel(ev.slot, make_double2(vx, vy));
    const int npairs = tx + ty;
    for (int k = 0; k < kWallDoubles; ++k) {
        W.contrib[(size_t)first * kWallDoubles + k] = acc[k];
        if (npairs > 1) W.contrib[(size_t)(first + 1) * kWallDoubles + k] = 0.0;
    }
    for (int k = 0; k < 4; ++k)
        if (nhit[k]) atomicAdd(&W.ints[k], nhit[k]);
}

// WallInfo doubles: block partials of k_stream_bc then per-pair contributions, in order.
__global__ void k_wall_reduce(const double* __restrict__ partial, int nPartial, const double* __restrict__ contrib,
                              const uint64_t* __restrict__ totalPairs, int cap, double* __restrict__ out) {
    const int k = threadIdx.x;
    if (k >= kWallDoubles) return;
    double a = 0.0;
    for (int b = 0; b < nPartial; ++b) a = __dadd_rn(a, partial[b * kWallDoubles + k]);
    const int np = min((int)*totalPairs, cap);
    for (int q = 0; q < np; ++q) a = __dadd_rn(a, contrib[(size_t)q * kWallDoubles + k]);
    out[k] = a;
}

}  // namespace mpcd_dev
