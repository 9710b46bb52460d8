// The fast form of the step: FP32 cell-relative state in per-cell bins, exact int64 cell sums,
// and a redistribution whose decisions use counter-based draws.
//
// The plain form reproduces the reference's draws one by one, which ties every zone to the
// serial order of one generator. The fast form keeps the reference's physics and rules:
//   - stream and body force, the wall modes of apply_bc_general (src/boundary_conditions.cpp:19-203);
//   - the SRD rotation by +-alpha on a randomly shifted grid with the isokinetic thermostat
//     (src/srd_collision.cpp:9-140);
//   - the zone redistribution (src/zone_pass.cpp:669-973): dense passes with ranked range-2
//     targets in 8 angular bins, round-robin quotas, relief targets, the sparse phase with
//     donors ranked by the smoothed-occupancy gradient, the transfer masks and the per-cell
//     momentum correction, on the base tiles and then on tiles shifted by half a tile;
//   - the liquid closure (src/liquid_closure.cpp:329-444): repair kick with beta_opt, pressure
//     drive smoothed on the interzone mask, EOS kick;
// but draws every random number from a hash of (run seed, step, what the draw is for), so that
// zones, cells and particles proceed independently.
//
// Order-free by construction: no result depends on the order of particles inside a bin, which
// atomics make arbitrary. Cell sums are exact integer sums; a choice between particles uses
// their particle ids; per-particle draws are keyed by particle id. So the state, read in
// particle-id order, is the same from run to run.
//
// State. Each cell c owns the bin of slots [c K, c K + cnt[c]) in three arrays: the position
// inside the cell in cell units (float2 in [0, 1)), the velocity (float2) and the particle id.
// Velocities are kept on the grid of 2^-20: q = v 2^20 is an integer (exact in FP32 while
// |v| < 16), so momentum sums are exact int64 sums and a conserving update can restore them to
// the last unit. K is fixed per context (a few times the mean occupancy); a cell above K
// particles fails the step with a capacity error.
#pragma once

#include <cstdint>

#include "closure.cuh"
#include "common.cuh"

namespace mpcd_dev {

constexpr double kFastQ = 1048576.0;           // grid units per velocity unit (2^20)
constexpr double kFastInvQ = 1.0 / 1048576.0;
constexpr float kFastOffMax = 0x1.fffffep-1f;  // largest float below 1
constexpr int kFastMaxK = 128;                 // bin capacity limit (removal masks of 4 words)
constexpr int kFastMaxZoneCells = 128;         // zone cells (dense/low orders sort 128 keys)
constexpr int kFastZoneWarps = 8;              // zones per block of the zone decision kernel
constexpr int kErrBinCapacity = 13;            // a cell above its bin capacity
constexpr int kErrRecordCapacity = 14;         // a zone's moves outgrew its record area

struct FastBins {
    float2* off;
    float2* vel;
    int* pid;
    int* cnt;
};

// Values of the running step, derived on the device by k_fast_step_begin (graph replay keeps
// the step number on the device).
struct FastStep {
    long long step;
    int fqx, fqy;                // body-force increments of this step, grid units
    double sx, sy;               // SRD grid shift in cell units, in [-1/2, 1/2)
    unsigned long long seed;     // hash seed of this step
};

struct FastParams {
    int K;
    int zoneWY;                  // unused padding for alignment
    double fqx, fqy;             // body force * dt in grid units (fractional)
    float dtqx, dtqy;            // cell units moved per grid unit of velocity in one step
    double sigmaQ, UtopQ, UbottomQ;  // wall temperature and wall speeds in grid units
    double lowMapEmpty, highMapEmpty;  // threshold maps of empty cells (src/zone_pass.cpp:321-345)
    unsigned long long seed;     // run seed
};

// Wall hits and the wall energy change (int64, grid^2 units) of a step
struct FastWall {
    unsigned long long n[4];     // left, right, bottom, top
    unsigned long long dE2;      // sum of (|q'|^2 - |q|^2) over the hits, two's complement
};

// ------------------------------------------------------------------ counter-based draws
// SplitMix64's output function (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): a bijective 64-bit mixer, here applied to combined keys.
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t fhash(uint64_t a, uint64_t b, uint64_t c) {
    return fmix64(fmix64(fmix64(a) ^ b) ^ c);
}
// uniform in [0, 1) with 53 random bits
__device__ __forceinline__ double fu01(uint64_t h) { return (double)(h >> 11) * 0x1.0p-53; }
// standard normal by the Box-Muller transform of two uniforms of h1, h2
__device__ __forceinline__ double fnormal(uint64_t h1, uint64_t h2) {
    const double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53;  // (0, 1]
    const double u2 = (double)(h2 >> 11) * 0x1.0p-53;
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

__device__ __forceinline__ int fq_of(float v) { return __float2int_rn(v * 1048576.0f); }
// q / 2^20 rounded once to FP32 (scaling by a power of two commutes with the rounding)
__device__ __forceinline__ float fv_of(long long q) { return __ll2float_rn(q) * 0x1.0p-20f; }

// floor(a / b) for b > 0
__device__ __forceinline__ long long floor_div_ll(long long a, long long b) {
    long long q = a / b;
    if ((a % b != 0) && (a < 0)) --q;
    return q;
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_min_u64_c(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, v, o);
        v = x < v ? x : v;
    }
    return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Full-warp int64 sum with redux.sync: the two's-complement words summed in four 16-bit limbs
// (a limb's sum over 32 lanes stays below 2^21), exact modulo 2^64.
__device__ __forceinline__ long long warp_sum_i64(long long v) {
    const unsigned long long u = (unsigned long long)v;
    unsigned long long s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        s += (unsigned long long)__reduce_add_sync(0xffffffffu, (unsigned)(u >> (16 * k)) & 0xFFFFu) << (16 * k);
    return (long long)s;
}
// Full-warp u64 minimum with redux.sync: the high words' minimum, then the low words' among the
// lanes that hold it.
__device__ __forceinline__ unsigned long long warp_min_u64_r(unsigned long long v) {
    const unsigned hi = (unsigned)(v >> 32);
    const unsigned mh = __reduce_min_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_min_sync(0xffffffffu, hi == mh ? (unsigned)v : 0xFFFFFFFFu);
    return ((unsigned long long)mh << 32) | ml;
}

// ------------------------------------------------------------------ step begin
__device__ __forceinline__ void fast_step_begin(const FastParams& F, FastStep* S, FastWall* W, int* nSpill) {
    *nSpill = 0;
    const long long s = S->step + 1;
    S->step = s;
    // the long-run force is exact: the increments of steps 1..s add up to round(s f)
    S->fqx = (int)(llrint((double)s * F.fqx) - llrint((double)(s - 1) * F.fqx));
    S->fqy = (int)(llrint((double)s * F.fqy) - llrint((double)(s - 1) * F.fqy));
    const uint64_t h = fhash(F.seed, (uint64_t)s, 0x535244ULL);
    S->sx = fu01(h) - 0.5;
    S->sy = fu01(fmix64(h)) - 0.5;
    S->seed = fhash(F.seed, (uint64_t)s, 0x5354ULL);
    for (int k = 0; k < 4; ++k) W->n[k] = 0;
    W->dE2 = 0;
}

__global__ void k_fast_step_begin(FastParams F, FastStep* S, FastWall* W, int* nSpill) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    fast_step_begin(F, S, W, nSpill);
}

// ------------------------------------------------------------------ stream + walls + binning
constexpr int kStreamCells = 8;  // cells per warp of the stream kernel

// A coordinate along one axis as (cell, offset in [0, 1)): integer arithmetic for the cell,
// FP32 for the offset. Moving the integer part of the offset into the cell is exact for
// offsets of at least 0; below 0 it rounds once (at most half a unit of 2^-24).
__device__ __forceinline__ void fix_cell(int& c, float& r) {
    const float f = floorf(r);
    c += (int)f;
    r -= f;
    if (r >= 1.0f) {
        ++c;
        r = 0.0f;
    }
}
// x -> -x
__device__ __forceinline__ void reflect_low(int& c, float& r) {
    if (r > 0.0f) {
        c = -c - 1;
        r = 1.0f - r;
        fix_cell(c, r);
    } else {
        c = -c;
    }
}
// x -> 2 L - x
__device__ __forceinline__ void reflect_high(int& c, float& r, int L) {
    if (r > 0.0f) {
        c = 2 * L - c - 1;
        r = 1.0f - r;
        fix_cell(c, r);
    } else {
        c = 2 * L - c;
    }
}

// One warp per run of kStreamCells consecutive source cells, the lanes over the run's particles
// in order. Applies the pending closure kick of the previous step (kick[c], grid units,
// nullable), then body force, streaming and the walls of apply_bc_general
// (src/boundary_conditions.cpp:37-202: up to four sweeps of left, right, bottom, top, then the
// final wrap or clamp), and files each particle into the bin of its new cell (warp-aggregated
// slot claims).
__device__ __forceinline__ void fast_stream_block(int bx, const DevParams& P, const FastParams& F,
                                                  const FastStep* __restrict__ S, const FastBins& in,
                                                  const FastBins& out, const int2* __restrict__ kick,
                                                  FastWall* __restrict__ W, DevStatus* st) {
    const int c0 = (int)((bx * (size_t)blockDim.x + threadIdx.x) >> 5) * kStreamCells;
    const int lane = threadIdx.x & 31;
    if (c0 >= P.Nc) return;
    // lanes below kStreamCells: their cell's count and the exclusive prefix of the counts
    int n = 0;
    if (lane < kStreamCells && c0 + lane < P.Nc) n = min(in.cnt[c0 + lane], F.K);
    int incl = n;
#pragma unroll
    for (int o = 1; o < kStreamCells; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    const int excl = incl - n;
    const int total = __shfl_sync(0xffffffffu, incl, kStreamCells - 1);
    const int ix0 = c0 / P.Ny, iy0 = c0 - ix0 * P.Ny;
    const int fqx = S->fqx, fqy = S->fqy;
    const uint64_t seed = S->seed;
    const int Nx = P.Nx, Ny = P.Ny;
    int hits[4] = {0, 0, 0, 0};
    long long dE2 = 0;
    // the particle i of the run: its cell g (the last whose start is at most i, by a binary
    // search over the starts held in lanes 0 .. 7) and slot; each round's loads are issued
    // before the previous round is processed
    auto locate = [&](int i, int& g, int& slot) {
        g = 0;
#pragma unroll
        for (int st = kStreamCells / 2; st >= 1; st >>= 1) {
            const int sv = __shfl_sync(0xffffffffu, excl, g + st);
            if (i >= sv) g += st;
        }
        slot = i - __shfl_sync(0xffffffffu, excl, g);
    };
    float2 offA = make_float2(0.f, 0.f), velA = offA;
    int pidA = 0, gA = 0;
    int2 kickA = make_int2(0, 0);
    auto fetch = [&](int i) {
        int g, slot;
        locate(i, g, slot);
        gA = g;
        if (i < total) {
            const size_t s = (size_t)(c0 + g) * F.K + slot;
            offA = in.off[s];
            velA = in.vel[s];
            pidA = in.pid[s];
            if (kick) kickA = kick[c0 + g];
        }
    };
    fetch(lane);
    for (int i0 = 0; i0 < total; i0 += 32) {
        const int i = i0 + lane;
        const bool live = i < total;
        const float2 off = offA, w = velA;
        const int g = gA;
        int pid = pidA;
        const int2 kq = kickA;
        fetch(i + 32);
        int newc = 0, qx = 0, qy = 0;
        float2 o = make_float2(0.f, 0.f);
        if (live) {
            const int c = c0 + g;
            int cx = ix0, cy = iy0 + g;
            while (cy >= Ny) {
                cy -= Ny;
                ++cx;
            }
            qx = fq_of(w.x) + kq.x + fqx;
            qy = fq_of(w.y) + kq.y + fqy;
            float rx = off.x + (float)qx * F.dtqx, ry = off.y + (float)qy * F.dtqy;
            fix_cell(cx, rx);
            fix_cell(cy, ry);
            // x < 0 is cx < 0; x > L is cx > L or (cx == L and r > 0)
            auto below = [](int cc) { return cc < 0; };
            auto above = [](int cc, float r, int L) { return cc > L || (cc == L && r > 0.0f); };
            bool inside = !below(cx) && !above(cx, rx, Nx) && !below(cy) && !above(cy, ry, Ny);
            for (int sweep = 0; sweep < 4 && !inside; ++sweep) {
                const long long e0 = (long long)qx * qx + (long long)qy * qy;
                bool hit = false;
                const uint64_t hk = fhash(seed, (uint64_t)(uint32_t)pid, (uint64_t)sweep);
                if (below(cx)) {
                    if (P.bc[0] == MPCD_BC_PERIODIC) {
                        cx += Nx;
                    } else {
                        reflect_low(cx, rx);
                        if (P.bc[0] == MPCD_BC_THERMALIZE) {
                            qx = (int)llrint(fabs(F.sigmaQ * fnormal(fmix64(hk ^ 1), fmix64(hk ^ 2))));
                            qy = (int)llrint(F.sigmaQ * fnormal(fmix64(hk ^ 3), fmix64(hk ^ 4)));
                        } else if (P.bc[0] == MPCD_BC_BOUNCEBACK) {
                            qx = abs(qx);
                            qy = -qy;
                        } else if (P.bc[0] == MPCD_BC_SPECULAR) {
                            qx = abs(qx);
                        } else if (st) {
                            raise_error(st, kErrUnsupportedBcLeft, c);
                        }
                        ++hits[0];
                        hit = true;
                    }
                }
                if (above(cx, rx, Nx)) {
                    if (P.bc[1] == MPCD_BC_PERIODIC) {
                        cx -= Nx;
                    } else {
                        reflect_high(cx, rx, Nx);
                        if (P.bc[1] == MPCD_BC_THERMALIZE) {
                            qx = -(int)llrint(fabs(F.sigmaQ * fnormal(fmix64(hk ^ 5), fmix64(hk ^ 6))));
                            qy = (int)llrint(F.sigmaQ * fnormal(fmix64(hk ^ 7), fmix64(hk ^ 8)));
                        } else if (P.bc[1] == MPCD_BC_BOUNCEBACK) {
                            qx = -abs(qx);
                            qy = -qy;
                        } else if (P.bc[1] == MPCD_BC_SPECULAR) {
                            qx = -abs(qx);
                        } else if (st) {
                            raise_error(st, kErrUnsupportedBcRight, c);
                        }
                        ++hits[1];
                        hit = true;
                    }
                }
                if (below(cy)) {
                    if (P.bc[2] == MPCD_BC_PERIODIC) {
                        cy += Ny;
                    } else {
                        reflect_low(cy, ry);
                        if (P.bc[2] == MPCD_BC_THERMALIZE) {
                            qx = (int)llrint(F.UbottomQ + F.sigmaQ * fnormal(fmix64(hk ^ 9), fmix64(hk ^ 10)));
                            qy = (int)llrint(fabs(F.sigmaQ * fnormal(fmix64(hk ^ 11), fmix64(hk ^ 12))));
                        } else if (P.bc[2] == MPCD_BC_BOUNCEBACK) {
                            qx = (int)llrint(2.0 * F.UbottomQ) - qx;
                            qy = abs(qy);
                        } else if (P.bc[2] == MPCD_BC_SPECULAR) {
                            qy = abs(qy);
                        } else if (st) {
                            raise_error(st, kErrUnsupportedBcBottom, c);
                        }
                        ++hits[2];
                        hit = true;
                    }
                }
                if (above(cy, ry, Ny)) {
                    if (P.bc[3] == MPCD_BC_PERIODIC) {
                        cy -= Ny;
                    } else {
                        reflect_high(cy, ry, Ny);
                        if (P.bc[3] == MPCD_BC_THERMALIZE) {
                            qx = (int)llrint(F.UtopQ + F.sigmaQ * fnormal(fmix64(hk ^ 13), fmix64(hk ^ 14)));
                            qy = -(int)llrint(fabs(F.sigmaQ * fnormal(fmix64(hk ^ 15), fmix64(hk ^ 16))));
                        } else if (P.bc[3] == MPCD_BC_BOUNCEBACK) {
                            qx = (int)llrint(2.0 * F.UtopQ) - qx;
                            qy = -abs(qy);
                        } else if (P.bc[3] == MPCD_BC_SPECULAR) {
                            qy = -abs(qy);
                        } else if (st) {
                            raise_error(st, kErrUnsupportedBcTop, c);
                        }
                        ++hits[3];
                        hit = true;
                    }
                }
                if (hit) dE2 += (long long)qx * qx + (long long)qy * qy - e0;
                inside = !below(cx) && !above(cx, rx, Nx) && !below(cy) && !above(cy, ry, Ny);
            }
            // the final wrap x - floor(x / L) L or clamp (src/boundary_conditions.cpp:178-202);
            // after the sweeps a particle is within one period of the box
            if (P.perx) {
                if (cx < 0) cx += Nx;
                if (cx >= Nx) cx -= Nx;
            } else if (cx < 0) {
                cx = 0;
                rx = 0.0f;
            } else if (cx >= Nx) {
                cx = Nx - 1;
                rx = kFastOffMax;
            }
            if (P.pery) {
                if (cy < 0) cy += Ny;
                if (cy >= Ny) cy -= Ny;
            } else if (cy < 0) {
                cy = 0;
                ry = 0.0f;
            } else if (cy >= Ny) {
                cy = Ny - 1;
                ry = kFastOffMax;
            }
            cx = min(max(cx, 0), Nx - 1);
            cy = min(max(cy, 0), Ny - 1);
            o = make_float2(fminf(rx, kFastOffMax), fminf(ry, kFastOffMax));
            newc = cy + Ny * cx;
        }
        // warp-aggregated slot claims in the destination bins
        const unsigned act = __ballot_sync(0xffffffffu, live);
        if (live) {
            const unsigned grp = __match_any_sync(act, newc);
            const int leader = __ffs(grp) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(out.cnt + newc, __popc(grp));
            base = __shfl_sync(grp, base, leader);
            const int slot = base + __popc(grp & lanemask_lt());
            if (slot < F.K) {
                const size_t d = (size_t)newc * F.K + slot;
                out.off[d] = o;
                out.vel[d] = make_float2(fv_of(qx), fv_of(qy));
                out.pid[d] = pid;
            } else if (st) {
                raise_error(st, kErrBinCapacity, newc);
            }
        }
    }
    if (W) {
        for (int k = 0; k < 4; ++k) {
            const int h = warp_sum_i(hits[k]);
            if (lane == 0 && h) atomicAdd(&W->n[k], (unsigned long long)h);
        }
        const long long e = warp_sum_ll(dE2);
        if (lane == 0 && e) atomicAdd(&W->dE2, (unsigned long long)e);
    }
}

__global__ void __launch_bounds__(256, 4) k_fast_stream(DevParams P, FastParams F, const FastStep* __restrict__ S,
                                                     FastBins in, FastBins out, const int2* __restrict__ kick,
                                                     FastWall* __restrict__ W, DevStatus* st) {
    fast_stream_block((int)blockIdx.x, P, F, S, in, out, kick, W, st);
}

// ------------------------------------------------------------------ SRD collision
// The SRD cell along one axis of a particle at standard cell g with offset r: the grid shifted
// by ss in [-1/2, 1/2) cells (srd_cell_id_with_random_shift, src/srd_collision.cpp:9-45:
// wrapped on periodic axes, clamped on the others). SRD cell s thus holds particles of the
// standard cells s - 1 and s (ss >= 0) or s and s + 1 (ss < 0).
__device__ __forceinline__ int srd_axis(int g, float r, float ss, int N, bool per) {
    int s = g + (int)floorf(r + ss);
    if (s < 0) s = per ? s + N : 0;
    if (s >= N) s = per ? s - N : N - 1;
    return s;
}

// Rotation of one SRD cell (src/srd_collision.cpp:47-140) from its exact sums in grid units:
// velocities relative to the cell mean turned by +-alpha (the sign drawn per SRD cell) and
// scaled by the isokinetic thermostat's factor.
struct SrdRot {
    double ux, uy, lam, ct, sn;
};
__device__ __forceinline__ SrdRot srd_rotation(const DevParams& P, uint64_t seed, int w, int N, long long Sx,
                                               long long Sy, long long Sqq) {
    SrdRot R;
    R.ux = (double)Sx / N;
    R.uy = (double)Sy / N;
    R.ct = 1.0;
    R.sn = 0.0;
    if (N >= 2) {
        const uint64_t h = fhash(seed, (uint64_t)w, 0x5349474EULL);
        const int rr = (h >> 63) ? 1 : 2;  // +alpha or -alpha
        R.ct = P.rotCos[rr];
        R.sn = P.rotSin[rr];
    }
    R.lam = 1.0;
    if (P.useThermostat && N > 1) {
        // sum |q - u|^2 = (N sum|q|^2 - |sum q|^2) / N, an exact integer numerator (in 64 bits
        // when its terms stay below 2^62, else in 128)
        double numd;
        if (N < 512 && Sqq < (1LL << 53) && llabs(Sx) < (1LL << 31) && llabs(Sy) < (1LL << 31))
            numd = (double)((long long)N * Sqq - Sx * Sx - Sy * Sy);
        else
            numd = (double)((__int128)N * Sqq - (__int128)Sx * Sx - (__int128)Sy * Sy);
        const double s2 = numd / (double)N;
        if (s2 > 0.0) R.lam = sqrt(2.0 * (double)(N - 1) * P.kBT * kFastQ * kFastQ / s2);
    }
    return R;
}
__device__ __forceinline__ void srd_rotate(const SrdRot& R, int qx, int qy, long long& nx, long long& ny) {
    const double rx = (double)qx - R.ux, ry = (double)qy - R.uy;
    nx = llrint(R.ux + R.lam * (R.ct * rx - R.sn * ry));
    ny = llrint(R.uy + R.lam * (R.sn * rx + R.ct * ry));
}
// the members that may take an SRD cell's rounding residual: new velocities of |n| < 2^22
__device__ __forceinline__ bool srd_eligible(long long nx, long long ny) {
    return llabs(nx) < (1LL << 22) && llabs(ny) < (1LL << 22);
}

// SRD collision tiles: kCollTX x TY SRD cells per block of kCollThreads threads. The block
// gathers the standard cells under its tile (one column and one row of halo on the side the
// shift points to) into shared memory, sorts their particles by SRD cell, collides each SRD
// cell with 32 / TY threads and writes the new velocities back in place. Each cell keeps its
// momentum exactly: the rounding of the new velocities to the grid leaves an integer residual
// that goes to the eligible member with the smallest particle id. A tile whose standard cells
// hold more than pcap particles is left to k_fast_collide_spill.
constexpr int kCollTX = 8;
constexpr int kCollThreads = 256;
constexpr int kCollMaxStd = (kCollTX + 1) * (32 + 1);  // standard cells under a tile (TY <= 32)

struct CollideArgs {
    DevParams P;
    FastParams F;
    const FastStep* S;
    FastBins b;
    int TY, tilesY, nTiles, pcap;
    int* spill;   // tiles left to the spill kernel
    int* nSpill;  // their number (zeroed by k_fast_step_begin)
};

// the shared layout of a tile: standard-cell tables, then per staged particle its velocity,
// id, SRD cell and rank, home (local cell << 7 | slot) and the SRD-ordered member list
struct CollideMem {
    int* cstart;    // kCollMaxStd + 1
    int* gcell;     // kCollMaxStd
    short2* gxy;    // kCollMaxStd
    int* scnt;      // 256
    int* sstart;    // 257
    int* wsum;      // 32
    int2* q;        // pcap
    int* pid;       // pcap
    uint32_t* sr;   // pcap: (SRD cell << 16) | rank, ~0 outside the tile
    uint16_t* home; // pcap
    uint16_t* list; // pcap
    __host__ __device__ static size_t bytes(int pcap) {
        return (size_t)(kCollMaxStd + 1) * 4 + kCollMaxStd * 4 + kCollMaxStd * 4 + 256 * 4 + 257 * 4 + 32 * 4 +
               (size_t)pcap * (8 + 4 + 4 + 2 + 2) + 64;
    }
    __device__ void carve(char* base, int pcap) {
        char* p = base;
        auto take = [&](size_t n, size_t a) {
            p = (char*)(((uintptr_t)p + a - 1) / a * a);
            char* r = p;
            p += n;
            return r;
        };
        q = (int2*)take((size_t)pcap * 8, 8);
        pid = (int*)take((size_t)pcap * 4, 4);
        sr = (uint32_t*)take((size_t)pcap * 4, 4);
        cstart = (int*)take((size_t)(kCollMaxStd + 1) * 4, 4);
        gcell = (int*)take((size_t)kCollMaxStd * 4, 4);
        gxy = (short2*)take((size_t)kCollMaxStd * 4, 4);
        scnt = (int*)take(256 * 4, 4);
        sstart = (int*)take(257 * 4, 4);
        wsum = (int*)take(32 * 4, 4);
        home = (uint16_t*)take((size_t)pcap * 2, 2);
        list = (uint16_t*)take((size_t)pcap * 2, 2);
    }
};

// exclusive prefix of v[0..n) into out[0..n] (out[n] the total), n <= 512, all threads of a
// kCollThreads block; v and out may alias
__device__ void block_scan(const int* v, int* out, int n, int* wsum) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    int carry = 0;
    for (int b0 = 0; b0 < n; b0 += kCollThreads) {
        const int t = b0 + tid;
        const int x = t < n ? v[t] : 0;
        int incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            const int w = lane < kCollThreads / 32 ? wsum[lane] : 0;
            int wi = w;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += u;
            }
            if (lane < kCollThreads / 32) wsum[lane] = wi - w;
            if (lane == kCollThreads / 32 - 1) wsum[kCollThreads / 32] = wi;
        }
        __syncthreads();
        if (t < n) out[t] = carry + wsum[wid] + incl - x;
        carry += wsum[kCollThreads / 32];
        __syncthreads();
    }
    if (tid == 0) out[n] = carry;
    __syncthreads();
}

__device__ __forceinline__ void fast_collide_tile_block(int bx, const CollideArgs& A, char* smem) {
    const DevParams& P = A.P;
    const int K = A.F.K;
    const int tid = threadIdx.x;
    CollideMem M;
    M.carve(smem, A.pcap);
    const int tile = bx;
    const int X0 = (tile / A.tilesY) * kCollTX, Y0 = (tile % A.tilesY) * A.TY;
    const int TXc = min(kCollTX, P.Nx - X0), TYc = min(A.TY, P.Ny - Y0);
    const float ssx = (float)A.S->sx, ssy = (float)A.S->sy;
    // the halo column: X0 - 1 for a shift >= 0, X0 + TXc for a shift < 0 (when that column
    // exists and is not in the tile)
    const bool upx = ssx < 0.0f, upy = ssy < 0.0f;
    const int hx = (TXc < P.Nx && (P.perx || (upx ? X0 + TXc < P.Nx : X0 > 0))) ? 1 : 0;
    const int hy = (TYc < P.Ny && (P.pery || (upy ? Y0 + TYc < P.Ny : Y0 > 0))) ? 1 : 0;
    const int LX = TXc + hx, LY = TYc + hy, NL = LX * LY, NS = TXc * TYc;
    const int gx0 = X0 - (upx ? 0 : hx), gy0 = Y0 - (upy ? 0 : hy);
    for (int t = tid; t < NL; t += kCollThreads) {
        const int lx = t / LY, ly = t - lx * LY;
        int gx = gx0 + lx, gy = gy0 + ly;
        if (gx < 0) gx += P.Nx;
        if (gx >= P.Nx) gx -= P.Nx;
        if (gy < 0) gy += P.Ny;
        if (gy >= P.Ny) gy -= P.Ny;
        const int gc = gy + P.Ny * gx;
        M.gcell[t] = gc;
        M.gxy[t] = make_short2((short)gx, (short)gy);
        M.cstart[t] = min(A.b.cnt[gc], K);
    }
    for (int t = tid; t < NS; t += kCollThreads) M.scnt[t] = 0;
    __syncthreads();
    block_scan(M.cstart, M.cstart, NL, M.wsum);
    const int total = M.cstart[NL];
    if (total > A.pcap) {
        if (tid == 0) A.spill[atomicAdd(A.nSpill, 1)] = tile;
        return;
    }
    // each particle's home (local cell << 7 | slot), cell by cell
    for (int lc = tid; lc < NL; lc += kCollThreads) {
        const int a = M.cstart[lc], e = M.cstart[lc + 1];
        for (int f = a; f < e; ++f) M.home[f] = (uint16_t)((lc << 7) | (f - a));
    }
    __syncthreads();
    // stage every particle of the standard cells; count the tile's members per SRD cell
    // (four particles per thread and iteration, their loads issued together)
    constexpr int kU = 4;
    for (int fb = tid; fb < total; fb += kU * kCollThreads) {
        int lcs[kU], js[kU];
        float2 off[kU], vv[kU];
        int pp[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int f = fb + u * kCollThreads;
            const int h = f < total ? M.home[f] : 0;
            lcs[u] = h >> 7;
            js[u] = h & 127;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (fb + u * kCollThreads < total) {
                const size_t s = (size_t)M.gcell[lcs[u]] * K + js[u];
                off[u] = A.b.off[s];
                vv[u] = A.b.vel[s];
                pp[u] = A.b.pid[s];
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int f = fb + u * kCollThreads;
            if (f >= total) break;
            const short2 g = M.gxy[lcs[u]];
            const int sx = srd_axis(g.x, off[u].x, ssx, P.Nx, P.perx) - X0;
            const int sy = srd_axis(g.y, off[u].y, ssy, P.Ny, P.pery) - Y0;
            uint32_t code = 0xFFFFFFFFu;
            if (sx >= 0 && sx < TXc && sy >= 0 && sy < TYc) {
                const int k = sx * TYc + sy;
                code = ((uint32_t)k << 16) | (uint32_t)atomicAdd(M.scnt + k, 1);
            }
            M.q[f] = make_int2(fq_of(vv[u].x), fq_of(vv[u].y));
            M.pid[f] = pp[u];
            M.sr[f] = code;
        }
    }
    __syncthreads();
    block_scan(M.scnt, M.sstart, NS, M.wsum);
    for (int f = tid; f < total; f += kCollThreads) {
        const uint32_t code = M.sr[f];
        if (code != 0xFFFFFFFFu) M.list[M.sstart[code >> 16] + (code & 0xFFFFu)] = (uint16_t)f;
    }
    __syncthreads();
    // collide: tpc threads per SRD cell (aligned lane groups)
    const int tpc = kCollThreads / (kCollTX * A.TY);
    const int k = tid / tpc, sub = tid - k * tpc;
    const bool own = k < NS;
    const int N = own ? M.scnt[k] : 0;
    const int b0 = own ? M.sstart[k] : 0;
    long long Sx = 0, Sy = 0, Sqq = 0;
    for (int m = sub; m < N; m += tpc) {
        const int2 q = M.q[M.list[b0 + m]];
        Sx += q.x;
        Sy += q.y;
        Sqq += (long long)q.x * q.x + (long long)q.y * q.y;
    }
    for (int o = 1; o < tpc; o <<= 1) {
        Sx += __shfl_xor_sync(0xffffffffu, Sx, o);
        Sy += __shfl_xor_sync(0xffffffffu, Sy, o);
        Sqq += __shfl_xor_sync(0xffffffffu, Sqq, o);
    }
    const int w = own ? (Y0 + k % TYc) + P.Ny * (X0 + k / TYc) : 0;
    SrdRot R{};
    if (N > 0) R = srd_rotation(P, A.S->seed, w, N, Sx, Sy, Sqq);
    long long Tx = 0, Ty = 0;
    int minPid = 0x7fffffff;
    for (int m = sub; m < N; m += tpc) {
        const int f = M.list[b0 + m];
        const int2 q = M.q[f];
        long long nx, ny;
        srd_rotate(R, q.x, q.y, nx, ny);
        Tx += nx;
        Ty += ny;
        if (srd_eligible(nx, ny)) minPid = min(minPid, M.pid[f]);
        M.q[f] = make_int2((int)nx, (int)ny);
    }
    for (int o = 1; o < tpc; o <<= 1) {
        Tx += __shfl_xor_sync(0xffffffffu, Tx, o);
        Ty += __shfl_xor_sync(0xffffffffu, Ty, o);
        minPid = min(minPid, __shfl_xor_sync(0xffffffffu, minPid, o));
    }
    const long long rx = Sx - Tx, ry = Sy - Ty;
    for (int m = sub; m < N; m += tpc) {
        const int f = M.list[b0 + m];
        const int2 q = M.q[f];
        long long nx = q.x, ny = q.y;
        if (M.pid[f] == minPid) {
            nx += rx;
            ny += ry;
        }
        const int h = M.home[f];
        A.b.vel[(size_t)M.gcell[h >> 7] * K + (h & 127)] = make_float2(fv_of(nx), fv_of(ny));
    }
}

__global__ void __launch_bounds__(kCollThreads) k_fast_collide_tile(CollideArgs A) {
    extern __shared__ __align__(16) char smem[];
    fast_collide_tile_block((int)blockIdx.x, A, smem);
}

// The tiles the tile kernel left (more particles than its shared memory holds): one warp per
// SRD cell, its members found among the particles of the two-by-two standard cells under it
// and read twice from global memory. The same arithmetic as the tile kernel.
__device__ __forceinline__ void fast_collide_spill_block(int bx, int gx, const CollideArgs& A) {
    const DevParams& P = A.P;
    const int K = A.F.K;
    const int lane = threadIdx.x & 31;
    const int nsp = *A.nSpill;
    if (nsp == 0) return;
    const float ssx = (float)A.S->sx, ssy = (float)A.S->sy;
    const int ex = ssx < 0.0f ? 1 : 0, ey = ssy < 0.0f ? 1 : 0;
    const int cellsPerTile = kCollTX * A.TY;
    const long long items = (long long)nsp * cellsPerTile;
    const long long wstep = (long long)gx * (blockDim.x >> 5);
    for (long long it = (bx * (long long)blockDim.x + threadIdx.x) >> 5; it < items; it += wstep) {
        const int tile = A.spill[it / cellsPerTile];
        const int kk = (int)(it % cellsPerTile);
        const int X0 = (tile / A.tilesY) * kCollTX, Y0 = (tile % A.tilesY) * A.TY;
        const int TXc = min(kCollTX, P.Nx - X0), TYc = min(A.TY, P.Ny - Y0);
        if (kk >= TXc * TYc) continue;
        const int sx = X0 + kk / TYc, sy = Y0 + kk % TYc;
        // the standard cells that can hold members: sx - 1 + ex .. sx + ex (wrapped; missing ones skipped)
        int cells[4];
        int nc = 0;
        for (int a = 0; a < 2; ++a)
            for (int bb = 0; bb < 2; ++bb) {
                int gx = sx - 1 + ex + a, gy = sy - 1 + ey + bb;
                if (gx < 0 || gx >= P.Nx) {
                    if (!P.perx) continue;
                    gx = gx < 0 ? gx + P.Nx : gx - P.Nx;
                }
                if (gy < 0 || gy >= P.Ny) {
                    if (!P.pery) continue;
                    gy = gy < 0 ? gy + P.Ny : gy - P.Ny;
                }
                cells[nc++] = gy + P.Ny * gx;
            }
        long long Sx = 0, Sy = 0, Sqq = 0;
        int N = 0;
        // pass 1: sums
        for (int ci = 0; ci < nc; ++ci) {
            const int gc = cells[ci];
            const int gx = gc / P.Ny, gy = gc - gx * P.Ny;
            const int n = min(A.b.cnt[gc], K);
            for (int j = lane; j < n; j += 32) {
                const size_t s = (size_t)gc * K + j;
                const float2 off = A.b.off[s];
                if (srd_axis(gx, off.x, ssx, P.Nx, P.perx) != sx || srd_axis(gy, off.y, ssy, P.Ny, P.pery) != sy) continue;
                const float2 v = A.b.vel[s];
                const long long qx = fq_of(v.x), qy = fq_of(v.y);
                Sx += qx;
                Sy += qy;
                Sqq += qx * qx + qy * qy;
                ++N;
            }
        }
        Sx = warp_sum_ll(Sx);
        Sy = warp_sum_ll(Sy);
        Sqq = warp_sum_ll(Sqq);
        N = warp_sum_i(N);
        if (N == 0) continue;
        const SrdRot R = srd_rotation(P, A.S->seed, sy + P.Ny * sx, N, Sx, Sy, Sqq);
        // pass 2: the rounding residual and its taker
        long long Tx = 0, Ty = 0;
        int minPid = 0x7fffffff;
        for (int ci = 0; ci < nc; ++ci) {
            const int gc = cells[ci];
            const int gx = gc / P.Ny, gy = gc - gx * P.Ny;
            const int n = min(A.b.cnt[gc], K);
            for (int j = lane; j < n; j += 32) {
                const size_t s = (size_t)gc * K + j;
                const float2 off = A.b.off[s];
                if (srd_axis(gx, off.x, ssx, P.Nx, P.perx) != sx || srd_axis(gy, off.y, ssy, P.Ny, P.pery) != sy) continue;
                const float2 v = A.b.vel[s];
                long long nx, ny;
                srd_rotate(R, fq_of(v.x), fq_of(v.y), nx, ny);
                Tx += nx;
                Ty += ny;
                if (srd_eligible(nx, ny)) minPid = min(minPid, A.b.pid[s]);
            }
        }
        Tx = warp_sum_ll(Tx);
        Ty = warp_sum_ll(Ty);
        minPid = (int)__reduce_min_sync(0xffffffffu, (unsigned)minPid);
        const long long rx = Sx - Tx, ry = Sy - Ty;
        // pass 3: the new velocities (every lane reads its members before the warp writes)
        for (int ci = 0; ci < nc; ++ci) {
            const int gc = cells[ci];
            const int gx = gc / P.Ny, gy = gc - gx * P.Ny;
            const int n = min(A.b.cnt[gc], K);
            for (int j0 = 0; j0 < n; j0 += 32) {
                const int j = j0 + lane;
                const size_t s = (size_t)gc * K + j;
                bool mem = false;
                float2 nv = make_float2(0.f, 0.f);
                if (j < n) {
                    const float2 off = A.b.off[s];
                    mem = srd_axis(gx, off.x, ssx, P.Nx, P.perx) == sx && srd_axis(gy, off.y, ssy, P.Ny, P.pery) == sy;
                    if (mem) {
                        const float2 v = A.b.vel[s];
                        long long nx, ny;
                        srd_rotate(R, fq_of(v.x), fq_of(v.y), nx, ny);
                        if (A.b.pid[s] == minPid) {
                            nx += rx;
                            ny += ry;
                        }
                        nv = make_float2(fv_of(nx), fv_of(ny));
                    }
                }
                __syncwarp();
                if (mem) A.b.vel[s] = nv;
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_fast_collide_spill(CollideArgs A) {
    fast_collide_spill_block((int)blockIdx.x, (int)gridDim.x, A);
}

// ------------------------------------------------------------------ zone redistribution
// One warp per zone (a cell rectangle of at most kFastMaxZoneCells cells, kFastZoneWarps zones
// per block). The zone reads its own cells' bins and the pass-input counts of a two-cell halo
// (snapshot semantics: src/zone_pass_openmp.cpp:34-172), and writes its cells' bins to the
// output buffers. Particles move only between cells of the zone.
struct FastZoneArgs {
    DevParams P;
    FastParams F;
    const int4* rects;         // (x0, x1, y0, y1) per zone
    int nZones;
    int pass;                  // 0 base, 1 shifted (salts the draws)
    const FastStep* S;
    FastBins b;                // the bins, updated in place (cnt unused: cntIn / cntOut)
    const int* cntIn;          // pass-input counts (the snapshot every zone reads)
    int* cntOut;               // pass-output counts
    const longlong2* sumsIn;   // nullable: per cell the input's momentum (cells left unchanged pass it on)
    longlong2* sumsOut;        // per cell the output's momentum (the next pass's input; red state: closure)
    longlong4* ref;            // nullable: per cell the input's (sum qx, sum qy, sum |q|^2, N): the
                               // closure's reference fields (stateRef is the collided state,
                               // src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:241-251)
    int* moved;                // (dense, sparse) over all zones
    int* recOverflow;          // zones that ran out of records (their remaining moves are skipped)
    DevStatus* st;
    int maxCells, winCap, nsmCap, recCap;
    // what the decision kernel hands the apply kernel: per cell a summary (bit 63 changed,
    // bit 48 corrected, bits 32-47 arrivals, bits 0-31 its first arrival record) and the removal
    // masks of changed cells; per zone (recCap records from z * recCap) the arrivals in cell
    // order: id, position in the cell, velocity (grid units)
    unsigned long long* meta;
    uint4* cellRm;
    int* recPidG;
    float2* recOffG;
    int2* recQG;
    // nullable: the zone each slot of the decision kernel runs (slot = block * zones per block +
    // warp), heaviest zones first, so that the zones of one block finish their phases together
    const int* order;
};

// The 24 range-2 neighbour offsets grouped by the angular bin of atan2(dy, dx)
// (src/zone_pass.cpp:447-457: bin = floor((angle + pi) / (pi / 4)) mod 8): three per bin, bin b
// in lanes 3b .. 3b + 2. For |d| <= 2 on axes of at least 5 cells the minimal-image step is
// the offset itself.
__constant__ signed char kFastNb[24][2] = {
    {-2, -1}, {-2, 0}, {-1, 0},  {-2, -2}, {-1, -2}, {-1, -1}, {0, -2}, {1, -2}, {0, -1}, {2, -2}, {1, -1}, {2, -1},
    {1, 0},   {2, 0},  {2, 1},   {1, 1},   {1, 2},   {2, 2},   {0, 1},  {-1, 2}, {0, 2},  {-2, 1}, {-1, 1}, {-2, 2}};

// zone working set layout (bytes), carved per warp
struct FastZoneMem {
    short* win;        // winCap: counts of the window (zone + 2-cell halo); -1 outside the domain
    uint16_t* wi;      // cell: its window index
    uint8_t* cx;       // cell: local x
    uint8_t* cy;       // cell: local y
    uint8_t* n0;       // cell: particles at the pass start
    uint8_t* flg;      // cell: flags
    uint8_t* nrecv;    // cell: records currently in the cell
    uint32_t* rm;      // cell x 4: originals removed
    int* recPid;       // recCap
    uint16_t* recStart;// cell + 1: start of each cell's arrivals in the exported records
    int* rfill;        // cell: records filed so far
    uint16_t* recSrc;  // recCap: (origin cell << 7) | slot
    uint8_t* recCur;   // recCap: current cell
    uint32_t* recDraw; // recCap: the draw of the position in the current cell (salt << 8 | k)
    float* nsm;        // nsmCap: smoothed occupancy of the zone and a one-cell ring
    uint32_t* keys;    // 128: order keys of the dense / low cells; the output's hole slots
    uint8_t* ord;      // 128: those cells in key order
    int* tgt;          // 32: ordered targets or donors
    int* tgt2;         // 32: receivers of a dense cell's first phase

    template <class F>
    __host__ __device__ static void layout(int maxCells, int winCap, int nsmCap, int recCap, F&& take) {
        take((size_t)winCap * 2, 2);
        take((size_t)maxCells * 2, 2);
        for (int k = 0; k < 5; ++k) take((size_t)maxCells, 1);
        take((size_t)maxCells * 16, 4);
        take((size_t)recCap * 4, 4);
        take((size_t)(maxCells + 1) * 2, 2);
        take((size_t)maxCells * 4, 4);
        take((size_t)recCap * 2, 2);
        take((size_t)recCap, 1);
        take((size_t)recCap * 4, 4);
        take((size_t)nsmCap * 4, 4);
        take(128 * 4, 4);
        take(128, 1);
        take(32 * 4, 4);
        take(32 * 4, 4);
    }
    __host__ __device__ static size_t bytes(int maxCells, int winCap, int nsmCap, int recCap) {
        size_t b = 0;
        layout(maxCells, winCap, nsmCap, recCap, [&](size_t n, size_t a) { b = (b + a - 1) / a * a + n; });
        return (b + 15) / 16 * 16;
    }
    __device__ void carve(char* base, int maxCells, int winCap, int nsmCap, int recCap) {
        size_t b = 0;
        char* p[19];
        int i = 0;
        layout(maxCells, winCap, nsmCap, recCap, [&](size_t n, size_t a) {
            b = (b + a - 1) / a * a;
            p[i++] = base + b;
            b += n;
        });
        win = (short*)p[0];
        wi = (uint16_t*)p[1];
        cx = (uint8_t*)p[2];
        cy = (uint8_t*)p[3];
        n0 = (uint8_t*)p[4];
        flg = (uint8_t*)p[5];
        nrecv = (uint8_t*)p[6];
        rm = (uint32_t*)p[7];
        recPid = (int*)p[8];
        recStart = (uint16_t*)p[9];
        rfill = (int*)p[10];
        recSrc = (uint16_t*)p[11];
        recCur = (uint8_t*)p[12];
        recDraw = (uint32_t*)p[13];
        nsm = (float*)p[14];
        keys = (uint32_t*)p[15];
        ord = (uint8_t*)p[16];
        tgt = (int*)p[17];
        tgt2 = (int*)p[18];
        // all of them in shared memory (lets the compiler use shared-space accesses)
        __builtin_assume(__isShared(win) && __isShared(wi) && __isShared(cx) && __isShared(cy) && __isShared(n0) &&
                         __isShared(flg) && __isShared(nrecv) && __isShared(rm) && __isShared(recPid) &&
                         __isShared(recStart) && __isShared(rfill) && __isShared(recSrc) && __isShared(recCur) &&
                         __isShared(recDraw) && __isShared(nsm) && __isShared(keys) && __isShared(ord) &&
                         __isShared(tgt) && __isShared(tgt2));
    }
};

constexpr uint8_t kZBulkD = 1, kZBulkS = 2, kZRecv = 4, kZBB = 8, kZSkip = 16;

// A source cell's candidates, one per original slot j in lane j % 32: register j / 32 holds
// slot lane + 32 (j / 32). Four named registers (an indexed array would live in local memory).
struct Cands {
    unsigned long long r0, r1, r2, r3;
    __device__ __forceinline__ unsigned long long lowest() const {
        const unsigned long long x = r0 < r1 ? r0 : r1, y = r2 < r3 ? r2 : r3;
        return x < y ? x : y;
    }
    __device__ __forceinline__ void set(int r, unsigned long long v) {
        r0 = r == 0 ? v : r0;
        r1 = r == 1 ? v : r1;
        r2 = r == 2 ? v : r2;
        r3 = r == 3 ? v : r3;
    }
    // removes original slot j (its lane clears it)
    __device__ __forceinline__ void take(int j, int lane) {
        if ((j & 31) == lane) set(j >> 5, ~0ULL);
    }
};

// A moved particle's position in its new cell: two 24-bit uniforms of one draw of the zone's
// stream, keyed by the operation's salt and the move's index k in it (draw = salt << 8 | k)
__device__ __forceinline__ float2 zone_draw_pos(uint64_t zseed, uint32_t draw) {
    const uint64_t hp = fmix64(zseed ^ ((uint64_t)(draw >> 8) << 20) ^ (0x504F53ULL + (uint64_t)(draw & 0xFFu)));
    return make_float2(fminf((float)(hp >> 40) * 0x1.0p-24f, kFastOffMax),
                       fminf((float)((hp >> 8) & 0xFFFFFFu) * 0x1.0p-24f, kFastOffMax));
}

struct FastZone {
    const FastZoneArgs* A;
    FastZoneMem M;
    int lane, z;
    int x0, x1, y0, y1, TX, TY, nl, WY;
    uint64_t zseed;
    uint32_t op;        // operation counter (salts the draws)
    int nrec;
    bool failed;        // out of records: remaining moves skipped
    int movedDense, movedSparse;

    __device__ __forceinline__ int cnt(int l) const { return M.win[M.wi[l]]; }
    __device__ __forceinline__ void add_cnt(int l, int d) { M.win[M.wi[l]] += (short)d; }
    __device__ __forceinline__ int gcell(int l) const { return (y0 + M.cy[l]) + A->P.Ny * (x0 + M.cx[l]); }
    __device__ __forceinline__ double low_map(bool bulk) const { return bulk ? A->P.lowThrBulk : A->F.lowMapEmpty; }
    __device__ __forceinline__ double high_map(bool bulk) const { return bulk ? A->P.highThr : A->F.highMapEmpty; }

    // the zone cell at local (lx + dx, ly + dy), wrapping periodic axes; -1 outside the domain
    // or outside the zone
    __device__ __forceinline__ int neighbour(int l, int dx, int dy) const {
        const DevParams& P = A->P;
        int gx = x0 + M.cx[l] + dx, gy = y0 + M.cy[l] + dy;
        if (P.perx) gx = gx < 0 ? gx + P.Nx : (gx >= P.Nx ? gx - P.Nx : gx);
        else if (gx < 0 || gx >= P.Nx) return -1;
        if (P.pery) gy = gy < 0 ? gy + P.Ny : (gy >= P.Ny ? gy - P.Ny : gy);
        else if (gy < 0 || gy >= P.Ny) return -1;
        if (gx < x0 || gx >= x1 || gy < y0 || gy >= y1) return -1;
        return (gx - x0) * TY + (gy - y0);
    }

    __device__ __forceinline__ uint64_t member_key(bool dense, uint32_t salt, uint32_t pid, int rec) const {
        if (dense) return rec < 0 ? (uint64_t)pid : ((1ULL << 31) + (uint64_t)rec);
        return ((fmix64(zseed ^ ((uint64_t)salt << 32) ^ (uint64_t)pid) >> 41) << 31) | (uint64_t)(pid & 0x7fffffffu);
    }

    // The candidates of source cell l, one key per original not yet removed: slot j in lane
    // j % 32, register j / 32. A candidate is (key << 10) | (record flag << 9) | index: keys of at
    // most 54 bits whose low 31 bits are the particle id, original slots below 128 and records
    // below 512.
    __device__ __forceinline__ void load_candidates(int l, bool dense, uint32_t salt, Cands& cand) const {
        const FastBins& B = A->b;
        const size_t ib = (size_t)gcell(l) * A->F.K;
        const int n0 = M.n0[l];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int j = lane + 32 * r;
            unsigned long long v = ~0ULL;
            if (j < n0 && !(M.rm[4 * l + r] & (1u << lane)))
                v = (member_key(dense, salt, (uint32_t)B.pid[ib + j], -1) << 10) | (unsigned long long)j;
            cand.set(r, v);
        }
    }

    // Removes nt members of cell l and files them into cell t at fresh uniform positions.
    // dense: the members in the reference's list order (the cell's particles in ascending id,
    // then the arrivals in order: src/zone_pass.cpp:541-583 takes the first ids), from the
    // candidates the caller loaded once for the cell; otherwise members chosen uniformly at
    // random (the sparse phase shuffles the donor's list) from candidates keyed afresh.
    __device__ __forceinline__ void move_members(int l, int t, int nt, bool dense, Cands& cand) {
        const uint32_t salt = ++op;
        if (!dense) load_candidates(l, false, salt, cand);
        for (int k = 0; k < nt; ++k) {
            if (failed) return;
            unsigned long long best = cand.lowest();
            if (M.nrecv[l] > 0) {
                for (int r = lane; r < nrec; r += 32) {
                    if (M.recCur[r] != l) continue;
                    const unsigned long long v =
                        (member_key(dense, salt, (uint32_t)M.recPid[r], r) << 10) | 512ULL | (unsigned long long)r;
                    best = v < best ? v : best;
                }
            }
            best = warp_min_u64_r(best);
            if (best == ~0ULL) return;  // no member left (cannot happen while counts agree)
            // the new position: the draw (salt, k), evaluated when the record is exported
            const uint32_t draw = (salt << 8) | (uint32_t)k;
            if (!(best & 512ULL)) {  // an original of cell l
                const int j = (int)(best & 511ULL);
                if (nrec >= A->recCap) {
                    failed = true;
                    return;
                }
                cand.take(j, lane);
                if (lane == 0) {
                    M.rm[4 * l + (j >> 5)] |= 1u << (j & 31);
                    M.recPid[nrec] = (int)((best >> 10) & 0x7fffffffULL);
                    M.recSrc[nrec] = (uint16_t)((l << 7) | j);
                    M.recCur[nrec] = (uint8_t)t;
                    M.recDraw[nrec] = draw;
                    M.nrecv[t] += 1;
                }
                ++nrec;
            } else if (lane == 0) {  // an arrival in cell l moves on
                const int r = (int)(best & 511ULL);
                M.recCur[r] = (uint8_t)t;
                M.recDraw[r] = draw;
                M.nrecv[l] -= 1;
                M.nrecv[t] += 1;
            }
            __syncwarp();
        }
    }

    // spread_particles_from_dense_source_round_robin (src/zone_pass.cpp:527-589) over the
    // targets ranked as rank_dense_targets_unified does (:436-490); map: 0 low, 1 high.
    // Returns the particles moved; the receivers go to rcv[*nr ...].
    __device__ __forceinline__ int spread(int l, int needOut, int mapKind, int* rcv, int* nr, Cands& cand) {
        // lane k < 24: the k-th neighbour of the bin-grouped offset table
        const int k = lane;
        int t = -1, ddx = 0, ddy = 0;
        double map = 0.0;
        bool adm = false;
        if (k < 24) {
            ddx = kFastNb[k][0];
            ddy = kFastNb[k][1];
            t = neighbour(l, ddx, ddy);
            if (t >= 0) {
                const bool bulk = M.flg[t] & kZBulkD;
                map = mapKind ? high_map(bulk) : low_map(bulk);
                adm = (double)cnt(t) < map;
            }
        }
        const unsigned admMask = __ballot_sync(0xffffffffu, adm);
        const int T = __popc(admMask);
        if (T == 0) return 0;
        const uint32_t salt = ++op;
        const int startBin = (int)(fmix64(zseed ^ ((uint64_t)salt << 12) ^ 0x42494EULL) >> 61);
        // sort key (-deficit, cnt, chebyshev, distance^2, random); inward weight is 0 here
        unsigned long long key = ~0ULL;
        if (adm) {
            const double deficit = fmax(0.0, map - (double)cnt(t));
            const unsigned long long dq = (unsigned long long)min(llrint(deficit * 4096.0), (long long)0xFFFFF);
            const int cheb = max(abs(ddx), abs(ddy)), d2 = ddx * ddx + ddy * ddy;
            key = ((0xFFFFFULL - dq) << 44) | ((unsigned long long)min(cnt(t), 255) << 36) |
                  ((unsigned long long)cheb << 34) | ((unsigned long long)d2 << 30) |
                  (fmix64(zseed ^ ((uint64_t)salt << 8) ^ (uint64_t)k) & 0x3FFFFFFFULL);
        }
        // rank inside the bin: the two other lanes of the bin
        const int b = k / 3, base = 3 * b;
        const unsigned long long ka = __shfl_sync(0xffffffffu, key, base + ((k - base + 1) % 3));
        const unsigned long long kb = __shfl_sync(0xffffffffu, key, base + ((k - base + 2) % 3));
        const int rank = (ka < key) + (kb < key);
        const int pos = rank * 8 + ((b - startBin + 8) & 7);
        const unsigned posMask = __reduce_or_sync(0xffffffffu, adm ? (1u << pos) : 0u);
        const int ord = __popc(posMask & ((1u << pos) - 1u));
        if (adm) M.tgt[ord] = t;
        __syncwarp();
        // per ordered target (lane o < T): its current integer deficit
        int def = 0;
        double mapO = 0.0;
        int tO = -1;
        if (lane < T) {
            tO = M.tgt[lane];
            const bool bulk = M.flg[tO] & kZBulkD;
            mapO = mapKind ? high_map(bulk) : low_map(bulk);
            def = max(0, (int)floor(mapO - (double)cnt(tO)));
        }
        int avail = cnt(l);
        // With at most as many particles to move as targets with a deficit, the round-robin
        // quota stays 1: the first needOut of those targets (in order) take one particle each,
        // the i-th the i-th member in list order, drawn as the general loop below draws them
        // (its i-th call's salt, first draw). Done in one step when the source holds no records.
        const unsigned defMask = __ballot_sync(0xffffffffu, lane < T && def > 0);
        if (needOut > 0 && needOut <= __popc(defMask) && needOut <= avail && M.nrecv[l] == 0 && !failed &&
            nrec + needOut <= A->recCap) {
            unsigned long long mine = ~0ULL;
            for (int i = 0; i < needOut; ++i) {
                const unsigned long long best = warp_min_u64_r(cand.lowest());
                const int j = (int)(best & 511ULL);
                cand.take(j, lane);
                if (lane == i) mine = best;
            }
            const int drank = __popc(defMask & lanemask_lt());
            __syncwarp();
            if (lane < T && def > 0 && drank < needOut) M.tgt[drank] = tO;
            __syncwarp();
            if (lane < needOut) {
                const int t = M.tgt[lane];
                const int j = (int)(mine & 511ULL);
                const uint32_t salt = op + 1 + (uint32_t)lane;
                const int rec = nrec + lane;
                M.recPid[rec] = (int)((mine >> 10) & 0x7fffffffULL);
                M.recSrc[rec] = (uint16_t)((l << 7) | j);
                M.recCur[rec] = (uint8_t)t;
                M.recDraw[rec] = salt << 8;
                M.nrecv[t] += 1;
                add_cnt(t, 1);
                atomicOr(&M.rm[4 * l + (j >> 5)], 1u << (j & 31));
                rcv[*nr + lane] = t;
            }
            if (lane == 0) add_cnt(l, -needOut);
            op += (uint32_t)needOut;
            nrec += needOut;
            *nr += needOut;
            __syncwarp();
            return needOut;
        }
        int moved = 0;
        unsigned got = 0;
        while (needOut > 0 && avail > 0 && !failed) {
            bool progressed = false;
            for (int kk = 0; kk < T; ++kk) {
                const int d = __shfl_sync(0xffffffffu, def, kk);
                if (d <= 0) continue;
                const int rem = __popc(__ballot_sync(0xffffffffu, lane >= kk && lane < T && def > 0));
                const int quota = max(1, (needOut + max(1, rem) - 1) / max(1, rem));
                const int nt = max(1, min(min(quota, d), min(needOut, avail)));
                const int tt = __shfl_sync(0xffffffffu, tO, kk);
                move_members(l, tt, nt, true, cand);
                if (failed) break;
                if (lane == 0) {
                    add_cnt(l, -nt);
                    add_cnt(tt, nt);
                }
                __syncwarp();
                if (lane == kk) def = max(0, (int)floor(mapO - (double)cnt(tO)));
                got |= 1u << kk;
                avail -= nt;
                needOut -= nt;
                moved += nt;
                progressed = true;
                if (needOut <= 0 || avail <= 0) break;
            }
            if (!progressed) break;
        }
        // receivers, in target order
        if ((got >> lane) & 1u) rcv[*nr + __popc(got & ((1u << lane) - 1u))] = tO;
        *nr += __popc(got);
        __syncwarp();
        return moved;
    }

    // the transfer masks (src/zone_pass.cpp:492-525) for a source and its nr receivers (lane
    // k < nr holds the k-th in myRcv), bulk flag bit bf
    __device__ void masks(int src, int myRcv, int nr, uint8_t bf) {
        bool allBulk = (M.flg[src] & bf) != 0;
        const bool mine = lane < nr;
        const int rc = mine ? myRcv : src;
        allBulk = allBulk && __all_sync(0xffffffffu, !mine || (M.flg[rc] & bf));
        __syncwarp();
        if (lane <= nr) {
            const int cc = lane < nr ? rc : src;
            uint8_t f = M.flg[cc];
            if (lane < nr) f |= kZRecv;
            f = allBulk ? (uint8_t)(f | kZBB) : (uint8_t)((f | kZSkip) & ~kZBB);
            M.flg[cc] = f;
        }
        __syncwarp();
    }

    // redistribute_dense_cell_at_range_zone_local (src/zone_pass.cpp:591-634) and the mask
    // update of the dense loop (:745-750)
    __device__ void dense_cell(int l) {
        const bool bulk = M.flg[l] & kZBulkD;
        const double hi = high_map(bulk);
        const int nc = cnt(l);
        if (nc <= 0 || (double)nc <= hi) return;
        const int needOut = max(0, (int)ceil((double)nc - hi));
        int nr = 0;
        int moved = 0;
        Cands cand;
        load_candidates(l, true, 0, cand);
        // the low map first, then the high map for what is left (one call site: code size)
#pragma unroll 1
        for (int phase = 0; phase < 2; ++phase) {
            const int out = phase == 0 ? needOut : max(0, (int)ceil((double)cnt(l) - hi));
            if (out <= 0 || failed) continue;
            moved += spread(l, out, phase, M.tgt2, &nr, cand);
        }
        // the receivers of the two phases may repeat a cell; flags are idempotent
        const int nrc = min(nr, 31);
        masks(l, lane < nrc ? M.tgt2[lane] : l, nrc, kZBulkD);
        movedDense += moved;
    }

    // smoothed occupancy (src/zone_pass.cpp:296-319, non-periodic) of the zone and a one-cell
    // ring, from the window counts
    __device__ void compute_nsm() {
        const DevParams& P = A->P;
        const int RY = TY + 2, total = (TX + 2) * RY;
        for (int i = lane; i < total; i += 32) {
            const int rx = i / RY - 1, ry = i % RY - 1;  // local coordinates, -1 .. TX
            int cxx = x0 + rx, cyy = y0 + ry;
            if (P.perx) cxx = cxx < 0 ? cxx + P.Nx : (cxx >= P.Nx ? cxx - P.Nx : cxx);
            if (P.pery) cyy = cyy < 0 ? cyy + P.Ny : (cyy >= P.Ny ? cyy - P.Ny : cyy);
            float v = 0.0f;
            if (cxx >= 0 && cxx < P.Nx && cyy >= 0 && cyy < P.Ny) {
                float acc = 0.0f, ws = 0.0f;
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (cxx + dx < 0 || cxx + dx >= P.Nx || cyy + dy < 0 || cyy + dy >= P.Ny) continue;
                        const float w = (float)((2 - abs(dx)) * (2 - abs(dy))) * 0.0625f;
                        acc += w * (float)M.win[(rx + dx + 2) * WY + (ry + dy + 2)];
                        ws += w;
                    }
                v = acc / ws;
            }
            M.nsm[i] = v;
        }
        __syncwarp();
    }
    __device__ __forceinline__ float nsm_at(int rx, int ry) const { return M.nsm[(rx + 1) * (TY + 2) + (ry + 1)]; }

    // the sparse phase for low cell l (src/zone_pass.cpp:803-854)
    __device__ void sparse_cell(int l) {
        const DevParams& P = A->P;
        const int nc = cnt(l);
        if (nc <= 0) return;
        int need = max(0, P.lowThrBulkInt - nc);
        if (need <= 0) return;
        const int lx = M.cx[l], ly = M.cy[l];
        // inward direction from the local gradient of the smoothed occupancy (:375-411)
        const int gx = x0 + lx, gy = y0 + ly;
        float dirx, diry;
        if (P.perx) dirx = 0.5f * (nsm_at(lx + 1, ly) - nsm_at(lx - 1, ly));
        else if (gx == 0) dirx = nsm_at(lx + 1, ly) - nsm_at(lx, ly);
        else if (gx == P.Nx - 1) dirx = nsm_at(lx, ly) - nsm_at(lx - 1, ly);
        else dirx = 0.5f * (nsm_at(lx + 1, ly) - nsm_at(lx - 1, ly));
        if (P.pery) diry = 0.5f * (nsm_at(lx, ly + 1) - nsm_at(lx, ly - 1));
        else if (gy == 0) diry = nsm_at(lx, ly + 1) - nsm_at(lx, ly);
        else if (gy == P.Ny - 1) diry = nsm_at(lx, ly) - nsm_at(lx, ly - 1);
        else diry = 0.5f * (nsm_at(lx, ly + 1) - nsm_at(lx, ly - 1));
        const float ndir = hypotf(dirx, diry);
        // donors: in-zone 8-neighbours above ceil(lowThrBulk), ranked by
        // 100 align + Nsm (+ a random tie-break) descending (rank_admissible_neighbors_inward, :636-667)
        const int k = lane;
        int d = -1, ddx = 0, ddy = 0;
        bool don = false;
        if (k < 8) {
            const int idx = k < 4 ? k : k + 1;
            ddx = idx % 3 - 1;
            ddy = idx / 3 - 1;
            d = neighbour(l, ddx, ddy);
            don = d >= 0 && cnt(d) > P.lowThrBulkInt;
        }
        const unsigned donMask = __ballot_sync(0xffffffffu, don);
        if (!donMask) return;
        const uint32_t salt = ++op;
        float score = -1e30f;
        uint32_t tie = 0;
        if (don) {
            const float nstep = (ddx != 0 && ddy != 0) ? 1.41421356f : 1.0f;
            float align = 0.0f;
            if (ndir >= 1e-14f) align = ((float)ddx * dirx + (float)ddy * diry) / (ndir * nstep);
            score = 100.0f * align + nsm_at(lx + ddx, ly + ddy);
            tie = (uint32_t)fmix64(zseed ^ ((uint64_t)salt << 8) ^ (uint64_t)k);
        }
        int ord = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float sj = __shfl_sync(0xffffffffu, score, j);
            const uint32_t tj = __shfl_sync(0xffffffffu, tie, j);
            if (don && ((donMask >> j) & 1u) && (sj > score || (sj == score && tj < tie))) ++ord;
        }
        if (don) M.tgt[ord] = d;
        __syncwarp();
        const int nd = __popc(donMask);
        for (int q = 0; q < nd && need > 0 && !failed; ++q) {
            const int dn = M.tgt[q];
            const int avail = cnt(dn) - P.lowThrBulkInt;
            if (avail <= 0) continue;
            const int nt = min(need, min(avail, cnt(dn)));
            if (nt <= 0) continue;
            Cands cand;
            move_members(dn, l, nt, false, cand);
            if (failed) break;
            if (lane == 0) {
                add_cnt(dn, -nt);
                add_cnt(l, nt);
            }
            __syncwarp();
            // update_transfer_correction_masks(d, {c}, bulkMaskLowBefore), recvMask[c]
            masks(dn, l, 1, kZBulkS);
            movedSparse += nt;
            need -= nt;
        }
    }

    // The cells with a key (keyOf(l) != ~0) in ascending key order into M.ord: compacted by
    // ballot, each placed by counting the smaller keys (keys are distinct: the cell index is
    // their low byte). Returns how many.
    template <class KeyOf>
    __device__ int order_cells(KeyOf&& keyOf) {
        int D = 0;
        for (int l0 = 0; l0 < nl; l0 += 32) {
            const int l = l0 + lane;
            const uint32_t key = l < nl ? keyOf(l) : 0xFFFFFFFFu;
            const bool on = key != 0xFFFFFFFFu;
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (on) M.keys[D + __popc(m & lanemask_lt())] = key;
            D += __popc(m);
        }
        __syncwarp();
        for (int i = lane; i < D; i += 32) {
            const uint32_t k = M.keys[i];
            int rank = 0;
            for (int j = 0; j < D; ++j) rank += M.keys[j] < k;
            M.ord[rank] = (uint8_t)(k & 0xFFu);
        }
        __syncwarp();
        return D;
    }
};

// The zone's decisions for the apply kernel: its arrival records in cell order (with the moved
// particles' velocities, read here, before any bin is rewritten) and per cell the summary and
// removal masks.
__device__ void fast_zone_export(FastZone& Z) {
    const FastZoneArgs& A = *Z.A;
    FastZoneMem& M = Z.M;
    const int lane = Z.lane, K = A.F.K, nl = Z.nl;
    for (int l = lane; l < nl; l += 32) M.rfill[l] = 0;
    // records grouped by cell (exclusive prefix of the arrivals per cell)
    int base = 0;
    for (int l0 = 0; l0 < nl; l0 += 32) {
        const int l = l0 + lane;
        const int v = l < nl ? M.nrecv[l] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (l < nl) M.recStart[l] = (uint16_t)(base + incl - v);
        base += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();
    const size_t zb = (size_t)Z.z * A.recCap;
    for (int r = lane; r < Z.nrec; r += 32) {
        const int src = M.recSrc[r];
        const int l = M.recCur[r];
        const float2 v = A.b.vel[(size_t)Z.gcell(src >> 7) * K + (src & 127)];
        const size_t g = zb + M.recStart[l] + atomicAdd(M.rfill + l, 1);
        A.recPidG[g] = M.recPid[r];
        A.recOffG[g] = zone_draw_pos(Z.zseed, M.recDraw[r]);
        A.recQG[g] = make_int2(fq_of(v.x), fq_of(v.y));
    }
    for (int l = lane; l < nl; l += 32) {
        const int c = Z.gcell(l);
        const uint4 rm = make_uint4(M.rm[4 * l], M.rm[4 * l + 1], M.rm[4 * l + 2], M.rm[4 * l + 3]);
        const int nr = M.nrecv[l];
        const bool changed = (rm.x | rm.y | rm.z | rm.w) != 0 || nr > 0;
        unsigned long long meta = 0;
        if (changed) {
            const uint8_t f = M.flg[l];
            const bool corr = A.P.momCorr != 0 && !(f & kZSkip) && !((f & kZRecv) && !(f & kZBB));
            meta = (1ULL << 63) | ((unsigned long long)corr << 48) | ((unsigned long long)nr << 32) |
                   (unsigned long long)(zb + M.recStart[l]);
            A.cellRm[c] = rm;
        }
        A.meta[c] = meta;
    }
}

// floor(a / b) for b > 0, in 32 bits when a fits
__device__ __forceinline__ long long floor_div_small(long long a, int b) {
    if (a >= -2147483647LL - 1 && a <= 2147483647LL) {
        const int ai = (int)a;
        int q = ai / b;
        if ((ai % b != 0) && (ai < 0)) --q;
        return q;
    }
    return floor_div_ll(a, b);
}

// Output of a zone pass (src/zone_pass.cpp:870-909), in place, one thread per cell: only the
// cells whose members changed are rewritten. A changed cell's final members are its kept
// particles and its arrivals; the kept particles above the new count and then the arrivals fill
// the holes the departed left (in slot order), then the slots from the old count on. The
// momentum correction restores each corrected cell's pass-input momentum exactly: an integer
// share per member, the remainder to the member of smallest id. A cell is read four slots at a
// time (32-byte loads: bins start on 128-byte boundaries, K being a multiple of 16) before it is
// written; no thread reads another cell's slots (the arrivals come from the exported records).
__device__ __forceinline__ void fast_zone_apply_block(int blk, const FastZoneArgs& A) {
    const int c = (int)(blk * (size_t)blockDim.x + threadIdx.x);
    if (c >= A.P.Nc) return;
    const int K = A.F.K;
    const FastBins& B = A.b;
    const int n0 = min(A.cntIn[c], K);
    const unsigned long long meta = A.meta[c];
    const bool changed = (meta >> 63) != 0;
    if (!changed && A.sumsIn) {  // nothing to read: the input passes through
        A.cntOut[c] = n0;
        A.sumsOut[c] = A.sumsIn[c];
        return;
    }
    const uint4 rmv = changed ? A.cellRm[c] : make_uint4(0u, 0u, 0u, 0u);
    const uint32_t rm0 = rmv.x, rm1 = rmv.y, rm2 = rmv.z, rm3 = rmv.w;
    const int nr = (int)((meta >> 32) & 0xFFFFu);
    const size_t rs = (size_t)(meta & 0xFFFFFFFFULL);
    // the removal bits of slots j0 .. j0 + 3 (j0 a multiple of 4)
    auto rbits = [&](int j0) -> uint32_t {
        const uint32_t w = j0 < 32 ? rm0 : (j0 < 64 ? rm1 : (j0 < 96 ? rm2 : rm3));
        return (w >> (j0 & 31)) & 0xFu;
    };
    const size_t ib = (size_t)c * K;
    const float4* v4 = reinterpret_cast<const float4*>(B.vel + ib);
    const int4* p4 = reinterpret_cast<const int4*>(B.pid + ib);
    long long bx = 0, by = 0, qq = 0, ax = 0, ay = 0;
    int mp = 0x7fffffff;
#pragma unroll 2
    for (int j0 = 0; j0 < n0; j0 += 4) {
        const float4 va = v4[j0 >> 1], vb = v4[(j0 >> 1) + 1];
        const int4 pp = changed ? p4[j0 >> 2] : make_int4(0, 0, 0, 0);
        const float vx[4] = {va.x, va.z, vb.x, vb.z}, vy[4] = {va.y, va.w, vb.y, vb.w};
        const int pv[4] = {pp.x, pp.y, pp.z, pp.w};
        const uint32_t rb = rbits(j0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (j0 + u >= n0) break;
            const long long qx = fq_of(vx[u]), qy = fq_of(vy[u]);
            bx += qx;
            by += qy;
            qq += qx * qx + qy * qy;
            if (changed && !((rb >> u) & 1u)) {
                ax += qx;
                ay += qy;
                mp = min(mp, pv[u]);
            }
        }
    }
    if (A.ref) A.ref[c] = make_longlong4(bx, by, qq, n0);
    if (!changed) {
        A.cntOut[c] = n0;
        A.sumsOut[c] = make_longlong2(bx, by);
        return;
    }
    for (int k = 0; k < nr; ++k) {
        const int2 q = A.recQG[rs + k];
        ax += q.x;
        ay += q.y;
        mp = min(mp, A.recPidG[rs + k]);
    }
    const int kept = n0 - (__popc(rm0) + __popc(rm1) + __popc(rm2) + __popc(rm3));
    const int nAll = kept + nr;
    long long shx = 0, shy = 0, remx = 0, remy = 0;
    if (((meta >> 48) & 1ULL) && nAll > 0) {
        const long long dx = bx - ax, dy = by - ay;
        shx = floor_div_small(dx, nAll);
        shy = floor_div_small(dy, nAll);
        remx = dx - shx * nAll;
        remy = dy - shy * nAll;
    }
    A.sumsOut[c] = make_longlong2(ax + shx * nAll + remx, ay + shy * nAll + remy);
    if (nAll > K) raise_error(A.st, kErrBinCapacity, c);
    A.cntOut[c] = min(nAll, K);
    const int below = min(n0, nAll);
    // kept particles that stay: velocity corrected in place (whole 32-byte groups are
    // rewritten; the other slots in them keep their values or are filled below)
    if (shx | shy | remx | remy) {
        float4* w4 = reinterpret_cast<float4*>(B.vel + ib);
        const bool rem = (remx | remy) != 0;
        for (int j0 = 0; j0 < below; j0 += 4) {
            float4 va = w4[j0 >> 1], vb = w4[(j0 >> 1) + 1];
            const int4 pp = rem ? p4[j0 >> 2] : make_int4(-1, -1, -1, -1);
            const uint32_t rb = rbits(j0);
            auto fix = [&](float& x, float& y, int p, int u) {
                if (j0 + u >= below || ((rb >> u) & 1u)) return;
                long long qx = fq_of(x) + shx, qy = fq_of(y) + shy;
                if (p == mp) {
                    qx += remx;
                    qy += remy;
                }
                x = fv_of(qx);
                y = fv_of(qy);
            };
            fix(va.x, va.y, pp.x, 0);
            fix(va.z, va.w, pp.y, 1);
            fix(vb.x, vb.y, pp.z, 2);
            fix(vb.z, vb.w, pp.w, 3);
            w4[j0 >> 1] = va;
            w4[(j0 >> 1) + 1] = vb;
        }
    }
    // holes below the new count, in slot order, then the slots from the old count on
    int hw = 0;
    uint32_t hbits = rm0;
    int app = n0;
    auto next_free = [&]() -> int {
        for (;;) {
            if (hbits) {
                const int j = 32 * hw + __ffs(hbits) - 1;
                hbits &= hbits - 1;
                if (j < below) return j;
                hbits = 0;
                hw = 4;
            }
            if (++hw >= 4) return app++;
            hbits = hw == 1 ? rm1 : (hw == 2 ? rm2 : rm3);
        }
    };
    // kept particles above the new count
    for (int j = nAll; j < n0; ++j) {
        if ((rbits(j & ~3) >> (j & 3)) & 1u) continue;
        const size_t s = ib + j;
        const float2 v = B.vel[s];
        const float2 o = B.off[s];
        const int p = B.pid[s];
        long long qx = fq_of(v.x) + shx, qy = fq_of(v.y) + shy;
        if (p == mp) {
            qx += remx;
            qy += remy;
        }
        const int d = next_free();
        B.off[ib + d] = o;
        B.vel[ib + d] = make_float2(fv_of(qx), fv_of(qy));
        B.pid[ib + d] = p;
    }
    // arrivals
    for (int k = 0; k < nr; ++k) {
        const int p = A.recPidG[rs + k];
        const int2 q = A.recQG[rs + k];
        long long qx = q.x + shx, qy = q.y + shy;
        if (p == mp) {
            qx += remx;
            qy += remy;
        }
        const int d = next_free();
        if (d < K) {
            B.off[ib + d] = A.recOffG[rs + k];
            B.vel[ib + d] = make_float2(fv_of(qx), fv_of(qy));
            B.pid[ib + d] = p;
        }
    }
}

__global__ void __launch_bounds__(256) k_fast_zone_apply(FastZoneArgs A) {
    fast_zone_apply_block((int)blockIdx.x, A);
}

// kW zones per block, in step: a block barrier after the set-up, after each dense pass and
// after the sparse phase, so that the resident warps of an SM execute the same phase's code
template <int kW>
__device__ __forceinline__ void fast_zone_block(int bx, const FastZoneArgs& A, char* smem) {
    const int wib = threadIdx.x >> 5;
    const int slot = bx * kW + wib;
    const int z = A.order && slot < A.nZones ? A.order[slot] : slot;
    FastZone Z;
    Z.A = &A;
    Z.lane = threadIdx.x & 31;
    Z.z = z;
    const int lane = Z.lane;
    const DevParams& P = A.P;
    Z.failed = false;
    bool ok = z < A.nZones;
    if (ok) {
        const int4 R = A.rects[z];
        Z.x0 = R.x; Z.x1 = R.y; Z.y0 = R.z; Z.y1 = R.w;
        Z.TX = Z.x1 - Z.x0; Z.TY = Z.y1 - Z.y0; Z.nl = Z.TX * Z.TY; Z.WY = Z.TY + 4;
        Z.zseed = fhash(A.S->seed, (uint64_t)z, 0x5A4F4E45ULL + (uint64_t)A.pass);
        Z.op = 0;
        Z.nrec = 0;
        Z.movedDense = Z.movedSparse = 0;
        if (Z.nl > A.maxCells || (Z.TX + 4) * Z.WY > A.winCap || (Z.TX + 2) * (Z.TY + 2) > A.nsmCap) {
            if (lane == 0) raise_error(A.st, kErrZoneCapacity, z);
            ok = false;
        }
    }
    FastZoneMem& M = Z.M;
    if (ok) {
        const size_t per = FastZoneMem::bytes(A.maxCells, A.winCap, A.nsmCap, A.recCap);
        Z.M.carve(smem + per * wib, A.maxCells, A.winCap, A.nsmCap, A.recCap);
        // pass-input counts of the window (wrapped on periodic axes, -1 outside the domain)
        const int W = (Z.TX + 4) * Z.WY;
        for (int w = lane; w < W; w += 32) {
            int gx = Z.x0 - 2 + w / Z.WY, gy = Z.y0 - 2 + w % Z.WY;
            if (P.perx) gx = wrap_index(gx, P.Nx);
            if (P.pery) gy = wrap_index(gy, P.Ny);
            const bool in = gx >= 0 && gx < P.Nx && gy >= 0 && gy < P.Ny;
            M.win[w] = in ? (short)min(A.cntIn[gy + P.Ny * gx], A.F.K) : (short)-1;
        }
        for (int l = lane; l < Z.nl; l += 32) {
            const int lx = l / Z.TY, ly = l - lx * Z.TY;
            M.cx[l] = (uint8_t)lx;
            M.cy[l] = (uint8_t)ly;
            M.wi[l] = (uint16_t)((lx + 2) * Z.WY + (ly + 2));
        }
        __syncwarp();
        for (int l = lane; l < Z.nl; l += 32) {
            M.n0[l] = (uint8_t)Z.cnt(l);
            M.flg[l] = 0;
            M.nrecv[l] = 0;
            M.rm[4 * l] = M.rm[4 * l + 1] = M.rm[4 * l + 2] = M.rm[4 * l + 3] = 0;
        }
        __syncwarp();
    }
    __syncthreads();
    // dense passes (src/zone_pass.cpp:708-781): cells above their high map, in random order
    for (int pass = 0; pass < P.maxPasses; ++pass) {
        if (ok && !Z.failed) {
            for (int l = lane; l < Z.nl; l += 32) {
                const bool bulk = Z.cnt(l) > 0;
                M.flg[l] = (uint8_t)((M.flg[l] & ~kZBulkD) | (bulk ? kZBulkD : 0));
            }
            __syncwarp();
            const int D = Z.order_cells([&](int i) -> uint32_t {
                const bool bulk = M.flg[i] & kZBulkD;
                if ((double)Z.cnt(i) > Z.high_map(bulk))
                    return ((uint32_t)fhash(Z.zseed, 0x44454EULL + (uint64_t)pass, (uint64_t)i) & 0xFFFFFF00u) | (uint32_t)i;
                return 0xFFFFFFFFu;
            });
            for (int q = 0; q < D && !Z.failed; ++q) Z.dense_cell(M.ord[q]);
            __syncwarp();
        }
        __syncthreads();
    }
    // sparse phase (src/zone_pass.cpp:783-854)
    if (ok && !Z.failed) {
        for (int l = lane; l < Z.nl; l += 32) {
            const bool bulk = Z.cnt(l) > 0;
            M.flg[l] = (uint8_t)((M.flg[l] & ~kZBulkS) | (bulk ? kZBulkS : 0));
        }
        __syncwarp();
        Z.compute_nsm();
        const int L = Z.order_cells([&](int i) -> uint32_t {
            const int cn = Z.cnt(i);
            if (cn > 0 && (double)cn < Z.low_map(true))
                return ((uint32_t)fhash(Z.zseed, 0x4C4F57ULL, (uint64_t)i) & 0xFFFFFF00u) | (uint32_t)i;
            return 0xFFFFFFFFu;
        });
        for (int q = 0; q < L && !Z.failed; ++q) Z.sparse_cell(M.ord[q]);
    }
    __syncthreads();
    if (!ok) return;
    // the decisions for the apply kernel
    fast_zone_export(Z);
    if (lane == 0) {
        if (Z.movedDense || Z.movedSparse) {
            atomicAdd(A.moved, Z.movedDense);
            atomicAdd(A.moved + 1, Z.movedSparse);
        }
        if (Z.failed) atomicAdd(A.recOverflow, 1);
    }
}

template <int kW>
__global__ void __launch_bounds__(32 * kW, 24 / kW) k_fast_zone(FastZoneArgs A) {
    extern __shared__ __align__(16) char smem[];
    fast_zone_block<kW>((int)blockIdx.x, A, smem);
}

// Launch order of the decision kernel. The work of a zone is its particles above the high map
// plus its cells below the low map (its dense and sparse phases), from the pass-input counts;
// one warp per zone. A zone's decisions do not depend on when it runs, so the order changes
// only how evenly the zones of a block (which run their phases together) are loaded.
constexpr int kFastCostBuckets = 256;
constexpr int kFastOrderWindow = 1024;  // zones sorted together (one block of k_fast_zone_rank)
__device__ __forceinline__ void fast_zone_cost_block(int bx, const FastZoneArgs& A, int* __restrict__ cost) {
    const int z = (int)((bx * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (z >= A.nZones) return;
    const DevParams& P = A.P;
    const int4 R = A.rects[z];
    const int TY = R.w - R.z, nl = (R.y - R.x) * TY;
    int w = 0;
    for (int l = lane; l < nl; l += 32) {
        int gx = R.x + l / TY, gy = R.z + l % TY;
        if (P.perx) gx = wrap_index(gx, P.Nx);
        if (P.pery) gy = wrap_index(gy, P.Ny);
        if (gx < 0 || gx >= P.Nx || gy < 0 || gy >= P.Ny) continue;
        const int n = min(A.cntIn[gy + P.Ny * gx], A.F.K);
        if (n > 0 && (double)n > P.highThr) w += (int)ceil((double)n - P.highThr);
        else if (n > 0 && (double)n < P.lowThrBulk) ++w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (lane == 0) cost[z] = min(kFastCostBuckets - 1, w);
}

__global__ void k_fast_zone_cost(FastZoneArgs A, int* __restrict__ cost) { fast_zone_cost_block((int)blockIdx.x, A, cost); }

// The zones of each window of kFastOrderWindow slots in descending cost: a counting sort in
// shared memory (places within a bucket come from shared atomics, in no fixed order).
__device__ __forceinline__ void fast_zone_rank_block(int bx, const int* __restrict__ cost, int nZones,
                                                     int* __restrict__ order) {
    __shared__ int hist[kFastCostBuckets];
    const int t = threadIdx.x;
    const int z = bx * kFastOrderWindow + t;
    const bool live = z < nZones;
    if (t < kFastCostBuckets) hist[t] = 0;
    __syncthreads();
    const int b = live ? cost[z] : 0;
    const int r = live ? atomicAdd(hist + b, 1) : 0;
    __syncthreads();
    if (t < 32) {  // exclusive offsets, buckets in descending cost: 8 buckets per lane
        int v[kFastCostBuckets / 32], acc = 0;
#pragma unroll
        for (int k = 0; k < kFastCostBuckets / 32; ++k) {
            v[k] = hist[kFastCostBuckets - 1 - (8 * t + k)];
            acc += v[k];
        }
        int incl = acc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (t >= o) incl += u;
        }
        int run = incl - acc;
#pragma unroll
        for (int k = 0; k < kFastCostBuckets / 32; ++k) {
            const int bucket = kFastCostBuckets - 1 - (8 * t + k);
            const int cnt = v[k];
            hist[bucket] = run;
            run += cnt;
        }
    }
    __syncthreads();
    if (live) order[bx * kFastOrderWindow + hist[b] + r] = z;
}

__global__ void __launch_bounds__(kFastOrderWindow) k_fast_zone_rank(const int* __restrict__ cost, int nZones,
                                                                     int* __restrict__ order) {
    fast_zone_rank_block((int)blockIdx.x, cost, nZones, order);
}

// ------------------------------------------------------------------ closure
// Per cell, from the exact sums: the reference fields of stateRef, the collided state the base
// pass read (N, Ux, Uy, T, rho, Pkin, Pvir: src/common_grid.cpp:32-100), and pdriveRaw = Pkin + Pvir
// (src/liquid_closure.cpp:401-405); the red momenta, duRepair = (P_ref - P_red) / gamma and the
// beta_opt terms (:343-360) into cols (num term, den term).
__device__ __forceinline__ void fast_closure_cells_block(int bx, const DevParams& P, const longlong4* __restrict__ ref,
                                                         const longlong2* __restrict__ red, const int* __restrict__ redN,
                                                         double* __restrict__ pdRaw, double* __restrict__ duRX,
                                                         double* __restrict__ duRY, double* __restrict__ cols,
                                                         float4* __restrict__ feat) {
    const int c = bx * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    const longlong4 r = ref[c];
    const int n = (int)r.w;
    double uxr = 0.0, uyr = 0.0, T = 0.0;
    if (n > 0) {
        uxr = (double)r.x / n * kFastInvQ;
        uyr = (double)r.y / n * kFastInvQ;
    }
    if (n > 1) {
        const __int128 num = (__int128)n * r.z - (__int128)r.x * r.x - (__int128)r.y * r.y;
        T = (double)num / (double)n * kFastInvQ * kFastInvQ / (double)(2 * (n - 1));
    }
    const double rho = (double)n / P.Vc;
    const double pk = rho * T;
    const double pv = P.Kvirial * (rho - P.rhoTarget);
    pdRaw[c] = pk + pv;
    const longlong2 q = red[c];
    const int m = redN[c];
    double uxd = 0.0, uyd = 0.0;
    if (m > 0) {
        uxd = (double)q.x / m * kFastInvQ;
        uyd = (double)q.y / m * kFastInvQ;
    }
    const double ax = (double)(r.x - q.x) * kFastInvQ / P.gamma;
    const double ay = (double)(r.y - q.y) * kFastInvQ / P.gamma;
    const double ex = uxd - uxr, ey = uyd - uyr;
    duRX[c] = ax;
    duRY[c] = ay;
    cols[2 * (size_t)c] = -(ex * ax + ey * ay);
    cols[2 * (size_t)c + 1] = ax * ax + ay * ay;
    // the learned closure's stencil input: occupancy, kinetic pressure relative to the target
    // rho* kBT, and the mean velocity along x (the network predicts the EOS kick, which the
    // pressure drive Pkin + Pvir of these fields determines)
    if (feat) {  // .w: the red count, the weight of the cell's kick in the momentum sum
        const double pkRel = pk / (P.rhoTarget * P.kBT) - 1.0;
        feat[c] = make_float4((float)((double)n / P.gamma - 1.0), (float)pkRel, (float)uxr, (float)m);
    }
}

__global__ void k_fast_closure_cells(DevParams P, const longlong4* __restrict__ ref, const longlong2* __restrict__ red,
                                     const int* __restrict__ redN, double* __restrict__ pdRaw, double* __restrict__ duRX,
                                     double* __restrict__ duRY, double* __restrict__ cols, float4* __restrict__ feat) {
    fast_closure_cells_block((int)blockIdx.x, P, ref, red, redN, pdRaw, duRX, duRY, cols, feat);
}

// EOS kick from the blended pressure drive (src/liquid_closure.cpp:243-295, :424-430) plus
// beta_applied * duRepair, rounded per cell to the grid (the pending kick of the next step).
// learned (nullable): per cell (duX, duY) of the learned closure replacing the EOS kick where
// it is a number and the step's mode (nullable) is learned; elsewhere the plain EOS kick. The
// learned kicks are taken less their particle-weighted mean (learnedSum: sum of N du at 2^-32
// and the particles kicked), so they carry no net momentum: the plain EOS kick is the gradient
// of a field and moves the mean flow by a negligible amount, while a network's residual bias,
// though small against the kick, is of the size of the body force per step.
// eosX, eosY (nullable): the plain EOS kick per cell (training samples).
__device__ __forceinline__ void fast_kick_cells_block(int bx, const DevParams& P, const double* __restrict__ pd,
                                                      const double* __restrict__ duRX, const double* __restrict__ duRY,
                                                      const double* __restrict__ numDen,
                                                      const double* __restrict__ learnedX,
                                                      const double* __restrict__ learnedY,
                                                      const long long* __restrict__ learnedSum,
                                                      const int* __restrict__ mode, int2* __restrict__ kick,
                                                      double* __restrict__ eosX, double* __restrict__ eosY) {
    const int c = bx * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    const double beta = beta_applied(P, numDen[0], numDen[1]);
    double ex, ey;
    if (learnedX && (!mode || *mode) && !isnan(learnedX[c])) {
        const double nk = learnedSum ? (double)learnedSum[2] : 0.0;
        const double mx = nk > 0.0 ? (double)learnedSum[0] * 0x1p-32 / nk : 0.0;
        const double my = nk > 0.0 ? (double)learnedSum[1] * 0x1p-32 / nk : 0.0;
        ex = learnedX[c] - mx;
        ey = learnedY[c] - my;
    } else {
        const int ix = c / P.Ny, iy = c - ix * P.Ny;
        double gx, gy;
        if (P.perx) gx = (pd[iy + P.Ny * wrap_index(ix + 1, P.Nx)] - pd[iy + P.Ny * wrap_index(ix - 1, P.Nx)]) / (2.0 * P.dx);
        else if (ix == 0) gx = (pd[iy + P.Ny * (ix + 1)] - pd[c]) / P.dx;
        else if (ix == P.Nx - 1) gx = (pd[c] - pd[iy + P.Ny * (ix - 1)]) / P.dx;
        else gx = (pd[iy + P.Ny * (ix + 1)] - pd[iy + P.Ny * (ix - 1)]) / (2.0 * P.dx);
        if (P.pery) gy = (pd[wrap_index(iy + 1, P.Ny) + P.Ny * ix] - pd[wrap_index(iy - 1, P.Ny) + P.Ny * ix]) / (2.0 * P.dy);
        else if (iy == 0) gy = (pd[(iy + 1) + P.Ny * ix] - pd[c]) / P.dy;
        else if (iy == P.Ny - 1) gy = (pd[c] - pd[(iy - 1) + P.Ny * ix]) / P.dy;
        else gy = (pd[(iy + 1) + P.Ny * ix] - pd[(iy - 1) + P.Ny * ix]) / (2.0 * P.dy);
        const double k = -P.dt / P.rhoTarget * P.betaEOS;
        ex = k * gx;
        ey = k * gy;
        if (eosX) {
            eosX[c] = ex;
            eosY[c] = ey;
        }
    }
    const double dx = beta * duRX[c] + ex, dy = beta * duRY[c] + ey;
    kick[c] = make_int2((int)llrint(dx * kFastQ), (int)llrint(dy * kFastQ));
}

__global__ void k_fast_kick_cells(DevParams P, const double* __restrict__ pd, const double* __restrict__ duRX,
                                  const double* __restrict__ duRY, const double* __restrict__ numDen,
                                  const double* __restrict__ learnedX, const double* __restrict__ learnedY,
                                  const long long* __restrict__ learnedSum, const int* __restrict__ mode,
                                  int2* __restrict__ kick, double* __restrict__ eosX, double* __restrict__ eosY) {
    fast_kick_cells_block((int)blockIdx.x, P, pd, duRX, duRY, numDen, learnedX, learnedY, learnedSum, mode, kick, eosX,
                          eosY);
}

// per cell of the bins: count and count^2 (the learned closure's occupancy-variance check)
__global__ void k_fast_count_cols(const int* __restrict__ cnt, int Nc, double* __restrict__ cols) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nc) return;
    const double n = (double)cnt[c];
    cols[2 * (size_t)c] = n;
    cols[2 * (size_t)c + 1] = n * n;
}

// Applies the pending kick to the bins in place (before the state is read out).
__global__ void k_fast_apply_kick(DevParams P, FastParams F, FastBins b, const int2* __restrict__ kick) {
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= P.Nc) return;
    const int n = min(b.cnt[c], F.K);
    const int2 kq = kick[c];
    if (kq.x == 0 && kq.y == 0) return;
    for (int j = lane; j < n; j += 32) {
        const size_t s = (size_t)c * F.K + j;
        const float2 v = b.vel[s];
        b.vel[s] = make_float2(fv_of(fq_of(v.x) + kq.x), fv_of(fq_of(v.y) + kq.y));
    }
}

// Per cell of the current bins: count, count^2, out-of-band flag, sum |q|^2 (as doubles of
// exact integers), sum qx, sum qy, Ux and Uy (for mean Ux / Qx): the metrics row's columns.
__global__ void k_fast_metric_cols(DevParams P, FastParams F, FastBins b, double* __restrict__ cols) {
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= P.Nc) return;
    const int n = min(b.cnt[c], F.K);
    long long sx = 0, sy = 0, sqq = 0;
    for (int j = lane; j < n; j += 32) {
        const float2 v = b.vel[(size_t)c * F.K + j];
        const long long qx = fq_of(v.x), qy = fq_of(v.y);
        sx += qx;
        sy += qy;
        sqq += qx * qx + qy * qy;
    }
    sx = warp_sum_ll(sx);
    sy = warp_sum_ll(sy);
    sqq = warp_sum_ll(sqq);
    if (lane == 0) {
        const double nn = (double)n;
        double* o = cols + 8 * (size_t)c;
        o[0] = nn;
        o[1] = nn * nn;
        o[2] = ((nn > P.highThr) || (nn > 0.0 && nn < P.lowThrBulk)) ? 1.0 : 0.0;
        o[3] = 0.5 * (double)sqq * kFastInvQ * kFastInvQ;
        o[4] = (double)sx * kFastInvQ;
        o[5] = (double)sy * kFastInvQ;
        o[6] = n > 0 ? (double)sx / n * kFastInvQ : 0.0;
        o[7] = n > 0 ? (double)sy / n * kFastInvQ : 0.0;
    }
}

// Poiseuille profile: per row iy, the sum over steps of the row's momentum (int64 at 2^-32)
// and particle count, from the current bins plus a pending kick (nullable).
__global__ void k_fast_profile(DevParams P, FastParams F, FastBins b, const int2* __restrict__ kick,
                               unsigned long long* __restrict__ rowP, unsigned long long* __restrict__ rowN) {
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= P.Nc) return;
    const int n = min(b.cnt[c], F.K);
    long long sx = 0;
    for (int j = lane; j < n; j += 32) sx += fq_of(b.vel[(size_t)c * F.K + j].x);
    sx = warp_sum_ll(sx);
    if (lane == 0 && n > 0) {
        if (kick) sx += (long long)n * kick[c].x;
        const int iy = c % P.Ny;
        atomicAdd(rowP + iy, (unsigned long long)(sx * 4096LL));  // grid units (2^-20) -> 2^-32
        atomicAdd(rowN + iy, (unsigned long long)n);
    }
}

// ------------------------------------------------------------------ state I/O
// FP64 positions and velocities in particle-id order into the bins (claims per cell)
__global__ void k_fast_load(DevParams P, FastParams F, const double2* __restrict__ x, const double2* __restrict__ v, int n,
                            FastBins b, DevStatus* st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 X = x[i];
    const int c = cell_of(X.x, X.y, P);
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
    const int slot = atomicAdd(b.cnt + c, 1);
    if (slot >= F.K) {
        raise_error(st, kErrBinCapacity, c);
        return;
    }
    const size_t s = (size_t)c * F.K + slot;
    const float ox = fminf(fmaxf((float)(X.x / P.dx - (double)ix), 0.0f), kFastOffMax);
    const float oy = fminf(fmaxf((float)(X.y / P.dy - (double)iy), 0.0f), kFastOffMax);
    b.off[s] = make_float2(ox, oy);
    const double2 V = v[i];
    b.vel[s] = make_float2(fv_of(llrint(V.x * kFastQ)), fv_of(llrint(V.y * kFastQ)));
    b.pid[s] = i;
}

// the bins into FP64 positions and velocities in particle-id order
__global__ void k_fast_store(DevParams P, FastParams F, FastBins b, double2* __restrict__ x, double2* __restrict__ v) {
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= P.Nc) return;
    const int n = min(b.cnt[c], F.K);
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
    for (int j = lane; j < n; j += 32) {
        const size_t s = (size_t)c * F.K + j;
        const int p = b.pid[s];
        if (p < 0 || p >= P.n) continue;
        const float2 o = b.off[s];
        const float2 w = b.vel[s];
        x[p] = make_double2(((double)ix + (double)o.x) * P.dx, ((double)iy + (double)o.y) * P.dy);
        v[p] = make_double2((double)w.x, (double)w.y);
    }
}

}  // namespace mpcd_dev
