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
constexpr int kFastZoneWarps = 4;              // zones per block of the zone kernel
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
    double dtqx, dtqy;           // cell units moved per grid unit of velocity in one step
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
__device__ __forceinline__ float fv_of(long long q) { return (float)((double)q * kFastInvQ); }

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
__device__ __forceinline__ int warp_sum_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ step begin
__global__ void k_fast_step_begin(FastParams F, FastStep* S, FastWall* W) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
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

// ------------------------------------------------------------------ stream + walls + binning
// One warp per source cell. Applies the pending closure kick of the previous step (kick[c],
// grid units, nullable), sums the kicked state per cell (the closure's reference fields:
// ref[c] = (sum qx, sum qy, sum |q|^2, N)), then body force, streaming and the walls of
// apply_bc_general (src/boundary_conditions.cpp:37-202: up to four sweeps of left, right,
// bottom, top, then the final wrap or clamp), and files each particle into the bin of its new
// cell (warp-aggregated slot claims).
__global__ void __launch_bounds__(256) k_fast_stream(DevParams P, FastParams F, const FastStep* __restrict__ S,
                                                     FastBins in, FastBins out, const int2* __restrict__ kick,
                                                     longlong4* __restrict__ ref, FastWall* __restrict__ W,
                                                     DevStatus* st) {
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= P.Nc) return;
    const int n = min(in.cnt[c], F.K);  // a count above K (a failed step) reads no further
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
    const int fqx = S->fqx, fqy = S->fqy;
    const uint64_t seed = S->seed;
    const int2 kq = kick ? kick[c] : make_int2(0, 0);
    long long sx = 0, sy = 0, sqq = 0;
    int hits[4] = {0, 0, 0, 0};
    long long dE2 = 0;
    const double Nx = (double)P.Nx, Ny = (double)P.Ny;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        const bool live = j < n;
        int newc = 0;
        float2 o = make_float2(0.f, 0.f);
        int qx = 0, qy = 0, pid = 0;
        if (live) {
            const size_t s = (size_t)c * F.K + j;
            const float2 off = in.off[s];
            const float2 w = in.vel[s];
            pid = in.pid[s];
            qx = fq_of(w.x) + kq.x;
            qy = fq_of(w.y) + kq.y;
            sx += qx;
            sy += qy;
            sqq += (long long)qx * qx + (long long)qy * qy;
            qx += fqx;
            qy += fqy;
            double X = (double)ix + (double)off.x + (double)qx * F.dtqx;
            double Y = (double)iy + (double)off.y + (double)qy * F.dtqy;
            for (int sweep = 0; sweep < 4; ++sweep) {
                const long long e0 = (long long)qx * qx + (long long)qy * qy;
                bool hit = false;
                const uint64_t hk = fhash(seed, (uint64_t)(uint32_t)pid, (uint64_t)sweep);
                if (X < 0.0) {
                    if (P.bc[0] == MPCD_BC_PERIODIC) {
                        X += Nx;
                    } else {
                        X = -X;
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
                if (X > Nx) {
                    if (P.bc[1] == MPCD_BC_PERIODIC) {
                        X -= Nx;
                    } else {
                        X = 2.0 * Nx - X;
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
                if (Y < 0.0) {
                    if (P.bc[2] == MPCD_BC_PERIODIC) {
                        Y += Ny;
                    } else {
                        Y = -Y;
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
                if (Y > Ny) {
                    if (P.bc[3] == MPCD_BC_PERIODIC) {
                        Y -= Ny;
                    } else {
                        Y = 2.0 * Ny - Y;
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
                if (X >= 0.0 && X <= Nx && Y >= 0.0 && Y <= Ny) break;
            }
            if (P.perx) X = X - floor(X / Nx) * Nx;
            else X = fmin(fmax(X, 0.0), Nx);
            if (P.pery) Y = Y - floor(Y / Ny) * Ny;
            else Y = fmin(fmax(Y, 0.0), Ny);
            int jx = (int)floor(X), jy = (int)floor(Y);
            jx = min(max(jx, 0), P.Nx - 1);
            jy = min(max(jy, 0), P.Ny - 1);
            o.x = fminf(fmaxf((float)(X - (double)jx), 0.0f), kFastOffMax);
            o.y = fminf(fmaxf((float)(Y - (double)jy), 0.0f), kFastOffMax);
            newc = jy + P.Ny * jx;
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
    sx = warp_sum_ll(sx);
    sy = warp_sum_ll(sy);
    sqq = warp_sum_ll(sqq);
    if (lane == 0 && ref) ref[c] = make_longlong4(sx, sy, sqq, n);
    if (W) {
        for (int k = 0; k < 4; ++k) {
            const int h = warp_sum_i(hits[k]);
            if (lane == 0 && h) atomicAdd(&W->n[k], (unsigned long long)h);
        }
        const long long e = warp_sum_ll(dE2);
        if (lane == 0 && e) atomicAdd(&W->dE2, (unsigned long long)e);
    }
}

// ------------------------------------------------------------------ SRD collision
// One warp per SRD cell (jx, jy) of the grid shifted by (sx, sy) cell units: its particles
// come from the 2 x 2 standard cells that overlap it (a particle in cell (ix, iy) at offset
// (ox, oy) lies in SRD cell (ix + floor(ox + sx), iy + floor(oy + sy)), wrapped on periodic
// axes and clamped on the others, as srd_cell_id_with_random_shift does, src/srd_collision.cpp:9-45).
// Rotation of the velocities relative to the cell mean by +-alpha, the sign drawn per SRD cell,
// and the isokinetic thermostat (src/srd_collision.cpp:47-140). Sums are exact in grid units;
// the rounding of the new velocities to the grid leaves an integer residual that goes to the
// member with the smallest particle id, so every SRD cell keeps its momentum exactly.
__device__ __forceinline__ int fast_srd_index(int i, double o, double s, int N, bool per) {
    int j = i + (int)floor((double)o + s);
    if (per) j = wrap_index(j, N);
    else j = min(max(j, 0), N - 1);
    return j;
}

__global__ void __launch_bounds__(256) k_fast_collide(DevParams P, FastParams F, const FastStep* __restrict__ S,
                                                      FastBins b) {
    const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= P.Nc) return;
    const int jx = w / P.Ny, jy = w - jx * P.Ny;
    const double sxs = S->sx, sys = S->sy;
    const int fx = (sxs < 0.0) ? -1 : 0, fy = (sys < 0.0) ? -1 : 0;
    int src[4], n[4];
    int total = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int ax = jx - fx - 1 + (k & 1), ay = jy - fy - 1 + (k >> 1);
        bool ok = true;
        if (P.perx) ax = wrap_index(ax, P.Nx);
        else ok = ok && ax >= 0 && ax < P.Nx;
        if (P.pery) ay = wrap_index(ay, P.Ny);
        else ok = ok && ay >= 0 && ay < P.Ny;
        src[k] = ok ? ay + P.Ny * ax : -1;
        n[k] = ok ? min(b.cnt[src[k]], F.K) : 0;
        total += n[k];
    }
    // duplicate sources (a periodic axis of one or two cells) are read once
    if (src[1] == src[0]) n[1] = 0;
    if (src[2] == src[0] || src[2] == src[1]) n[2] = 0;
    if (src[3] == src[0] || src[3] == src[1] || src[3] == src[2]) n[3] = 0;
    total = n[0] + n[1] + n[2] + n[3];
    // pass 1: membership and exact sums
    long long Sx = 0, Sy = 0, Sqq = 0;
    int N = 0;
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        bool mem = false;
        int qx = 0, qy = 0;
        if (t < total) {
            int k = 0, j = t;
            while (j >= n[k]) { j -= n[k]; ++k; }
            const size_t s = (size_t)src[k] * F.K + j;
            const int ix = src[k] / P.Ny, iy = src[k] - ix * P.Ny;
            const float2 o = b.off[s];
            mem = fast_srd_index(ix, o.x, sxs, P.Nx, P.perx) == jx && fast_srd_index(iy, o.y, sys, P.Ny, P.pery) == jy;
            if (mem) {
                const float2 v = b.vel[s];
                qx = fq_of(v.x);
                qy = fq_of(v.y);
            }
        }
        N += __popc(__ballot_sync(0xffffffffu, mem));
        Sx += qx;
        Sy += qy;
        Sqq += (long long)qx * qx + (long long)qy * qy;
    }
    if (N == 0) return;
    Sx = warp_sum_ll(Sx);
    Sy = warp_sum_ll(Sy);
    Sqq = warp_sum_ll(Sqq);
    const double ux = (double)Sx / N, uy = (double)Sy / N;
    double ct = 1.0, sn = 0.0;
    if (N >= 2) {
        const uint64_t h = fhash(S->seed, (uint64_t)w, 0x5349474EULL);
        const int r = (h >> 63) ? 1 : 2;  // +alpha or -alpha
        ct = P.rotCos[r];
        sn = P.rotSin[r];
    }
    double lam = 1.0;
    if (P.useThermostat && N > 1) {
        // sum |q - u|^2 = (N sum|q|^2 - |sum q|^2) / N, an exact integer numerator
        const __int128 num = (__int128)N * Sqq - (__int128)Sx * Sx - (__int128)Sy * Sy;
        const double s2 = (double)num / (double)N;
        if (s2 > 0.0) lam = sqrt(2.0 * (double)(N - 1) * P.kBT * kFastQ * kFastQ / s2);
    }
    // pass 2: new velocities rounded to the grid; their sum and the smallest-id member
    long long Tx = 0, Ty = 0;
    unsigned long long best = ~0ULL;  // (pid, slot) of the member that takes the residual
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        if (t < total) {
            int k = 0, j = t;
            while (j >= n[k]) { j -= n[k]; ++k; }
            const size_t s = (size_t)src[k] * F.K + j;
            const int ix = src[k] / P.Ny, iy = src[k] - ix * P.Ny;
            const float2 o = b.off[s];
            if (fast_srd_index(ix, o.x, sxs, P.Nx, P.perx) == jx && fast_srd_index(iy, o.y, sys, P.Ny, P.pery) == jy) {
                const float2 v = b.vel[s];
                const double rx = (double)fq_of(v.x) - ux, ry = (double)fq_of(v.y) - uy;
                const long long nx = llrint(ux + lam * (ct * rx - sn * ry));
                const long long ny = llrint(uy + lam * (sn * rx + ct * ry));
                Tx += nx;
                Ty += ny;
                b.vel[s] = make_float2(fv_of(nx), fv_of(ny));
                if (llabs(nx) < (1LL << 22) && llabs(ny) < (1LL << 22)) {
                    const unsigned long long key = ((unsigned long long)(uint32_t)b.pid[s] << 32) | (unsigned long long)t;
                    best = key < best ? key : best;
                }
            }
        }
    }
    Tx = warp_sum_ll(Tx);
    Ty = warp_sum_ll(Ty);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
        best = x < best ? x : best;
    }
    __syncwarp();
    const long long rx = Sx - Tx, ry = Sy - Ty;
    if (lane == 0 && best != ~0ULL && (rx != 0 || ry != 0)) {
        int k = 0, j = (int)(best & 0xffffffffu);
        while (j >= n[k]) { j -= n[k]; ++k; }
        const size_t s = (size_t)src[k] * F.K + j;
        const float2 v = b.vel[s];
        b.vel[s] = make_float2(fv_of(fq_of(v.x) + rx), fv_of(fq_of(v.y) + ry));
    }
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
    FastBins in, out;
    longlong2* red;            // nullable: per cell the output's momentum sum (closure input)
    int* moved;                // (dense, sparse) over all zones
    int* recOverflow;          // zones that ran out of records (their remaining moves are skipped)
    DevStatus* st;
    int maxCells, winCap, nsmCap, recCap;
};

// zone working set layout (bytes), carved per warp
struct FastZoneMem {
    short* win;       // winCap: counts of the window (zone + 2-cell halo); -1 outside the domain
    uint8_t* n0;      // cell: particles at the pass start
    uint8_t* flg;     // cell: flags
    uint8_t* nrecv;   // cell: records currently in the cell
    uint32_t* rm;     // cell x 4: originals removed
    int* recPid;      // recCap
    uint16_t* recSrc; // recCap: (origin cell << 7) | slot
    uint8_t* recCur;  // recCap: current cell
    float2* recOff;   // recCap: position in the current cell
    float* nsm;       // nsmCap: smoothed occupancy of the zone and a one-cell ring
    uint32_t* keys;   // 128: order keys (dense / low cells), sort scratch
    int* tgt;         // 32: ordered targets or donors
    float* tgtMap;    // 32
    int* pidBuf;      // kFastMaxK: member ids (momentum correction)

    __host__ __device__ static size_t bytes(int maxCells, int winCap, int nsmCap, int recCap) {
        size_t b = 0;
        auto add = [&](size_t n, size_t a) { b = (b + a - 1) / a * a + n; };
        add((size_t)winCap * 2, 2);
        add((size_t)maxCells, 1);
        add((size_t)maxCells, 1);
        add((size_t)maxCells, 1);
        add((size_t)maxCells * 16, 4);
        add((size_t)recCap * 4, 4);
        add((size_t)recCap * 2, 2);
        add((size_t)recCap, 1);
        add((size_t)recCap * 8, 8);
        add((size_t)nsmCap * 4, 4);
        add(128 * 4, 4);
        add(32 * 4, 4);
        add(32 * 4, 4);
        add((size_t)kFastMaxK * 4, 4);
        return (b + 15) / 16 * 16;
    }
    __device__ void carve(char* base, int maxCells, int winCap, int nsmCap, int recCap) {
        size_t b = 0;
        auto take = [&](size_t n, size_t a) {
            b = (b + a - 1) / a * a;
            char* p = base + b;
            b += n;
            return p;
        };
        win = (short*)take((size_t)winCap * 2, 2);
        n0 = (uint8_t*)take((size_t)maxCells, 1);
        flg = (uint8_t*)take((size_t)maxCells, 1);
        nrecv = (uint8_t*)take((size_t)maxCells, 1);
        rm = (uint32_t*)take((size_t)maxCells * 16, 4);
        recPid = (int*)take((size_t)recCap * 4, 4);
        recSrc = (uint16_t*)take((size_t)recCap * 2, 2);
        recCur = (uint8_t*)take((size_t)recCap, 1);
        recOff = (float2*)take((size_t)recCap * 8, 8);
        nsm = (float*)take((size_t)nsmCap * 4, 4);
        keys = (uint32_t*)take(128 * 4, 4);
        tgt = (int*)take(32 * 4, 4);
        tgtMap = (float*)take(32 * 4, 4);
        pidBuf = (int*)take((size_t)kFastMaxK * 4, 4);
    }
};

constexpr uint8_t kZBulkD = 1, kZBulkS = 2, kZRecv = 4, kZBB = 8, kZSkip = 16;

// ascending sort of 128 u32 keys in shared memory by one warp (bitonic network)
__device__ __forceinline__ void warp_sort128(uint32_t* a, int lane) {
    for (int k = 2; k <= 128; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            __syncwarp();
            for (int i = lane; i < 128; i += 32) {
                const int p = i ^ j;
                if (p > i) {
                    const uint32_t x = a[i], y = a[p];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        a[i] = y;
                        a[p] = x;
                    }
                }
            }
        }
    }
    __syncwarp();
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

    __device__ __forceinline__ int widx(int lx, int ly) const { return (lx + 2) * WY + (ly + 2); }
    __device__ __forceinline__ int cnt(int l) const { return M.win[widx(l / TY, l % TY)]; }
    __device__ __forceinline__ void add_cnt(int l, int d) { M.win[widx(l / TY, l % TY)] += (short)d; }
    __device__ __forceinline__ int gcell(int l) const { return (y0 + l % TY) + A->P.Ny * (x0 + l / TY); }
    __device__ __forceinline__ double low_map(bool bulk) const { return bulk ? A->P.lowThrBulk : A->F.lowMapEmpty; }
    __device__ __forceinline__ double high_map(bool bulk) const { return bulk ? A->P.highThr : A->F.highMapEmpty; }

    // local cell of the zone cell at local (lx, ly) moved by (dx, dy), wrapping periodic axes;
    // -1 outside the domain or outside the zone
    __device__ __forceinline__ int neighbour(int l, int dx, int dy) const {
        const DevParams& P = A->P;
        int gx = x0 + l / TY + dx, gy = y0 + l % TY + dy;
        if (P.perx) gx = wrap_index(gx, P.Nx);
        else if (gx < 0 || gx >= P.Nx) return -1;
        if (P.pery) gy = wrap_index(gy, P.Ny);
        else if (gy < 0 || gy >= P.Ny) return -1;
        if (gx < x0 || gx >= x1 || gy < y0 || gy >= y1) return -1;
        return (gx - x0) * TY + (gy - y0);
    }

    // Removes nt members of cell l and files them into cell t at fresh uniform positions.
    // dense: the members in the reference's list order (the cell's particles in ascending id,
    // then the arrivals in order: src/zone_pass.cpp:541-583 takes the first ids); otherwise
    // members chosen uniformly at random (the sparse phase shuffles the donor's list). A
    // candidate is (key << 10) | (record flag << 9) | index: keys of at most 54 bits, original
    // slots below 128 and records below 512.
    __device__ __forceinline__ uint64_t member_key(bool dense, uint32_t salt, uint32_t pid, int rec) const {
        if (dense) return rec < 0 ? (uint64_t)pid : ((1ULL << 31) + (uint64_t)rec);
        return ((fhash(zseed, salt, pid) >> 41) << 31) | (uint64_t)(pid & 0x7fffffffu);
    }
    __device__ void move_members(int l, int t, int nt, bool dense) {
        const FastBins& B = A->in;
        const int c = gcell(l);
        const int n0 = M.n0[l];
        const uint32_t salt = ++op;
        for (int k = 0; k < nt; ++k) {
            if (failed) return;
            unsigned long long best = ~0ULL;
            for (int j = lane; j < n0; j += 32) {
                if (M.rm[4 * l + (j >> 5)] & (1u << (j & 31))) continue;
                const uint32_t pid = (uint32_t)B.pid[(size_t)c * A->F.K + j];
                const unsigned long long v = (member_key(dense, salt, pid, -1) << 10) | (unsigned long long)j;
                best = v < best ? v : best;
            }
            if (M.nrecv[l] > 0) {
                for (int r = lane; r < nrec; r += 32) {
                    if (M.recCur[r] != l) continue;
                    const unsigned long long v =
                        (member_key(dense, salt, (uint32_t)M.recPid[r], r) << 10) | 512ULL | (unsigned long long)r;
                    best = v < best ? v : best;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
                best = x < best ? x : best;
            }
            if (best == ~0ULL) return;  // no member left (cannot happen while counts agree)
            const uint64_t hp = fhash(zseed, salt, 0x504F53ULL + (uint64_t)k);
            const float2 pos = make_float2(fminf((float)fu01(hp), kFastOffMax), fminf((float)fu01(fmix64(hp)), kFastOffMax));
            if (!(best & 512ULL)) {  // an original of cell l
                const int j = (int)(best & 511ULL);
                if (nrec >= A->recCap) {
                    failed = true;
                    return;
                }
                if (lane == 0) {
                    M.rm[4 * l + (j >> 5)] |= 1u << (j & 31);
                    M.recPid[nrec] = B.pid[(size_t)c * A->F.K + j];
                    M.recSrc[nrec] = (uint16_t)((l << 7) | j);
                    M.recCur[nrec] = (uint8_t)t;
                    M.recOff[nrec] = pos;
                    M.nrecv[t] += 1;
                }
                ++nrec;
            } else if (lane == 0) {  // an arrival in cell l moves on
                const int r = (int)(best & 511ULL);
                M.recCur[r] = (uint8_t)t;
                M.recOff[r] = pos;
                M.nrecv[l] -= 1;
                M.nrecv[t] += 1;
            }
            __syncwarp();
        }
    }

    // update_transfer_correction_masks (src/zone_pass.cpp:492-525) for source l and the
    // receivers recv (bit k: target k of tgt[]), bulk flag bit `bf`
    __device__ void update_masks(int l, unsigned recvBits, uint8_t bf) {
        bool allBulk = (M.flg[l] & bf) != 0;
        for (int k = 0; k < 32; ++k)
            if (recvBits & (1u << k)) allBulk = allBulk && (M.flg[M.tgt[k]] & bf);
        if (lane == 0) {
            auto set = [&](int c) {
                if (allBulk) M.flg[c] |= kZBB;
                else M.flg[c] = (uint8_t)((M.flg[c] | kZSkip) & ~kZBB);
            };
            set(l);
            for (int k = 0; k < 32; ++k)
                if (recvBits & (1u << k)) set(M.tgt[k]);
        }
        __syncwarp();
    }

    // spread_particles_from_dense_source_round_robin (src/zone_pass.cpp:527-589) over the
    // targets ranked as rank_dense_targets_unified does (:436-490); map: 0 low, 1 high.
    // Returns the particles moved; receivers are added to *recvBits (bits index M.tgt).
    __device__ int spread(int l, int needOut, int mapKind, unsigned* recvBits) {
        const DevParams& P = A->P;
        // candidates: range-2 neighbours in dy-outer, dx-inner order (lane k < 24)
        const int k = lane;
        int t = -1, ddx = 0, ddy = 0;
        double map = 0.0;
        bool adm = false;
        if (k < 24) {
            const int idx = k < 12 ? k : k + 1;
            ddx = idx % 5 - 2;
            ddy = idx / 5 - 2;
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
        const int startBin = (int)(fhash(zseed, salt, 0x42494EULL) & 7);
        // sort key (-deficit, cnt, chebyshev, distance^2, random); inward weight is 0 here
        unsigned long long key = ~0ULL;
        int bin = 0;
        if (adm) {
            const double deficit = fmax(0.0, map - (double)cnt(t));
            const unsigned long long dq = (unsigned long long)min(llrint(deficit * 4096.0), (long long)0xFFFFF);
            const int cheb = max(abs(ddx), abs(ddy)), d2 = ddx * ddx + ddy * ddy;
            key = ((0xFFFFFULL - dq) << 44) | ((unsigned long long)min(cnt(t), 255) << 36) |
                  ((unsigned long long)cheb << 34) | ((unsigned long long)d2 << 30) |
                  (fhash(zseed, salt, (uint64_t)k) & 0x3FFFFFFFULL);
            bin = P.atanBin[(ddx + 2) + 5 * (ddy + 2)];
        }
        int rank = 0;
        for (int j = 0; j < 24; ++j) {
            const unsigned long long kj = __shfl_sync(0xffffffffu, key, j);
            const int bj = __shfl_sync(0xffffffffu, bin, j);
            if (adm && ((admMask >> j) & 1u) && bj == bin && kj < key) ++rank;
        }
        const int pos = rank * 8 + ((bin - startBin + 8) & 7);
        int ord = 0;
        for (int j = 0; j < 24; ++j) {
            const int pj = __shfl_sync(0xffffffffu, pos, j);
            if (adm && ((admMask >> j) & 1u) && pj < pos) ++ord;
        }
        if (adm) {
            M.tgt[ord] = t;
            M.tgtMap[ord] = (float)map;
        }
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
        int moved = 0;
        while (needOut > 0 && avail > 0 && !failed) {
            bool progressed = false;
            for (int kk = 0; kk < T; ++kk) {
                const int d = __shfl_sync(0xffffffffu, def, kk);
                if (d <= 0) continue;
                const int rem = __popc(__ballot_sync(0xffffffffu, lane >= kk && lane < T && def > 0));
                const int quota = max(1, (needOut + max(1, rem) - 1) / max(1, rem));
                const int nt = max(1, min(min(quota, d), min(needOut, avail)));
                const int tt = __shfl_sync(0xffffffffu, tO, kk);
                move_members(l, tt, nt, true);
                if (failed) break;
                if (lane == 0) {
                    add_cnt(l, -nt);
                    add_cnt(tt, nt);
                }
                __syncwarp();
                if (lane == kk) def = max(0, (int)floor(mapO - (double)cnt(tO)));
                // the receiver's index in M.tgt for the masks
                *recvBits |= 1u << kk;
                avail -= nt;
                needOut -= nt;
                moved += nt;
                progressed = true;
                if (needOut <= 0 || avail <= 0) break;
            }
            if (!progressed) break;
        }
        return moved;
    }

    // redistribute_dense_cell_at_range_zone_local (src/zone_pass.cpp:591-634) and the mask
    // update of the dense loop (:745-750)
    __device__ void dense_cell(int l) {
        const bool bulk = M.flg[l] & kZBulkD;
        const double hi = high_map(bulk);
        const int nc = cnt(l);
        if (nc <= 0 || (double)nc <= hi) return;
        int needOut = max(0, (int)ceil((double)nc - hi));
        unsigned recvPoor = 0, recvRelief = 0;
        int moved = 0;
        if (needOut > 0) moved += spread(l, needOut, 0, &recvPoor);
        // the poor targets are in M.tgt now; keep their cells before the relief ranking
        int poorCells[24];
        int np = 0;
        for (int k = 0; k < 24; ++k)
            if (recvPoor & (1u << k)) poorCells[np++] = M.tgt[k];
        const int remainingOut = max(0, (int)ceil((double)cnt(l) - hi));
        if (remainingOut > 0 && !failed) moved += spread(l, remainingOut, 1, &recvRelief);
        // masks over the union of both phases' receivers
        bool allBulk = (M.flg[l] & kZBulkD) != 0;
        for (int k = 0; k < np; ++k) allBulk = allBulk && (M.flg[poorCells[k]] & kZBulkD);
        for (int k = 0; k < 24; ++k)
            if (recvRelief & (1u << k)) allBulk = allBulk && (M.flg[M.tgt[k]] & kZBulkD);
        __syncwarp();
        if (lane == 0) {
            auto set = [&](int c) {
                if (allBulk) M.flg[c] |= kZBB;
                else M.flg[c] = (uint8_t)((M.flg[c] | kZSkip) & ~kZBB);
            };
            set(l);
            for (int k = 0; k < np; ++k) {
                M.flg[poorCells[k]] |= kZRecv;
                set(poorCells[k]);
            }
            for (int k = 0; k < 24; ++k)
                if (recvRelief & (1u << k)) {
                    M.flg[M.tgt[k]] |= kZRecv;
                    set(M.tgt[k]);
                }
        }
        __syncwarp();
        movedDense += moved;
    }

    // smoothed occupancy (src/zone_pass.cpp:296-319, non-periodic) of the zone and a one-cell
    // ring, from the window counts
    __device__ void compute_nsm() {
        const DevParams& P = A->P;
        const int RY = TY + 2, total = (TX + 2) * RY;
        for (int i = lane; i < total; i += 32) {
            const int rx = i / RY - 1, ry = i % RY - 1;  // local coordinates, -1 .. TX
            int cx = x0 + rx, cy = y0 + ry;
            if (P.perx) cx = wrap_index(cx, P.Nx);
            if (P.pery) cy = wrap_index(cy, P.Ny);
            float v = 0.0f;
            if (cx >= 0 && cx < P.Nx && cy >= 0 && cy < P.Ny) {
                double acc = 0.0, ws = 0.0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (cx + dx < 0 || cx + dx >= P.Nx || cy + dy < 0 || cy + dy >= P.Ny) continue;
                        const double w = (double)((2 - abs(dx)) * (2 - abs(dy))) * 0.0625;
                        acc += w * (double)M.win[(rx + dx + 2) * WY + (ry + dy + 2)];
                        ws += w;
                    }
                v = (float)(acc / fmax(ws, 1e-30));
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
        const int lx = l / TY, ly = l % TY;
        // inward direction from the local gradient of the smoothed occupancy (:375-411)
        const int gx = x0 + lx, gy = y0 + ly;
        double dirx, diry;
        if (P.perx) dirx = 0.5 * ((double)nsm_at(lx + 1, ly) - (double)nsm_at(lx - 1, ly));
        else if (gx == 0) dirx = (double)nsm_at(lx + 1, ly) - (double)nsm_at(lx, ly);
        else if (gx == P.Nx - 1) dirx = (double)nsm_at(lx, ly) - (double)nsm_at(lx - 1, ly);
        else dirx = 0.5 * ((double)nsm_at(lx + 1, ly) - (double)nsm_at(lx - 1, ly));
        if (P.pery) diry = 0.5 * ((double)nsm_at(lx, ly + 1) - (double)nsm_at(lx, ly - 1));
        else if (gy == 0) diry = (double)nsm_at(lx, ly + 1) - (double)nsm_at(lx, ly);
        else if (gy == P.Ny - 1) diry = (double)nsm_at(lx, ly) - (double)nsm_at(lx, ly - 1);
        else diry = 0.5 * ((double)nsm_at(lx, ly + 1) - (double)nsm_at(lx, ly - 1));
        const double ndir = hypot(dirx, diry);
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
        double score = -1e300;
        uint32_t tie = 0;
        if (don) {
            const double nstep = P.hypotTab[(ddx + 2) + 5 * (ddy + 2)];
            double align = 0.0;
            if (ndir >= 1e-14 && nstep >= 1e-14) align = ((double)ddx * dirx + (double)ddy * diry) / (ndir * nstep);
            score = 100.0 * align + (double)nsm_at(lx + ddx, ly + ddy);
            tie = (uint32_t)fhash(zseed, salt, (uint64_t)k);
        }
        int ord = 0;
        for (int j = 0; j < 8; ++j) {
            const double sj = __shfl_sync(0xffffffffu, score, j);
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
            move_members(dn, l, nt, false);
            if (failed) break;
            if (lane == 0) {
                add_cnt(dn, -nt);
                add_cnt(l, nt);
                M.flg[l] |= kZRecv;
            }
            __syncwarp();
            // update_transfer_correction_masks(d, {c}, bulkMaskLowBefore)
            const bool allBulk = (M.flg[dn] & kZBulkS) && (M.flg[l] & kZBulkS);
            if (lane == 0) {
                for (int c2 : {dn, l}) {
                    if (allBulk) M.flg[c2] |= kZBB;
                    else M.flg[c2] = (uint8_t)((M.flg[c2] | kZSkip) & ~kZBB);
                }
            }
            __syncwarp();
            movedSparse += nt;
            need -= nt;
        }
    }
};

// Output of one zone cell: its members (the originals still there, then the arrivals), with
// the momentum correction of src/zone_pass.cpp:870-909 restoring the cell's momentum exactly
// (an integer share per member, the remainder one unit each to the members of smallest id).
__device__ void fast_zone_output_cell(FastZone& Z, int l) {
    const FastZoneArgs& A = *Z.A;
    FastZoneMem& M = Z.M;
    const int lane = Z.lane, K = A.F.K;
    const int c = Z.gcell(l);
    const int n0 = M.n0[l];
    const size_t ib = (size_t)c * K;
    const uint32_t* rm = M.rm + 4 * l;
    const bool changed = (rm[0] | rm[1] | rm[2] | rm[3]) != 0 || M.nrecv[l] > 0;
    long long fx = 0, fy = 0;  // final momentum of the cell
    if (!changed) {
        for (int j = lane; j < n0; j += 32) {
            const float2 o = A.in.off[ib + j];
            const float2 v = A.in.vel[ib + j];
            const int p = A.in.pid[ib + j];
            A.out.off[ib + j] = o;
            A.out.vel[ib + j] = v;
            A.out.pid[ib + j] = p;
            fx += fq_of(v.x);
            fy += fq_of(v.y);
        }
        if (lane == 0) A.out.cnt[c] = n0;
    } else {
        // members: originals not removed (compacted), then records in this cell
        long long bx = 0, by = 0, ax = 0, ay = 0;
        int nOrig = 0;
        for (int j0 = 0; j0 < n0; j0 += 32) {
            const int j = j0 + lane;
            const bool in0 = j < n0;
            const bool keep = in0 && !(rm[j >> 5] & (1u << (j & 31)));
            const unsigned kb = __ballot_sync(0xffffffffu, keep);
            if (in0) {
                const float2 v = A.in.vel[ib + j];
                bx += fq_of(v.x);
                by += fq_of(v.y);
                if (keep) {
                    ax += fq_of(v.x);
                    ay += fq_of(v.y);
                    M.pidBuf[nOrig + __popc(kb & lanemask_lt())] = A.in.pid[ib + j];
                }
            }
            nOrig += __popc(kb);
        }
        int nAll = nOrig;
        for (int r0 = 0; r0 < Z.nrec; r0 += 32) {
            const int r = r0 + lane;
            const bool here = r < Z.nrec && M.recCur[r] == l;
            const unsigned hb = __ballot_sync(0xffffffffu, here);
            if (here) {
                const int src = M.recSrc[r];
                const float2 v = A.in.vel[(size_t)Z.gcell(src >> 7) * K + (src & 127)];
                ax += fq_of(v.x);
                ay += fq_of(v.y);
                const int slot = nAll + __popc(hb & lanemask_lt());
                if (slot < kFastMaxK) M.pidBuf[slot] = M.recPid[r];
            }
            nAll += __popc(hb);
        }
        bx = warp_sum_ll(bx);
        by = warp_sum_ll(by);
        ax = warp_sum_ll(ax);
        ay = warp_sum_ll(ay);
        __syncwarp();
        if (nAll > K) {
            if (lane == 0) raise_error(A.st, kErrBinCapacity, c);
            nAll = K;
        }
        const uint8_t f = M.flg[l];
        bool doCorr = A.P.momCorr != 0;
        if (doCorr && (f & kZSkip)) doCorr = false;
        if (doCorr && (f & kZRecv) && !(f & kZBB)) doCorr = false;
        long long shx = 0, shy = 0, remx = 0, remy = 0;
        if (doCorr && nAll > 0) {
            const long long dx = bx - ax, dy = by - ay;
            shx = floor_div_ll(dx, nAll);
            shy = floor_div_ll(dy, nAll);
            remx = dx - shx * nAll;
            remy = dy - shy * nAll;
        }
        // rank of a member by id among the cell's members (the remainder goes to the lowest)
        auto id_rank = [&](int p) {
            int r = 0;
            for (int i = 0; i < nAll; ++i) r += M.pidBuf[i] < p;
            return r;
        };
        int k = 0;
        for (int j0 = 0; j0 < n0; j0 += 32) {
            const int j = j0 + lane;
            const bool keep = j < n0 && !(rm[j >> 5] & (1u << (j & 31)));
            const unsigned kb = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int slot = k + __popc(kb & lanemask_lt());
                if (slot < K) {
                    const int p = A.in.pid[ib + j];
                    const float2 v = A.in.vel[ib + j];
                    long long qx = fq_of(v.x) + shx, qy = fq_of(v.y) + shy;
                    if (remx || remy) {
                        const int rk = id_rank(p);
                        if (rk < remx) ++qx;
                        if (rk < remy) ++qy;
                    }
                    A.out.off[ib + slot] = A.in.off[ib + j];
                    A.out.vel[ib + slot] = make_float2(fv_of(qx), fv_of(qy));
                    A.out.pid[ib + slot] = p;
                    fx += qx;
                    fy += qy;
                }
            }
            k += __popc(kb);
        }
        for (int r0 = 0; r0 < Z.nrec; r0 += 32) {
            const int r = r0 + lane;
            const bool here = r < Z.nrec && M.recCur[r] == l;
            const unsigned hb = __ballot_sync(0xffffffffu, here);
            if (here) {
                const int slot = k + __popc(hb & lanemask_lt());
                if (slot < K) {
                    const int src = M.recSrc[r];
                    const size_t s = (size_t)Z.gcell(src >> 7) * K + (src & 127);
                    const int p = M.recPid[r];
                    const float2 v = A.in.vel[s];
                    long long qx = fq_of(v.x) + shx, qy = fq_of(v.y) + shy;
                    if (remx || remy) {
                        const int rk = id_rank(p);
                        if (rk < remx) ++qx;
                        if (rk < remy) ++qy;
                    }
                    A.out.off[ib + slot] = M.recOff[r];
                    A.out.vel[ib + slot] = make_float2(fv_of(qx), fv_of(qy));
                    A.out.pid[ib + slot] = p;
                    fx += qx;
                    fy += qy;
                }
            }
            k += __popc(hb);
        }
        if (lane == 0) A.out.cnt[c] = nAll;
    }
    if (A.red) {
        fx = warp_sum_ll(fx);
        fy = warp_sum_ll(fy);
        if (lane == 0) A.red[c] = make_longlong2(fx, fy);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32 * kFastZoneWarps) k_fast_zone(FastZoneArgs A) {
    extern __shared__ __align__(16) char smem[];
    const int wib = threadIdx.x >> 5;
    const int z = blockIdx.x * kFastZoneWarps + wib;
    if (z >= A.nZones) return;
    FastZone Z;
    Z.A = &A;
    Z.lane = threadIdx.x & 31;
    Z.z = z;
    const int lane = Z.lane;
    const DevParams& P = A.P;
    const int4 R = A.rects[z];
    Z.x0 = R.x; Z.x1 = R.y; Z.y0 = R.z; Z.y1 = R.w;
    Z.TX = Z.x1 - Z.x0; Z.TY = Z.y1 - Z.y0; Z.nl = Z.TX * Z.TY; Z.WY = Z.TY + 4;
    Z.zseed = fhash(A.S->seed, (uint64_t)z, 0x5A4F4E45ULL + (uint64_t)A.pass);
    Z.op = 0;
    Z.nrec = 0;
    Z.failed = false;
    Z.movedDense = Z.movedSparse = 0;
    if (Z.nl > A.maxCells || (Z.TX + 4) * Z.WY > A.winCap || (Z.TX + 2) * (Z.TY + 2) > A.nsmCap) {
        if (lane == 0) raise_error(A.st, kErrZoneCapacity, z);
        return;
    }
    const size_t per = FastZoneMem::bytes(A.maxCells, A.winCap, A.nsmCap, A.recCap);
    Z.M.carve(smem + per * wib, A.maxCells, A.winCap, A.nsmCap, A.recCap);
    FastZoneMem& M = Z.M;
    // pass-input counts of the window (wrapped on periodic axes, -1 outside the domain)
    const int W = (Z.TX + 4) * Z.WY;
    for (int w = lane; w < W; w += 32) {
        int gx = Z.x0 - 2 + w / Z.WY, gy = Z.y0 - 2 + w % Z.WY;
        if (P.perx) gx = wrap_index(gx, P.Nx);
        if (P.pery) gy = wrap_index(gy, P.Ny);
        const bool ok = gx >= 0 && gx < P.Nx && gy >= 0 && gy < P.Ny;
        M.win[w] = ok ? (short)min(A.in.cnt[gy + P.Ny * gx], A.F.K) : (short)-1;
    }
    __syncwarp();
    for (int l = lane; l < Z.nl; l += 32) {
        M.n0[l] = (uint8_t)Z.cnt(l);
        M.flg[l] = 0;
        M.nrecv[l] = 0;
        M.rm[4 * l] = M.rm[4 * l + 1] = M.rm[4 * l + 2] = M.rm[4 * l + 3] = 0;
    }
    __syncwarp();
    // dense passes (src/zone_pass.cpp:708-781): cells above their high map, in random order
    for (int pass = 0; pass < P.maxPasses && !Z.failed; ++pass) {
        for (int l = lane; l < Z.nl; l += 32) {
            const bool bulk = Z.cnt(l) > 0;
            M.flg[l] = (uint8_t)((M.flg[l] & ~kZBulkD) | (bulk ? kZBulkD : 0));
        }
        __syncwarp();
        for (int i = lane; i < 128; i += 32) {
            uint32_t key = 0xFFFFFFFFu;
            if (i < Z.nl) {
                const bool bulk = M.flg[i] & kZBulkD;
                if ((double)Z.cnt(i) > Z.high_map(bulk))
                    key = ((uint32_t)fhash(Z.zseed, 0x44454EULL + (uint64_t)pass, (uint64_t)i) & 0xFFFFFF00u) | (uint32_t)i;
            }
            M.keys[i] = key;
        }
        warp_sort128(M.keys, lane);
        for (int q = 0; q < 128 && !Z.failed; ++q) {
            const uint32_t key = M.keys[q];
            if (key == 0xFFFFFFFFu) break;
            Z.dense_cell((int)(key & 0xFFu));
        }
        __syncwarp();
    }
    // sparse phase (src/zone_pass.cpp:783-854)
    if (!Z.failed) {
        for (int l = lane; l < Z.nl; l += 32) {
            const bool bulk = Z.cnt(l) > 0;
            M.flg[l] = (uint8_t)((M.flg[l] & ~kZBulkS) | (bulk ? kZBulkS : 0));
        }
        __syncwarp();
        Z.compute_nsm();
        for (int i = lane; i < 128; i += 32) {
            uint32_t key = 0xFFFFFFFFu;
            if (i < Z.nl) {
                const int cn = Z.cnt(i);
                if (cn > 0 && (double)cn < Z.low_map(true))
                    key = ((uint32_t)fhash(Z.zseed, 0x4C4F57ULL, (uint64_t)i) & 0xFFFFFF00u) | (uint32_t)i;
            }
            M.keys[i] = key;
        }
        warp_sort128(M.keys, lane);
        for (int q = 0; q < 128 && !Z.failed; ++q) {
            const uint32_t key = M.keys[q];
            if (key == 0xFFFFFFFFu) break;
            Z.sparse_cell((int)(key & 0xFFu));
        }
    }
    __syncwarp();
    // output with the momentum correction
    for (int l = 0; l < Z.nl; ++l) fast_zone_output_cell(Z, l);
    if (lane == 0) {
        if (Z.movedDense || Z.movedSparse) {
            atomicAdd(A.moved, Z.movedDense);
            atomicAdd(A.moved + 1, Z.movedSparse);
        }
        if (Z.failed) atomicAdd(A.recOverflow, 1);
    }
}

// ------------------------------------------------------------------ closure
// Per cell, from the exact sums: the reference fields of the step-start state (N, Ux, Uy, T,
// rho, Pkin, Pvir: src/common_grid.cpp:32-100) and pdriveRaw = Pkin + Pvir
// (src/liquid_closure.cpp:401-405); the red momenta, duRepair = (P_ref - P_red) / gamma and the
// beta_opt terms (:343-360) into cols (num term, den term).
__global__ void k_fast_closure_cells(DevParams P, const longlong4* __restrict__ ref, const longlong2* __restrict__ red,
                                     const int* __restrict__ redN, double* __restrict__ pdRaw, double* __restrict__ duRX,
                                     double* __restrict__ duRY, double* __restrict__ cols, float4* __restrict__ feat) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
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
    if (feat) feat[c] = make_float4((float)((double)n / P.gamma - 1.0), (float)uxr, (float)uyr, (float)n);
}

// EOS kick from the blended pressure drive (src/liquid_closure.cpp:243-295, :424-430) plus
// beta_applied * duRepair, rounded per cell to the grid (the pending kick of the next step).
// learned (nullable): per cell (duX, duY) of the learned closure replacing the EOS kick.
__global__ void k_fast_kick_cells(DevParams P, const double* __restrict__ pd, const double* __restrict__ duRX,
                                  const double* __restrict__ duRY, const double* __restrict__ numDen,
                                  const double* __restrict__ learnedX, const double* __restrict__ learnedY,
                                  int2* __restrict__ kick) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    const double beta = beta_applied(P, numDen[0], numDen[1]);
    double ex, ey;
    if (learnedX) {
        ex = learnedX[c];
        ey = learnedY[c];
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
    }
    const double dx = beta * duRX[c] + ex, dy = beta * duRY[c] + ey;
    kick[c] = make_int2((int)llrint(dx * kFastQ), (int)llrint(dy * kFastQ));
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
