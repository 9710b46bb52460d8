// One zone pass of the incompressible redistribution: one warp per zone.
//
// Reference: run_zone_pass_openmp -> run_zone_pass_snapshot_impl
// (src/zone_pass_openmp.cpp:34-172) running run_zone_kernel (src/zone_pass.cpp:669-973)
// on a private copy of the pass input for every zone, then merging zone by zone.
//
// What a zone kernel reads and writes (this is what makes one warp per zone exact):
//   - it moves particles only between cells of its own rectangle (targets and donors are
//     filtered to the zone: src/zone_pass.cpp:611,625,274,819);
//   - outside its rectangle it reads only cell counts of the pass input, up to two cells
//     away (3x3 smoothing of src/zone_pass.cpp:296-319 around the 4-neighbour gradient of
//     :375-411), which never change during the pass;
//   - the particle lists it needs are those of its own cells, in ascending particle id
//     (src/zone_pass.cpp:112-118), and their velocities from the pass input.
// The merge writes each particle from the LAST zone whose rectangle holds the particle's
// input cell (zone ids grow in merge order), i.e. from ownerMap[input cell]. Shifted layouts
// overlap (tiles start at 0 and at tile/2, src/zone_pass.cpp:160-221), so every zone
// processes its full rectangle but writes only the particles it owns, out of place.
//
// Warp discipline: every lane runs the same control flow with identical scalar values
// (the RNG stream is warp-uniform); lane-parallel sections are candidate evaluation,
// position sampling, list copies and the final per-particle writes. Shared-memory scalars
// written by lane 0 are followed by __syncwarp() before any lane reads them.
#pragma once

#include "common.cuh"

namespace mpcd_dev {

constexpr uint8_t kPMoved = 1, kPOwned = 2;
constexpr uint8_t kCRecv = 1, kCBulkBulk = 2, kCSkip = 4, kCBulkBefore = 8, kCChanged = 16, kCApply = 32;

struct ZoneArgs {
    DevParams P;
    const int4* rects;        // (xs, xe, ys, ye) per zone, zone id = index + 1
    const int* owner;         // ownerMap of the layout
    const uint64_t* start;    // cell index of the pass input (packed starts)
    const int* slots;
    const double2* xin;
    const double2* vin;
    double2* xout;
    double2* vout;
    int* cid;                 // standard-grid cell per slot; moved owned particles updated
    const uint64_t* seeds;    // seeded MT19937-64 state per zone (312 words each)
    int nZones;
    int maxCells, winCap, nlocCap, arenaCap;  // capacities of the per-zone working set
    int* overflow;            // zones left to the overflow kernel
    int* nOverflow;
    int2* zoneMoved;          // (dense, sparse) per zone
    double2* zoneCorr;        // (stats[4], stats[5]) per zone
    DevStatus* st;
};

// Working set of one zone; carved from shared memory (fast path) or global memory.
template <typename Idx>
struct ZoneMem {
    uint64_t* mt;      // 2 * 312
    double* lowA;      // maxCells (reused as du.x at the end)
    double* highA;     // maxCells (reused as du.y)
    double* nsm;       // (TX+2)(TY+2) <= winCap (reused as dU2)
    int* slot;         // nlocCap
    int* win;          // winCap: pass-input counts around the zone (-1 = outside)
    int* cnt;          // maxCells: live counts
    int* cnt0;         // maxCells
    int* base0;        // maxCells: first local index of the cell's input list
    int* abase;        // maxCells: list storage start in the arena
    int* head;         // maxCells
    int* len;          // maxCells
    int* cap;          // maxCells
    Idx* arena;        // arenaCap
    Idx* scratch;      // nlocCap: compaction buffer, then final cell per local particle
    uint8_t* pflags;   // nlocCap
    uint8_t* cflags;   // maxCells
    Idx* list;         // maxCells: dense / low cell order
    int* small;        // 128 ints: candidates, targets, receivers, donors
    double* smallD;    // 16 doubles: donor scores

    __host__ __device__ static size_t bytes(int maxCells, int winCap, int nlocCap, int arenaCap) {
        size_t b = 0;
        auto add = [&](size_t n, size_t a) { b = (b + a - 1) / a * a + n; };
        add(2 * kMtN * 8, 8);
        add((size_t)maxCells * 8, 8);
        add((size_t)maxCells * 8, 8);
        add((size_t)winCap * 8, 8);
        add((size_t)nlocCap * 4, 4);
        add((size_t)winCap * 4, 4);
        for (int k = 0; k < 7; ++k) add((size_t)maxCells * 4, 4);
        add((size_t)arenaCap * sizeof(Idx), sizeof(Idx));
        add((size_t)nlocCap * sizeof(Idx), sizeof(Idx));
        add((size_t)nlocCap, 1);
        add((size_t)maxCells, 1);
        add((size_t)maxCells * sizeof(Idx), sizeof(Idx));
        add(128 * 4, 4);
        add(16 * 8, 8);
        return (b + 15) / 16 * 16;
    }
    __device__ void carve(char* base, int maxCells, int winCap, int nlocCap, int arenaCap) {
        size_t b = 0;
        auto take = [&](size_t n, size_t a) {
            b = (b + a - 1) / a * a;
            char* p = base + b;
            b += n;
            return p;
        };
        mt = (uint64_t*)take(2 * kMtN * 8, 8);
        lowA = (double*)take((size_t)maxCells * 8, 8);
        highA = (double*)take((size_t)maxCells * 8, 8);
        nsm = (double*)take((size_t)winCap * 8, 8);
        slot = (int*)take((size_t)nlocCap * 4, 4);
        win = (int*)take((size_t)winCap * 4, 4);
        cnt = (int*)take((size_t)maxCells * 4, 4);
        cnt0 = (int*)take((size_t)maxCells * 4, 4);
        base0 = (int*)take((size_t)maxCells * 4, 4);
        abase = (int*)take((size_t)maxCells * 4, 4);
        head = (int*)take((size_t)maxCells * 4, 4);
        len = (int*)take((size_t)maxCells * 4, 4);
        cap = (int*)take((size_t)maxCells * 4, 4);
        arena = (Idx*)take((size_t)arenaCap * sizeof(Idx), sizeof(Idx));
        scratch = (Idx*)take((size_t)nlocCap * sizeof(Idx), sizeof(Idx));
        pflags = (uint8_t*)take((size_t)nlocCap, 1);
        cflags = (uint8_t*)take((size_t)maxCells, 1);
        list = (Idx*)take((size_t)maxCells * sizeof(Idx), sizeof(Idx));
        small = (int*)take(128 * 4, 4);
        smallD = (double*)take(16 * 8, 8);
    }
};

// Scalar (warp-uniform) state of one zone.
template <typename Idx>
struct ZoneState {
    ZoneMem<Idx> M;
    WarpMt rng;
    const ZoneArgs* A;
    int lane, zone;
    int xs, xe, ys, ye, TX, TY, nl, WY;  // rectangle, sizes, window height
    int nloc, arenaTop;
    int movedDense, movedSparse;
    bool failed;

    __device__ __forceinline__ const DevParams& P() const { return A->P; }
    __device__ __forceinline__ bool in_zone(int ix, int iy) const { return ix >= xs && ix < xe && iy >= ys && iy < ye; }
    __device__ __forceinline__ int loc(int ix, int iy) const { return (ix - xs) * TY + (iy - ys); }
    __device__ __forceinline__ int gx_of(int l) const { return xs + l / TY; }
    __device__ __forceinline__ int gy_of(int l) const { return ys + l % TY; }

    // pass-input or live count of an in-range cell within two cells of the zone
    __device__ __forceinline__ int cnt_at(int ix, int iy) const {
        if (in_zone(ix, iy)) return M.cnt[loc(ix, iy)];
        int wx = ix - (xs - 2), wy = iy - (ys - 2);
        if (wx < 0) wx += P().Nx;
        else if (wx >= TX + 4) wx -= P().Nx;
        if (wy < 0) wy += P().Ny;
        else if (wy >= WY) wy -= P().Ny;
        return M.win[wx * WY + wy];
    }
    __device__ __forceinline__ int nsm_index(int ix, int iy) const {
        int lx = ix - (xs - 1), ly = iy - (ys - 1);
        if (lx < 0) lx += P().Nx;
        if (lx >= TX + 2) lx -= P().Nx;
        if (ly < 0) ly += P().Ny;
        if (ly >= TY + 2) ly -= P().Ny;
        return lx * (TY + 2) + ly;
    }
    // src/zone_pass.cpp:246-261
    __device__ __forceinline__ bool shift_index(int iy, int ix, int dy, int dx, int& jy, int& jx) const {
        jy = iy + dy;
        if (P().pery) jy = wrap_index(jy, P().Ny);
        else if (jy < 0 || jy >= P().Ny) return false;
        jx = ix + dx;
        if (P().perx) jx = wrap_index(jx, P().Nx);
        else if (jx < 0 || jx >= P().Nx) return false;
        return true;
    }
    // src/zone_pass.cpp:229-244 -> index into the 5x5 step tables (-1 if outside)
    __device__ __forceinline__ int step_index(int sx, int sy, int tx, int ty, int& ddx, int& ddy) const {
        int a = tx - sx, b = ty - sy;
        if (P().perx) {
            if (a > P().Nx / 2) a -= P().Nx;
            if (a < -P().Nx / 2) a += P().Nx;
        }
        if (P().pery) {
            if (b > P().Ny / 2) b -= P().Ny;
            if (b < -P().Ny / 2) b += P().Ny;
        }
        ddx = a;
        ddy = b;
        if (a < -2 || a > 2 || b < -2 || b > 2) return -1;
        return (a + 2) + 5 * (b + 2);
    }

    // ------------------------------------------------------------------ smoothing, maps
    __device__ void compute_nsm() {
        const DevParams& p = P();
        const int GX = TX + 2, GY = TY + 2;
        for (int g = lane; g < GX * GY; g += kWarp) {
            int ix = xs - 1 + g / GY, iy = ys - 1 + g % GY;
            if (p.perx) ix = wrap_index(ix, p.Nx);
            if (p.pery) iy = wrap_index(iy, p.Ny);
            double val = 0.0;
            if (ix >= 0 && ix < p.Nx && iy >= 0 && iy < p.Ny) {
                double acc = 0.0, ws = 0.0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int jy = iy + dy, jx = ix + dx;
                        if (jy < 0 || jy >= p.Ny || jx < 0 || jx >= p.Nx) continue;
                        const double w = ((dx == 0) ? 2.0 : 1.0) * ((dy == 0) ? 2.0 : 1.0) * 0.0625;
                        acc = __dadd_rn(acc, __dmul_rn(w, (double)cnt_at(jx, jy)));
                        ws = __dadd_rn(ws, w);
                    }
                val = __ddiv_rn(acc, smax(ws, 1e-30));
            }
            M.nsm[g] = val;
        }
        __syncwarp();
    }

    // threshold maps of zone cells (src/zone_pass.cpp:321-345, :715-725) + bulk flags
    __device__ void build_maps() {
        const DevParams& p = P();
        for (int l = lane; l < nl; l += kWarp) {
            double f = 1.0;
            if (p.useLFF) {
                const double fraw = __ddiv_rn(M.nsm[nsm_index(gx_of(l), gy_of(l))], smax(p.gamma, 1e-12));
                const double g = __dmul_rn(p.fluidFracGain, fraw);
                f = (g < 0.0) ? 0.0 : ((1.0 < g) ? 1.0 : g);
            }
            const double gl = __dmul_rn(p.gamma, f);
            double lo = smax(__dmul_rn(p.lowFrac, gl), p.lowThrFloor);
            double hi = smax(__dmul_rn(p.highFrac, gl), p.highThrFloor);
            const bool bulk = M.cnt[l] > 0;
            if (bulk) {
                lo = p.lowThrBulk;
                hi = p.highThr;
            }
            M.lowA[l] = lo;
            M.highA[l] = hi;
            M.cflags[l] = (uint8_t)((M.cflags[l] & ~kCBulkBefore) | (bulk ? kCBulkBefore : 0));
        }
        __syncwarp();
    }

    // ordered list of zone cells satisfying pred (ascending cell index); returns the count
    template <typename Pred>
    __device__ int collect(Pred pred) {
        int total = 0;
        for (int b = 0; b < nl; b += kWarp) {
            const int l = b + lane;
            const bool ok = (l < nl) && pred(l);
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) M.list[total + __popc(m & lanemask_lt())] = (Idx)l;
            total += __popc(m);
        }
        __syncwarp();
        return total;
    }

    // ------------------------------------------------------------------ arena lists
    // tightly repack every list into the arena (rare: only when the arena top is reached)
    __device__ void compact() {
        int off = 0;
        for (int l = 0; l < nl; ++l) {
            const int a = M.abase[l] + M.head[l], n = M.len[l];
            for (int j = lane; j < n; j += kWarp) M.scratch[off + j] = M.arena[a + j];
            off += n;
        }
        __syncwarp();
        off = 0;
        for (int l = 0; l < nl; ++l) {
            const int n = M.len[l];
            for (int j = lane; j < n; j += kWarp) M.arena[off + j] = M.scratch[off + j];
            if (lane == 0) {
                M.abase[l] = off;
                M.head[l] = 0;
                M.cap[l] = n;
            }
            off += n;
        }
        arenaTop = off;
        __syncwarp();
    }

    // make room to append `extra` entries to list t (may relocate or repack lists)
    __device__ bool ensure_room(int t, int extra) {
        if (M.head[t] + M.len[t] + extra <= M.cap[t]) return true;
        const int want = M.len[t] + extra + 8;
        if (arenaTop + want > A->arenaCap) {
            compact();
            if (arenaTop + want > A->arenaCap) {
                if (lane == 0) raise_error(A->st, kErrZoneCapacity, zone);
                failed = true;
                return false;
            }
        }
        const int a = M.abase[t] + M.head[t], n = M.len[t];
        for (int j = lane; j < n; j += kWarp) M.arena[arenaTop + j] = M.arena[a + j];
        __syncwarp();
        if (lane == 0) {
            M.abase[t] = arenaTop;
            M.head[t] = 0;
            M.cap[t] = want;
        }
        arenaTop += want;
        __syncwarp();
        return true;
    }

    // Move `nt` particles from list position srcPos (arena index, read before any
    // relocation) into cell t, drawing their positions with sample_in_cell
    // (src/zone_pass.cpp:280-294): per particle U for x then U for y.
    __device__ bool move_into(int s, int srcOff, int nt, int t) {
        if (!ensure_room(t, nt)) return false;
        const DevParams& p = P();
        const int tix = gx_of(t), tiy = gy_of(t);
        const double x0 = __dmul_rn((double)tix, p.dx), y0 = __dmul_rn((double)tiy, p.dy);
        const int src = M.abase[s] + M.head[s] + srcOff;
        const int dst = M.abase[t] + M.head[t] + M.len[t];
        for (int q0 = 0; q0 < nt; q0 += 128) {
            const int c = min(128, nt - q0);
            rng.ensure(2 * c);
            for (int q = q0 + lane; q < q0 + c; q += kWarp) {
                const int k = (int)M.arena[src + q];
                const double px = __dadd_rn(x0, __dmul_rn(p.dx, canon(rng.peek(2 * (q - q0)))));
                const double py = __dadd_rn(y0, __dmul_rn(p.dy, canon(rng.peek(2 * (q - q0) + 1))));
                const uint8_t fl = M.pflags[k];
                if (fl & kPOwned) {
                    const int sl = M.slot[k];
                    A->xout[sl] = make_double2(px, py);
                    A->cid[sl] = cell_of(px, py, p);
                }
                M.pflags[k] = fl | kPMoved;
                M.arena[dst + q] = (Idx)k;
            }
            rng.consume(2 * c);
            __syncwarp();
        }
        if (lane == 0) {
            M.len[t] += nt;
            M.cnt[t] += nt;
        }
        __syncwarp();
        return true;
    }

    __device__ __forceinline__ void push_recv(int* recv, int& nrecv, int c) {
        bool seen = false;
        for (int q = 0; q < nrecv; ++q) seen |= (recv[q] == c);
        if (!seen) {
            if (lane == 0) recv[nrecv] = c;
            ++nrecv;
        }
        __syncwarp();
    }

    // update_transfer_correction_masks (src/zone_pass.cpp:492-525), forceSkip = false
    __device__ void update_masks(int src, const int* recv, int nrecv) {
        // touched = unique_stable([src] + recv); src is never a receiver here
        bool allBulk = (M.cflags[src] & kCBulkBefore) != 0;
        for (int q = 0; q < nrecv; ++q) allBulk &= (M.cflags[recv[q]] & kCBulkBefore) != 0;
        if (lane <= nrecv) {
            const int c = (lane == 0) ? src : recv[lane - 1];
            uint8_t f = M.cflags[c];
            if (allBulk) f |= kCBulkBulk;
            else f = (uint8_t)((f | kCSkip) & ~kCBulkBulk);
            M.cflags[c] = f;
        }
        __syncwarp();
    }

    // ------------------------------------------------------------------ dense phase
    // admissible_dense_targets_rangeR (src/zone_pass.cpp:413-434) + the zone filter;
    // writes the ordered candidates to cand and returns their number
    __device__ int admissible(int l, const double* map, int* cand) {
        const int ix = gx_of(l), iy = gy_of(l);
        int nb = -1;
        if (lane < 24) {
            const int kk = (lane < 12) ? lane : lane + 1;
            const int dy = kk / 5 - 2, dx = kk % 5 - 2;
            int jy, jx;
            if (shift_index(iy, ix, dy, dx, jy, jx) && in_zone(jx, jy)) {
                const int t = loc(jx, jy);
                if ((double)M.cnt[t] < map[t]) nb = t;
            }
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, nb >= 0);
        const unsigned same = __match_any_sync(0xffffffffu, nb >= 0 ? nb : -1 - lane);
        const bool keep = (nb >= 0) && ((same & m0 & lanemask_lt()) == 0);
        const unsigned mk = __ballot_sync(0xffffffffu, keep);
        if (keep) cand[__popc(mk & lanemask_lt())] = nb;
        __syncwarp();
        return __popc(mk);
    }

    // rank_dense_targets_unified (src/zone_pass.cpp:436-490) with inwardWeight = 0:
    // per-bin insertion sort (stable) on (-deficit, cnt, cheb, dist2, U01), round robin
    __device__ int rank_dense(int l, const int* cand, int m, const double* map, int* T) {
        if (m == 0) return 0;
        const DevParams& p = P();
        const int startBin = (int)rng.uint_in(1, 8) - 1;
        rng.ensure(m);
        int nb = -1, bin = -1, key2 = 0, cheb = 0, d2 = 0;
        double dneg = 0.0, tie = 0.0;
        if (lane < m) {
            nb = cand[lane];
            int ddx, ddy;
            const int idx = step_index(gx_of(l), gy_of(l), gx_of(nb), gy_of(nb), ddx, ddy);
            if (idx < 0) {
                raise_error(A->st, kErrTableRange, zone);
                bin = 0;
            } else {
                bin = p.atanBin[idx];
            }
            dneg = -smax(0.0, __dsub_rn(map[nb], (double)M.cnt[nb]));
            key2 = M.cnt[nb];
            cheb = max(abs(ddx), abs(ddy));
            d2 = ddx * ddx + ddy * ddy;
            tie = canon(rng.peek(lane));
        }
        rng.consume(m);
        int r = 0;
        for (int j = 0; j < m; ++j) {
            const int bj = __shfl_sync(0xffffffffu, bin, j);
            const double dj = __shfl_sync(0xffffffffu, dneg, j);
            const int cj = __shfl_sync(0xffffffffu, key2, j);
            const int hj = __shfl_sync(0xffffffffu, cheb, j);
            const int ej = __shfl_sync(0xffffffffu, d2, j);
            const double tj = __shfl_sync(0xffffffffu, tie, j);
            if (lane < m && j != lane && bj == bin) {
                bool less, eq = false;
                if (dj != dneg) less = dj < dneg;
                else if (cj != key2) less = cj < key2;
                else if (hj != cheb) less = hj < cheb;
                else if (ej != d2) less = ej < d2;
                else if (tj != tie) less = tj < tie;
                else { less = false; eq = true; }
                if (less || (eq && j < lane)) ++r;
            }
        }
        int pos = 0;
        for (int b = 0; b < 8; ++b) {
            const int cb = __popc(__ballot_sync(0xffffffffu, lane < m && bin == b));
            if (lane < m) {
                pos += min(cb, r);
                const int rb = (b - startBin + 8) & 7, rq = (bin - startBin + 8) & 7;
                if (rb < rq && cb > r) ++pos;
            }
        }
        if (lane < m) T[pos] = nb;
        __syncwarp();
        return m;
    }

    // spread_particles_from_dense_source_round_robin (src/zone_pass.cpp:527-589)
    __device__ int spread(int s, const int* T, int nT, const double* map, int needOut, int* recv, int& nrecv) {
        if (needOut <= 0 || nT == 0) return 0;
        const int srcLen = M.len[s];
        if (srcLen == 0) return 0;
        int taken = 0, moved = 0;
        while (needOut > 0 && taken < srcLen) {
            bool progressed = false;
            for (int kk = 0; kk < nT; ++kk) {
                int defj = 0;
                if (lane < nT) {
                    const int t = T[lane];
                    defj = max(0, (int)floor(__dsub_rn(map[t], (double)M.cnt[t])));
                }
                const unsigned pm = __ballot_sync(0xffffffffu, lane < nT && defj > 0);
                const int deficit = __shfl_sync(0xffffffffu, defj, kk);
                if (deficit <= 0) continue;
                const int remaining = __popc(pm >> kk);
                const int quota = max(1, (int)ceil(__ddiv_rn((double)needOut, (double)max(1, remaining))));
                const int nt = max(1, min(min(quota, deficit), min(needOut, srcLen - taken)));
                const int t = T[kk];
                if (t == s) {
                    if (lane == 0) raise_error(A->st, kErrTargetIsSource, zone);
                    failed = true;
                    return moved;
                }
                if (!move_into(s, taken, nt, t)) return moved;
                push_recv(recv, nrecv, t);
                taken += nt;
                moved += nt;
                needOut -= nt;
                progressed = true;
                if (needOut <= 0 || taken >= srcLen) break;
            }
            if (!progressed) break;
        }
        if (moved > 0 && lane == 0) {
            M.head[s] += taken;
            M.len[s] -= taken;
            M.cnt[s] = M.len[s];
        }
        __syncwarp();
        return moved;
    }

    // one dense cell (src/zone_pass.cpp:734-753 calling :591-634)
    __device__ void dense_cell(int l) {
        int* cand = M.small;        // 24
        int* T = M.small + 32;      // 24
        int* recv = M.small + 64;   // <= 24 unique
        const int ncc = M.cnt[l];
        if (ncc <= 0) return;
        const double hl = M.highA[l];
        if ((double)ncc <= hl) return;
        int nrecv = 0, moved = 0;
        const int needOut = max(0, (int)ceil(__dsub_rn((double)M.cnt[l], hl)));
        if (needOut > 0) {
            int m = admissible(l, M.lowA, cand);
            int nT = rank_dense(l, cand, m, M.lowA, T);
            moved += spread(l, T, nT, M.lowA, needOut, recv, nrecv);
            if (failed) return;
            const int rem = max(0, (int)ceil(__dsub_rn((double)M.cnt[l], hl)));
            if (rem > 0) {
                m = admissible(l, M.highA, cand);
                nT = rank_dense(l, cand, m, M.highA, T);
                moved += spread(l, T, nT, M.highA, rem, recv, nrecv);
                if (failed) return;
            }
        }
        if (lane < nrecv) M.cflags[recv[lane]] |= (kCRecv | kCChanged);
        if (lane == 0 && moved > 0) M.cflags[l] |= kCChanged;
        __syncwarp();
        update_masks(l, recv, nrecv);
        movedDense += moved;
    }

    // ------------------------------------------------------------------ sparse phase
    // inward_direction_from_local_gradient (src/zone_pass.cpp:375-411)
    __device__ void inward(int l, double& gx, double& gy) const {
        const DevParams& p = P();
        const int ix = gx_of(l), iy = gy_of(l);
#define NS(jx, jy) M.nsm[nsm_index((jx), (jy))]
        if (p.perx) gx = __dmul_rn(0.5, __dsub_rn(NS(wrap_index(ix + 1, p.Nx), iy), NS(wrap_index(ix - 1, p.Nx), iy)));
        else if (ix == 0) gx = __dsub_rn(NS(ix + 1, iy), NS(ix, iy));
        else if (ix == p.Nx - 1) gx = __dsub_rn(NS(ix, iy), NS(ix - 1, iy));
        else gx = __dmul_rn(0.5, __dsub_rn(NS(ix + 1, iy), NS(ix - 1, iy)));
        if (p.pery) gy = __dmul_rn(0.5, __dsub_rn(NS(ix, wrap_index(iy + 1, p.Ny)), NS(ix, wrap_index(iy - 1, p.Ny))));
        else if (iy == 0) gy = __dsub_rn(NS(ix, iy + 1), NS(ix, iy));
        else if (iy == p.Ny - 1) gy = __dsub_rn(NS(ix, iy), NS(ix, iy - 1));
        else gy = __dmul_rn(0.5, __dsub_rn(NS(ix, iy + 1), NS(ix, iy - 1)));
#undef NS
    }

    // one sparse cell (src/zone_pass.cpp:804-854)
    __device__ void sparse_cell(int l) {
        const DevParams& p = P();
        int* don = M.small + 96;  // <= 8
        const int ncc = M.cnt[l];
        if (ncc <= 0) return;
        if (M.len[l] == 0) return;
        // local_neighbors_in_zone, range 1 (src/zone_pass.cpp:263-278)
        const int ix = gx_of(l), iy = gy_of(l);
        int nb = -1;
        if (lane < 8) {
            const int kk = (lane < 4) ? lane : lane + 1;
            const int dy = kk / 3 - 1, dx = kk % 3 - 1;
            int jy, jx;
            if (shift_index(iy, ix, dy, dx, jy, jx) && in_zone(jx, jy)) nb = loc(jx, jy);
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, nb >= 0);
        if (m0 == 0) return;
        const unsigned same = __match_any_sync(0xffffffffu, nb >= 0 ? nb : -1 - lane);
        const bool uniq = (nb >= 0) && ((same & m0 & lanemask_lt()) == 0);
        const int lowInt = p.lowThrBulkInt;
        int need = max(0, lowInt - ncc);
        if (need <= 0) return;
        const bool isDonor = uniq && M.cnt[nb] > lowInt;
        const unsigned md = __ballot_sync(0xffffffffu, isDonor);
        const int nd = __popc(md);
        if (nd == 0) return;
        if (isDonor) don[__popc(md & lanemask_lt())] = nb;
        __syncwarp();
        // rank_admissible_neighbors_inward (src/zone_pass.cpp:636-667)
        double gx, gy;
        inward(l, gx, gy);
        warp_shuffle(don, nd, rng, lane);
        const double ndir = mpcd_dd::hypot_cr(gx, gy);
        PolarNormal N;
        N.reset();
        double* score = M.smallD;
        for (int k = 0; k < nd; ++k) {
            const int d = don[k];
            int ddx, ddy;
            const int idx = step_index(ix, iy, gx_of(d), gy_of(d), ddx, ddy);
            const double nstep = (idx >= 0) ? p.hypotTab[idx] : 0.0;
            double align = 0.0;
            if (ndir >= 1e-14 && nstep >= 1e-14)
                align = __ddiv_rn(__dadd_rn(__dmul_rn((double)ddx, gx), __dmul_rn((double)ddy, gy)), __dmul_rn(ndir, nstep));
            const double noise = __dmul_rn(1e-9, N.next(rng));
            const double sc = __dadd_rn(__dadd_rn(__dmul_rn(100.0, align), M.nsm[nsm_index(gx_of(d), gy_of(d))]), noise);
            if (lane == 0) score[k] = sc;
        }
        __syncwarp();
        if (lane == 0) {  // stable insertion sort, descending
            for (int i = 1; i < nd; ++i) {
                const double sv = score[i];
                const int ov = don[i];
                int j = i;
                while (j > 0 && sv > score[j - 1]) {
                    score[j] = score[j - 1];
                    don[j] = don[j - 1];
                    --j;
                }
                score[j] = sv;
                don[j] = ov;
            }
        }
        __syncwarp();
        for (int k = 0; k < nd; ++k) {
            const int d = don[k];
            const int ld = M.len[d];
            if (ld == 0) continue;
            const int avail = M.cnt[d] - lowInt;
            if (avail <= 0) continue;
            const int nt = min(min(need, avail), ld);
            if (nt <= 0) continue;
            warp_shuffle(M.arena + M.abase[d] + M.head[d], ld, rng, lane);
            if (!move_into(d, 0, nt, l)) return;
            if (lane == 0) {
                M.head[d] += nt;
                M.len[d] -= nt;
                M.cnt[d] = M.len[d];
                M.cflags[l] |= (kCRecv | kCChanged);
                M.cflags[d] |= kCChanged;
            }
            __syncwarp();
            int one = l;
            update_masks(d, &one, 1);
            movedSparse += nt;
            need -= nt;
            if (need <= 0) break;
        }
    }
};

// ------------------------------------------------------------------ the zone body
template <typename Idx>
__device__ void zone_body(const ZoneArgs& A, int z, char* mem, bool overflowPath) {
    ZoneState<Idx> S;
    S.A = &A;
    S.lane = threadIdx.x & 31;
    S.zone = z;
    S.failed = false;
    S.movedDense = S.movedSparse = 0;
    const int lane = S.lane;
    const DevParams& p = A.P;
    const int4 R = A.rects[z];
    S.xs = R.x; S.xe = R.y; S.ys = R.z; S.ye = R.w;
    S.TX = S.xe - S.xs; S.TY = S.ye - S.ys; S.nl = S.TX * S.TY; S.WY = S.TY + 4;
    const int W = (S.TX + 4) * S.WY;
    if (S.nl > A.maxCells || W > A.winCap || (S.TX + 2) * (S.TY + 2) > A.winCap) {
        if (!overflowPath && lane == 0) A.overflow[atomicAdd(A.nOverflow, 1)] = z;
        if (overflowPath && lane == 0) raise_error(A.st, kErrZoneCapacity, z);
        return;
    }
    S.M.carve(mem, A.maxCells, A.winCap, A.nlocCap, A.arenaCap);
    ZoneMem<Idx>& M = S.M;
    // pass-input counts around the zone
    for (int w = lane; w < W; w += kWarp) {
        int ix = S.xs - 2 + w / S.WY, iy = S.ys - 2 + w % S.WY;
        if (p.perx) ix = wrap_index(ix, p.Nx);
        if (p.pery) iy = wrap_index(iy, p.Ny);
        int c = -1;
        if (ix >= 0 && ix < p.Nx && iy >= 0 && iy < p.Ny) {
            const int cc = iy + p.Ny * ix;
            c = (int)((uint32_t)A.start[cc + 1] - (uint32_t)A.start[cc]);
        }
        M.win[w] = c;
    }
    __syncwarp();
    // zone cell counts and their prefix (local particle numbering in input order)
    int total = 0;
    for (int b = 0; b < S.nl; b += kWarp) {
        const int l = b + lane;
        int c = 0;
        if (l < S.nl) c = M.win[(l / S.TY + 2) * S.WY + (l % S.TY + 2)];
        int x = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (l < S.nl) {
            M.cnt0[l] = c;
            M.cnt[l] = c;
            M.base0[l] = total + x - c;
            M.len[l] = c;
            M.head[l] = 0;
            M.cflags[l] = 0;
        }
        total += __shfl_sync(0xffffffffu, x, 31);
    }
    S.nloc = total;
    if (total > A.nlocCap || total > A.arenaCap) {
        if (!overflowPath && lane == 0) A.overflow[atomicAdd(A.nOverflow, 1)] = z;
        if (overflowPath && lane == 0) raise_error(A.st, kErrZoneCapacity, z);
        return;
    }
    __syncwarp();
    for (int l = lane; l < S.nl; l += kWarp) {
        M.abase[l] = M.base0[l];
        M.cap[l] = M.cnt0[l];
    }
    S.arenaTop = total;
    // slots of the zone's particles: one contiguous run of the cell index per zone column
    for (int col = 0; col < S.TX; ++col) {
        const int c0 = S.ys + p.Ny * (S.xs + col);
        const int g0 = (int)(uint32_t)A.start[c0], g1 = (int)(uint32_t)A.start[c0 + S.TY];
        const int b0 = M.base0[col * S.TY];
        for (int j = lane; j < g1 - g0; j += kWarp) M.slot[b0 + j] = A.slots[g0 + j];
    }
    for (int k = lane; k < total; k += kWarp) M.arena[k] = (Idx)k;
    __syncwarp();
    for (int l = 0; l < S.nl; ++l) {
        const int c = S.gy_of(l) + p.Ny * S.gx_of(l);
        const uint8_t fl = (A.owner[c] == z + 1) ? kPOwned : 0;
        for (int j = lane; j < M.cnt0[l]; j += kWarp) M.pflags[M.base0[l] + j] = fl;
    }
    for (int i = lane; i < kMtN; i += kWarp) M.mt[i] = A.seeds[(size_t)z * kMtN + i];
    __syncwarp();
    S.rng.buf = M.mt;
    S.rng.init_from_seeded(lane);

    // dense passes (src/zone_pass.cpp:708-781)
    for (int pass = 0; pass < p.maxPasses && !S.failed; ++pass) {
        if (p.useLFF) S.compute_nsm();
        S.build_maps();
        const int nd = S.collect([&](int l) { return (double)M.cnt[l] > M.highA[l]; });
        warp_shuffle(M.list, nd, S.rng, lane);
        for (int q = 0; q < nd && !S.failed; ++q) S.dense_cell((int)M.list[q]);
    }
    // sparse phase (src/zone_pass.cpp:783-854)
    if (!S.failed) {
        S.compute_nsm();
        S.build_maps();
        const int nlow = S.collect([&](int l) { return M.cnt[l] > 0 && (double)M.cnt[l] < M.lowA[l]; });
        warp_shuffle(M.list, nlow, S.rng, lane);
        for (int q = 0; q < nlow && !S.failed; ++q) S.sparse_cell((int)M.list[q]);
    }
    if (S.failed) return;

    // momentum correction (src/zone_pass.cpp:870-922)
    double* dux = M.lowA;
    double* duy = M.highA;
    double* du2 = M.nsm;
    for (int l = lane; l < S.nl; l += kWarp) {
        double d2 = 0.0, ux = 0.0, uy = 0.0;
        uint8_t f = M.cflags[l] & ~kCApply;
        const int n = M.len[l];
        if ((f & kCChanged) && n > 0) {
            double bx = 0.0, by = 0.0, axs = 0.0, ays = 0.0;
            for (int j = 0; j < M.cnt0[l]; ++j) {
                const double2 w = A.vin[M.slot[M.base0[l] + j]];
                bx = __dadd_rn(bx, w.x);
                by = __dadd_rn(by, w.y);
            }
            const int a = M.abase[l] + M.head[l];
            for (int j = 0; j < n; ++j) {
                const double2 w = A.vin[M.slot[(int)M.arena[a + j]]];
                axs = __dadd_rn(axs, w.x);
                ays = __dadd_rn(ays, w.y);
            }
            ux = __ddiv_rn(__dsub_rn(bx, axs), (double)n);
            uy = __ddiv_rn(__dsub_rn(by, ays), (double)n);
            d2 = __dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy));
            bool doCorr = p.momCorr != 0;
            if (doCorr && (f & kCSkip)) doCorr = false;
            if (doCorr && (f & kCRecv) && !(f & kCBulkBulk)) doCorr = false;
            if (doCorr && (ux != 0.0 || uy != 0.0)) f |= kCApply;
        }
        dux[l] = ux;
        duy[l] = uy;
        du2[l] = d2;
        M.cflags[l] = f;
    }
    __syncwarp();
    // zone stats[4], stats[5] in ascending cell order (src/zone_pass.cpp:911-922)
    if (lane == 0) {
        double acc = 0.0, mx = 0.0;
        int cntDU = 0;
        for (int l = 0; l < S.nl; ++l) {
            const double d2 = du2[l];
            mx = smax(mx, sqrt(d2));
            if (d2 > 0.0) {
                acc = __dadd_rn(acc, d2);
                ++cntDU;
            }
        }
        A.zoneCorr[z] = make_double2((cntDU > 0) ? sqrt(__ddiv_rn(acc, (double)cntDU)) : 0.0, (cntDU > 0) ? mx : 0.0);
        A.zoneMoved[z] = make_int2(S.movedDense, S.movedSparse);
    }
    // final cell of every local particle
    for (int l = lane; l < S.nl; l += kWarp) {
        const int a = M.abase[l] + M.head[l];
        for (int j = 0; j < M.len[l]; ++j) M.scratch[(int)M.arena[a + j]] = (Idx)l;
    }
    __syncwarp();
    // owned particles: corrected velocities, unmoved positions copied
    for (int k = lane; k < S.nloc; k += kWarp) {
        const uint8_t fl = M.pflags[k];
        if (!(fl & kPOwned)) continue;
        const int sl = M.slot[k];
        const int fc = (int)M.scratch[k];
        double2 w = A.vin[sl];
        if (M.cflags[fc] & kCApply) w = make_double2(__dadd_rn(w.x, dux[fc]), __dadd_rn(w.y, duy[fc]));
        A.vout[sl] = w;
        if (!(fl & kPMoved)) A.xout[sl] = A.xin[sl];
    }
}

__global__ void __launch_bounds__(32) k_zone_pass(ZoneArgs A) {
    extern __shared__ __align__(16) char smem[];
    const int z = blockIdx.x;
    if (z >= A.nZones) return;
    zone_body<uint16_t>(A, z, smem, false);
}

// zones that did not fit the shared-memory working set, one at a time per block, with a
// global-memory working set per block
__global__ void __launch_bounds__(32) k_zone_overflow(ZoneArgs A, char* gmem, size_t perBlock) {
    const int nov = *A.nOverflow;
    for (int i = blockIdx.x; i < nov; i += gridDim.x) zone_body<uint32_t>(A, A.overflow[i], gmem + perBlock * blockIdx.x, true);
}

// Seeded MT19937-64 state of every zone: seed = seedBase + 104729 (iz + 1)
// (src/zone_pass_openmp.cpp:78). One thread per zone runs the sequential seeding
// recurrence; states are staged in shared memory and written zone-major, coalesced.
constexpr int kSeedZonesPerBlock = 16;
__global__ void __launch_bounds__(kSeedZonesPerBlock * 2) k_zone_seeds(uint64_t seedBase, int nZones, uint64_t* out) {
    __shared__ uint64_t st[kSeedZonesPerBlock][kMtN];
    const int t = threadIdx.x;
    const int z0 = blockIdx.x * kSeedZonesPerBlock;
    if (t < kSeedZonesPerBlock && z0 + t < nZones) {
        uint64_t w = seedBase + 104729ULL * (uint64_t)(z0 + t + 1);
        st[t][0] = w;
        for (int i = 1; i < kMtN; ++i) {
            w = mt_seed_next(w, i);
            st[t][i] = w;
        }
    }
    __syncthreads();
    const int nz = min(kSeedZonesPerBlock, nZones - z0);
    for (int i = t; i < nz * kMtN; i += blockDim.x) out[(size_t)z0 * kMtN + i] = st[i / kMtN][i % kMtN];
}

// pass metrics: integer sums and a fixed-order reduction of the per-zone correction stats
__global__ void k_zone_metrics(const int2* __restrict__ moved, const double2* __restrict__ corr, int nZones,
                               double* __restrict__ out /* movedDense, movedSparse, corrRms, corrMax */) {
    __shared__ double sa[256], sm[256];
    __shared__ long long sd[256], ss[256];
    __shared__ int sc[256];
    const int t = threadIdx.x;
    double acc = 0.0, mx = 0.0;
    long long d = 0, s = 0;
    int c = 0;
    for (int z = t; z < nZones; z += blockDim.x) {
        const double2 q = corr[z];
        if (q.x > 0.0) {
            acc = __dadd_rn(acc, __dmul_rn(q.x, q.x));
            ++c;
        }
        mx = smax(mx, q.y);
        d += moved[z].x;
        s += moved[z].y;
    }
    sa[t] = acc; sm[t] = mx; sd[t] = d; ss[t] = s; sc[t] = c;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (t < o) {
            sa[t] = __dadd_rn(sa[t], sa[t + o]);
            sm[t] = smax(sm[t], sm[t + o]);
            sd[t] += sd[t + o];
            ss[t] += ss[t + o];
            sc[t] += sc[t + o];
        }
        __syncthreads();
    }
    if (t == 0) {
        out[0] = (double)sd[0];
        out[1] = (double)ss[0];
        out[2] = (sc[0] > 0) ? sqrt(__ddiv_rn(sa[0], (double)sc[0])) : 0.0;
        out[3] = sm[0];
    }
}

}  // namespace mpcd_dev
