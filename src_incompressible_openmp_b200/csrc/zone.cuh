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
// processes its full rectangle and writes only the particles it owns. The pass is out of
// place: the output buffers start as a copy of the input, and a zone writes only what it
// changes (positions of moved particles, velocities of corrected cells).
//
// Lists: a cell's list starts as its input segment of the cell index (ascending id) and
// stays implicit -- a head offset into that segment -- until the cell receives particles or
// is shuffled; then it is materialised in a small arena. List entries encode
// (input cell << 20 | position in its input segment), so a particle's slot is read from the
// cell index when needed.
//
// Warp discipline: every lane runs the same control flow with identical scalar values (the
// RNG stream is warp-uniform); lane-parallel sections are candidate evaluation, position
// sampling, list copies and the final momentum correction. Shared-memory scalars written by
// lane 0 are followed by __syncwarp() before any lane reads them.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace mpcd_dev {

// cell flags
constexpr uint8_t kCRecv = 1, kCBulkBulk = 2, kCSkip = 4, kCBulkBefore = 8, kCChanged = 16, kCOwned = 32,
                  kCMat = 64;
constexpr int kEntryShift = 20;  // entry = cell << 20 | position (cells < 4096, positions < 2^20)

struct ZoneArgs {
    DevParams P;
    const int4* rects;        // (xs, xe, ys, ye) per zone, zone id = index + 1
    const int* owner;         // ownerMap of the layout
    const uint64_t* start;    // cell index of the pass input (packed starts)
    const int* slots;
    const double2* vin;
    double2* xout;            // pre-filled with the input positions
    double2* vout;            // pre-filled with the input velocities
    int* cid;                 // standard-grid cell per slot; moved owned particles updated
    const uint64_t* seeds;    // seeded MT19937-64 state per zone (312 words each)
    int nZones;
    int maxCells, winCap, arenaCap, nsmCap;  // capacities of the per-zone working set
    int* overflow;            // zones left to the overflow kernel
    int* nOverflow;
    int2* zoneMoved;          // (dense, sparse) per zone
    double2* zoneCorr;        // (stats[4], stats[5]) per zone
    const int* order;         // launch order of the zones (heaviest first); nullptr = by id
    DevStatus* st;
    // run_zone_pass (serial, in place): zones one after another on the live state. slots[]
    // then holds the pass-input lists followed by an area where each zone appends the new
    // lists (ascending particle id) of the cells it changed; liveStart/liveCnt point to the
    // current list of every cell.
    int serial;
    int* slotsW;              // slots[], writable (the live-list area)
    int* liveCnt;
    int* liveStart;
    int* liveTop;             // next free entry of the live-list area
    int liveEnd;
    const int* pid;           // particle id per slot
    double2* duScratch;       // momentum correction per cell of the running zone
    // single-zone in-place API (serial kernel only; nullptr otherwise): per zone, the kernel-side
    // diagnostics of run_zone_kernel (src/zone_pass.cpp:857-972): sum of uxNow^2, sum of uyNow^2
    // over the zone's non-empty cells, sum and count of the non-zero dPx^2, the same for dPy,
    // the dense cells handled over the passes (nHigh) and the sparse ones (nLow)
    double* zoneDiag;
    // FP32 precision form (f32 != 0): the pass input and output states are these views and
    // vin, xout, vout are unused
    int f32;
    View32 in32, out32;
};

// pass input / output velocities of slot s (kF32: the FP32 views, instantiated separately)
template <bool kF32>
__device__ __forceinline__ double2 zone_vin(const ZoneArgs& A, int s) { return kF32 ? A.in32.vel(s) : A.vin[s]; }
template <bool kF32>
__device__ __forceinline__ void zone_vout(const ZoneArgs& A, int s, double2 w) {
    if (kF32)
        A.out32.set_vel(s, w);
    else
        A.vout[s] = w;
}

// Working set of one zone; carved from shared memory (fast path, I = uint16_t: 16-bit
// per-cell counts and arena offsets) or global memory (overflow path, I = int).
template <typename I>
struct ZoneMem {
    using W = typename std::conditional<sizeof(I) == 2, int16_t, int>::type;
    uint64_t* mt;      // 312: MT19937-64 state
    uint64_t* carry;   // 64: untwisted words of the previous block still to be drawn
    double* nsm;       // (TX+2)(TY+2): smoothed occupancy; reused for dU2 at the end
    W* win;            // (TX+4)(TY+4): pass-input counts around the zone (-1 = outside)
    int* gstart;       // cell: start of its input segment in the cell index
    I* cnt0;           // cell: input count
    I* head;           // cell: list head (implicit: offset into the input segment)
    I* len;            // cell: list length = live count
    I* abase;          // cell: arena start of a materialised list
    I* cap;            // cell: arena capacity of a materialised list
    uint8_t* cflags;   // cell
    uint16_t* list;    // cell: dense / low cell order
    uint16_t* order;   // cell: arena order of materialised lists (compaction)
    uint32_t* arena;   // arenaCap
    int* small;        // 64 ints: ranked targets, donors
    double* smallD;    // 24 doubles: donor normals, their polar components and radii

    __host__ __device__ static size_t bytes(int maxCells, int winCap, int arenaCap, int nsmCap) {
        size_t b = 0;
        auto add = [&](size_t n, size_t a) { b = (b + a - 1) / a * a + n; };
        add((size_t)kMtN * 8, 8);
        add(64 * 8, 8);
        add((size_t)nsmCap * 8, 8);
        add((size_t)winCap * sizeof(W), sizeof(W));
        add((size_t)maxCells * 4, 4);
        for (int k = 0; k < 5; ++k) add((size_t)maxCells * sizeof(I), sizeof(I));
        add((size_t)maxCells, 1);
        add((size_t)maxCells * 2, 2);
        add((size_t)maxCells * 2, 2);
        add((size_t)arenaCap * 4, 4);
        add(64 * 4, 4);
        add(24 * 8, 8);
        return (b + 15) / 16 * 16;
    }
    __device__ void carve(char* base, int maxCells, int winCap, int arenaCap, int nsmCap) {
        size_t b = 0;
        auto take = [&](size_t n, size_t a) {
            b = (b + a - 1) / a * a;
            char* p = base + b;
            b += n;
            return p;
        };
        mt = (uint64_t*)take((size_t)kMtN * 8, 8);
        carry = (uint64_t*)take(64 * 8, 8);
        nsm = (double*)take((size_t)nsmCap * 8, 8);
        win = (W*)take((size_t)winCap * sizeof(W), sizeof(W));
        gstart = (int*)take((size_t)maxCells * 4, 4);
        cnt0 = (I*)take((size_t)maxCells * sizeof(I), sizeof(I));
        head = (I*)take((size_t)maxCells * sizeof(I), sizeof(I));
        len = (I*)take((size_t)maxCells * sizeof(I), sizeof(I));
        abase = (I*)take((size_t)maxCells * sizeof(I), sizeof(I));
        cap = (I*)take((size_t)maxCells * sizeof(I), sizeof(I));
        cflags = (uint8_t*)take((size_t)maxCells, 1);
        list = (uint16_t*)take((size_t)maxCells * 2, 2);
        order = (uint16_t*)take((size_t)maxCells * 2, 2);
        arena = (uint32_t*)take((size_t)arenaCap * 4, 4);
        small = (int*)take(64 * 4, 4);
        smallD = (double*)take(24 * 8, 8);
    }
};

// In-place twist of a 312-word MT19937-64 state by one warp (reads of each half are staged
// in registers before its writes).
__device__ __noinline__ void mt_twist_inplace_warp(uint64_t* A, int lane) {
    uint64_t nv[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int i = lane + k * kWarp;
        nv[k] = (i < kMtN - kMtM) ? (A[i + kMtM] ^ mt_mix(A[i], A[i + 1])) : 0ULL;
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int i = lane + k * kWarp;
        if (i < kMtN - kMtM) A[i] = nv[k];
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int i = kMtN - kMtM + lane + k * kWarp;
        nv[k] = 0ULL;
        if (i < kMtN - 1) nv[k] = A[i - (kMtN - kMtM)] ^ mt_mix(A[i], A[i + 1]);
        else if (i == kMtN - 1) nv[k] = A[kMtM - 1] ^ mt_mix(A[kMtN - 1], A[0]);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int i = kMtN - kMtM + lane + k * kWarp;
        if (i < kMtN) A[i] = nv[k];
    }
    __syncwarp();
}

// copy a seeded 312-word state from global memory (one warp, 10 loads per lane in flight)
__device__ __noinline__ void mt_load_warp(uint64_t* buf, const uint64_t* seeded, int lane) {
    uint64_t w[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        const int i = lane + k * kWarp;
        w[k] = (i < kMtN) ? seeded[i] : 0ULL;
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        const int i = lane + k * kWarp;
        if (i < kMtN) buf[i] = w[k];
    }
    __syncwarp();
}

// 64-bit division and remainder on rare paths, out of line to keep the zone kernel small
__device__ __noinline__ uint64_t umod64_slow(uint64_t a, uint64_t b) { return a % b; }
__device__ __noinline__ uint64_t udiv64_slow(uint64_t a, uint64_t b) { return a / b; }

// Next block of a zone's stream (out of line, once per 312 draws): loads the seeded state
// on first use, keeps the kMtN - pos words not yet drawn in `carry`, twists in place.
// Returns the number of carried words.
__device__ __noinline__ int mt_refill(uint64_t* buf, uint64_t* carry, const uint64_t* seeded, int pos, int lane) {
    if (seeded) mt_load_warp(buf, seeded, lane);
    const int left = kMtN - pos;  // 0..63 words still to draw from the old block
    for (int i = lane; i < left; i += kWarp) carry[i] = buf[pos + i];
    __syncwarp();
    mt_twist_inplace_warp(buf, lane);
    return left;
}

// Warp-uniform MT19937-64 stream with a single state buffer. Batches of up to 64 draws
// may cross a block boundary: the words left in the old block move to `carry` first.
struct ZoneMt {
    uint64_t* buf;
    uint64_t* carry;
    const uint64_t* seeded;  // the zone's seeded state, loaded at the first draw
    int pos;     // next draw: carry[ncarry + pos] if pos < 0, else buf[pos]
    int ncarry;
    int lane;

    __device__ __forceinline__ void init(uint64_t* b, uint64_t* c, const uint64_t* s, int lane_) {
        buf = b;
        carry = c;
        seeded = s;
        pos = kMtN;
        ncarry = 0;
        lane = lane_;
    }
    __device__ __forceinline__ void ensure(int k) {  // k <= 64
        if (pos + k <= kMtN) return;
        const int left = mt_refill(buf, carry, seeded, pos, lane);
        seeded = nullptr;
        ncarry = left;
        pos = -left;
    }
    __device__ __forceinline__ uint64_t peek(int i) const {
        const int j = pos + i;
        return mt_temper((j < 0) ? carry[ncarry + j] : buf[j]);
    }
    __device__ __forceinline__ void consume(int k) { pos += k; }
    __device__ __forceinline__ uint64_t next() {
        ensure(1);
        const uint64_t u = peek(0);
        consume(1);
        return u;
    }
    __device__ __forceinline__ double u01() { return canon(next()); }
    __device__ __forceinline__ uint64_t uint_in(uint64_t lo, uint64_t hi) {
        const uint64_t range = hi - lo + 1ULL;
        uint64_t u = next();
        uint64_t low = u * range;
        uint64_t high = __umul64hi(u, range);
        if (low < range) {
            const uint64_t thr = umod64_slow(0ULL - range, range);
            while (low < thr) {
                u = next();
                low = u * range;
                high = __umul64hi(u, range);
            }
        }
        return high + lo;
    }
};

// std::shuffle of m entries at a (warp-uniform; lane 0 performs the swaps)
template <typename T>
__device__ __forceinline__ void zone_shuffle(T* a, int m, ZoneMt& r, int lane) {
    if (m <= 0) return;
    int i = 1;
    if ((m % 2) == 0) {
        const int j = (int)r.uint_in(0, 1);
        if (lane == 0) {
            const T t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
        ++i;
    }
    while (i != m) {
        const uint64_t sr = (uint64_t)i + 1ULL;
        const uint64_t x = r.uint_in(0, sr * (sr + 1ULL) - 1ULL);
        // x < sr (sr + 1) < 2^32 for the list sizes here: 32-bit division is exact
        int p1, p2;
        if (sr < 65535ULL) {
            const uint32_t x32 = (uint32_t)x, b1 = (uint32_t)sr + 1u;
            const uint32_t q = x32 / b1;
            p1 = (int)q;
            p2 = (int)(x32 - q * b1);
        } else {
            const uint64_t q = udiv64_slow(x, sr + 1ULL);
            p1 = (int)q;
            p2 = (int)(x - q * (sr + 1ULL));
        }
        if (lane == 0) {
            T t = a[i];
            a[i] = a[p1];
            a[p1] = t;
            t = a[i + 1];
            a[i + 1] = a[p2];
            a[p2] = t;
        }
        i += 2;
    }
    __syncwarp();
}

// The same shuffle for m <= 32 entries, with every draw taken from the stream at once: lane
// k computes draw k, and the swaps are applied in draw order to one value per lane. If some
// draw would need Lemire's rejection step (probability ~ range / 2^64), nothing is consumed
// and the sequential version runs instead.
template <typename T>
__device__ __forceinline__ void zone_shuffle_fast(T* a, int m, ZoneMt& r, int lane) {
    if (m <= 1) return;
    if (m > kWarp) {
        zone_shuffle(a, m, r, lane);
        return;
    }
    const bool even = (m % 2) == 0;
    const int D = (even ? 1 : 0) + (m - (even ? 2 : 1)) / 2;  // <= 16 draws
    r.ensure(D);
    int i = 0, p1 = 0, p2 = -1;
    bool rej = false;
    if (lane < D) {
        const bool first2 = even && lane == 0;
        i = first2 ? 1 : (even ? 2 : 1) + 2 * (lane - (even ? 1 : 0));
        const uint64_t R = first2 ? 2ULL : (uint64_t)(i + 1) * (uint64_t)(i + 2);
        const uint64_t u = r.peek(lane);
        const uint64_t low = u * R;
        if (low < R) rej = low < umod64_slow(0ULL - R, R);
        const uint32_t x = (uint32_t)__umul64hi(u, R);
        if (first2) {
            p1 = (int)x;
        } else {
            const uint32_t b1 = (uint32_t)(i + 2), q = x / b1;
            p1 = (int)q;
            p2 = (int)(x - q * b1);
        }
    }
    if (__any_sync(0xffffffffu, rej)) {
        zone_shuffle(a, m, r, lane);
        return;
    }
    r.consume(D);
    unsigned v = (lane < m) ? (unsigned)a[lane] : 0u;
    for (int k = 0; k < D; ++k) {
        const int ik = __shfl_sync(0xffffffffu, i, k);
        const int a1 = __shfl_sync(0xffffffffu, p1, k);
        const int a2 = __shfl_sync(0xffffffffu, p2, k);
        v = __shfl_sync(0xffffffffu, v, (lane == ik) ? a1 : ((lane == a1) ? ik : lane));
        if (a2 >= 0) {
            const int i2 = ik + 1;
            v = __shfl_sync(0xffffffffu, v, (lane == i2) ? a2 : ((lane == a2) ? i2 : lane));
        }
    }
    if (lane < m) a[lane] = (T)v;
    __syncwarp();
}

// sqrt(-2 ln r2 / r2) of the polar method, out of line
__device__ __noinline__ double polar_scale(double r2) { return sqrt(__ddiv_rn(__dmul_rn(-2.0, log_cr_dev(r2)), r2)); }

// polar-method normal deviate (libstdc++ normal_distribution), one cached value
struct ZoneNormal {
    double saved;
    int has;
    __device__ __forceinline__ double next(ZoneMt& r) {
        if (has) {
            has = 0;
            return saved;
        }
        double x, y, r2;
        do {
            x = __dsub_rn(__dmul_rn(2.0, r.u01()), 1.0);
            y = __dsub_rn(__dmul_rn(2.0, r.u01()), 1.0);
            r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = polar_scale(r2);
        saved = __dmul_rn(x, mult);
        has = 1;
        return __dmul_rn(y, mult);
    }
};

// Repacks the materialised lists of a zone at the bottom of its arena, in arena order;
// returns the new arena top. Out of line: it runs only when the arena is full.
template <typename I>
__device__ __noinline__ int zone_compact(uint8_t* cflags, I* abase, I* head, const I* len, I* cap,
                                         uint16_t* order, uint32_t* arena, int nl, int lane) {
    for (int l = lane; l < nl; l += kWarp) {
        int r = 0;
        if (cflags[l] & kCMat)
            for (int q = 0; q < nl; ++q)
                if ((cflags[q] & kCMat) && (abase[q] < abase[l] || (abase[q] == abase[l] && q < l))) ++r;
        order[l] = (uint16_t)r;
    }
    __syncwarp();
    int nmat = 0;
    for (int l = 0; l < nl; ++l) nmat += (cflags[l] & kCMat) ? 1 : 0;
    int off = 0;
    for (int r = 0; r < nmat; ++r) {
        int l = 0;
        for (int q = 0; q < nl; ++q)
            if ((cflags[q] & kCMat) && order[q] == r) l = q;
        const int a = abase[l] + head[l], n = len[l];
        // off <= a: copy down in ascending chunks (reads of a chunk precede its writes)
        for (int j0 = 0; j0 < n; j0 += kWarp) {
            const int j = j0 + lane;
            const uint32_t v = (j < n) ? arena[a + j] : 0u;
            __syncwarp();
            if (j < n) arena[off + j] = v;
            __syncwarp();
        }
        if (lane == 0) {
            abase[l] = off;
            head[l] = 0;
            cap[l] = n;
        }
        off += n;
        __syncwarp();
    }
    __syncwarp();
    return off;
}

// smoothed occupancy on the zone plus a one-cell ring (src/zone_pass.cpp:296-319):
// 3x3 binomial weights, renormalised over the in-domain neighbours. Out of line (called at
// most twice per pass).
template <typename W, typename I>
__device__ __noinline__ void zone_compute_nsm(double* nsm, const W* win, const I* cnt, int xs, int ys, int TX,
                                              int TY, int Nx, int Ny, int perx, int pery, int lane) {
    const int GX = TX + 2, GY = TY + 2, WY = TY + 4;
    for (int g = lane; g < GX * GY; g += kWarp) {
        int ix = xs - 1 + g / GY, iy = ys - 1 + g % GY;
        if (perx) ix = wrap_index(ix, Nx);
        if (pery) iy = wrap_index(iy, Ny);
        double val = 0.0;
        if (ix >= 0 && ix < Nx && iy >= 0 && iy < Ny) {
            double acc = 0.0, ws = 0.0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int jy = iy + dy, jx = ix + dx;
                    if (jy < 0 || jy >= Ny || jx < 0 || jx >= Nx) continue;
                    const double w = ((dx == 0) ? 2.0 : 1.0) * ((dy == 0) ? 2.0 : 1.0) * 0.0625;
                    int c;
                    if (jx >= xs && jx < xs + TX && jy >= ys && jy < ys + TY) {
                        c = cnt[(jx - xs) * TY + (jy - ys)];
                    } else {
                        int wx = jx - (xs - 2), wy = jy - (ys - 2);
                        if (wx < 0) wx += Nx;
                        else if (wx >= TX + 4) wx -= Nx;
                        if (wy < 0) wy += Ny;
                        else if (wy >= WY) wy -= Ny;
                        c = win[wx * WY + wy];
                    }
                    acc = __dadd_rn(acc, __dmul_rn(w, (double)c));
                    ws = __dadd_rn(ws, w);
                }
            val = __ddiv_rn(acc, smax(ws, 1e-30));
        }
        nsm[g] = val;
    }
    __syncwarp();
}

// hypot, out of line (once per sparse cell)
__device__ __noinline__ double zone_hypot(double a, double b) { return mpcd_dd::hypot_cr(a, b); }

// cnt deviates of one fresh normal_distribution (polar method: pairs of uniforms in stream
// order until r2 is in (0, 1]; each accepted pair gives y*m, then the cached x*m) into out[].
// Lane c examines candidate pair c of the batch; the accepted ones are ranked by ballot. The
// polar scale m uses the CUDA log (a few ulp from the correctly rounded one); comp and rad
// keep each deviate's polar component and r2, so that the exact deviate can be rebuilt as
// comp * polar_scale(r2).
__device__ __forceinline__ void zone_normals_fast(double* out, double* comp, double* rad, int cnt, ZoneMt& r, int lane) {
    int got = 0;
    while (got < cnt) {
        r.ensure(2 * kWarp);
        const double x = __dsub_rn(__dmul_rn(2.0, canon(r.peek(2 * lane))), 1.0);
        const double y = __dsub_rn(__dmul_rn(2.0, canon(r.peek(2 * lane + 1))), 1.0);
        const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
        const bool acc = !(r2 > 1.0 || r2 == 0.0);
        const unsigned am = __ballot_sync(0xffffffffu, acc);
        const int need = (cnt - got + 1) / 2;
        const int rank = __popc(am & lanemask_lt());
        const int used = min(__popc(am), need);
        int last = kWarp - 1;
        if (__popc(am) >= need) last = __ffs(__ballot_sync(0xffffffffu, acc && rank == need - 1)) - 1;
        if (acc && rank < need) {
            const double mult = sqrt(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
            const int k0 = got + 2 * rank;
            out[k0] = __dmul_rn(y, mult);
            comp[k0] = y;
            rad[k0] = r2;
            if (k0 + 1 < cnt) {
                out[k0 + 1] = __dmul_rn(x, mult);
                comp[k0 + 1] = x;
                rad[k0 + 1] = r2;
            }
        }
        r.consume(2 * (last + 1));
        got += 2 * used;
    }
    __syncwarp();
}

// Scalar (warp-uniform) state of one zone.
template <typename I, bool kF32 = false>
struct ZoneState {
    ZoneMem<I> M;
    ZoneMt rng;
    const ZoneArgs* A;
    int lane, zone;
    int xs, xe, ys, ye, TX, TY, nl, WY;
    // l / TY as (l * tyMagic) >> 32, tyMagic = ceil(2^32 / TY) (2^32 for TY = 1): exact for
    // l * TY < 2^32, which the 16-bit working set guarantees (l, TY < 2^16); the int path divides
    unsigned long long tyMagic;
    int arenaTop, arenaCap;
    int movedDense, movedSparse;
    int atanLane;   // lane k < 25 holds the angular bin of step k (DevParams::atanBin)
    double hypLane; // lane k < 25 holds the length of step k (DevParams::hypotTab)
    bool nbDirect;  // no wrapped neighbour (|offset| <= 2) of a zone cell lies in the zone
    bool dupNb5;    // a periodic axis shorter than 5 cells: range-2 neighbours can coincide
    bool dupNb3;    // a periodic axis shorter than 3 cells: 8-neighbours can coincide
    bool failed;   // capacity exhausted: the zone is handed to the overflow path
    bool fatal;    // a device error was raised

    __device__ __forceinline__ const DevParams& P() const { return A->P; }
    __device__ __forceinline__ bool in_zone(int ix, int iy) const { return ix >= xs && ix < xe && iy >= ys && iy < ye; }
    __device__ __forceinline__ int loc(int ix, int iy) const { return (ix - xs) * TY + (iy - ys); }
    __device__ __forceinline__ int lx_of(int l) const {
        return (sizeof(I) == 2) ? (int)(((unsigned long long)(unsigned)l * tyMagic) >> 32) : l / TY;
    }
    __device__ __forceinline__ int gx_of(int l) const { return xs + lx_of(l); }
    __device__ __forceinline__ int gy_of(int l) const { return ys + (l - lx_of(l) * TY); }

    __device__ __forceinline__ int cnt_at(int ix, int iy) const {
        if (in_zone(ix, iy)) return M.len[loc(ix, iy)];
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
    __device__ __forceinline__ bool shift_index(int iy, int ix, int dy, int dx, int& jy, int& jx) const {
        jy = iy + dy;
        if (P().pery) jy = wrap_index(jy, P().Ny);
        else if (jy < 0 || jy >= P().Ny) return false;
        jx = ix + dx;
        if (P().perx) jx = wrap_index(jx, P().Nx);
        else if (jx < 0 || jx >= P().Nx) return false;
        return true;
    }
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

    // threshold maps (src/zone_pass.cpp:321-345, :715-725) from the cell's bulk flag at
    // the last map build and the smoothed occupancy then
    __device__ __forceinline__ double frac(int l) const {
        const DevParams& p = P();
        if (!p.useLFF) return 1.0;
        const double fraw = __ddiv_rn(M.nsm[nsm_index(gx_of(l), gy_of(l))], smax(p.gamma, 1e-12));
        const double g = __dmul_rn(p.fluidFracGain, fraw);
        return (g < 0.0) ? 0.0 : ((1.0 < g) ? 1.0 : g);
    }
    __device__ __forceinline__ double map_low(int l) const {
        const DevParams& p = P();
        if (M.cflags[l] & kCBulkBefore) return p.lowThrBulk;
        return smax(__dmul_rn(p.lowFrac, __dmul_rn(p.gamma, frac(l))), p.lowThrFloor);
    }
    __device__ __forceinline__ double map_high(int l) const {
        const DevParams& p = P();
        if (M.cflags[l] & kCBulkBefore) return p.highThr;
        return smax(__dmul_rn(p.highFrac, __dmul_rn(p.gamma, frac(l))), p.highThrFloor);
    }
    __device__ __forceinline__ double map_val(int l, bool low) const { return low ? map_low(l) : map_high(l); }

    // ------------------------------------------------------------------ smoothing, maps
    __device__ void compute_nsm() {
        zone_compute_nsm(M.nsm, M.win, M.len, xs, ys, TX, TY, P().Nx, P().Ny, P().perx, P().pery, lane);
    }

    // start of a map build: record which cells are bulk (cnt > 0)
    __device__ void mark_bulk() {
        for (int l = lane; l < nl; l += kWarp) {
            const uint8_t f = M.cflags[l];
            M.cflags[l] = (uint8_t)((f & ~kCBulkBefore) | ((M.len[l] > 0) ? kCBulkBefore : 0));
        }
        __syncwarp();
    }

    template <typename Pred>
    __device__ int collect(Pred pred) {
        int total = 0;
        for (int b = 0; b < nl; b += kWarp) {
            const int l = b + lane;
            const bool ok = (l < nl) && pred(l);
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) M.list[total + __popc(m & lanemask_lt())] = (uint16_t)l;
            total += __popc(m);
        }
        __syncwarp();
        return total;
    }

    // ------------------------------------------------------------------ lists
    __device__ __forceinline__ uint32_t elem(int l, int i) const {
        if (M.cflags[l] & kCMat) return M.arena[M.abase[l] + M.head[l] + i];
        return ((uint32_t)l << kEntryShift) | (uint32_t)(M.head[l] + i);
    }

    // repack the materialised lists at the bottom of the arena (rare: out of line)
    __device__ void compact() {
        arenaTop = zone_compact(M.cflags, M.abase, M.head, M.len, M.cap, M.order, M.arena, nl, lane);
    }

    // materialise or grow list t so that `extra` entries can be appended
    __device__ bool ensure_room(int t, int extra) {
        const bool mat = (M.cflags[t] & kCMat) != 0;
        if (mat && M.head[t] + M.len[t] + extra <= M.cap[t]) return true;
        const int n = M.len[t];
        const int want = n + extra + 4;
        if (arenaTop + want > arenaCap) {
            compact();
            if (arenaTop + want > arenaCap) {
                failed = true;
                return false;
            }
        }
        for (int j = lane; j < n; j += kWarp) M.arena[arenaTop + j] = elem(t, j);
        __syncwarp();
        if (lane == 0) {
            M.abase[t] = arenaTop;
            M.head[t] = 0;
            M.cap[t] = want;
            M.cflags[t] |= kCMat;
        }
        arenaTop += want;
        __syncwarp();
        return true;
    }

    // Move `nt` particles from positions srcOff.. of list s into cell t, drawing positions
    // with sample_in_cell (src/zone_pass.cpp:280-294): per particle U for x then U for y.
    // slotPre/preOff: lane k holds the slot of entry preOff + k of list s if it was loaded
    // ahead (owned entries only); entries outside that window are loaded here.
    __device__ bool move_into(int s, int srcOff, int nt, int t, int slotPre = -1, int preOff = 1 << 29) {
        if (!ensure_room(t, nt)) return false;
        const DevParams& p = P();
        const double x0 = __dmul_rn((double)gx_of(t), p.dx), y0 = __dmul_rn((double)gy_of(t), p.dy);
        const int dst = M.abase[t] + M.head[t] + M.len[t];
        for (int q0 = 0; q0 < nt; q0 += kWarp) {
            const int c = min(kWarp, nt - q0);
            rng.ensure(2 * c);
            const int q = q0 + lane;
            const int w = preOff + srcOff + q;  // position in the prefetched window
            const int pre = __shfl_sync(0xffffffffu, slotPre, w & (kWarp - 1));
            if (lane < c) {
                const uint32_t e = elem(s, srcOff + q);
                const double px = __dadd_rn(x0, __dmul_rn(p.dx, canon(rng.peek(2 * lane))));
                const double py = __dadd_rn(y0, __dmul_rn(p.dy, canon(rng.peek(2 * lane + 1))));
                const int lc = (int)(e >> kEntryShift);
                if (M.cflags[lc] & kCOwned) {
                    const int sl = (w < kWarp) ? pre : A->slots[M.gstart[lc] + (int)(e & ((1u << kEntryShift) - 1))];
                    const int cc = cell_of(px, py, p);
                    if (kF32)
                        A->out32.set_pos(sl, make_double2(px, py), cc, p);
                    else
                        A->xout[sl] = make_double2(px, py);
                    A->cid[sl] = cc;
                }
                M.arena[dst + q] = e;
            }
            rng.consume(2 * c);
            __syncwarp();
        }
        if (lane == 0) {
            M.len[t] += nt;
        }
        __syncwarp();
        return true;
    }

    // receivers of a source cell, lane k < nrecv holding the k-th (at most 24 targets)
    __device__ __forceinline__ void push_recv(int& recvReg, int& nrecv, int c) {
        if (!__any_sync(0xffffffffu, lane < nrecv && recvReg == c)) {
            if (lane == nrecv) recvReg = c;
            ++nrecv;
        }
    }

    // update_transfer_correction_masks (src/zone_pass.cpp:492-525), forceSkip = false
    __device__ void update_masks(int src, int recvReg, int nrecv) {
        const bool ok = lane >= nrecv || (M.cflags[recvReg] & kCBulkBefore) != 0;
        const bool allBulk = ((M.cflags[src] & kCBulkBefore) != 0) && __all_sync(0xffffffffu, ok);
        const int prevRecv = __shfl_up_sync(0xffffffffu, recvReg, 1);
        if (lane <= nrecv) {
            const int c = (lane == 0) ? src : prevRecv;
            uint8_t f = M.cflags[c];
            if (allBulk) f |= kCBulkBulk;
            else f = (uint8_t)((f | kCSkip) & ~kCBulkBulk);
            M.cflags[c] = f;
        }
        __syncwarp();
    }

    // ------------------------------------------------------------------ dense phase
    // Targets of dense cell l, ranked, into T[0..m): admissible_dense_targets_rangeR
    // (src/zone_pass.cpp:413-434) with the zone filter, then rank_dense_targets_unified
    // (:436-490, inwardWeight = 0): angular bins, per-bin order on (-deficit, cnt, cheb,
    // dist2, U01) (a stable insertion sort), round robin over the bins from a random start.
    // Lane k < 24 examines neighbour k; the kept ones keep their order (compacted index ci).
    __device__ int select_targets(int l, bool low, int* T) {
        const int ix = gx_of(l), iy = gy_of(l);
        int nb = -1, ddx = 0, ddy = 0, idx = 0;
        if (lane < 24) {
            const int kk = (lane < 12) ? lane : lane + 1;
            const int dy = kk / 5 - 2, dx = kk % 5 - 2;
            int jy, jx;
            if (nbDirect ? in_zone(jx = ix + dx, jy = iy + dy) : (shift_index(iy, ix, dy, dx, jy, jx) && in_zone(jx, jy))) {
                const int t = loc(jx, jy);
                if ((double)M.len[t] < map_val(t, low)) nb = t;
            }
        }
        bool keep = nb >= 0;
        if (dupNb5) {  // wrapped offsets can coincide: keep the first occurrence of each cell
            const unsigned m0 = __ballot_sync(0xffffffffu, nb >= 0);
            const unsigned same = __match_any_sync(0xffffffffu, nb >= 0 ? nb : -1 - lane);
            keep = keep && ((same & m0 & lanemask_lt()) == 0);
        }
        const unsigned mk = __ballot_sync(0xffffffffu, keep);
        const int m = __popc(mk);
        if (m == 0) return 0;
        const int ci = __popc(mk & lanemask_lt());
        // draws: uniform_int(1, 8) for the start bin (range 8: Lemire never rejects), then one
        // U01 per target in compacted order
        rng.ensure(m + 1);
        const int startBin = (int)__umul64hi(rng.peek(0), 8ULL);
        int key2 = 0;
        double dneg = 0.0, tie = 0.0;
        if (keep) {
            idx = step_index(ix, iy, gx_of(nb), gy_of(nb), ddx, ddy);
            if (idx < 0) raise_error(A->st, kErrTableRange, zone);
            dneg = -smax(0.0, __dsub_rn(map_val(nb, low), (double)M.len[nb]));
            const int cheb = max(abs(ddx), abs(ddy)), d2 = ddx * ddx + ddy * ddy;
            key2 = (M.len[nb] << 8) | (cheb << 4) | d2;  // lexicographic (cnt, cheb, dist2)
            tie = canon(rng.peek(1 + ci));
        }
        rng.consume(m + 1);
        // angular bin of the step (table held in lanes 0..24)
        const int tb = __shfl_sync(0xffffffffu, atanLane, idx < 0 ? 0 : idx);
        const int bin = keep ? ((idx < 0) ? 0 : tb) : 8 + lane;
        // rank within the bin: compare only with the other kept lanes of the same bin
        unsigned others = __match_any_sync(0xffffffffu, bin) & ~(1u << lane);
        int r = 0;
        while (__any_sync(0xffffffffu, others != 0u)) {
            const int j = others ? (__ffs(others) - 1) : lane;
            others &= others - 1u;
            const double dj = __shfl_sync(0xffffffffu, dneg, j);
            const int kj = __shfl_sync(0xffffffffu, key2, j);
            const double tj = __shfl_sync(0xffffffffu, tie, j);
            if (j != lane) {
                bool less, eq = false;
                if (dj != dneg) less = dj < dneg;
                else if (kj != key2) less = kj < key2;
                else if (tj != tie) less = tj < tie;
                else { less = false; eq = true; }
                if (less || (eq && j < lane)) ++r;  // lane order = compacted order
            }
        }
        // round robin over the bins from startBin: position = entries of rank < r in every
        // bin, plus the bins before this one (in rotated order) that still hold rank r
        int pos = 0;
        for (int b = 0; b < 8; ++b) {
            const int cb = __popc(__ballot_sync(0xffffffffu, bin == b));
            if (keep) {
                pos += min(cb, r);
                const int rb = (b - startBin + 8) & 7, rq = (bin - startBin + 8) & 7;
                if (rb < rq && cb > r) ++pos;
            }
        }
        if (keep) T[pos] = nb;
        __syncwarp();
        return m;
    }

    // spread_particles_from_dense_source_round_robin (src/zone_pass.cpp:527-589). Lane k holds
    // target k's map value and deficit; a move changes only the deficit of its own target, so
    // each round walks the targets whose deficit was positive at the start of the round.
    __device__ int spread(int s, const int* T, int nT, bool low, int needOut, int& recvReg, int& nrecv, int slotPre,
                          int preOff) {
        if (needOut <= 0 || nT == 0) return 0;
        const int srcLen = M.len[s];
        if (srcLen == 0) return 0;
        int tl = -1, defj = 0;
        double mv = 0.0;
        if (lane < nT) {
            tl = T[lane];
            mv = map_val(tl, low);
            defj = max(0, (int)floor(__dsub_rn(mv, (double)M.len[tl])));
        }
        int taken = 0, moved = 0;
        bool stop = false;
        while (!stop && needOut > 0 && taken < srcLen) {
            const unsigned pm = __ballot_sync(0xffffffffu, lane < nT && defj > 0);
            if (pm == 0) break;  // no target can take a particle: no progress
            unsigned rest = pm;
            while (rest) {
                const int kk = __ffs(rest) - 1;
                rest &= rest - 1;
                const int deficit = __shfl_sync(0xffffffffu, defj, kk);
                const int t = __shfl_sync(0xffffffffu, tl, kk);
                const int remaining = __popc(pm >> kk);
                // ceil(needOut / remaining): integer division gives the same value as the
                // reference's ceil of the double quotient for these magnitudes
                const int rem1 = max(1, remaining);
                const int quota = max(1, (needOut + rem1 - 1) / rem1);
                const int nt = max(1, min(min(quota, deficit), min(needOut, srcLen - taken)));
                if (t == s) {
                    if (lane == 0) raise_error(A->st, kErrTargetIsSource, zone);
                    fatal = true;
                    return moved;
                }
                if (!move_into(s, taken, nt, t, slotPre, preOff)) return moved;
                push_recv(recvReg, nrecv, t);
                if (lane == kk) defj = max(0, (int)floor(__dsub_rn(mv, (double)M.len[tl])));
                taken += nt;
                moved += nt;
                needOut -= nt;
                if (needOut <= 0 || taken >= srcLen) {
                    stop = true;
                    break;
                }
            }
        }
        if (moved > 0 && lane == 0) {
            M.head[s] += taken;
            M.len[s] -= taken;
        }
        __syncwarp();
        return moved;
    }

    // one dense cell (src/zone_pass.cpp:734-753 calling :591-634)
    __device__ void dense_cell(int l) {
        int* T = M.small;
        int recvReg = -1;
        const int ncc = M.len[l];
        if (ncc <= 0) return;
        const double hl = map_high(l);
        if ((double)ncc <= hl) return;
        int nrecv = 0, moved = 0;
        // The two rounds take at most ceil(cnt - high) entries from the front of the list:
        // load the slots of the owned ones now, so the loads overlap the target ranking.
        int slotPre = -1;
        {
            const int take = min(min(M.len[l], max(0, (int)ceil(__dsub_rn((double)ncc, hl)))), kWarp);
            if (lane < take) {
                const uint32_t e = elem(l, lane);
                const int lc = (int)(e >> kEntryShift);
                if (M.cflags[lc] & kCOwned) slotPre = A->slots[M.gstart[lc] + (int)(e & ((1u << kEntryShift) - 1))];
            }
        }
        // first towards the low-threshold map, then whatever is left towards the high one
        // (one copy of the code for both rounds)
#pragma unroll 1
        for (int round = 0; round < 2; ++round) {
            const int need = max(0, (int)ceil(__dsub_rn((double)M.len[l], hl)));
            if (need <= 0) break;
            const bool low = (round == 0);
            const int nT = select_targets(l, low, T);
            moved += spread(l, T, nT, low, need, recvReg, nrecv, slotPre, moved);
            if (failed || fatal) return;
        }
        if (lane < nrecv) M.cflags[recvReg] |= (kCRecv | kCChanged);
        if (lane == 0 && moved > 0) M.cflags[l] |= kCChanged;
        __syncwarp();
        update_masks(l, recvReg, nrecv);
        movedDense += moved;
    }

    // ------------------------------------------------------------------ sparse phase
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
        int* don = M.small + 32;
        const int ncc = M.len[l];
        if (ncc <= 0) return;
        if (M.len[l] == 0) return;
        const int ix = gx_of(l), iy = gy_of(l);
        int nb = -1;
        if (lane < 8) {
            const int kk = (lane < 4) ? lane : lane + 1;
            const int dy = kk / 3 - 1, dx = kk % 3 - 1;
            int jy, jx;
            if (nbDirect ? in_zone(jx = ix + dx, jy = iy + dy) : (shift_index(iy, ix, dy, dx, jy, jx) && in_zone(jx, jy)))
                nb = loc(jx, jy);
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, nb >= 0);
        if (m0 == 0) return;
        bool uniq = nb >= 0;
        if (dupNb3) {  // wrapped offsets can coincide: keep the first occurrence of each cell
            const unsigned same = __match_any_sync(0xffffffffu, nb >= 0 ? nb : -1 - lane);
            uniq = uniq && ((same & m0 & lanemask_lt()) == 0);
        }
        const int lowInt = p.lowThrBulkInt;
        int need = max(0, lowInt - ncc);
        if (need <= 0) return;
        const bool isDonor = uniq && M.len[nb] > lowInt;
        const unsigned md = __ballot_sync(0xffffffffu, isDonor);
        const int nd = __popc(md);
        if (nd == 0) return;
        if (isDonor) don[__popc(md & lanemask_lt())] = nb;
        __syncwarp();
        double gx, gy;
        inward(l, gx, gy);
        zone_shuffle_fast(don, nd, rng, lane);
        // one N(0,1) per donor in shuffled order, then scores in parallel (lane k = donor k).
        // The scores only rank the donors: they are computed first with the CUDA hypot and
        // log, and again with the correctly rounded ones (the reference's values) only if two
        // scores lie closer than those functions' few-ulp differences could move them.
        double* nrm = M.smallD;
        zone_normals_fast(nrm, M.smallD + 8, M.smallD + 16, nd, rng, lane);
        int dk = -1, idx = 0, ddx = 0, ddy = 0;
        if (lane < nd) {
            dk = don[lane];
            idx = step_index(ix, iy, gx_of(dk), gy_of(dk), ddx, ddy);
        }
        const double hs = __shfl_sync(0xffffffffu, hypLane, idx < 0 ? 0 : idx);
        const double nsmd = (lane < nd) ? M.nsm[nsm_index(gx_of(dk), gy_of(dk))] : 0.0;
        auto score = [&](double ndir, double nv) {
            const double nstep = (idx >= 0) ? hs : 0.0;
            double align = 0.0;
            if (ndir >= 1e-14 && nstep >= 1e-14)
                align = __ddiv_rn(__dadd_rn(__dmul_rn((double)ddx, gx), __dmul_rn((double)ddy, gy)), __dmul_rn(ndir, nstep));
            const double noise = __dmul_rn(1e-9, nv);
            return __dadd_rn(__dadd_rn(__dmul_rn(100.0, align), nsmd), noise);
        };
        const double ndirF = hypot(gx, gy);
        double sc = (lane < nd) ? score(ndirF, nrm[lane]) : 0.0;
        // the fast and exact scores differ by under 2e-13 (1 + |score|): distinct ranks are
        // certain when every gap exceeds 1e-12 (1 + |score|) and the norm is clear of 1e-14
        bool sure = !(ndirF > 0.5e-14 && ndirF < 2e-14);
        for (int j = 0; j < nd; ++j) {
            const double sj = __shfl_sync(0xffffffffu, sc, j);
            if (lane < nd && j != lane && fabs(sj - sc) <= 1e-12 * (1.0 + fabs(sc))) sure = false;
        }
        if (!__all_sync(0xffffffffu, sure)) {
            const double ndir = zone_hypot(gx, gy);
            if (lane < nd) sc = score(ndir, __dmul_rn(M.smallD[8 + lane], polar_scale(M.smallD[16 + lane])));
        }
        // descending, ties in shuffled order (std::sort of <= 16 elements is an insertion sort)
        int rk = 0;
        for (int j = 0; j < nd; ++j) {
            const double sj = __shfl_sync(0xffffffffu, sc, j);
            if (lane < nd && j != lane && (sj > sc || (sj == sc && j < lane))) ++rk;
        }
        __syncwarp();
        if (lane < nd) don[rk] = dk;
        __syncwarp();
        for (int k = 0; k < nd; ++k) {
            const int d = don[k];
            const int ld = M.len[d];
            if (ld == 0) continue;
            const int avail = M.len[d] - lowInt;
            if (avail <= 0) continue;
            const int nt = min(min(need, avail), ld);
            if (nt <= 0) continue;
            if (!ensure_room(d, 0)) return;  // materialise the donor list to shuffle it
            zone_shuffle_fast(M.arena + M.abase[d] + M.head[d], ld, rng, lane);
            if (!move_into(d, 0, nt, l)) return;
            if (lane == 0) {
                M.head[d] += nt;
                M.len[d] -= nt;
                M.cflags[l] |= (kCRecv | kCChanged);
                M.cflags[d] |= kCChanged;
            }
            __syncwarp();
            update_masks(d, (lane == 0) ? l : -1, 1);
            movedSparse += nt;
            need -= nt;
            if (need <= 0) break;
        }
    }
};

// global cell of window position w (zone rectangle plus a 2-cell ring, wrapped)
template <typename I, bool kF32>
__device__ __forceinline__ int iy_ix_cell(const ZoneState<I, kF32>& S, int w, const DevParams& p) {
    int ix = S.xs - 2 + w / S.WY, iy = S.ys - 2 + w % S.WY;
    if (p.perx) ix = wrap_index(ix, p.Nx);
    if (p.pery) iy = wrap_index(iy, p.Ny);
    return iy + p.Ny * ix;
}

// End of a zone of the serial pass: apply the deferred momentum corrections, then publish
// the new list (ascending particle id) and count of every cell the zone changed.
template <typename I, bool kF32>
__device__ __forceinline__ void serial_finish(ZoneState<I, kF32>& S, const ZoneArgs& A, const DevParams& p) {
    ZoneMem<I>& M = S.M;
    const int lane = S.lane;
    for (int l = lane; l < S.nl; l += kWarp) {
        const double2 du = A.duScratch[l];
        if (du.x != 0.0 || du.y != 0.0) {
            const int n = M.len[l];
            for (int j = 0; j < n; ++j) {
                const uint32_t e = S.elem(l, j);
                const int sl = A.slots[M.gstart[(int)(e >> kEntryShift)] + (int)(e & ((1u << kEntryShift) - 1))];
                const double2 w = zone_vin<false>(A, sl);
                zone_vout<false>(A, sl, make_double2(__dadd_rn(w.x, du.x), __dadd_rn(w.y, du.y)));
            }
        }
    }
    __syncwarp();
    int top = *A.liveTop;
    for (int b = 0; b < S.nl; b += kWarp) {
        const int l = b + lane;
        const bool ch = l < S.nl && (M.cflags[l] & kCChanged);
        const int n = ch ? M.len[l] : 0;
        int off = n;  // inclusive scan of the list lengths
        for (int o = 1; o < kWarp; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += t;
        }
        const int total = __shfl_sync(0xffffffffu, off, kWarp - 1);
        off -= n;
        if (top + total > A.liveEnd) {
            if (lane == 0) raise_error(A.st, kErrZoneCapacity, S.zone);
            return;
        }
        if (ch) {
            const int dst = top + off;
            for (int j = 0; j < n; ++j) {
                const uint32_t e = S.elem(l, j);
                A.slotsW[dst + j] = A.slots[M.gstart[(int)(e >> kEntryShift)] + (int)(e & ((1u << kEntryShift) - 1))];
            }
            for (int i = dst + 1; i < dst + n; ++i) {  // insertion sort by particle id
                const int v = A.slotsW[i];
                const int pv = A.pid[v];
                int j = i;
                while (j > dst && A.pid[A.slotsW[j - 1]] > pv) {
                    A.slotsW[j] = A.slotsW[j - 1];
                    --j;
                }
                A.slotsW[j] = v;
            }
            const int gc = S.gy_of(l) + p.Ny * S.gx_of(l);
            A.liveStart[gc] = dst;
            A.liveCnt[gc] = n;
        }
        top += total;
    }
    __syncwarp();
    if (lane == 0) *A.liveTop = top;
    __syncwarp();
}

// ------------------------------------------------------------------ the zone body
// The zone body in four phases: set-up (the pass-input counts around the zone, the cells'
// segments and ownership, the draw stream), one dense pass, the sparse phase, and the output
// (momentum correction and the zone's stats). zone_body runs them back to back; the
// phase-synchronous kernel runs the zones of a block in step, a barrier between phases.

// Set-up; false if the zone must be re-run on the overflow path.
template <bool kSerial, typename I, bool kF32>
__device__ __forceinline__ bool zone_setup(ZoneState<I, kF32>& S, const ZoneArgs& A, int z, char* mem, int maxCells,
                                           int winCap, int arenaCap, int nsmCap) {
    S.A = &A;
    S.lane = threadIdx.x & 31;
    S.zone = z;
    S.failed = false;
    S.fatal = false;
    S.movedDense = S.movedSparse = 0;
    const int lane = S.lane;
    const DevParams& p = A.P;
    const int4 R = A.rects[z];
    S.xs = R.x; S.xe = R.y; S.ys = R.z; S.ye = R.w;
    S.TX = S.xe - S.xs; S.TY = S.ye - S.ys; S.nl = S.TX * S.TY; S.WY = S.TY + 4;
    S.tyMagic = (S.TY > 0) ? ((1ULL << 32) + (unsigned long long)S.TY - 1ULL) / (unsigned long long)S.TY : 0ULL;
    S.atanLane = (lane < 25) ? p.atanBin[lane] : 0;
    S.hypLane = (lane < 25) ? p.hypotTab[lane] : 0.0;
    S.dupNb5 = (p.perx && p.Nx < 5) || (p.pery && p.Ny < 5);
    S.nbDirect = (!p.perx || S.TX < p.Nx - 2) && (!p.pery || S.TY < p.Ny - 2);
    S.dupNb3 = (p.perx && p.Nx < 3) || (p.pery && p.Ny < 3);
    const int W = (S.TX + 4) * S.WY;
    if (S.nl > maxCells || W > winCap || (S.TX + 2) * (S.TY + 2) > nsmCap || S.nl >= (1 << (32 - kEntryShift)) ||
        (sizeof(I) == 2 && S.nl > 65535))
        return false;
    S.M.carve(mem, maxCells, winCap, arenaCap, nsmCap);
    constexpr bool kNarrow = sizeof(I) == 2;  // 16-bit counts: window counts <= 32767, zone total <= 65535
    bool wide = false;
    S.arenaCap = arenaCap;
    S.arenaTop = 0;
    ZoneMem<I>& M = S.M;
    // pass-input counts around the zone
    for (int w0 = 0; w0 < W; w0 += 4 * kWarp) {
        uint64_t a[4], b[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int w = w0 + lane + k * kWarp;
            int ix = S.xs - 2 + w / S.WY, iy = S.ys - 2 + w % S.WY;
            if (p.perx) ix = wrap_index(ix, p.Nx);
            if (p.pery) iy = wrap_index(iy, p.Ny);
            ok[k] = w < W && ix >= 0 && ix < p.Nx && iy >= 0 && iy < p.Ny;
            const int cc = ok[k] ? iy + p.Ny * ix : 0;
            a[k] = ok[k] ? A.start[cc] : 0ULL;
            b[k] = ok[k] ? A.start[cc + 1] : 0ULL;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int w = w0 + lane + k * kWarp;
            if (w < W) {
                int cv = ok[k] ? (int)((uint32_t)b[k] - (uint32_t)a[k]) : -1;
                if (kSerial && ok[k]) cv = A.liveCnt[iy_ix_cell(S, w, p)];
                if (kNarrow && cv > 32767) wide = true;
                M.win[w] = cv;
            }
        }
    }
    // zone cells: segment starts and ownership
    for (int l0 = 0; l0 < S.nl; l0 += 4 * kWarp) {
        int own[4];
        uint64_t st[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int l = l0 + lane + k * kWarp;
            const int c = (l < S.nl) ? S.gy_of(l) + p.Ny * S.gx_of(l) : 0;
            own[k] = (l < S.nl) ? A.owner[c] : 0;
            st[k] = (l < S.nl) ? A.start[c] : 0ULL;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int l = l0 + lane + k * kWarp;
            if (l < S.nl) {
                M.gstart[l] = kSerial ? A.liveStart[S.gy_of(l) + p.Ny * S.gx_of(l)] : (int)(uint32_t)st[k];
                M.cflags[l] = (kSerial || own[k] == z + 1) ? kCOwned : 0;
            }
        }
    }
    __syncwarp();
    int tot = 0;
    for (int l = lane; l < S.nl; l += kWarp) {
        const int c = M.win[(l / S.TY + 2) * S.WY + (l % S.TY + 2)];
        tot += c;
        M.cnt0[l] = c;
        M.len[l] = c;
        M.head[l] = 0;
        M.abase[l] = 0;
        M.cap[l] = 0;
    }
    if (kNarrow) {  // counts too large for the 16-bit working set: the overflow path takes the zone
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
        if (__any_sync(0xffffffffu, wide) || tot > 65535) return false;
    }
    __syncwarp();
    S.rng.init(M.mt, M.carry, A.seeds + (size_t)z * kMtN, lane);
    return true;
}

// One dense pass (src/zone_pass.cpp:708-781): the cells above their high map, in shuffled
// order. Returns how many.
template <typename I, bool kF32>
__device__ __forceinline__ int zone_dense_pass(ZoneState<I, kF32>& S) {
    const int lane = S.lane;
    const DevParams& p = S.A->P;
    ZoneMem<I>& M = S.M;
    if (p.useLFF) S.compute_nsm();
    S.mark_bulk();
    const int nd = S.collect([&](int l) { return (double)M.len[l] > S.map_high(l); });
    zone_shuffle_fast(M.list, nd, S.rng, lane);
    for (int q = 0; q < nd && !S.failed && !S.fatal; ++q) S.dense_cell((int)M.list[q]);
    return nd;
}

// The sparse phase (src/zone_pass.cpp:783-854). Returns the sparse cells.
template <typename I, bool kF32>
__device__ __forceinline__ int zone_sparse(ZoneState<I, kF32>& S) {
    const int lane = S.lane;
    const DevParams& p = S.A->P;
    ZoneMem<I>& M = S.M;
    // the smoothed occupancy feeds the maps only with local fluid-fraction thresholds;
    // otherwise it is needed only if some cell is sparse (inward gradient, donor scores)
    if (p.useLFF) S.compute_nsm();
    S.mark_bulk();
    const int nlow = S.collect([&](int l) { return M.len[l] > 0 && (double)M.len[l] < S.map_low(l); });
    if (!p.useLFF && nlow > 0) S.compute_nsm();
    zone_shuffle_fast(M.list, nlow, S.rng, lane);
    for (int q = 0; q < nlow && !S.failed && !S.fatal; ++q) S.sparse_cell((int)M.list[q]);
    return nlow;
}

// Output: the momentum correction and the zone's stats; false if the zone must be re-run on the
// overflow path.
template <bool kSerial, typename I, bool kF32>
__device__ __forceinline__ bool zone_finish(ZoneState<I, kF32>& S, const ZoneArgs& A, int z, int nHighAll, int nLowAll) {
    const int lane = S.lane;
    const DevParams& p = A.P;
    ZoneMem<I>& M = S.M;
    if (S.fatal) return true;
    if (S.failed) return false;

    // momentum correction (src/zone_pass.cpp:870-922): per changed cell, the momentum of
    // its input list and of its final list, both in list order; owned particles of
    // corrected cells get v + du
    double* du2 = M.nsm;
    const bool wantDiag = kSerial && A.zoneDiag != nullptr;
    double dgUx2 = 0.0, dgUy2 = 0.0, dgPx2 = 0.0, dgPy2 = 0.0;
    int dgNPx = 0, dgNPy = 0;
    for (int l = lane; l < S.nl; l += kWarp) {
        double d2 = 0.0;
        const uint8_t f = M.cflags[l];
        const int n = M.len[l];
        if (kSerial) A.duScratch[l] = make_double2(0.0, 0.0);  // cells left unchanged get none
        if (wantDiag && !(f & kCChanged) && n > 0) {
            // an unchanged cell: uxNow from its input list (ascending id), no momentum error
            double sx = 0.0, sy = 0.0;
            for (int j = 0; j < n; ++j) {
                const double2 w = zone_vin<kF32>(A, A.slots[M.gstart[l] + j]);
                sx = __dadd_rn(sx, w.x);
                sy = __dadd_rn(sy, w.y);
            }
            const double ux = __ddiv_rn(sx, (double)n), uy = __ddiv_rn(sy, (double)n);
            dgUx2 = __dadd_rn(dgUx2, __dmul_rn(ux, ux));
            dgUy2 = __dadd_rn(dgUy2, __dmul_rn(uy, uy));
        }
        if ((f & kCChanged) && n > 0) {
            double bx = 0.0, by = 0.0, axs = 0.0, ays = 0.0;
            const int n0 = M.cnt0[l], g0 = M.gstart[l];
            for (int j0 = 0; j0 < n0; j0 += 8) {
                int sl[8];
                double2 w[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) sl[u] = (j0 + u < n0) ? A.slots[g0 + j0 + u] : 0;
#pragma unroll
                for (int u = 0; u < 8; ++u) w[u] = (j0 + u < n0) ? zone_vin<kF32>(A, sl[u]) : make_double2(0.0, 0.0);
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (j0 + u < n0) {
                        bx = __dadd_rn(bx, w[u].x);
                        by = __dadd_rn(by, w[u].y);
                    }
            }
            for (int j0 = 0; j0 < n; j0 += 8) {
                int sl[8];
                double2 w[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    sl[u] = 0;
                    if (j0 + u < n) {
                        const uint32_t e = S.elem(l, j0 + u);
                        sl[u] = A.slots[M.gstart[e >> kEntryShift] + (int)(e & ((1u << kEntryShift) - 1))];
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) w[u] = (j0 + u < n) ? zone_vin<kF32>(A, sl[u]) : make_double2(0.0, 0.0);
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (j0 + u < n) {
                        axs = __dadd_rn(axs, w[u].x);
                        ays = __dadd_rn(ays, w[u].y);
                    }
            }
            const double ux = __ddiv_rn(__dsub_rn(bx, axs), (double)n);
            const double uy = __ddiv_rn(__dsub_rn(by, ays), (double)n);
            d2 = __dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy));
            if (wantDiag) {
                const double ax = __ddiv_rn(axs, (double)n), ay = __ddiv_rn(ays, (double)n);
                dgUx2 = __dadd_rn(dgUx2, __dmul_rn(ax, ax));
                dgUy2 = __dadd_rn(dgUy2, __dmul_rn(ay, ay));
                const double dpx = __dsub_rn(bx, axs), dpy = __dsub_rn(by, ays);
                const double ex = __dmul_rn(dpx, dpx), ey = __dmul_rn(dpy, dpy);
                if (ex > 0.0) { dgPx2 = __dadd_rn(dgPx2, ex); ++dgNPx; }
                if (ey > 0.0) { dgPy2 = __dadd_rn(dgPy2, ey); ++dgNPy; }
            }
            bool doCorr = p.momCorr != 0;
            if (doCorr && (f & kCSkip)) doCorr = false;
            if (doCorr && (f & kCRecv) && !(f & kCBulkBulk)) doCorr = false;
            if (kSerial) {
                // in place: every cell's sums must read the velocities of the zone's start
                A.duScratch[l] = (doCorr && (ux != 0.0 || uy != 0.0)) ? make_double2(ux, uy) : make_double2(0.0, 0.0);
            } else if (doCorr && (ux != 0.0 || uy != 0.0)) {
                for (int j = 0; j < n; ++j) {
                    const uint32_t e = S.elem(l, j);
                    const int lc = (int)(e >> kEntryShift);
                    if (!(M.cflags[lc] & kCOwned)) continue;
                    const int sl = A.slots[M.gstart[lc] + (int)(e & ((1u << kEntryShift) - 1))];
                    const double2 w = zone_vin<kF32>(A, sl);
                    zone_vout<kF32>(A, sl, make_double2(__dadd_rn(w.x, ux), __dadd_rn(w.y, uy)));
                }
            }
        }
        du2[l] = d2;
    }
    __syncwarp();
    if (wantDiag) {
        for (int o = 16; o > 0; o >>= 1) {
            dgUx2 = __dadd_rn(dgUx2, __shfl_xor_sync(0xffffffffu, dgUx2, o));
            dgUy2 = __dadd_rn(dgUy2, __shfl_xor_sync(0xffffffffu, dgUy2, o));
            dgPx2 = __dadd_rn(dgPx2, __shfl_xor_sync(0xffffffffu, dgPx2, o));
            dgPy2 = __dadd_rn(dgPy2, __shfl_xor_sync(0xffffffffu, dgPy2, o));
            dgNPx += __shfl_xor_sync(0xffffffffu, dgNPx, o);
            dgNPy += __shfl_xor_sync(0xffffffffu, dgNPy, o);
        }
        if (lane == 0) {
            double* d = A.zoneDiag + 8 * (size_t)z;
            d[0] = dgUx2; d[1] = dgUy2; d[2] = dgPx2; d[3] = (double)dgNPx; d[4] = dgPy2; d[5] = (double)dgNPy;
            d[6] = (double)nHighAll; d[7] = (double)nLowAll;
        }
        __syncwarp();
    }
    if (kSerial) serial_finish(S, A, p);
    // zone stats[4], stats[5] (src/zone_pass.cpp:911-922): the sum of positive dU2 in
    // ascending cell order and their maximum (zero entries change neither)
    double acc = 0.0, mx = 0.0;
    int cntDU = 0;
    for (int b = 0; b < S.nl; b += kWarp) {
        const int l = b + lane;
        const double d2 = (l < S.nl) ? du2[l] : 0.0;
        unsigned pos = __ballot_sync(0xffffffffu, d2 > 0.0);
        while (pos) {
            const int q = __ffs(pos) - 1;
            pos &= pos - 1;
            const double v = __shfl_sync(0xffffffffu, d2, q);
            acc = __dadd_rn(acc, v);
            mx = smax(mx, sqrt(v));
            ++cntDU;
        }
    }
    if (lane == 0) {
        A.zoneCorr[z] = make_double2((cntDU > 0) ? sqrt(__ddiv_rn(acc, (double)cntDU)) : 0.0, (cntDU > 0) ? mx : 0.0);
        A.zoneMoved[z] = make_int2(S.movedDense, S.movedSparse);
    }
    return true;
}

// Returns false if the zone must be re-run on the overflow path.
template <bool kSerial, typename I, bool kF32 = false>
__device__ bool zone_body(const ZoneArgs& A, int z, char* mem, int maxCells, int winCap, int arenaCap, int nsmCap) {
    ZoneState<I, kF32> S;
    if (!zone_setup<kSerial>(S, A, z, mem, maxCells, winCap, arenaCap, nsmCap)) return false;
    int nHighAll = 0, nLowAll = 0;  // dense cells over the passes, sparse cells (stats[0], stats[1])
    for (int pass = 0; pass < A.P.maxPasses && !S.failed && !S.fatal; ++pass) nHighAll += zone_dense_pass(S);
    if (!S.failed && !S.fatal) nLowAll = zone_sparse(S);
    return zone_finish<kSerial>(S, A, z, nHighAll, nLowAll);
}

// kF32: the FP32 precision form's state (A.in32, A.out32)
template <bool kF32>
__global__ void __launch_bounds__(32, 20) k_zone_pass(ZoneArgs A) {
    extern __shared__ __align__(16) char smem[];
    if ((int)blockIdx.x >= A.nZones) return;
    const int z = A.order ? A.order[blockIdx.x] : (int)blockIdx.x;
    if (!zone_body<false, uint16_t, kF32>(A, z, smem, A.maxCells, A.winCap, A.arenaCap, A.nsmCap) && (threadIdx.x & 31) == 0)
        A.overflow[atomicAdd(A.nOverflow, 1)] = z;
}

// Phase-synchronous zone pass: kW zones per block, consecutive entries of the launch order
// (heaviest first, so the zones of a block cost about the same), run in step with a block
// barrier after the set-up, after each dense pass and after the sparse phase. The resident
// warps of an SM then execute the same phase's code (the body is too large for the
// instruction cache as a whole). Each warp carves its working set at perWarp bytes.
template <bool kF32, int kW>
__global__ void __launch_bounds__(32 * kW) k_zone_pass_sync(ZoneArgs A, int perWarp) {
    extern __shared__ __align__(16) char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = (int)blockIdx.x * kW + w;
    const bool have = slot < A.nZones;
    const int z = have ? (A.order ? A.order[slot] : slot) : 0;
    ZoneState<uint16_t, kF32> S;
    S.failed = S.fatal = false;
    const bool ok = have && zone_setup<false>(S, A, z, smem + (size_t)perWarp * w, A.maxCells, A.winCap, A.arenaCap,
                                               A.nsmCap);
    int nHighAll = 0, nLowAll = 0;
    __syncthreads();
    for (int pass = 0; pass < A.P.maxPasses; ++pass) {
        if (ok && !S.failed && !S.fatal) nHighAll += zone_dense_pass(S);
        __syncthreads();
    }
    if (ok && !S.failed && !S.fatal) nLowAll = zone_sparse(S);
    __syncthreads();
    if (have && !(ok && zone_finish<false>(S, A, z, nHighAll, nLowAll)) && lane == 0)
        A.overflow[atomicAdd(A.nOverflow, 1)] = z;
}

// The zone pass of several replicas in one launch. Block b runs the zone at launch position
// b - offs[r] of replica r, offs being the prefix sums of the replicas' zone counts; the
// replica's arguments are copied into shared memory ahead of the zone's working set.
constexpr int kZoneArgsSmem = (int)((sizeof(ZoneArgs) + 15) / 16 * 16);
template <bool kF32>
__global__ void __launch_bounds__(32, 20) k_zone_pass_batch(const ZoneArgs* __restrict__ args, const int* __restrict__ offs,
                                                            int nRep) {
    extern __shared__ __align__(16) char smem[];
    const int b = (int)blockIdx.x;
    if (nRep <= 0 || b >= offs[nRep]) return;
    int lo = 0, hi = nRep - 1;  // the replica r with offs[r] <= b < offs[r + 1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    static_assert(sizeof(ZoneArgs) % 8 == 0, "ZoneArgs is copied in 8-byte words");
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(args + lo);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(smem);
    for (int i = (int)threadIdx.x; i < (int)(sizeof(ZoneArgs) / 8); i += 32) dst[i] = src[i];
    __syncwarp();
    const ZoneArgs& A = *reinterpret_cast<const ZoneArgs*>(smem);
    const int local = b - offs[lo];
    const int z = A.order ? A.order[local] : local;
    if (!zone_body<false, uint16_t, kF32>(A, z, smem + kZoneArgsSmem, A.maxCells, A.winCap, A.arenaCap, A.nsmCap) &&
        (threadIdx.x & 31) == 0)
        A.overflow[atomicAdd(A.nOverflow, 1)] = z;
}

// Launch order of the zones, heaviest first, so that the last wave of blocks holds the
// cheapest zones. The cost estimate is the number of particles above the bulk high threshold
// in the zone's cells (the dense-phase work); ties keep no particular order, which is fine:
// a zone's result does not depend on when it runs.
constexpr int kCostBuckets = 256;
__global__ void k_zone_cost(DevParams P, const int4* __restrict__ rects, const uint64_t* __restrict__ start, int nZones,
                            int* __restrict__ cost, int* __restrict__ hist) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nZones) return;
    const int4 R = rects[z];
    double ex = 0.0;
    for (int ix = R.x; ix < R.y; ++ix)
        for (int iy = R.z; iy < R.w; ++iy) {
            const int c = iy + P.Ny * ix;
            const double n = (double)(int)((uint32_t)start[c + 1] - (uint32_t)start[c]);
            if (n > P.highThr) ex += n - P.highThr;
        }
    const int b = min(kCostBuckets - 1, (int)ex);
    cost[z] = b;
    atomicAdd(hist + b, 1);
}

// one block: bucket offsets in descending cost, then each zone takes a place in its bucket
__global__ void __launch_bounds__(1024) k_zone_order(const int* __restrict__ cost, int* __restrict__ hist, int nZones,
                                                     int* __restrict__ order) {
    __shared__ int off[kCostBuckets];
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int b = kCostBuckets - 1; b >= 0; --b) {
            off[b] = acc;
            acc += hist[b];
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kCostBuckets; b += blockDim.x) hist[b] = 0;  // ready for the next pass
    for (int z = threadIdx.x; z < nZones; z += blockDim.x) order[atomicAdd(&off[cost[z]], 1)] = z;
}

// zones that did not fit the shared-memory working set, re-run from their seed with a
// global-memory working set per block (deterministic: identical decisions and writes)
// The last of its blocks to finish then computes the pass metrics (zone_metrics_warp) and
// resets the overflow and block counters for the next pass.
__device__ void zone_metrics_warp(const int2* __restrict__ moved, const double2* __restrict__ corr, int nZones,
                                  double* __restrict__ out);
// block blk of nblk: the overflow zones blk, blk + nblk, ...; the last block to finish
// computes the pass metrics (when metricsOut is given) and resets the counters
template <bool kF32>
__device__ __forceinline__ void zone_overflow_block(const ZoneArgs& A, char* gmem, size_t perBlock, int* blocksDone,
                                                    double* metricsOut, int blk, int nblk) {
    const int nov = *A.nOverflow;
    for (int i = blk; i < nov; i += nblk)
        if (!zone_body<false, int, kF32>(A, A.overflow[i], gmem + perBlock * blk, A.maxCells, A.winCap, A.arenaCap,
                                         A.nsmCap) &&
            (threadIdx.x & 31) == 0)
            raise_error(A.st, kErrZoneCapacity, A.overflow[i]);
    __syncwarp();
    int last = 0;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(blocksDone, 1) == nblk - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    if (metricsOut) zone_metrics_warp(A.zoneMoved, A.zoneCorr, A.nZones, metricsOut);
    if (threadIdx.x == 0) {
        *blocksDone = 0;
        *A.nOverflow = 0;
    }
}

template <bool kF32>
__global__ void __launch_bounds__(32) k_zone_overflow(ZoneArgs A, char* gmem, size_t perBlock, int* blocksDone,
                                                      double* metricsOut) {
    zone_overflow_block<kF32>(A, gmem, perBlock, blocksDone, metricsOut, (int)blockIdx.x, (int)gridDim.x);
}

// The overflow kernels of many contexts (a batch's replicas) as one launch: job r takes
// blocks [r * perJob, (r + 1) * perJob).
struct OverflowJob {
    ZoneArgs A;  // with the overflow path's capacities
    char* gmem;
    size_t perBlock;
    int* blocksDone;
    double* metricsOut;
};

__global__ void __launch_bounds__(32) k_zone_overflow_batch(const OverflowJob* __restrict__ jobs, int perJob) {
    const OverflowJob& J = jobs[blockIdx.x / perJob];
    zone_overflow_block<false>(J.A, J.gmem, J.perBlock, J.blocksDone, J.metricsOut, (int)(blockIdx.x % perJob), perJob);
}

// run_zone_pass (src/zone_pass.cpp:1096-1163): one warp runs the zones in id order on the
// live state; a zone that outgrows the shared-memory working set is re-run at once with the
// global one (B's capacities), which is safe since a failed zone has published nothing.
__global__ void __launch_bounds__(32) k_zone_serial(ZoneArgs A, ZoneArgs B, char* gmem) {
    extern __shared__ __align__(16) char smem[];
    for (int z = 0; z < A.nZones; ++z) {
        bool ok = zone_body<true, uint16_t>(A, z, smem, A.maxCells, A.winCap, A.arenaCap, A.nsmCap);
        if (!ok) ok = zone_body<true, int>(B, z, gmem, B.maxCells, B.winCap, B.arenaCap, B.nsmCap);
        if (!ok) {
            if ((threadIdx.x & 31) == 0) raise_error(A.st, kErrZoneCapacity, z);
            return;
        }
        __syncwarp();
    }
}

// Seeded MT19937-64 state of every zone: seed = seedBase + 104729 (iz + 1)
// (src/zone_pass_openmp.cpp:78). One thread per zone runs the sequential seeding
// recurrence; states are staged in shared memory and written zone-major, coalesced.
constexpr int kSeedZonesPerBlock = 16;
__global__ void __launch_bounds__(kSeedZonesPerBlock * 2) k_zone_seeds(uint64_t seedBase, int nZones, uint64_t* out,
                                                                       const uint64_t* seedDev, int which) {
    if (seedDev) seedBase = seedDev[which];
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

// pass metrics as in k_zone_metrics, by one warp (fixed order: lane stride, then a shuffle tree)
__device__ void zone_metrics_warp(const int2* __restrict__ moved, const double2* __restrict__ corr, int nZones,
                                  double* __restrict__ out) {
    const int t = threadIdx.x & 31;
    double acc = 0.0, mx = 0.0;
    long long d = 0, s = 0;
    int c = 0;
    for (int z = t; z < nZones; z += 32) {
        const double2 q = __ldcg(corr + z);
        const int2 m = __ldcg(moved + z);
        if (q.x > 0.0) {
            acc = __dadd_rn(acc, __dmul_rn(q.x, q.x));
            ++c;
        }
        mx = smax(mx, q.y);
        d += m.x;
        s += m.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc = __dadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, o));
        mx = smax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        d += __shfl_down_sync(0xffffffffu, d, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if (t == 0) {
        out[0] = (double)d;
        out[1] = (double)s;
        out[2] = (c > 0) ? sqrt(__ddiv_rn(acc, (double)c)) : 0.0;
        out[3] = mx;
    }
}

// pass metrics: integer sums and a fixed-order reduction of the per-zone correction stats
// (also clears the overflow-zone counter for the next pass, which starts after this kernel)
__global__ void k_zone_metrics(const int2* __restrict__ moved, const double2* __restrict__ corr, int nZones,
                               double* __restrict__ out /* movedDense, movedSparse, corrRms, corrMax */,
                               int* __restrict__ nOverflow) {
    if (threadIdx.x == 0 && nOverflow) *nOverflow = 0;
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
