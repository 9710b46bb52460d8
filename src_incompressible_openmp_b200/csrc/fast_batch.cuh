// Batched replicas of the fast form: one launch per phase for many independent channels of
// their own sizes, densities, forcings and seeds. Blocks [offs[r], offs[r + 1]) of a launch
// run replica r's blocks 0, 1, ... of the single-context kernel (the same per-block body, so
// each replica's state is bit-identical to the replica stepped alone). Each block first copies
// its replica's arguments into shared memory, which its threads then read as uniform values.
#pragma once
#include "closure.cuh"
#include "fast.cuh"

namespace mpcd_dev {

// replica r with offs[r] <= b < offs[r + 1] (offs ascending, offs[0] = 0); -1 past the end
__device__ __forceinline__ int fb_replica(const int* __restrict__ offs, int n, int b) {
    if (n <= 0 || b >= offs[n]) return -1;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// copies jobs[r] into dst (8-byte words) for the whole block
template <class T>
__device__ __forceinline__ const T& fb_stage(const T* __restrict__ jobs, int r, void* dst) {
    static_assert(sizeof(T) % 8 == 0, "batch jobs are copied in 8-byte words");
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(jobs + r);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
    for (int i = (int)threadIdx.x; i < (int)(sizeof(T) / 8); i += (int)blockDim.x) d[i] = s[i];
    __syncthreads();
    return *reinterpret_cast<const T*>(dst);
}
template <class T>
__host__ __device__ constexpr int fb_bytes() {
    return (int)((sizeof(T) + 15) / 16 * 16);
}

// step begin (block 0 of a replica, thread 0), the pass counters, and the stream's output
// counts zeroed (one thread per cell)
struct FastBeginJob {
    FastParams F;
    FastStep* S;
    FastWall* W;
    int* nSpill;
    int* moved;   // 8 counters
    int* cntOut;  // the stream's output bins
    int Nc, pad;
};

// stream (k_fast_stream's arguments)
struct FastStreamJob {
    DevParams P;
    FastParams F;
    const FastStep* S;
    FastBins in, out;
    const int2* kick;
    FastWall* W;
    DevStatus* st;
};

// a zone pass: the decision and apply kernels' arguments, the launch-order buffers
struct FastZoneJob {
    FastZoneArgs A;
    int* cost;
    int* order;
};

// closure: cells, the beta reduction, pressure drive and kick
struct FastClosureJob {
    DevParams P;
    const longlong4* ref;
    const longlong2* red;
    const int* redN;
    double* pdRaw;
    double* duRX;
    double* duRY;
    double* cols;
    double* partial;
    double* numDen;  // the reduction's output (beta num, den)
    const int* mask;
    double* pdrive;
    int2* kick;
    int anyMask, nbRed;  // the reduction's partial blocks
};
constexpr int kFastBatchRedRows = 8192;  // rows per partial block (reduce_cols' choice)

__global__ void __launch_bounds__(256) k_fb_begin(const FastBeginJob* __restrict__ jobs, const int* __restrict__ offs,
                                                  int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastBeginJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastBeginJob& J = fb_stage(jobs, r, sj);
    const int blk = (int)blockIdx.x - offs[r];
    if (blk == 0 && threadIdx.x == 0) fast_step_begin(J.F, J.S, J.W, J.nSpill);
    if (blk == 0 && threadIdx.x < 8) J.moved[threadIdx.x] = 0;
    const int c = blk * (int)blockDim.x + (int)threadIdx.x;
    if (c < J.Nc) J.cntOut[c] = 0;
}

__global__ void __launch_bounds__(256, 4) k_fb_stream(const FastStreamJob* __restrict__ jobs, const int* __restrict__ offs,
                                                     int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastStreamJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastStreamJob& J = fb_stage(jobs, r, sj);
    fast_stream_block((int)blockIdx.x - offs[r], J.P, J.F, J.S, J.in, J.out, J.kick, J.W, J.st);
}

// dynamic shared memory: the arguments, then the tile's working set
__global__ void __launch_bounds__(kCollThreads) k_fb_collide_tile(const CollideArgs* __restrict__ jobs,
                                                                  const int* __restrict__ offs, int n) {
    extern __shared__ __align__(16) char smem[];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const CollideArgs& A = fb_stage(jobs, r, smem);
    fast_collide_tile_block((int)blockIdx.x - offs[r], A, smem + fb_bytes<CollideArgs>());
}

// blocksPer blocks per replica
__global__ void __launch_bounds__(256) k_fb_collide_spill(const CollideArgs* __restrict__ jobs, int n, int blocksPer) {
    __shared__ __align__(16) char sj[fb_bytes<CollideArgs>()];
    const int r = (int)blockIdx.x / blocksPer;
    if (r >= n) return;
    const CollideArgs& A = fb_stage(jobs, r, sj);
    fast_collide_spill_block((int)blockIdx.x - r * blocksPer, blocksPer, A);
}

__global__ void k_fb_zone_cost(const FastZoneJob* __restrict__ jobs, const int* __restrict__ offs, int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastZoneJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastZoneJob& J = fb_stage(jobs, r, sj);
    fast_zone_cost_block((int)blockIdx.x - offs[r], J.A, J.cost);
}

__global__ void __launch_bounds__(kFastOrderWindow) k_fb_zone_rank(const FastZoneJob* __restrict__ jobs,
                                                                   const int* __restrict__ offs, int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastZoneJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastZoneJob& J = fb_stage(jobs, r, sj);
    fast_zone_rank_block((int)blockIdx.x - offs[r], J.cost, J.A.nZones, J.order);
}

// dynamic shared memory: the arguments, then the zones' working sets
__global__ void __launch_bounds__(32 * kFastZoneWarps, 24 / kFastZoneWarps)
    k_fb_zone(const FastZoneJob* __restrict__ jobs, const int* __restrict__ offs, int n) {
    extern __shared__ __align__(16) char smem[];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastZoneJob& J = fb_stage(jobs, r, smem);
    fast_zone_block<kFastZoneWarps>((int)blockIdx.x - offs[r], J.A, smem + fb_bytes<FastZoneJob>());
}

__global__ void __launch_bounds__(256) k_fb_zone_apply(const FastZoneJob* __restrict__ jobs, const int* __restrict__ offs,
                                                       int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastZoneJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastZoneJob& J = fb_stage(jobs, r, sj);
    fast_zone_apply_block((int)blockIdx.x - offs[r], J.A);
}

__global__ void __launch_bounds__(256) k_fb_closure_cells(const FastClosureJob* __restrict__ jobs,
                                                          const int* __restrict__ offs, int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastClosureJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastClosureJob& J = fb_stage(jobs, r, sj);
    fast_closure_cells_block((int)blockIdx.x - offs[r], J.P, J.ref, J.red, J.redN, J.pdRaw, J.duRX, J.duRY, J.cols,
                             nullptr);
}

__global__ void __launch_bounds__(kRedThreads) k_fb_reduce_partial(const FastClosureJob* __restrict__ jobs,
                                                                   const int* __restrict__ offs, int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastClosureJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastClosureJob& J = fb_stage(jobs, r, sj);
    reduce_partial_block((int)blockIdx.x - offs[r], J.cols, (int64_t)J.P.Nc, 2, 0u, kFastBatchRedRows, J.partial);
}

// one block per replica
__global__ void __launch_bounds__(kRedThreads) k_fb_reduce_final(const FastClosureJob* __restrict__ jobs, int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastClosureJob>()];
    if ((int)blockIdx.x >= n) return;
    const FastClosureJob& J = fb_stage(jobs, (int)blockIdx.x, sj);
    reduce_final_block(J.partial, J.nbRed, 2, 0u, J.numDen);
}

__global__ void __launch_bounds__(256) k_fb_pdrive(const FastClosureJob* __restrict__ jobs, const int* __restrict__ offs,
                                                   int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastClosureJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastClosureJob& J = fb_stage(jobs, r, sj);
    pdrive_blend_block((int)blockIdx.x - offs[r], J.P, J.pdRaw, J.mask, J.anyMask, J.pdrive, nullptr);
}

__global__ void __launch_bounds__(256) k_fb_kick(const FastClosureJob* __restrict__ jobs, const int* __restrict__ offs,
                                                 int n) {
    __shared__ __align__(16) char sj[fb_bytes<FastClosureJob>()];
    const int r = fb_replica(offs, n, (int)blockIdx.x);
    if (r < 0) return;
    const FastClosureJob& J = fb_stage(jobs, r, sj);
    fast_kick_cells_block((int)blockIdx.x - offs[r], J.P, J.pdrive, J.duRX, J.duRY, J.numDen, nullptr, nullptr, nullptr,
                          nullptr, J.kick, nullptr, nullptr);
}

}  // namespace mpcd_dev
