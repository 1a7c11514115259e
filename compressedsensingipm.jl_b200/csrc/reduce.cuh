// Deterministic grid-wide reductions.
//
// Each block reduces its threads' values in a fixed tree order and writes one
// partial per block; the last block to finish (atomic ticket) reduces the
// partials in block order and writes the final values.  The result is the same
// bit pattern on every run, independent of scheduling, so iteration counts are
// reproducible.  Components are summed, or max-reduced when their index is in
// the MAXMASK bit set, or min-reduced when in MINMASK.
#pragma once
#include <cuda_runtime.h>
#include <float.h>

namespace csipm {

struct RedWorkspace {
    double* partials;        // [max_blocks * NV]
    unsigned int* ticket;    // one counter, zero between launches
    double* out;             // [NV] final values
    int xonly = 0;           // 1: the blocks of one blockIdx.y / z reduce on their own (batched launches,
                             // one instance per blockIdx.y, each with its own workspace)
};

__device__ __forceinline__ double red_op(double a, double b, int comp, unsigned maxmask, unsigned minmask) {
    if ((maxmask >> comp) & 1u) return fmax(a, b);
    if ((minmask >> comp) & 1u) return fmin(a, b);
    return a + b;
}

__device__ __forceinline__ double red_identity(int comp, unsigned maxmask, unsigned minmask) {
    if ((maxmask >> comp) & 1u) return -DBL_MAX;
    if ((minmask >> comp) & 1u) return DBL_MAX;
    return 0.0;
}

// Reduce NV values held by every thread of the block; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], unsigned maxmask, unsigned minmask) {
    __shared__ double sh[NV][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        double x = v[c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x = red_op(x, __shfl_down_sync(0xffffffffu, x, off), c, maxmask, minmask);
        if (lane == 0) sh[c][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            double x = lane < nwarps ? sh[c][lane] : red_identity(c, maxmask, minmask);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x = red_op(x, __shfl_down_sync(0xffffffffu, x, off), c, maxmask, minmask);
            v[c] = x;
        }
    }
    __syncthreads();
}

// Grid-wide: every block calls this exactly once with its threads' values.
// The last block writes ws.out[0..NV) and resets the ticket.  Returns true in
// the threads of the last block (after the result is written).
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], const RedWorkspace& ws, unsigned maxmask, unsigned minmask) {
    block_reduce<NV>(v, maxmask, minmask);
    const unsigned nblocks = ws.xonly ? gridDim.x : gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = ws.xonly ? blockIdx.x : blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) ws.partials[(size_t)bid * NV + c] = v[c];
        __threadfence();
        const unsigned t = atomicAdd(ws.ticket, 1u);
        last = (t == nblocks - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) acc[c] = red_identity(c, maxmask, minmask);
    // fixed order: thread t reduces blocks t, t+nthr, ... then the block tree
    for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            volatile double* p = ws.partials;
            acc[c] = red_op(acc[c], p[(size_t)b * NV + c], c, maxmask, minmask);
        }
    }
    block_reduce<NV>(acc, maxmask, minmask);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) ws.out[c] = acc[c];
        *ws.ticket = 0u;
        __threadfence();
    }
    __syncthreads();
    return true;
}

}  // namespace csipm
