// Deterministic FP64 grid reduction: every block sums its threads' values
// (warp shuffles, then the warps in order), writes one partial, and the last
// block to finish sums the partials in block order.  The result does not
// depend on which blocks ran when, unlike one atomic add per warp, and only
// one atomic per block touches a shared address.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbm {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums (a, b) over the grid into out[0], out[1].  scratch: 2 doubles per
// block, then a u32 ticket that starts at zero (the last block resets it).
// Every thread of every block calls this once, with NT threads per block.
template <int NT>
__device__ __forceinline__ void grid_sum2(double a, double b, double *scratch, double *out) {
    __shared__ double sh[NT / 32][2];
    __shared__ bool last;
    uint32_t *ticket = reinterpret_cast<uint32_t *>(scratch + 2 * (size_t)gridDim.x);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    a = warp_sum_d(a);
    b = warp_sum_d(b);
    if (lane == 0) { sh[warp][0] = a; sh[warp][1] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0, sb = 0;
        for (int w = 0; w < NT / 32; w++) { sa += sh[w][0]; sb += sh[w][1]; }
        scratch[2 * blockIdx.x] = sa;
        scratch[2 * blockIdx.x + 1] = sb;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double sa = 0, sb = 0;
    for (uint32_t k = threadIdx.x; k < gridDim.x; k += NT) {
        sa += __ldcg(&scratch[2 * k]);
        sb += __ldcg(&scratch[2 * k + 1]);
    }
    sa = warp_sum_d(sa);
    sb = warp_sum_d(sb);
    __syncthreads();
    if (lane == 0) { sh[warp][0] = sa; sh[warp][1] = sb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int w = 0; w < NT / 32; w++) { ta += sh[w][0]; tb += sh[w][1]; }
        out[0] = ta;
        out[1] = tb;
        *ticket = 0u;
    }
}

}  // namespace lbm
