// Force and moment sum over wall records without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need
// this sum: hosts whose device memory is all handed out by their own pool
// allocator, embedded callers that must keep a fixed device footprint, and
// latency-critical loops that cannot afford cudaMalloc/cudaFree, which may
// synchronise the whole device.  lbm_record_forces_noalloc sums the force and
// moment words of wall records that already live in device memory (the
// 40-word D3Q19 layout lbm_records returns) into six doubles in device
// memory, using only a scratch area that is part of this library's image: a
// file-scope __device__ array of a fixed, modest size that every GPU loading
// the library keeps until the process exits.  The caller passes the inputs
// and the output; nothing is allocated or freed.
//
// The sum is over the records' float force words (FP32 values summed in
// FP64), also for FP64-storage lattices, whose lbm_run forces sum the double
// copies instead; the two then differ at float rounding.
//
// The scratch is shared by every call on a device and keeps the last call's
// contents; each call clears the counter it needs before using it.  Two calls
// whose kernels overlap on the GPU (different streams, no ordering between
// them) race on the scratch and must not be issued.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/simlab_lbm.h"
#include "lbm_device.cuh"

namespace {

constexpr uint32_t NA_BLOCK = 256;
constexpr uint64_t NA_MAX_RECORDS = 1ull << 20;                   // 1,048,576 records
constexpr uint32_t NA_MAX_BLOCKS = (uint32_t)(NA_MAX_RECORDS / NA_BLOCK);  // 4096
// the engine's D3Q19 record layout (force at R_FT..R_FT+2, moment after it)
constexpr uint32_t REC_WORDS = lbm::RS, REC_FT = lbm::R_FT;
static_assert(REC_WORDS == 40 && REC_FT + 6 <= REC_WORDS, "wall record layout of lbm_records");

struct NoallocScratch {
    double partials[NA_MAX_BLOCKS * 8];  // per-block sums (6 used of 8), 256 KiB
    unsigned int ticket;                 // blocks finished; the last one reduces
};

static __device__ __align__(256) NoallocScratch g_scratch;

__device__ __forceinline__ double warp_sum_na(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// one record per thread; FP64 warp shuffles, then per block, then the last
// block sums the block partials in a fixed order
__global__ void __launch_bounds__(NA_BLOCK) k_record_sum(const uint32_t *recs, uint32_t nrec, NoallocScratch *scr, double *out) {
    const uint32_t r = blockIdx.x * NA_BLOCK + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (r < nrec)
        for (int j = 0; j < 6; j++) v[j] = (double)__uint_as_float(recs[(uint64_t)r * REC_WORDS + REC_FT + j]);
    __shared__ double sh[NA_BLOCK / 32][6];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = 0; j < 6; j++) v[j] = warp_sum_na(v[j]);
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = v[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < (int)(NA_BLOCK / 32); w++) t += sh[w][threadIdx.x];
        scr->partials[blockIdx.x * 8 + threadIdx.x] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&scr->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += NA_BLOCK)
        for (int j = 0; j < 6; j++) acc[j] += __ldcg(&scr->partials[b * 8 + j]);
    for (int j = 0; j < 6; j++) acc[j] = warp_sum_na(acc[j]);
    __syncthreads();
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = acc[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < (int)(NA_BLOCK / 32); w++) t += sh[w][threadIdx.x];
        out[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) scr->ticket = 0u;
}

std::mutex g_mu;
// scratch address per device ordinal, found once per device; this assumes
// the device's primary context lives as long as the process (a
// cudaDeviceReset would leave a stale address here)
NoallocScratch *g_ptr[64] = {};
thread_local std::string g_err;

}  // namespace

extern "C" {

int lbm_noalloc_error(char *buf, uint64_t len) {
    if (buf && len) {
        std::strncpy(buf, g_err.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return LBM_OK;
}

uint64_t lbm_record_forces_noalloc_max(void) { return NA_MAX_RECORDS; }

int lbm_record_forces_noalloc(const uint32_t *records_dev, uint64_t nrec, double *forces_dev, void *stream) {
    if (!forces_dev || (nrec && !records_dev)) {
        g_err = "null device pointer";
        return LBM_ERR_INVALID;
    }
    if (nrec > NA_MAX_RECORDS) {
        g_err = "too many records for the allocation-free sum: " + std::to_string(nrec) + " > " + std::to_string(NA_MAX_RECORDS);
        return LBM_ERR_INVALID;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        g_err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return LBM_ERR_CUDA;
    }
    NoallocScratch *scr;
    {
        // first call on this device: the scratch array's device address (a
        // host-side use of the symbol itself would be a host address)
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_ptr[dev]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_scratch);
            if (e != cudaSuccess || !ptr) {
                g_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return LBM_ERR_CUDA;
            }
            g_ptr[dev] = (NoallocScratch *)ptr;
        }
        scr = g_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (nrec == 0) {
        e = cudaMemsetAsync(forces_dev, 0, 6 * sizeof(double), st);
    } else {
        e = cudaMemsetAsync(&scr->ticket, 0, sizeof(unsigned int), st);  // start from zero whatever an earlier call left
        if (e == cudaSuccess) {
            const unsigned blocks = (unsigned)((nrec + NA_BLOCK - 1) / NA_BLOCK);
            k_record_sum<<<blocks, NA_BLOCK, 0, st>>>(records_dev, (uint32_t)nrec, scr, forces_dev);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess) {
        g_err = std::string("record sum: ") + cudaGetErrorString(e);
        return LBM_ERR_CUDA;
    }
    return LBM_OK;
}

}  // extern "C"
