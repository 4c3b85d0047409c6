// Host-side waits with a time limit: every wait of the library on device
// work polls and gives up after its limit instead of blocking for good.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <thread>

namespace lbm {

// Waits for the work queued on stream s, at most limit_s seconds.  Returns
// cudaSuccess, the stream's error, or cudaErrorTimeout when the limit passed.
inline cudaError_t stream_wait(cudaStream_t s, double limit_s) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaStreamQuery(s);
        if (q != cudaErrorNotReady) return q;
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit_s) return cudaErrorTimeout;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

}  // namespace lbm
