// Kernel launchers of the D3Q19 time step (d3q19_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "lbm_device.cuh"

namespace lbm {

// storage: 0 FP32, 1 FP16, 2 BF16, 3 FP64 (lbm_storage); coll: 0 regularized, 1 BGK
// side: null, or a second stream on which the wall-cell kernel overlaps the
// face kernel (fork/join: two events); ev: null, or 4 events recorded before
// the step, after faces, after walls, after bulk
cudaError_t launch_step(int storage, const LatParams &p, const StepParams &s, int parity, int coll, cudaStream_t st, cudaStream_t side,
                        cudaEvent_t fork, cudaEvent_t join, cudaEvent_t *ev = nullptr);
cudaError_t launch_init(int storage, const LatParams &p, cudaStream_t st);
cudaError_t launch_dump(int storage, const LatParams &p, int q, cudaStream_t st);
cudaError_t launch_sample(int storage, const LatParams &p, const StepParams &s, int q, const float *verts, uint32_t nvert, float voff,
                          double *vacc, const int32_t *slicedef, uint32_t nslices, uint32_t npix, double *sacc, cudaStream_t st);
// FP64 mass and non-finite count into out[0], out[1]; scratch: 2 doubles per
// block of mass_blocks() blocks, then a u32 ticket that starts at zero
uint32_t mass_blocks();
cudaError_t launch_mass(int storage, const LatParams &p, int q, double *scratch, double *out, cudaStream_t st);
// one thread waits limit_ns for a barrier phase nothing completes: status[0] = 1 if it gave up, status[1] = us waited
cudaError_t launch_wait_selftest(uint32_t *status, uint64_t limit_ns, cudaStream_t st);

}  // namespace lbm
