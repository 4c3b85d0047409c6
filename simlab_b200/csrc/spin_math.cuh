// f32 geometry of the GPU re-voxelizers (shared by the D3Q19 and D3Q27
// lattices): vector arithmetic rounded operation by operation (no fused
// multiply-add, IEEE division and square root), body-frame rotations and the
// segment-triangle test of crates/cfd/src/shader.rs:883-897, plus the
// occupancy lookup of shader.rs:866-871.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lbm {
namespace rv {

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return {fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)), fs(fm(a.x, b.y), fm(a.y, b.x))};
}
// rot is row-major with the body axes as columns: to_body = R^T v, from_body = R b
__device__ __forceinline__ V3 col(const float *rot, int k) { return {rot[k], rot[3 + k], rot[6 + k]}; }
__device__ __forceinline__ V3 to_body(const float *rot, V3 v) { return {dot(col(rot, 0), v), dot(col(rot, 1), v), dot(col(rot, 2), v)}; }
__device__ __forceinline__ V3 from_body(const float *rot, V3 b) {
    const V3 c0 = col(rot, 0), c1 = col(rot, 1), c2 = col(rot, 2);
    return {fa(fa(fm(c0.x, b.x), fm(c1.x, b.y)), fm(c2.x, b.z)), fa(fa(fm(c0.y, b.x), fm(c1.y, b.y)), fm(c2.y, b.z)),
            fa(fa(fm(c0.z, b.x), fm(c1.z, b.y)), fm(c2.z, b.z))};
}

// shader.rs:883-897: Moller-Trumbore, 9 when there is no hit
__device__ __forceinline__ float ray_tri(V3 o, V3 d, V3 v0, V3 e1, V3 e2) {
    const V3 pv = cross(d, e2);
    const float det = dot(e1, pv);
    if (fabsf(det) < 1e-12f) return 9.0f;
    const float inv = __fdiv_rn(1.0f, det);
    const V3 tv = sub(o, v0);
    const float a = fm(dot(tv, pv), inv);
    if (a < 0.0f || a > 1.0f) return 9.0f;
    const V3 qv = cross(tv, e1);
    const float b = fm(dot(d, qv), inv);
    if (b < 0.0f || fa(a, b) > 1.0f) return 9.0f;
    const float t = fm(dot(e2, qv), inv);
    if (t < -1e-4f || t > 1.0f) return 9.0f;
    return t > 0.0f ? t : 0.0f;  // +0 for -0 too: the hit bits are compared as integers
}

// the occupancy bit nearest to a body-frame point (shader.rs:866-871)
__device__ __forceinline__ bool occ_bit(const uint32_t *occ, const float *lo, float invh, const int32_t *n, V3 b) {
    const float gx = rintf(fm(fs(b.x, lo[0]), invh));
    const float gy = rintf(fm(fs(b.y, lo[1]), invh));
    const float gz = rintf(fm(fs(b.z, lo[2]), invh));
    if (!(gx >= 0.f && gy >= 0.f && gz >= 0.f) || gx >= (float)n[0] || gy >= (float)n[1] || gz >= (float)n[2]) return false;
    const uint32_t l = ((uint32_t)gz * (uint32_t)n[1] + (uint32_t)gy) * (uint32_t)n[0] + (uint32_t)gx;
    return ((__ldg(occ + (l >> 5)) >> (l & 31u)) & 1u) != 0u;
}

}  // namespace rv
}  // namespace lbm
