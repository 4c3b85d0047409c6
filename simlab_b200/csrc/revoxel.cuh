// GPU re-voxelizer of a spinning part (crates/cfd/src/shader.rs:865-1104):
// every step the part's triangles, rotated to the step's angle, are tested
// against the lattice links around them (k_tri_scatter, nearest and farthest
// hit and hit count per link, by atomics into a per-link scratch); then every
// cell of the swept box is classified (k_voxelize): solid or fluid from the
// body-frame occupancy grid, cut links and q from the scratch, a refill of
// the populations a just-uncovered cell would have sent out, and the momentum
// the part takes from cells it covers or gives to cells it uncovers; finally
// the scratch is reset for the next step (k_qclear).
//
// The geometric arithmetic is f32 rounded operation by operation (no fused
// multiply-add, IEEE division and square root), as the reference states it,
// so every cell asks "is this cell solid?" with the same arithmetic for
// itself and its neighbours (a disagreement would let a fluid cell read
// populations a solid cell never wrote), and the CPU oracle reproduces the
// classification bit for bit.
#pragma once

#include "lbm_device.cuh"
#include "spin_math.cuh"

namespace lbm {
namespace rv {

__device__ __forceinline__ bool occ_at(const LatParams &p, V3 b) { return occ_bit(p.occ, p.occ_lo, p.occ_invh, p.occ_n, b); }
// shader.rs:877-881
__device__ __forceinline__ bool solid_at(const LatParams &p, const StepParams &s, int x, int y, int z, bool before) {
    const V3 pc = {fs((float)x, p.kf.center[0]), fs((float)y, p.kf.center[1]), fs((float)z, p.kf.center[2])};
    return occ_at(p, to_body(before ? s.rot_prev : s.rot, pc));
}

}  // namespace rv

// shader.rs:902-940: one thread per triangle
__global__ void __launch_bounds__(BLOCK) k_tri_scatter(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s) {
    using namespace rv;
    // one warp per triangle, its lanes over the lattice points near it
    const uint32_t t = (blockIdx.x * BLOCK + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (t >= p.ntri) return;
    const float4 t0 = p.tris[3 * t], t1 = p.tris[3 * t + 1], t2 = p.tris[3 * t + 2];
    const V3 ctr = {p.kf.center[0], p.kf.center[1], p.kf.center[2]};
    const V3 a = add(ctr, from_body(s.rot, {t0.x, t0.y, t0.z}));
    const V3 e1 = from_body(s.rot, {t1.x, t1.y, t1.z});
    const V3 e2 = from_body(s.rot, {t2.x, t2.y, t2.z});
    const V3 nrm = cross(e1, e2);
    const float nl = __fsqrt_rn(dot(nrm, nrm));
    if (nl < 1e-12f) return;
    const V3 nn = {__fdiv_rn(nrm.x, nl), __fdiv_rn(nrm.y, nl), __fdiv_rn(nrm.z, nl)};
    const V3 b = add(a, e1), c = add(a, e2);
    const int lo[3] = {max((int)ceilf(fs(fminf(fminf(a.x, b.x), c.x), 1.415f)), p.box_lo[0]),
                       max((int)ceilf(fs(fminf(fminf(a.y, b.y), c.y), 1.415f)), p.box_lo[1]),
                       max((int)ceilf(fs(fminf(fminf(a.z, b.z), c.z), 1.415f)), p.box_lo[2])};
    const int hi[3] = {min((int)floorf(fa(fmaxf(fmaxf(a.x, b.x), c.x), 1.415f)), p.box_lo[0] + (int)p.box_n[0] - 1),
                       min((int)floorf(fa(fmaxf(fmaxf(a.y, b.y), c.y), 1.415f)), p.box_lo[1] + (int)p.box_n[1] - 1),
                       min((int)floorf(fa(fmaxf(fmaxf(a.z, b.z), c.z), 1.415f)), p.box_lo[2] + (int)p.box_n[2] - 1)};
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    const int npts = (nx > 0 && ny > 0 && nz > 0) ? nx * ny * nz : 0;
    for (int q = (int)lane; q < npts; q += 32) {
                const int x = lo[0] + q % nx, y = lo[1] + (q / nx) % ny, z = lo[2] + q / (nx * ny);
                const V3 pt = {(float)x, (float)y, (float)z};
                const float d0 = dot(nn, sub(pt, a));
                if (fabsf(d0) > 1.415f) continue;
                const uint32_t k = ((uint32_t)(z - p.box_lo[2]) * p.box_n[1] + (uint32_t)(y - p.box_lo[1])) * p.box_n[0] + (uint32_t)(x - p.box_lo[0]);
#pragma unroll
                for (int i = 1; i < 19; i += 2) {
                    const V3 cv = {(float)CX(i), (float)CY(i), (float)CZ(i)};
                    const float d1 = fa(d0, dot(nn, cv));
                    if (fm(d0, d1) > 0.0f && fabsf(d0) > 1e-6f) continue;
                    const float tt = ray_tri(pt, cv, a, e1, e2);
                    if (tt <= 1.0f) {
                        const uint64_t o = ((uint64_t)k * 9u + (uint32_t)(i - 1) / 2u) * 3u;
                        const uint32_t tb = __float_as_uint(tt > 0.0f ? tt : 0.0f);
                        atomicMin(p.qscr + o, tb);
                        atomicMax(p.qscr + o + 1, tb);
                        atomicAdd(p.qscr + o + 2, 1u);
                    }
                }
            }
}

// shader.rs:942-948
__global__ void __launch_bounds__(BLOCK) k_qclear(const __grid_constant__ LatParams p) {
    const uint64_t k = (uint64_t)blockIdx.x * BLOCK + threadIdx.x;
    if (k >= (uint64_t)p.nrec * 9u) return;
    p.qscr[3 * k] = 0x7f7fffffu;
    p.qscr[3 * k + 1] = 0u;
    p.qscr[3 * k + 2] = 0u;
}

// shader.rs:953-1104: one thread per swept-box cell (record k); Q is the
// parity of the previous step (the refill writes what the cell would have
// sent out then)
template <class S, int Q>
__global__ void __launch_bounds__(BLOCK) k_voxelize(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s) {
    using namespace rv;
    using R = typename Pop<S>::real;
    const uint32_t k = blockIdx.x * BLOCK + threadIdx.x;
    if (k >= p.nrec) return;
    const uint32_t lx = k % p.box_n[0], ly = (k / p.box_n[0]) % p.box_n[1], lz = k / (p.box_n[0] * p.box_n[1]);
    const int px = (int)lx + p.box_lo[0], py = (int)ly + p.box_lo[1], pz = (int)lz + p.box_lo[2];
    const uint32_t n = ((uint32_t)pz * p.NY + (uint32_t)py) * p.NX + (uint32_t)px;
    const Consts<R> &kk = K<R>(p);
    const R pc[3] = {(R)px - kk.center[0], (R)py - kk.center[1], (R)pz - kk.center[2]};
    const bool solid_now = solid_at(p, s, px, py, pz, false);
    const bool solid_before = solid_at(p, s, px, py, pz, true);
    R F[3] = {0, 0, 0};
    if (solid_now) {
        p.flags[n] = 1u | ((k + 1u) << 2);
        p.recs[k * RS + R_MASK] = 0u;
        if (!solid_before) {
            // covered this step: the part takes the cell's momentum
            const R rho = Rec<R>::macro(p, k, 0);
            for (int a = 0; a < 3; a++) F[a] = rho * Rec<R>::macro(p, k, 1 + a);
        }
        const R T[3] = {pc[1] * F[2] - pc[2] * F[1], pc[2] * F[0] - pc[0] * F[2], pc[0] * F[1] - pc[1] * F[0]};
        for (int a = 0; a < 3; a++) { Rec<R>::set_ft(p, k, a, F[a]); Rec<R>::set_ft(p, k, 3 + a, T[a]); }
        return;
    }
    // link hits of this step: each link is kept once, at the cell it leaves
    // in the positive direction; the cell at its other end reads it mirrored
    float qv[19], qx[19];
    uint32_t nh[19];
#pragma unroll
    for (int i = 1; i < 19; i++) {
        qv[i] = 9.0f; qx[i] = -1.0f; nh[i] = 0u;
        if (i & 1) {
            const uint64_t o = ((uint64_t)k * 9u + (uint32_t)(i - 1) / 2u) * 3u;
            const uint32_t c = p.qscr[o + 2];
            if (c) { qv[i] = __uint_as_float(p.qscr[o]); qx[i] = __uint_as_float(p.qscr[o + 1]); nh[i] = c; }
        } else {
            const int qxl = (int)lx + CX(i), qyl = (int)ly + CY(i), qzl = (int)lz + CZ(i);
            if (qxl >= 0 && qyl >= 0 && qzl >= 0 && qxl < (int)p.box_n[0] && qyl < (int)p.box_n[1] && qzl < (int)p.box_n[2]) {
                const uint32_t k2 = ((uint32_t)qzl * p.box_n[1] + (uint32_t)qyl) * p.box_n[0] + (uint32_t)qxl;
                const uint64_t o = ((uint64_t)k2 * 9u + (uint32_t)(i - 2) / 2u) * 3u;
                const uint32_t c = p.qscr[o + 2];
                if (c) { qv[i] = fs(1.0f, __uint_as_float(p.qscr[o + 1])); qx[i] = fs(1.0f, __uint_as_float(p.qscr[o])); nh[i] = c; }
            }
        }
    }
    uint32_t mask = 0;
#pragma unroll
    for (int i = 1; i < 19; i++) {
        // a wall where the neighbour is solid, or where the link crosses a
        // sheet thinner than a cell (two hits); q from the nearest hit
        if (solid_at(p, s, px + CX(i), py + CY(i), pz + CZ(i), false)) {
            if (nh[i] == 0u) qv[i] = 1.0f;
            mask |= 1u << i;
        } else if (nh[i] >= 2u && fs(qx[i], qv[i]) > 1e-5f) {
            mask |= 1u << i;
        } else {
            qv[i] = 1.0f;
        }
    }
#pragma unroll
    for (int w = 0; w < 9; w++) {
        const uint32_t lo = __half_as_ushort(__float2half_rn(fminf(qv[2 * w + 1], 1.0f)));
        const uint32_t hi = __half_as_ushort(__float2half_rn(fminf(qv[2 * w + 2], 1.0f)));
        p.recs[k * RS + R_Q + w] = lo | (hi << 16);
    }
    p.recs[k * RS + R_MASK] = mask;
    if (solid_before) {
        // uncovered this step: refill what the cell would have sent out last
        // step, the equilibrium at the wall velocity and the density of the
        // fluid neighbours plus their mean non-equilibrium stress; the part
        // gives up the refill's momentum
        R rs = 0, cnt = 0, pis[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 1; i < 19; i++) {
            const bool fluid_now = !solid_at(p, s, px + CX(i), py + CY(i), pz + CZ(i), false);
            const bool fluid_before = !solid_at(p, s, px + CX(i), py + CY(i), pz + CZ(i), true);
            if (!(fluid_now && fluid_before)) continue;
            const int qxl = (int)lx + CX(i), qyl = (int)ly + CY(i), qzl = (int)lz + CZ(i);
            if (!(qxl >= 0 && qyl >= 0 && qzl >= 0 && qxl < (int)p.box_n[0] && qyl < (int)p.box_n[1] && qzl < (int)p.box_n[2])) continue;
            const uint32_t k2 = ((uint32_t)qzl * p.box_n[1] + (uint32_t)qyl) * p.box_n[0] + (uint32_t)qxl;
            rs += Rec<R>::macro(p, k2, 0);
            cnt += (R)1;
            R fp[19];
            fp[0] = 0;
            for (int j = 1; j < 19; j++) fp[j] = Rec<R>::fpost(p, k2, j);
            const Moments<R> m2 = moments<R>(fp);
            const R r2 = Rec<R>::macro(p, k2, 0);
            const R u2[3] = {Rec<R>::macro(p, k2, 1), Rec<R>::macro(p, k2, 2), Rec<R>::macro(p, k2, 3)};
            pis[3] += m2.sxy - r2 * u2[0] * u2[1];
            pis[4] += m2.sxz - r2 * u2[0] * u2[2];
            pis[5] += m2.syz - r2 * u2[1] * u2[2];
            const R tr = (m2.sxx + m2.syy + m2.szz) / (R)3;
            const R uu = u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2];
            pis[0] += m2.sxx - tr - r2 * (u2[0] * u2[0] - uu / (R)3);
            pis[1] += m2.syy - tr - r2 * (u2[1] * u2[1] - uu / (R)3);
            pis[2] += m2.szz - tr - r2 * (u2[2] * u2[2] - uu / (R)3);
        }
        const R rho = cnt > (R)0 ? rs / cnt : (R)1;
        R om[3];
        if (sizeof(R) == 8) { om[0] = (R)s.omega_d[0]; om[1] = (R)s.omega_d[1]; om[2] = (R)s.omega_d[2]; }
        else { om[0] = (R)s.omega[0]; om[1] = (R)s.omega[1]; om[2] = (R)s.omega[2]; }
        const R uw[3] = {om[1] * pc[2] - om[2] * pc[1], om[2] * pc[0] - om[0] * pc[2], om[0] * pc[1] - om[1] * pc[0]};
        const R usq = (R)1.5 * (uw[0] * uw[0] + uw[1] * uw[1] + uw[2] * uw[2]);
        R fe[19];
#pragma unroll
        for (int i = 0; i < 19; i++) fe[i] = feq_i<R>(i, rho - (R)1, rho, uw[0], uw[1], uw[2], usq);
        if (cnt > (R)0) {
            for (int j = 0; j < 6; j++) pis[j] /= cnt;
            const R tr = (pis[0] + pis[1] + pis[2]) * (R)(1.0 / 3.0);
#pragma unroll
            for (int i = 0; i < 19; i++) fe[i] += fneq_i<R>(i, pis, tr);
        }
        const Nb nb = make_nb(p, (uint32_t)px, (uint32_t)py, (uint32_t)pz);
        Rng rng{sr_hash_mix(n, s.seed_mix)};
        store_prev_out<S, Q>(p, n, nb, 0x7ffffu, fe, rng);
        for (int a = 0; a < 3; a++) F[a] = -rho * uw[a];
        for (int i = 1; i < 19; i++) Rec<R>::set_fpost(p, k, i, fe[i]);
        Rec<R>::set_macro(p, k, 0, rho);
        for (int a = 0; a < 3; a++) Rec<R>::set_macro(p, k, 1 + a, uw[a]);
    }
    const R T[3] = {pc[1] * F[2] - pc[2] * F[1], pc[2] * F[0] - pc[0] * F[2], pc[0] * F[1] - pc[1] * F[0]};
    for (int a = 0; a < 3; a++) { Rec<R>::set_ft(p, k, a, F[a]); Rec<R>::set_ft(p, k, 3 + a, T[a]); }
    p.flags[n] = (k + 1u) << 2;
}

}  // namespace lbm
