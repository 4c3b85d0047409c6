// Multi-level D3Q27 kernels for sm_100a.
//
// One level step (crates/cfd/src/mshader.rs:612-699): each fluid cell pulls
// the post-collision populations of its 26 neighbours from the source set,
// applies Bouzidi bounce-back with moving-wall momentum exchange on its cut
// links (mshader.rs:364-403), takes moments, relaxes the deviatoric second
// central moments with the viscous rate (Smagorinsky and sponge on tau), sets
// the trace and every higher cumulant to equilibrium, rebuilds the
// populations of that Gaussian by backward central-moment transforms (`gauss`,
// mshader.rs:286-362), adds the absorbing layer and writes the result to the
// destination set.  Cells on a child box surface export their moments for the
// child's ghosts; even nodes of a refined level export theirs for the
// parent's restriction.
//
// Level kernels (mshader.rs:702-793): domain faces rebuilt from the interior
// cell, fine ghosts interpolated in space and time from the parent's surface
// moments with the Dupuis-Chopard stress rescale, coarse cells under the child
// box restricted from the coincident fine nodes.
//
// Memory-bound (220 B per cell update in FP32, 112 B in FP16/BF16): one thread
// per cell, 27 coalesced loads from the source planes (x-shifted loads served
// by L1), 27 coalesced stores.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>

#include "d3q27.h"
#include "spin_math.cuh"
#include "reduce.cuh"

namespace lbm27 {

using lbm::FastDiv;
using lbm::Pop;
using lbm::Rng;

constexpr int BLK = 256;

template <class R> __device__ __forceinline__ R W(int i) { return (R)WD(i); }
template <> __device__ __forceinline__ float W<float>(int i) { return (float)WD(i); }
template <class R> __device__ __forceinline__ R W45(int i) { return (R)(4.5 * WD(i)); }

template <class R> __device__ __forceinline__ const Consts27<R> &K(const LevelParams &p);
template <> __device__ __forceinline__ const Consts27<float> &K<float>(const LevelParams &p) { return p.kf; }
template <> __device__ __forceinline__ const Consts27<double> &K<double>(const LevelParams &p) { return p.kd; }

__device__ __forceinline__ void coords(const LevelParams &p, uint32_t n, uint32_t &x, uint32_t &y, uint32_t &z) {
    z = p.div_nxy.div(n);
    const uint32_t r = n - z * (p.NX * p.NY);
    y = p.div_nx.div(r);
    x = r - y * p.NX;
}

template <class S>
__device__ __forceinline__ const S *set_ptr(const LevelParams &p, uint32_t set) { return (const S *)p.pop + (uint64_t)set * 27u * p.NP; }
template <class S>
__device__ __forceinline__ S *set_ptr_w(const LevelParams &p, uint32_t set) { return (S *)p.pop + (uint64_t)set * 27u * p.NP; }

// own post-collision populations of cell n (mshader.rs:201-206)
template <class S>
__device__ __forceinline__ void own(const LevelParams &p, uint32_t set, uint32_t n, typename Pop<S>::real *f) {
    const S *s = set_ptr<S>(p, set);
#pragma unroll
    for (int i = 0; i < 27; i++) f[i] = Pop<S>::ld(s + (uint64_t)i * p.NP + n);
}
// writes a full post-collision state (mshader.rs:207-217)
template <class S>
__device__ __forceinline__ void put(const LevelParams &p, uint32_t set, uint32_t n, const typename Pop<S>::real *f, Rng &rng) {
    S *s = set_ptr_w<S>(p, set);
#pragma unroll
    for (int i = 0; i < 27; i++) s[(uint64_t)i * p.NP + n] = Pop<S>::enc(f[i], rng);
}

template <class R>
struct Mom {
    R rho1, j[3], s[6];
};

// mshader.rs:236-255
template <class R>
__device__ __forceinline__ Mom<R> moments(const R *f) {
    // sums over the x-rows (cy, cz fixed): row totals and x-differences
    R rs[9], rd[9];
#pragma unroll
    for (int r = 0; r < 9; r++) {
        rs[r] = (f[3 * r] + f[3 * r + 1]) + f[3 * r + 2];
        rd[r] = f[3 * r + 2] - f[3 * r];
    }
    Mom<R> m;
    // rows r = (cy + 1) + 3 (cz + 1)
    const R zm = (rs[0] + rs[1]) + rs[2], z0 = (rs[3] + rs[4]) + rs[5], zp = (rs[6] + rs[7]) + rs[8];
    m.rho1 = (zm + z0) + zp;
    m.j[0] = ((rd[0] + rd[1]) + rd[2]) + ((rd[3] + rd[4]) + rd[5]) + ((rd[6] + rd[7]) + rd[8]);
    const R ym = (rs[0] + rs[3]) + rs[6], yp = (rs[2] + rs[5]) + rs[8];
    m.j[1] = yp - ym;
    m.j[2] = zp - zm;
    // sxx: rows' f[+x] + f[-x]
    R sx = 0;
#pragma unroll
    for (int r = 0; r < 9; r++) sx += f[3 * r] + f[3 * r + 2];
    m.s[0] = sx;
    m.s[1] = ym + yp;
    m.s[2] = zm + zp;
    // sxy = sum cx cy f: rows with cy = +1 minus rows with cy = -1 of rd
    m.s[3] = ((rd[2] + rd[5]) + rd[8]) - ((rd[0] + rd[3]) + rd[6]);
    m.s[4] = ((rd[6] + rd[7]) + rd[8]) - ((rd[0] + rd[1]) + rd[2]);
    m.s[5] = (rs[8] - rs[6]) - (rs[2] - rs[0]);
    return m;
}

// mshader.rs:257-266: product-form equilibrium, shifted
template <class R>
__device__ __forceinline__ void feq(R rho, R ux, R uy, R uz, R *f) {
    const R third = (R)1 / (R)3, two3 = (R)2 / (R)3, h = (R)0.5;
    const R u[3] = {ux, uy, uz};
    R a[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const R uu = u[k] * u[k];
        a[k][0] = h * (third + uu - u[k]);
        a[k][1] = two3 - uu;
        a[k][2] = h * (third + uu + u[k]);
    }
#pragma unroll
    for (int i = 0; i < 27; i++) f[i] = rho * a[0][CX(i) + 1] * a[1][CY(i) + 1] * a[2][CZ(i) + 1] - W<R>(i);
}

// mshader.rs:268-280: 4.5 w (c c : p - tr p / 3)
template <class R>
__device__ __forceinline__ void fneq_add(const R *p, R *f) {
    const R tr = (p[0] + p[1] + p[2]) * ((R)1 / (R)3);
#pragma unroll
    for (int i = 0; i < 27; i++) {
        R t = -tr;
        if (CX(i) != 0) t = t + p[0];
        if (CY(i) != 0) t = t + p[1];
        if (CZ(i) != 0) t = t + p[2];
        if (CX(i) * CY(i) != 0) t = t + (R)(2 * CX(i) * CY(i)) * p[3];
        if (CX(i) * CZ(i) != 0) t = t + (R)(2 * CX(i) * CZ(i)) * p[4];
        if (CY(i) * CZ(i) != 0) t = t + (R)(2 * CY(i) * CZ(i)) * p[5];
        f[i] += W45<R>(i) * t;
    }
}

// mshader.rs:486-501
template <class R>
__device__ __forceinline__ void stress(const Mom<R> &mo, R rho, const R *u, R *p) {
    const R r3 = mo.rho1 / (R)3;
    p[0] = mo.s[0] - rho * u[0] * u[0] - r3;
    p[1] = mo.s[1] - rho * u[1] * u[1] - r3;
    p[2] = mo.s[2] - rho * u[2] * u[2] - r3;
    p[3] = mo.s[3] - rho * u[0] * u[1];
    p[4] = mo.s[4] - rho * u[0] * u[2];
    p[5] = mo.s[5] - rho * u[1] * u[2];
}
template <class R>
__device__ __forceinline__ void deviator(const R *p, R *d) {
    const R tr = (p[0] + p[1] + p[2]) / (R)3;
    d[0] = p[0] - tr; d[1] = p[1] - tr; d[2] = p[2] - tr;
    d[3] = p[3]; d[4] = p[4]; d[5] = p[5];
}
// mshader.rs:503-509: a post-collision state from rho, u and a stress
template <class R>
__device__ __forceinline__ void rebuild(R rho, const R *u, const R *pp, R *f) {
    feq<R>(rho, u[0], u[1], u[2], f);
    R d[6];
    deviator<R>(pp, d);
    fneq_add<R>(d, f);
}

template <class R>
__device__ __forceinline__ R sponge(const LevelParams &p, const Consts27<R> &k, uint32_t x, uint32_t y, uint32_t z) {
    const R pp[3] = {(R)(float)x, (R)(float)y, (R)(float)z};
    const R hi[3] = {(R)(float)(p.NX - 1) - pp[0], (R)(float)(p.NY - 1) - pp[1], (R)(float)(p.NZ - 1) - pp[2]};
    R s = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (k.sp_lo[a] > (R)0) s = max(s, (R)1 - pp[a] / k.sp_lo[a]);
        if (k.sp_hi[a] > (R)0) s = max(s, (R)1 - hi[a] / k.sp_hi[a]);
    }
    return min(max(s, (R)0), (R)1);
}

template <class S>
__device__ __forceinline__ Rng cell_rng(uint32_t n, uint32_t seed_mix) {
    Rng r;
    r.s = lbm::sr_hash_mix(n, seed_mix);
    return r;
}

// ------------------------------------------------------------ the step
// Storage in raw units: FP16 keeps (f - w) * 32768, the others f - w.  The
// step works on raw loads (no per-population rescale), scales the moments
// once, and folds the scale back into the last multiply of each output.
// Stochastic rounding converts two values per generator step.
template <class S> struct Raw;
template <> struct Raw<float> {
    static constexpr float SC = 1.0f;
    static __device__ __forceinline__ float ld(const float *p) { return *p; }
    static __device__ __forceinline__ void st2(float *a, float va, float *b, float vb, Rng &) { *a = va; *b = vb; }
    static __device__ __forceinline__ void st1(float *a, float va, Rng &) { *a = va; }
};
template <> struct Raw<double> {
    static constexpr double SC = 1.0;
    static __device__ __forceinline__ double ld(const double *p) { return *p; }
    static __device__ __forceinline__ void st2(double *a, double va, double *b, double vb, Rng &) { *a = va; *b = vb; }
    static __device__ __forceinline__ void st1(double *a, double va, Rng &) { *a = va; }
};
template <> struct Raw<__half> {
    static constexpr float SC = lbm::FP16_SCALE;
    static __device__ __forceinline__ float ld(const __half *p) { return __half2float(*p); }
    // one stochastically rounding conversion per pair
    static __device__ __forceinline__ void st2(__half *a, float va, __half *b, float vb, Rng &r) {
        const uint32_t h2 = lbm::cvt_rs_f16x2(va, vb, r.next2());
        *a = __ushort_as_half((unsigned short)(h2 >> 16));
        *b = __ushort_as_half((unsigned short)(h2 & 0xffffu));
    }
    static __device__ __forceinline__ void st1(__half *a, float va, Rng &r) {
        *a = __ushort_as_half((unsigned short)(lbm::cvt_rs_f16x2(va, 0.0f, r.next()) >> 16));
    }
};
template <> struct Raw<__nv_bfloat16> {
    static constexpr float SC = 1.0f;
    static __device__ __forceinline__ float ld(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ void st2(__nv_bfloat16 *a, float va, __nv_bfloat16 *b, float vb, Rng &r) {
        const uint32_t h2 = lbm::cvt_rs_bf16x2(va, vb, r.next2());
        *a = __ushort_as_bfloat16((unsigned short)(h2 >> 16));
        *b = __ushort_as_bfloat16((unsigned short)(h2 & 0xffffu));
    }
    static __device__ __forceinline__ void st1(__nv_bfloat16 *a, float va, Rng &r) {
        *a = __ushort_as_bfloat16((unsigned short)(lbm::cvt_rs_bf16x2(va, 0.0f, r.next()) >> 16));
    }
};

// backward transforms with the factor 1/2 of the outer two outputs deferred:
// returns (2 f-, f0, 2 f+) of mshader.rs:316-322; w2 = 2 w, ww = w^2
template <class R>
__device__ __forceinline__ void bk(R k0, R k1, R k2, R w, R w2, R ww, R &m, R &o, R &pl) {
    const R r1 = k1 + w * k0;
    const R r2 = k2 + w2 * k1 + ww * k0;
    m = r2 - r1; o = k0 - r2; pl = r2 + r1;
}
template <class R>  // k1 = 0
__device__ __forceinline__ void bk_even(R k0, R k2, R w, R ww, R &m, R &o, R &pl) {
    const R r1 = w * k0;
    const R r2 = k2 + ww * k0;
    m = r2 - r1; o = k0 - r2; pl = r2 + r1;
}
template <class R>  // k0 = k2 = 0
__device__ __forceinline__ void bk_odd(R k1, R w2, R &m, R &o, R &pl) {
    const R r2 = w2 * k1;
    m = r2 - k1; o = -r2; pl = r2 + k1;
}

// The Gaussian's populations (mshader.rs:286-362) with rho factored out of
// every central moment and the halves deferred: output (cx, cy, cz) carries
// the factor 2^(|cx|+|cy|+|cz|), removed with rho and the storage scale in
// the final multiply-add emit(i, X * rs[|c|] - SC w_i).
template <class R, bool FORCE, class Emit>
__device__ __forceinline__ void gauss_raw(const R *u, const R *sg, const R *m1, const R *rs, R SC, Emit &&emit) {
    const R a = sg[0], b = sg[1], cc = sg[2], d = sg[3], e = sg[4], g = sg[5];
    const R two = 2;
    const R k220 = a * b + two * d * d, k202 = a * cc + two * e * e, k022 = b * cc + two * g * g;
    const R k211 = a * g + two * d * e, k121 = b * e + two * d * g, k112 = cc * d + two * e * g;
    const R k222 = a * b * cc + two * (a * g * g + b * e * e + cc * d * d) + (R)8 * d * e * g;
    R w2[3], ww[3];
#pragma unroll
    for (int c = 0; c < 3; c++) { w2[c] = two * u[c]; ww[c] = u[c] * u[c]; }
    R Z[3][3][3];
    const R wz = u[2];
    if (FORCE) {
        bk<R>((R)1, m1[2], cc, wz, w2[2], ww[2], Z[0][0][0], Z[0][0][1], Z[0][0][2]);
        bk<R>(m1[0], e, (R)0, wz, w2[2], ww[2], Z[1][0][0], Z[1][0][1], Z[1][0][2]);
        bk<R>(m1[1], g, (R)0, wz, w2[2], ww[2], Z[0][1][0], Z[0][1][1], Z[0][1][2]);
    } else {
        bk_even<R>((R)1, cc, wz, ww[2], Z[0][0][0], Z[0][0][1], Z[0][0][2]);
        bk_odd<R>(e, w2[2], Z[1][0][0], Z[1][0][1], Z[1][0][2]);
        bk_odd<R>(g, w2[2], Z[0][1][0], Z[0][1][1], Z[0][1][2]);
    }
    bk_even<R>(a, k202, wz, ww[2], Z[2][0][0], Z[2][0][1], Z[2][0][2]);
    bk_even<R>(d, k112, wz, ww[2], Z[1][1][0], Z[1][1][1], Z[1][1][2]);
    bk_odd<R>(k211, w2[2], Z[2][1][0], Z[2][1][1], Z[2][1][2]);
    bk_even<R>(b, k022, wz, ww[2], Z[0][2][0], Z[0][2][1], Z[0][2][2]);
    bk_odd<R>(k121, w2[2], Z[1][2][0], Z[1][2][1], Z[1][2][2]);
    bk_even<R>(k220, k222, wz, ww[2], Z[2][2][0], Z[2][2][1], Z[2][2][2]);
    R Y[3][3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int c = 0; c < 3; c++) bk<R>(Z[i][0][c], Z[i][1][c], Z[i][2][c], u[1], w2[1], ww[1], Y[i][c][0], Y[i][c][1], Y[i][c][2]);
#pragma unroll
    for (int cyi = 0; cyi < 3; cyi++)
#pragma unroll
        for (int czi = 0; czi < 3; czi++) {
            R m, o, pl;
            bk<R>(Y[0][czi][cyi], Y[1][czi][cyi], Y[2][czi][cyi], u[0], w2[0], ww[0], m, o, pl);
            const int base = 3 * cyi + 9 * czi;  // direction (cx = -1, cy, cz)
            const int nz = (cyi != 1) + (czi != 1);
            emit(base, m * rs[nz + 1] - SC * W<R>(base));
            emit(base + 1, o * rs[nz] - SC * W<R>(base + 1));
            emit(base + 2, pl * rs[nz + 1] - SC * W<R>(base + 2));
        }
}

// Blocks of 256 threads per SM the step kernel is compiled for.  With the
// wall arithmetic in its own kernel, FP32, FP16 and BF16 fit 64 registers
// without spilling when the level has neither periodic axes nor sponges, so
// those run four blocks; sponges (the viscosity ramp and the absorbing
// layer) need 80 registers and run three, periodic wrap (offsets per thread)
// three, and both two.  The FP64 engine (a validation instrument) keeps the
// compiler's choice.
template <class S, bool WRAP, bool SPONGE> struct StepOcc {
    static constexpr int value = WRAP ? (SPONGE ? 2 : 3) : (SPONGE ? 3 : 4);
};
template <bool WRAP, bool SPONGE> struct StepOcc<double, WRAP, SPONGE> { static constexpr int value = 1; };

// WRAP: the level has periodic axes (neighbour offsets per thread); without
// them no stepped cell touches the boundary, and every neighbour offset is
// uniform across the grid
// One cell's update once its 27 pulled populations f (storage units) are
// in registers: walls, cumulant collision, stores into the other set, the
// moments the neighbouring levels read (mshader.rs:199-403,612-699).
// SPONGE: the level has sponge layers (viscosity ramp and absorbing layer);
// without them the code is left out, not predicated off per lane
template <class S, bool FORCE, bool SPONGE>
__device__ __forceinline__ void cell27(const LevelParams &p, const StepArgs &a, uint32_t n, uint32_t fg, uint32_t x, uint32_t y, uint32_t z,
                                       typename Pop<S>::real *f) {
    using R = typename Pop<S>::real;
    const Consts27<R> &k = K<R>(p);
    const R SC = (R)Raw<S>::SC, ISC = (R)1 / (R)Raw<S>::SC;
    const int64_t NP = (int64_t)p.NP;
    const uint32_t rec = fg >> 3;
    if (rec != 0) {
        // the wall populations k27_walls computed for this cell this step
        const uint32_t r = rec - 1;
        const uint32_t mask = p.recs[r * RS + R_MASK];
        const R *wf = (const R *)p.wallf + (uint64_t)r * 27;
#pragma unroll
        for (int i = 0; i < 27; i++)
            if (i != 13 && (mask & (1u << i))) f[26 - i] = wf[26 - i];
    }
    Mom<R> mo = moments<R>(f);
    if (Raw<S>::SC != 1) {
        mo.rho1 *= ISC;
#pragma unroll
        for (int c = 0; c < 3; c++) mo.j[c] *= ISC;
#pragma unroll
        for (int c = 0; c < 6; c++) mo.s[c] *= ISC;
    }
    const R rho = (R)1 + mo.rho1;
    const R inv_rho = (R)1 / rho;
    R G[3] = {0, 0, 0}, u[3];
    if (FORCE) {
#pragma unroll
        for (int c = 0; c < 3; c++) G[c] = rho * k.grav[c];
    }
#pragma unroll
    for (int c = 0; c < 3; c++) u[c] = FORCE ? (mo.j[c] + (R)0.5 * G[c]) * inv_rho : mo.j[c] * inv_rho;
    R pst[6];
    stress<R>(mo, rho, u, pst);
    R dv[6];
    deviator<R>(pst, dv);
    R tau = k.tau0;
    if (k.smag2 > (R)0) {
        const R pp = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2] + (R)2 * (dv[3] * dv[3] + dv[4] * dv[4] + dv[5] * dv[5]);
        tau = (R)0.5 * (k.tau0 + sqrt(k.tau0 * k.tau0 + (R)18 * k.smag2 * sqrt((R)2 * pp) * inv_rho));
    }
    R sp = 0;
    if (SPONGE && p.n_sponge) {
        sp = sponge<R>(p, k, x, y, z);
        if (sp > (R)0 && k.sponge_tau > tau) tau += sp * sp * (k.sponge_tau - tau);
    }
    const R om1 = (R)1 - (R)1 / tau;
    const R third = (R)1 / (R)3;
    R sg[6];
    const R om1r = om1 * inv_rho;
#pragma unroll
    for (int c = 0; c < 3; c++) sg[c] = third + om1r * dv[c];
#pragma unroll
    for (int c = 3; c < 6; c++) sg[c] = om1r * dv[c];
    R m1[3] = {0, 0, 0};
    if (FORCE) {
#pragma unroll
        for (int c = 0; c < 3; c++) m1[c] = (R)0.5 * G[c] * inv_rho;
    }
    // absorbing layer (mshader.rs:663-673): fo += sigma sp^2 (feq(1, ut) - feq(rho, u)),
    // both product-form equilibria, so per direction a product of axis factors
    const bool absorb = SPONGE && p.n_sponge && k.sigma > (R)0 && sp > (R)0;
    R at[3][3], ac[3][3], sgm = 0;
    if (absorb) {
        const R h = (R)0.5;
        const R ut[3] = {p.abs_u ? k.u_inf[0] : u[0], p.abs_u ? k.u_inf[1] : u[1], p.abs_u ? k.u_inf[2] : u[2]};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const R tt = ut[c] * ut[c], uu = u[c] * u[c];
            at[c][0] = h * (third + tt - ut[c]); at[c][1] = (R)2 / (R)3 - tt; at[c][2] = h * (third + tt + ut[c]);
            ac[c][0] = h * (third + uu - u[c]); ac[c][1] = (R)2 / (R)3 - uu; ac[c][2] = h * (third + uu + u[c]);
        }
        sgm = k.sigma * sp * sp * SC;
    }
    const R rs[4] = {rho * SC, rho * SC * (R)0.5, rho * SC * (R)0.25, rho * SC * (R)0.125};
    Rng rng = cell_rng<S>(n, a.seed_mix);
    S *dstn = set_ptr_w<S>(p, 1u - a.src) + n;
    R pend = 0;
    int pend_i = -1;
    gauss_raw<R, FORCE>(u, sg, m1, rs, SC, [&](int i, R v) {
        if (SPONGE && absorb) {
            const int ix = CX(i) + 1, iy = CY(i) + 1, iz = CZ(i) + 1;
            v += sgm * (at[0][ix] * at[1][iy] * at[2][iz] - rho * ac[0][ix] * ac[1][iy] * ac[2][iz]);
        }
        // stores go out in pairs (in emission order) so one generator step
        // rounds two values; the indices are compile-time after unrolling
        if (pend_i < 0) {
            pend = v;
            pend_i = i;
        } else {
            Raw<S>::st2(dstn + (int64_t)pend_i * NP, pend, dstn + (int64_t)i * NP, v, rng);
            pend_i = -1;
        }
    });
    if (pend_i >= 0) Raw<S>::st1(dstn + (int64_t)pend_i * NP, pend, rng);
    // moments for the finer level's ghosts (child box surface)
    if (p.has_child) {
        const int lx = (int)x - p.ch_lo[0], ly = (int)y - p.ch_lo[1], lz = (int)z - p.ch_lo[2];
        if (lx >= 0 && ly >= 0 && lz >= 0 && lx < (int)p.ch_n[0] && ly < (int)p.ch_n[1] && lz < (int)p.ch_n[2] &&
            (lx == 0 || ly == 0 || lz == 0 || lx == (int)p.ch_n[0] - 1 || ly == (int)p.ch_n[1] - 1 || lz == (int)p.ch_n[2] - 1)) {
            R *o = (R *)p.mom_child + ((uint64_t)a.mw * p.ch_nodes + ((uint64_t)lz * p.ch_n[1] + ly) * p.ch_n[0] + lx) * MW;
            o[0] = rho; o[1] = u[0]; o[2] = u[1]; o[3] = u[2];
#pragma unroll
            for (int c = 0; c < 6; c++) o[4 + c] = pst[c];
            o[10] = tau;
        }
    }
    // moments for the coarser level's restriction (the nodes it shares)
    if (p.has_parent && ((x | y | z) & 1u) == 0) {
        R *o = (R *)p.mom_up + (((uint64_t)(z >> 1) * p.pn[1] + (y >> 1)) * p.pn[0] + (x >> 1)) * MW;
        o[0] = rho; o[1] = u[0]; o[2] = u[1]; o[3] = u[2];
#pragma unroll
        for (int c = 0; c < 6; c++) o[4 + c] = pst[c];
        o[10] = tau;
    }
}


// Bouzidi bounce-back with moving-wall momentum exchange (mshader.rs:364-403),
// one thread per wall record, launched just before the step on the same
// stream.  For each cut link i of a cell the step will update, the
// population the step takes instead of the one it pulls from the solid side
// (direction 26 - i, storage units) goes to wallf, 27 slots per record; the
// force and moment on the wall go to the record.  Kept out of the step, the
// wall arithmetic (and the pulled values it needs next to the substituted
// ones) no longer shares the collision's register budget: the step compiled
// for four blocks per SM spilled with it inline.
// three blocks per SM: 80 registers hold the preloaded populations and link
// distances without spilling (FP64 keeps the compiler's choice)
template <class S> struct WallOcc { static constexpr int value = 3; };
template <> struct WallOcc<double> { static constexpr int value = 1; };

template <class S>
__global__ void __launch_bounds__(BLK, WallOcc<S>::value) k27_walls(const __grid_constant__ LevelParams p, const StepArgs a) {
    using R = typename Pop<S>::real;
    const uint32_t r = blockIdx.x * BLK + threadIdx.x;
    if (r >= p.nrec) return;
    const uint32_t n = p.recs[r * RS + R_CELL];
    const uint32_t fg = p.flags[n];
    // only the cells the step updates, each through its own record
    if ((fg & 7u) != 0 || (fg >> 3) != r + 1) return;
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    const Consts27<R> &k = K<R>(p);
    const R SC = (R)Raw<S>::SC, ISC = (R)1 / (R)Raw<S>::SC;
    const S *srcn = set_ptr<S>(p, a.src) + n;
    const int64_t NP = (int64_t)p.NP;
    // the step's pull offsets (with periodic wrap where an axis has it; a
    // stepped cell of a closed axis is never on its edge)
    const int32_t nx = (int32_t)p.NX, nxy = (int32_t)(p.NX * p.NY);
    const int32_t xo[3] = {x == 0 ? nx - 1 : -1, 0, x == p.NX - 1 ? -(nx - 1) : 1};
    const int32_t yo[3] = {y == 0 ? (int32_t)(p.NY - 1) * nx : -nx, 0, y == p.NY - 1 ? -(int32_t)(p.NY - 1) * nx : nx};
    const int32_t zo[3] = {z == 0 ? (int32_t)(p.NZ - 1) * nxy : -nxy, 0, z == p.NZ - 1 ? -(int32_t)(p.NZ - 1) * nxy : nxy};
    const uint32_t mask = p.recs[r * RS + R_MASK];
    R *wf = (R *)p.wallf + (uint64_t)r * 27;
    R Fv[3] = {0, 0, 0}, Tv[3] = {0, 0, 0};
    const R pc[3] = {(R)(float)x - k.center[0], (R)(float)y - k.center[1], (R)(float)z - k.center[2]};
    R om[3];
    if (sizeof(R) == 8) { om[0] = (R)a.omega_d[0]; om[1] = (R)a.omega_d[1]; om[2] = (R)a.omega_d[2]; }
    else { om[0] = (R)a.omega[0]; om[1] = (R)a.omega[1]; om[2] = (R)a.omega[2]; }
    if (mask != 0u) {
        // the link distances and the cell's own populations on the cut links
        // (both ends) first, all independent: loaded inside each link's
        // arithmetic, after the previous link's store (which the compiler
        // cannot tell from them), the links' memory latencies ran one after
        // another.  The pulled population, needed only by a short link whose
        // opposite is open, is still loaded where it is used.
        uint32_t qw[13];
#pragma unroll
        for (int w = 0; w < 13; w++) qw[w] = p.recs[r * RS + R_Q + w];
        R own[27];
#pragma unroll
        for (int i = 0; i < 27; i++)
            own[i] = (i != 13 && (mask & ((1u << i) | (1u << (26 - i))))) ? (R)Raw<S>::ld(srcn + (int64_t)i * NP) : (R)0;
#pragma unroll
        for (int i = 0; i < 27; i++) {
            if (i == 13) continue;
            if (!(mask & (1u << i))) continue;
            const int o = 26 - i;
            const uint32_t wq = qw[SLOT(i) / 2];
            const uint16_t hq = (SLOT(i) & 1) ? (uint16_t)(wq >> 16) : (uint16_t)(wq & 0xffffu);
            const R q = max((R)__half2float(__ushort_as_half(hq)), (R)0.001f);
            const R fpi = own[i] * ISC + W<R>(i);
            const R fpo = own[o] * ISC + W<R>(i);
            const R ci[3] = {(R)CX(i), (R)CY(i), (R)CZ(i)};
            const R xw[3] = {pc[0] + q * ci[0], pc[1] + q * ci[1], pc[2] + q * ci[2]};
            const R uw[3] = {om[1] * xw[2] - om[2] * xw[1], om[2] * xw[0] - om[0] * xw[2], om[0] * xw[1] - om[1] * xw[0]};
            const R cu = ci[0] * uw[0] + ci[1] * uw[1] + ci[2] * uw[2];
            const R w6 = (R)6 * W<R>(i);
            R fb;
            if (q >= (R)0.5) {
                fb = (fpi + ((R)2 * q - (R)1) * fpo - w6 * cu) / ((R)2 * q);
            } else if (!(mask & (1u << o))) {
                // the population pulled along c_i, as the step loads it
                const R fin = Raw<S>::ld(srcn + ((int64_t)i * NP + (xo[1 - CX(i)] + yo[1 - CY(i)] + zo[1 - CZ(i)]))) * ISC;
                fb = (R)2 * q * fpi + ((R)1 - (R)2 * q) * (fin + W<R>(i)) - w6 * cu;
            } else {
                fb = fpi - w6 * cu;
            }
            wf[o] = (fb - W<R>(i)) * SC;
            R flk[3];
#pragma unroll
            for (int c = 0; c < 3; c++) flk[c] = (ci[c] - uw[c]) * fpi + (ci[c] + uw[c]) * fb;
#pragma unroll
            for (int c = 0; c < 3; c++) Fv[c] += flk[c];
            Tv[0] += xw[1] * flk[2] - xw[2] * flk[1];
            Tv[1] += xw[2] * flk[0] - xw[0] * flk[2];
            Tv[2] += xw[0] * flk[1] - xw[1] * flk[0];
        }
    }
    if (p.moving) {
        // plus what the re-voxelizer booked for this cell this step
        for (int c = 0; c < 3; c++) {
            Fv[c] += p.recd ? (R)p.recd[r * 6 + c] : (R)__uint_as_float(p.recs[r * RS + R_FT + c]);
            Tv[c] += p.recd ? (R)p.recd[r * 6 + 3 + c] : (R)__uint_as_float(p.recs[r * RS + R_FT + 3 + c]);
        }
    }
    for (int c = 0; c < 3; c++) {
        p.recs[r * RS + R_FT + c] = __float_as_uint((float)Fv[c]);
        p.recs[r * RS + R_FT + 3 + c] = __float_as_uint((float)Tv[c]);
    }
    if (p.recd) {
        for (int c = 0; c < 3; c++) { p.recd[r * 6 + c] = (double)Fv[c]; p.recd[r * 6 + 3 + c] = (double)Tv[c]; }
    }
}

template <class S, bool FORCE, bool WRAP, bool SPONGE>
__global__ void __launch_bounds__(BLK, StepOcc<S, WRAP, SPONGE>::value) k27_step(const __grid_constant__ LevelParams p, const StepArgs a) {
    using R = typename Pop<S>::real;
    const uint32_t n = blockIdx.x * BLK + threadIdx.x;
    if (n >= p.N) return;
    const uint32_t fg = p.flags[n];
    if ((fg & 7u) != 0) return;
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    const S *src = set_ptr<S>(p, a.src);
    const S *srcn = src + n;
    const int64_t NP = (int64_t)p.NP, SX = 1, SY = (int64_t)p.NX, SZ = (int64_t)p.NX * p.NY;
    R f[27];
    if (WRAP) {
        // offsets of the axis neighbours with periodic wrap (mshader.rs:135-138)
        const int32_t nx = (int32_t)p.NX, nxy = (int32_t)(p.NX * p.NY);
        const int32_t xo[3] = {x == 0 ? nx - 1 : -1, 0, x == p.NX - 1 ? -(nx - 1) : 1};
        const int32_t yo[3] = {y == 0 ? (int32_t)(p.NY - 1) * nx : -nx, 0, y == p.NY - 1 ? -(int32_t)(p.NY - 1) * nx : nx};
        const int32_t zo[3] = {z == 0 ? (int32_t)(p.NZ - 1) * nxy : -nxy, 0, z == p.NZ - 1 ? -(int32_t)(p.NZ - 1) * nxy : nxy};
#pragma unroll
        for (int i = 0; i < 27; i++) f[i] = Raw<S>::ld(srcn + ((int64_t)i * NP + (xo[1 - CX(i)] + yo[1 - CY(i)] + zo[1 - CZ(i)])));
    } else {
        // pull: the population moving along c_i comes from n - c_i
#pragma unroll
        for (int i = 0; i < 27; i++) f[i] = Raw<S>::ld(srcn + ((int64_t)i * NP - CX(i) * SX - CY(i) * SY - CZ(i) * SZ));
    }
    cell27<S, FORCE, SPONGE>(p, a, n, fg, x, y, z, f);
}

// ------------------------------------------------------------ level kernels
// mshader.rs:702-733: domain faces of the coarsest level
template <class S>
__global__ void __launch_bounds__(BLK) k27_face(const __grid_constant__ LevelParams p, const StepArgs a) {
    using R = typename Pop<S>::real;
    const uint32_t kk = blockIdx.x * BLK + threadIdx.x;
    if (kk >= p.nface) return;
    const Consts27<R> &k = K<R>(p);
    const uint32_t b = p.faces[kk];
    uint32_t x, y, z;
    coords(p, b, x, y, z);
    if (!p.per[0]) x = min(max(x, 1u), p.NX - 2);
    if (!p.per[1]) y = min(max(y, 1u), p.NY - 2);
    if (!p.per[2]) z = min(max(z, 1u), p.NZ - 2);
    const uint32_t m = (z * p.NY + y) * p.NX + x;
    R rho = 1, u[3] = {k.u_inf[0], k.u_inf[1], k.u_inf[2]}, pp[6] = {0, 0, 0, 0, 0, 0};
    if ((p.flags[m] & 7u) == 0) {
        R f[27];
        own<S>(p, a.src, m, f);
        const Mom<R> mo = moments<R>(f);
        rho = (R)1 + mo.rho1;
#pragma unroll
        for (int c = 0; c < 3; c++) u[c] = mo.j[c] / rho;
        stress<R>(mo, rho, u, pp);
    }
    const uint32_t ty = (p.flags[b] >> 3) & 3u;
    if (ty == 1) {
        if (p.total_p) {
            const R third = (R)1 / (R)3;
            const R ui2 = k.u_inf[0] * k.u_inf[0] + k.u_inf[1] * k.u_inf[1] + k.u_inf[2] * k.u_inf[2];
            const R u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
            rho = (third + (R)0.5 * ui2) / (third + (R)0.5 * u2);
        } else {
            u[0] = k.u_inf[0]; u[1] = k.u_inf[1]; u[2] = k.u_inf[2];
        }
    } else {
        rho = 1;
    }
    R f[27];
    rebuild<R>(rho, u, pp, f);
    Rng rng = cell_rng<S>(b, a.seed_mix);
    put<S>(p, a.src, b, f, rng);
}

// mshader.rs:742-775: fine ghosts from the parent's surface moments, linear in
// space and time, stress rescaled for half the time step
template <class S>
__global__ void __launch_bounds__(BLK) k27_ghost(const __grid_constant__ LevelParams p, const StepArgs a) {
    using R = typename Pop<S>::real;
    const uint32_t kk = blockIdx.x * BLK + threadIdx.x;
    if (kk >= p.nghost) return;
    const uint32_t n = p.ghosts[kk];
    uint32_t xyz[3];
    coords(p, n, xyz[0], xyz[1], xyz[2]);
    const uint32_t h0[3] = {xyz[0] >> 1, xyz[1] >> 1, xyz[2] >> 1};
    const uint32_t odd[3] = {xyz[0] & 1u, xyz[1] & 1u, xyz[2] & 1u};
    const R *mp = (const R *)p.mom_parent;
    const uint64_t pnodes = (uint64_t)p.pn[0] * p.pn[1] * p.pn[2];
    R acc[11];
#pragma unroll
    for (int j = 0; j < 11; j++) acc[j] = 0;
    R wsum = 0;
    const R blend = (R)a.blend;
#pragma unroll
    for (uint32_t c = 0; c < 8; c++) {
        const uint32_t o[3] = {c & 1u, (c >> 1) & 1u, (c >> 2) & 1u};
        if ((o[0] & ~odd[0]) | (o[1] & ~odd[1]) | (o[2] & ~odd[2])) continue;
        const R w = (odd[0] ? (R)0.5 : (R)1) * (odd[1] ? (R)0.5 : (R)1) * (odd[2] ? (R)0.5 : (R)1);
        const uint64_t nd = ((uint64_t)(h0[2] + o[2]) * p.pn[1] + (h0[1] + o[1])) * p.pn[0] + (h0[0] + o[0]);
        const R *ma = mp + (a.mold * pnodes + nd) * MW;
        const R *mb = mp + (a.mnew * pnodes + nd) * MW;
#pragma unroll
        for (int j = 0; j < 11; j++) acc[j] += w * (((R)1 - blend) * ma[j] + blend * mb[j]);
        wsum += w;
    }
    const R rho = acc[0] / wsum;
    const R u[3] = {acc[1] / wsum, acc[2] / wsum, acc[3] / wsum};
    const R tc = acc[10] / wsum;
    const R tf = (R)0.5 + (R)2 * (tc - (R)0.5);
    const R sc = tf / ((R)2 * tc) * ((R)1 - (R)1 / tf);
    R pp[6];
#pragma unroll
    for (int j = 0; j < 6; j++) pp[j] = acc[4 + j] / wsum * sc;
    R f[27];
    rebuild<R>(rho, u, pp, f);
    Rng rng = cell_rng<S>(n, a.seed_mix);
    put<S>(p, a.src, n, f, rng);
}

// mshader.rs:777-793: coarse cells under the child box from its coincident nodes
template <class S>
__global__ void __launch_bounds__(BLK) k27_restrict(const __grid_constant__ LevelParams p, const StepArgs a) {
    using R = typename Pop<S>::real;
    const uint32_t kk = blockIdx.x * BLK + threadIdx.x;
    if (kk >= p.nrestrict) return;
    const uint32_t n = p.restricted[kk];
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    const uint32_t lx = x - (uint32_t)p.ch_lo[0], ly = y - (uint32_t)p.ch_lo[1], lz = z - (uint32_t)p.ch_lo[2];
    const R *m = (const R *)p.mom_child_up + (((uint64_t)lz * p.ch_n[1] + ly) * p.ch_n[0] + lx) * MW;
    const R rho = m[0];
    const R u[3] = {m[1], m[2], m[3]};
    const R tf = m[10];
    const R tc = (R)0.5 + (R)0.5 * (tf - (R)0.5);
    const R sc = (R)2 * tc / tf * ((R)1 - (R)1 / tc);
    R pp[6];
#pragma unroll
    for (int j = 0; j < 6; j++) pp[j] = m[4 + j] * sc;
    R f[27];
    rebuild<R>(rho, u, pp, f);
    Rng rng = cell_rng<S>(n, a.seed_mix);
    put<S>(p, a.src, n, f, rng);
}

// mshader.rs:520-527: feq(1, u_init) in both sets
template <class S>
__global__ void __launch_bounds__(BLK) k27_init(const __grid_constant__ LevelParams p) {
    using R = typename Pop<S>::real;
    const uint32_t n = blockIdx.x * BLK + threadIdx.x;
    if (n >= p.N) return;
    const Consts27<R> &k = K<R>(p);
    R f[27];
    feq<R>((R)1, k.u_init[0], k.u_init[1], k.u_init[2], f);
    Rng rng = cell_rng<S>(n, 0x632BE5ABu);
    put<S>(p, 0, n, f, rng);
    rng = cell_rng<S>(n, 0x632BE5ABu);
    put<S>(p, 1, n, f, rng);
}

// mshader.rs:495-505, 602-610
template <class S>
__global__ void __launch_bounds__(BLK) k27_dump(const __grid_constant__ LevelParams p, uint32_t src) {
    using R = typename Pop<S>::real;
    const uint32_t n = blockIdx.x * BLK + threadIdx.x;
    if (n >= p.N) return;
    const Consts27<R> &k = K<R>(p);
    if ((p.flags[n] & 7u) != 0) {
        const float nan = __int_as_float(0x7fc00000);
        p.dump[n] = make_float4(nan, nan, nan, nan);
        return;
    }
    R f[27];
    own<S>(p, src, n, f);
    const Mom<R> mo = moments<R>(f);
    const R rho = (R)1 + mo.rho1;
    p.dump[n] = make_float4((float)rho, (float)(mo.j[0] / rho - (R)0.5 * k.grav[0]), (float)(mo.j[1] / rho - (R)0.5 * k.grav[1]),
                            (float)(mo.j[2] / rho - (R)0.5 * k.grav[2]));
}

// Density and velocity of a cell of a level between steps, from its current
// source set (mshader.rs:495-505): every cell type but solid has them.
template <class S>
__device__ __forceinline__ bool cell_macro27(const LevelParams &p, uint32_t src, uint32_t n, float &rho, float &ux, float &uy, float &uz) {
    using R = typename Pop<S>::real;
    if ((p.flags[n] & 7u) == T_SOLID) return false;
    const Consts27<R> &k = K<R>(p);
    R f[27];
    own<S>(p, src, n, f);
    const Mom<R> mo = moments<R>(f);
    const R r = (R)1 + mo.rho1;
    rho = (float)r;
    ux = (float)(mo.j[0] / r - (R)0.5 * k.grav[0]);
    uy = (float)(mo.j[1] / r - (R)0.5 * k.grav[1]);
    uz = (float)(mo.j[2] / r - (R)0.5 * k.grav[2]);
    return true;
}

// Surface-pressure probes on the finest level (mshader.rs:563-588): each
// vertex (body coordinates relative to the centre, pushed out along its
// normal by voff) rotated by the step's rotation, the density trilinearly
// interpolated from the usable cells around it; FP64 running sums.
template <class S>
__global__ void __launch_bounds__(BLK) k27_sample_verts(const __grid_constant__ LevelParams p, const __grid_constant__ StepArgs a,
                                                        const float *verts, uint32_t nvert, float voff, double *vacc) {
    const uint32_t v = blockIdx.x * BLK + threadIdx.x;
    if (v >= nvert) return;
    const float bx = verts[8 * v] + voff * verts[8 * v + 4];
    const float by = verts[8 * v + 1] + voff * verts[8 * v + 5];
    const float bz = verts[8 * v + 2] + voff * verts[8 * v + 6];
    float sp[3];
    for (int c = 0; c < 3; c++) sp[c] = p.kf.center[c] + (a.rot[c * 3] * bx + a.rot[c * 3 + 1] * by + a.rot[c * 3 + 2] * bz);
    const float b0[3] = {floorf(sp[0]), floorf(sp[1]), floorf(sp[2])};
    const float fr[3] = {sp[0] - b0[0], sp[1] - b0[1], sp[2] - b0[2]};
    float acc = 0.f, wsum = 0.f;
    for (int c = 0; c < 8; c++) {
        const int o[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
        const int ci[3] = {(int)b0[0] + o[0], (int)b0[1] + o[1], (int)b0[2] + o[2]};
        if (ci[0] < 1 || ci[1] < 1 || ci[2] < 1 || ci[0] >= (int)p.NX - 1 || ci[1] >= (int)p.NY - 1 || ci[2] >= (int)p.NZ - 1) continue;
        const float w = (o[0] ? fr[0] : 1.f - fr[0]) * (o[1] ? fr[1] : 1.f - fr[1]) * (o[2] ? fr[2] : 1.f - fr[2]);
        float rho, ux, uy, uz;
        const uint32_t m = ((uint32_t)ci[2] * p.NY + (uint32_t)ci[1]) * p.NX + (uint32_t)ci[0];
        if (cell_macro27<S>(p, a.src, m, rho, ux, uy, uz) && w > 0.f) { acc += w * rho; wsum += w; }
    }
    if (wsum > 1e-6f) {
        vacc[2 * v] += (double)(acc / wsum);
        vacc[2 * v + 1] += 1.0;
    }
}

// Slice pixels this level owns (mshader.rs:590-602): pairs (pixel, cell),
// running FP64 sums of (rho, u) and a count per pixel.
template <class S>
__global__ void __launch_bounds__(BLK) k27_sample_slices(const __grid_constant__ LevelParams p, uint32_t src, const uint32_t *pix, uint32_t npix,
                                                         double *sacc) {
    const uint32_t k = blockIdx.x * BLK + threadIdx.x;
    if (k >= npix) return;
    const uint32_t px = pix[2 * k], cell = pix[2 * k + 1];
    float rho, ux, uy, uz;
    if (cell_macro27<S>(p, src, cell, rho, ux, uy, uz)) {
        double *b = sacc + 5ull * px;
        b[0] += rho; b[1] += ux; b[2] += uy; b[3] += uz; b[4] += 1.0;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// FP64 mass and non-finite count of the plain fluid cells of a level:
// grid-stride over the cells, then the deterministic grid sum of reduce.cuh
// (one atomic per block; the same result on every run).  out[0] = mass,
// out[1] = non-finite count.
template <class S>
__global__ void __launch_bounds__(BLK) k27_mass(const __grid_constant__ LevelParams p, uint32_t src, double *scratch, double *out) {
    using R = typename Pop<S>::real;
    double m = 0, nbad = 0;
    const uint32_t stride = gridDim.x * BLK;
#pragma unroll 1
    for (uint32_t n = blockIdx.x * BLK + threadIdx.x; n < p.N; n += stride) {
        if ((p.flags[n] & 7u) != 0) continue;
        R f[27];
        own<S>(p, src, n, f);
        double sum = 1.0;
#pragma unroll
        for (int i = 0; i < 27; i++) sum += (double)f[i];
        if (isfinite(sum)) m += sum;
        else nbad += 1.0;
    }
    lbm::grid_sum2<BLK>(m, nbad, scratch, out);
}

// ------------------------------------------------------------ spinning part
// The D3Q19 re-voxelizer (crates/cfd/src/shader.rs:865-1104) carried to the 27
// directions of this lattice (the reference spins parts on D3Q19 only): each
// link is kept once, at the cell it leaves along one of the 13 directions
// i = 14..26 (the partner -c of each has index 26 - i < 13).  In the pull
// scheme a just-uncovered cell's refill is written straight into the source
// set, where its neighbours pull it this step.
namespace sp27 {
using namespace lbm::rv;
__device__ __forceinline__ bool solid(const LevelParams &p, const float *rot, int x, int y, int z) {
    const V3 pc = {fs((float)x, p.kf.center[0]), fs((float)y, p.kf.center[1]), fs((float)z, p.kf.center[2])};
    return occ_bit(p.occ, p.occ_lo, p.occ_invh, p.occ_n, to_body(rot, pc));
}
__device__ __forceinline__ bool in_box(const LevelParams &p, int lx, int ly, int lz) {
    return lx >= 0 && ly >= 0 && lz >= 0 && lx < (int)p.box_n[0] && ly < (int)p.box_n[1] && lz < (int)p.box_n[2];
}
}  // namespace sp27

__global__ void __launch_bounds__(BLK) k27_tri_scatter(const __grid_constant__ LevelParams p, const StepArgs a) {
    using namespace lbm::rv;
    // one warp per triangle, its lanes over the lattice points near it
    const uint32_t t = (blockIdx.x * BLK + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (t >= p.ntri) return;
    const float4 t0 = p.tris[3 * t], t1 = p.tris[3 * t + 1], t2 = p.tris[3 * t + 2];
    const V3 ctr = {p.kf.center[0], p.kf.center[1], p.kf.center[2]};
    const V3 va = add(ctr, from_body(a.rot, {t0.x, t0.y, t0.z}));
    const V3 e1 = from_body(a.rot, {t1.x, t1.y, t1.z});
    const V3 e2 = from_body(a.rot, {t2.x, t2.y, t2.z});
    const V3 nrm = cross(e1, e2);
    const float nl = __fsqrt_rn(dot(nrm, nrm));
    if (nl < 1e-12f) return;
    const V3 nn = {__fdiv_rn(nrm.x, nl), __fdiv_rn(nrm.y, nl), __fdiv_rn(nrm.z, nl)};
    const V3 vb = add(va, e1), vc = add(va, e2);
    constexpr float REACH = 1.733f;  // the longest link, sqrt(3)
    const float mn[3] = {fminf(fminf(va.x, vb.x), vc.x), fminf(fminf(va.y, vb.y), vc.y), fminf(fminf(va.z, vb.z), vc.z)};
    const float mx[3] = {fmaxf(fmaxf(va.x, vb.x), vc.x), fmaxf(fmaxf(va.y, vb.y), vc.y), fmaxf(fmaxf(va.z, vb.z), vc.z)};
    int lo[3], hi[3];
    for (int c = 0; c < 3; c++) {
        lo[c] = max((int)ceilf(fs(mn[c], REACH)), p.box_lo[c]);
        hi[c] = min((int)floorf(fa(mx[c], REACH)), p.box_lo[c] + (int)p.box_n[c] - 1);
    }
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    const int npts = (nx > 0 && ny > 0 && nz > 0) ? nx * ny * nz : 0;
    for (int q = (int)lane; q < npts; q += 32) {
                const int x = lo[0] + q % nx, y = lo[1] + (q / nx) % ny, z = lo[2] + q / (nx * ny);
                const V3 pt = {(float)x, (float)y, (float)z};
                const float d0 = dot(nn, sub(pt, va));
                if (fabsf(d0) > REACH) continue;
                const uint32_t k = ((uint32_t)(z - p.box_lo[2]) * p.box_n[1] + (uint32_t)(y - p.box_lo[1])) * p.box_n[0] + (uint32_t)(x - p.box_lo[0]);
#pragma unroll
                for (int i = 14; i < 27; i++) {
                    const V3 cv = {(float)CX(i), (float)CY(i), (float)CZ(i)};
                    const float d1 = fa(d0, dot(nn, cv));
                    if (fm(d0, d1) > 0.0f && fabsf(d0) > 1e-6f) continue;
                    const float tt = ray_tri(pt, cv, va, e1, e2);
                    if (tt <= 1.0f) {
                        const uint64_t o = ((uint64_t)k * 13u + (uint32_t)(i - 14)) * 3u;
                        const uint32_t tb = __float_as_uint(tt > 0.0f ? tt : 0.0f);
                        atomicMin(p.qscr + o, tb);
                        atomicMax(p.qscr + o + 1, tb);
                        atomicAdd(p.qscr + o + 2, 1u);
                    }
                }
            }
}

__global__ void __launch_bounds__(BLK) k27_qclear(const __grid_constant__ LevelParams p) {
    const uint64_t k = (uint64_t)blockIdx.x * BLK + threadIdx.x;
    if (k >= (uint64_t)p.nrec * 13u) return;
    p.qscr[3 * k] = 0x7f7fffffu;
    p.qscr[3 * k + 1] = 0u;
    p.qscr[3 * k + 2] = 0u;
}

template <class S>
__global__ void __launch_bounds__(BLK) k27_voxelize(const __grid_constant__ LevelParams p, const StepArgs a) {
    using namespace lbm::rv;
    using R = typename Pop<S>::real;
    const uint32_t k = blockIdx.x * BLK + threadIdx.x;
    if (k >= p.nrec) return;
    const int lx = (int)(k % p.box_n[0]), ly = (int)((k / p.box_n[0]) % p.box_n[1]), lz = (int)(k / (p.box_n[0] * p.box_n[1]));
    const int px = lx + p.box_lo[0], py = ly + p.box_lo[1], pz = lz + p.box_lo[2];
    const uint32_t n = ((uint32_t)pz * p.NY + (uint32_t)py) * p.NX + (uint32_t)px;
    const Consts27<R> &kk = K<R>(p);
    const R pc[3] = {(R)px - kk.center[0], (R)py - kk.center[1], (R)pz - kk.center[2]};
    const bool solid_now = sp27::solid(p, a.rot, px, py, pz), solid_before = sp27::solid(p, a.rot_prev, px, py, pz);
    R F[3] = {0, 0, 0};
    if (solid_now) {
        p.flags[n] = T_SOLID | ((k + 1u) << 3);
        p.recs[k * RS + R_MASK] = 0u;
        if (!solid_before) {
            // covered this step: the part takes the cell's momentum
            R f[27];
            own<S>(p, a.src, n, f);
            const Mom<R> mo = moments<R>(f);
            for (int c = 0; c < 3; c++) F[c] = mo.j[c];
        }
    } else {
        float qv[27], qx[27];
        uint32_t nh[27];
#pragma unroll
        for (int i = 0; i < 27; i++) {
            qv[i] = 9.0f; qx[i] = -1.0f; nh[i] = 0u;
            if (i == 13) continue;
            if (i > 13) {
                const uint64_t o = ((uint64_t)k * 13u + (uint32_t)(i - 14)) * 3u;
                const uint32_t c = p.qscr[o + 2];
                if (c) { qv[i] = __uint_as_float(p.qscr[o]); qx[i] = __uint_as_float(p.qscr[o + 1]); nh[i] = c; }
            } else if (sp27::in_box(p, lx + CX(i), ly + CY(i), lz + CZ(i))) {
                const uint32_t k2 = ((uint32_t)(lz + CZ(i)) * p.box_n[1] + (uint32_t)(ly + CY(i))) * p.box_n[0] + (uint32_t)(lx + CX(i));
                const uint64_t o = ((uint64_t)k2 * 13u + (uint32_t)(26 - i - 14)) * 3u;
                const uint32_t c = p.qscr[o + 2];
                if (c) { qv[i] = fs(1.0f, __uint_as_float(p.qscr[o + 1])); qx[i] = fs(1.0f, __uint_as_float(p.qscr[o])); nh[i] = c; }
            }
        }
        uint32_t mask = 0;
#pragma unroll
        for (int i = 0; i < 27; i++) {
            if (i == 13) continue;
            if (sp27::solid(p, a.rot, px + CX(i), py + CY(i), pz + CZ(i))) {
                if (nh[i] == 0u) qv[i] = 1.0f;
                mask |= 1u << i;
            } else if (nh[i] >= 2u && fs(qx[i], qv[i]) > 1e-5f) {
                mask |= 1u << i;
            } else {
                qv[i] = 1.0f;
            }
        }
#pragma unroll
        for (int w = 0; w < 13; w++) {
            const int i0 = 2 * w < 13 ? 2 * w : 2 * w + 1, i1 = 2 * w + 1 < 13 ? 2 * w + 1 : 2 * w + 2;  // slots 2w, 2w+1
            const uint32_t lo = __half_as_ushort(__float2half_rn(fminf(qv[i0], 1.0f)));
            const uint32_t hi = __half_as_ushort(__float2half_rn(fminf(qv[i1], 1.0f)));
            p.recs[k * RS + R_Q + w] = lo | (hi << 16);
        }
        p.recs[k * RS + R_MASK] = mask;
        if (solid_before) {
            // uncovered this step: a post-collision state at the wall velocity
            // with the density and the mean non-equilibrium stress of the
            // neighbours that were fluid before and are now, written to the
            // source set its neighbours pull from; the part gives up its momentum
            R rs = 0, cnt = 0, pis[6] = {0, 0, 0, 0, 0, 0};
            for (int i = 0; i < 27; i++) {
                if (i == 13) continue;
                const int qx2 = px + CX(i), qy2 = py + CY(i), qz2 = pz + CZ(i);
                if (sp27::solid(p, a.rot, qx2, qy2, qz2) || sp27::solid(p, a.rot_prev, qx2, qy2, qz2)) continue;
                R f[27];
                own<S>(p, a.src, ((uint32_t)qz2 * p.NY + (uint32_t)qy2) * p.NX + (uint32_t)qx2, f);
                const Mom<R> mo = moments<R>(f);
                const R r2 = (R)1 + mo.rho1;
                const R u2[3] = {mo.j[0] / r2, mo.j[1] / r2, mo.j[2] / r2};
                R ps[6];
                stress<R>(mo, r2, u2, ps);
                for (int c = 0; c < 6; c++) pis[c] += ps[c];
                rs += r2;
                cnt += (R)1;
            }
            const R rho = cnt > (R)0 ? rs / cnt : (R)1;
            if (cnt > (R)0)
                for (int c = 0; c < 6; c++) pis[c] /= cnt;
            R om[3];
            if (sizeof(R) == 8) { om[0] = (R)a.omega_d[0]; om[1] = (R)a.omega_d[1]; om[2] = (R)a.omega_d[2]; }
            else { om[0] = (R)a.omega[0]; om[1] = (R)a.omega[1]; om[2] = (R)a.omega[2]; }
            const R uw[3] = {om[1] * pc[2] - om[2] * pc[1], om[2] * pc[0] - om[0] * pc[2], om[0] * pc[1] - om[1] * pc[0]};
            R f[27];
            rebuild<R>(rho, uw, pis, f);
            Rng rng = cell_rng<S>(n, a.seed_mix);
            put<S>(p, a.src, n, f, rng);
            for (int c = 0; c < 3; c++) F[c] = -rho * uw[c];
        }
        p.flags[n] = (k + 1u) << 3;
    }
    const R T[3] = {pc[1] * F[2] - pc[2] * F[1], pc[2] * F[0] - pc[0] * F[2], pc[0] * F[1] - pc[1] * F[0]};
    for (int c = 0; c < 3; c++) {
        p.recs[k * RS + R_FT + c] = __float_as_uint((float)F[c]);
        p.recs[k * RS + R_FT + 3 + c] = __float_as_uint((float)T[c]);
    }
    if (p.recd)
        for (int c = 0; c < 3; c++) { p.recd[k * 6 + c] = (double)F[c]; p.recd[k * 6 + 3 + c] = (double)T[c]; }
}

// FP64 sum of the records' force and moment: per-block partials in fixed
// order, the last block to finish sums the partials (mshader.rs:519-562 does
// the same sum in f32)
constexpr uint32_t RED_BLK = 256;
template <bool FP64>
__global__ void __launch_bounds__(RED_BLK) k27_reduce(const __grid_constant__ LevelParams p, double *partials, uint32_t *ticket, double *out) {
    const uint32_t r = blockIdx.x * RED_BLK + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (r < p.nrec) {
#pragma unroll
        for (int j = 0; j < 6; j++) v[j] = FP64 ? p.recd[(uint64_t)r * 6 + j] : (double)__uint_as_float(p.recs[(uint64_t)r * RS + R_FT + j]);
    }
    __shared__ double sh[RED_BLK / 32][6];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 6; j++) v[j] = warp_sum(v[j]);
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = v[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < (int)(RED_BLK / 32); w++) t += sh[w][threadIdx.x];
        partials[blockIdx.x * 8 + threadIdx.x] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += RED_BLK)
        for (int j = 0; j < 6; j++) acc[j] += __ldcg(&partials[b * 8 + j]);
    for (int j = 0; j < 6; j++) acc[j] = warp_sum(acc[j]);
    __syncthreads();
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = acc[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < (int)(RED_BLK / 32); w++) t += sh[w][threadIdx.x];
        out[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// ------------------------------------------------------------ launchers
static inline unsigned blocks_for(uint64_t n) { return (unsigned)((n + BLK - 1) / BLK); }

template <class F>
static cudaError_t dispatch(int storage, F &&fn) {
    switch (storage) {
        case 0: return fn((float *)nullptr);
        case 1: return fn((__half *)nullptr);
        case 2: return fn((__nv_bfloat16 *)nullptr);
        case 3: return fn((double *)nullptr);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch27_init(int storage, const LevelParams &p, cudaStream_t st) {
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_init<S><<<blocks_for(p.N), BLK, 0, st>>>(p);
        return cudaGetLastError();
    });
}

cudaError_t launch27_face(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st) {
    if (!p.nface) return cudaSuccess;
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_face<S><<<blocks_for(p.nface), BLK, 0, st>>>(p, a);
        return cudaGetLastError();
    });
}

cudaError_t launch27_step(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st) {
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        const bool wrap = p.per[0] || p.per[1] || p.per[2];
        const unsigned g = blocks_for(p.N);
        const bool sp = p.n_sponge != 0;
        if (p.nrec) k27_walls<S><<<blocks_for(p.nrec), BLK, 0, st>>>(p, a);
        if (p.forcing) {
            if (wrap) {
                if (sp) k27_step<S, true, true, true><<<g, BLK, 0, st>>>(p, a);
                else k27_step<S, true, true, false><<<g, BLK, 0, st>>>(p, a);
            } else {
                if (sp) k27_step<S, true, false, true><<<g, BLK, 0, st>>>(p, a);
                else k27_step<S, true, false, false><<<g, BLK, 0, st>>>(p, a);
            }
        } else {
            if (wrap) {
                if (sp) k27_step<S, false, true, true><<<g, BLK, 0, st>>>(p, a);
                else k27_step<S, false, true, false><<<g, BLK, 0, st>>>(p, a);
            } else {
                if (sp) k27_step<S, false, false, true><<<g, BLK, 0, st>>>(p, a);
                else k27_step<S, false, false, false><<<g, BLK, 0, st>>>(p, a);
            }
        }
        return cudaGetLastError();
    });
}

cudaError_t launch27_ghost(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st) {
    if (!p.nghost) return cudaSuccess;
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_ghost<S><<<blocks_for(p.nghost), BLK, 0, st>>>(p, a);
        return cudaGetLastError();
    });
}

cudaError_t launch27_restrict(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st) {
    if (!p.nrestrict) return cudaSuccess;
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_restrict<S><<<blocks_for(p.nrestrict), BLK, 0, st>>>(p, a);
        return cudaGetLastError();
    });
}

cudaError_t launch27_dump(int storage, const LevelParams &p, uint32_t src, cudaStream_t st) {
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_dump<S><<<blocks_for(p.N), BLK, 0, st>>>(p, src);
        return cudaGetLastError();
    });
}

cudaError_t launch27_sample_verts(int storage, const LevelParams &p, const StepArgs &a, const float *verts, uint32_t nvert, float voff,
                                  double *vacc, cudaStream_t st) {
    if (!nvert) return cudaSuccess;
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_sample_verts<S><<<blocks_for(nvert), BLK, 0, st>>>(p, a, verts, nvert, voff, vacc);
        return cudaGetLastError();
    });
}

cudaError_t launch27_sample_slices(int storage, const LevelParams &p, uint32_t src, const uint32_t *pix, uint32_t npix, double *sacc,
                                   cudaStream_t st) {
    if (!npix) return cudaSuccess;
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_sample_slices<S><<<blocks_for(npix), BLK, 0, st>>>(p, src, pix, npix, sacc);
        return cudaGetLastError();
    });
}

uint32_t mass27_blocks() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return (uint32_t)(4 * n);
}

cudaError_t launch27_mass(int storage, const LevelParams &p, uint32_t src, double *scratch, double *out, cudaStream_t st) {
    return dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        const unsigned g = std::min<unsigned>(mass27_blocks(), blocks_for(p.N));
        k27_mass<S><<<g, BLK, 0, st>>>(p, src, scratch, out);
        return cudaGetLastError();
    });
}

uint32_t reduce27_blocks(uint32_t nrec) { return (nrec + RED_BLK - 1) / RED_BLK; }

cudaError_t launch27_revoxel(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st) {
    if (!p.moving) return cudaSuccess;
    if (p.ntri) k27_tri_scatter<<<blocks_for((uint64_t)p.ntri * 32u), BLK, 0, st>>>(p, a);
    cudaError_t e = dispatch(storage, [&](auto *t) {
        using S = std::remove_pointer_t<decltype(t)>;
        k27_voxelize<S><<<blocks_for(p.nrec), BLK, 0, st>>>(p, a);
        return cudaGetLastError();
    });
    if (e != cudaSuccess) return e;
    k27_qclear<<<blocks_for((uint64_t)p.nrec * 13u), BLK, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch27_reduce(const LevelParams &p, int fp64, double *partials, uint32_t *ticket, double *out, cudaStream_t st) {
    if (p.nrec == 0) return cudaMemsetAsync(out, 0, 6 * sizeof(double), st);
    const uint32_t nb = reduce27_blocks(p.nrec);
    if (fp64) k27_reduce<true><<<nb, RED_BLK, 0, st>>>(p, partials, ticket, out);
    else k27_reduce<false><<<nb, RED_BLK, 0, st>>>(p, partials, ticket, out);
    return cudaGetLastError();
}

}  // namespace lbm27
