// D3Q19 time-step kernels for sm_100a.
//
// One step of parity P (crates/cfd/src/lattice.rs:715-737 dispatch order):
//   k_faces  -- face cells: rebuild the "previous" post-collision populations
//               from the inner neighbour (shader.rs:630-687; gather and write
//               fused, which is race free because a face cell's inner
//               neighbour is never a face cell), plus free-slip faces.
//   k_walls  -- wall-record cells: streaming + Bouzidi / moving-wall links +
//               collision (shader.rs:795-862 with $WALLS$ 399-436), and the
//               momentum-exchange force and moment summed in FP64 with warp
//               shuffles, per block, then by the last block in a fixed order
//               (replaces reduce1/reduce2, shader.rs:689-734).
//   k_bulk   -- every other fluid cell: fused AA stream + collide.
// k_walls and k_bulk touch disjoint cells; in the AA pattern every memory
// slot is read and written by exactly one thread per step, so they need no
// ordering between them.  The population layout is the reference's
// slot-major SoA (shader.rs:147-152): direction d of cell n at d * N + n,
// stored as f - w (FP32, FP64, FP16 x 32768 with stochastic rounding, BF16).
#include <algorithm>
#include <cstdio>
#include <type_traits>
#include <utility>

#include "lbm_device.cuh"
#include "lbm_kernels.h"
#include "tma.cuh"
#include "reduce.cuh"
#include "revoxel.cuh"

namespace lbm {

// compile-time loop: fn(std::integral_constant<int, I>) for I in [A, B)
template <int A, int B, class Fn>
__device__ __forceinline__ void constexpr_for(Fn &&fn) {
    if constexpr (A < B) {
        fn(std::integral_constant<int, A>{});
        constexpr_for<A + 1, B>(fn);
    }
}

// ---------------------------------------------------------------- collision
// Everything of shader.rs:815-847 after the wall links: moments, Smagorinsky
// tau from |Pi_neq| (825-828), wall model, sponge (832-833), regularized or
// plain BGK relaxation, absorbing layer (838-845), Guo forcing (442-455).
template <class R>
__device__ R wall_tau(const LatParams &p, const Consts<R> &k, uint32_t r, uint32_t mask, R pcx, R pcy, R pcz, R ux, R uy, R uz,
                      R tau_les, const R *om) {
    // Spalding wall model, shader.rs:540-597
    R ns[3] = {0, 0, 0};
#pragma unroll
    for (int i = 1; i < 19; i++) {
        if (mask & (1u << i)) {
            R q = (R)rec_q(p.recs, r, i);
            R w = i < 7 ? (R)(1.0 / 18.0) : (R)(1.0 / 36.0);
            ns[0] = ns[0] + (R)CX(i) * w * ((R)1.5 - q);
            ns[1] = ns[1] + (R)CY(i) * w * ((R)1.5 - q);
            ns[2] = ns[2] + (R)CZ(i) * w * ((R)1.5 - q);
        }
    }
    R nl = sqrt(ns[0] * ns[0] + ns[1] * ns[1] + ns[2] * ns[2]);
    if (nl < (R)1e-6) return tau_les;
    R nw[3] = {ns[0] / nl, ns[1] / nl, ns[2] / nl};
    R yy = 2;
#pragma unroll
    for (int i = 1; i < 19; i++) {
        if (mask & (1u << i)) {
            R cn = (R)CX(i) * nw[0] + (R)CY(i) * nw[1] + (R)CZ(i) * nw[2];
            if (cn > (R)0.3) {
                R q = (R)rec_q(p.recs, r, i);
                yy = min(yy, max(q, (R)0.02) * cn);
            }
        }
    }
    if (yy > (R)1.9) return tau_les;
    R xw[3] = {pcx + yy * nw[0], pcy + yy * nw[1], pcz + yy * nw[2]};
    R uwx = om[1] * xw[2] - om[2] * xw[1], uwy = om[2] * xw[0] - om[0] * xw[2], uwz = om[0] * xw[1] - om[1] * xw[0];
    R rx = ux - uwx, ry = uy - uwy, rz = uz - uwz;
    R un = rx * nw[0] + ry * nw[1] + rz * nw[2];
    R tx = rx - un * nw[0], ty = ry - un * nw[1], tz = rz - un * nw[2];
    R ut = sqrt(tx * tx + ty * ty + tz * tz);
    R nu0 = (k.tau0 - (R)0.5) / (R)3;
    if (ut < (R)1e-7) return tau_les;
    const R kap = (R)0.41;
    R eb = exp(-kap * (R)5.2);
    R ust = sqrt(nu0 * ut / yy);
    for (int it = 0; it < 12; it++) {
        R up = ut / ust;
        R yp = yy * ust / nu0;
        R ku = min(kap * up, (R)30);
        R eku = exp(ku);
        R g = up + eb * (eku - (R)1 - ku - (R)0.5 * ku * ku - ku * ku * ku / (R)6) - yp;
        R dgdup = (R)1 + eb * kap * (eku - (R)1 - ku - (R)0.5 * ku * ku);
        R dg = dgdup * (-up / ust) - yy / nu0;
        R step = g / dg;
        ust = min(max(ust - step, (R)0.1 * ust), (R)10 * ust);
        if (fabs(step) < (R)1e-5 * ust) break;
    }
    R nuw = ust * ust * yy / ut;
    return max((R)0.5 + (R)3 * max(nuw, nu0), tau_les);
}

// One cell's update after its populations f are loaded (and wall links
// applied): shader.rs:815-847 (regularized; plain BGK relaxes f itself and
// omits the forcing's regularization correction).  Returns rho and u (the u
// written to wall records).
//
// SC is the storage scale: f holds SC * (f_i - w_i) on entry and receives the
// post-collision values in the same units (SC = 32768 for FP16 storage, 1
// otherwise).  Scaling by a power of two is exact, so the collision can work
// on the scaled moments (rescaling only the density and 1/rho) and give the
// unscaled results times the scale bit for bit; the scale of the outputs
// rides on compile-time weights.
//
// The 9 opposite pairs (i = 2k+1, o = 2k+2) share c c, so the equilibrium,
// the non-equilibrium projection, the absorbing target and the forcing term
// are each split into a part even in c (the same for i and o) and a part odd
// in c (opposite signs); with per-weight-class coefficients a pair costs a
// handful of instructions.
//
// FEAT selects compile-time feature sets for the hot loop: 0 reads every
// switch from the parameters; odd values fix forcing and the u_inf absorbing
// target off and LES to bit 1.
//
// relax_m takes the moments m of f already computed (the regularized
// collision reads f only through them; plain BGK also reads f itself).
template <class R, int COLL, int SC = 1, int FEAT = 0>
__device__ __forceinline__ void relax_m(const LatParams &p, const Consts<R> &k, const Moments<R> &m, R *f, uint32_t x, uint32_t y,
                                        uint32_t z, bool wall, uint32_t r, uint32_t mask, R pcx, R pcy, R pcz, const R *om, R &rho_o,
                                        R &ux_o, R &uy_o, R &uz_o) {
    constexpr bool SPEC = (FEAT & 1) != 0;
    const bool les_on = SPEC ? (FEAT & 2) != 0 : (p.les_on != 0);
    const bool forcing = SPEC ? false : (p.forcing != 0);
    const bool abs_u = SPEC ? false : (p.abs_u != 0);
    // the moments stay in storage units; only rho1 and 1/rho are rescaled,
    // and the non-equilibrium stress pi (in storage units as well) meets
    // weights without the scale
    const R isc = (R)(1.0 / SC);
    const R rho1 = SC != 1 ? m.rho1 * isc : m.rho1;
    const R rho = (R)1 + rho1;
    const R irho = (R)1 / rho;
    const R irs = SC != 1 ? irho * isc : irho;
    const R ux = m.jx * irs + (R)0.5 * k.grav[0];
    const R uy = m.jy * irs + (R)0.5 * k.grav[1];
    const R uz = m.jz * irs + (R)0.5 * k.grav[2];
    R pi[6];
    pi_neq<R>(m, SC != 1 ? rho * (R)SC : rho, ux, uy, uz, pi);
    R tau = k.tau0;
    if (les_on) {
        // Smagorinsky tau from |Pi_neq| (shader.rs:825-828)
        const R pp = pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] + (R)2 * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]);
        const R qn = sqrt((R)2 * pp);
        tau = (R)0.5 * (k.tau0 + sqrt(k.tau0 * k.tau0 + (R)18 * k.smag2 * qn * irs));
    }
    if (wall && p.wall_model && mask != 0u) tau = wall_tau<R>(p, k, r, mask, pcx, pcy, pcz, ux, uy, uz, tau, om);
    R sp = 0;
    if (p.sponge_on) {
        sp = sponge_at<R>(k, p, x, y, z);
        if (sp > (R)0 && k.sponge_tau > tau) tau = tau + sp * sp * (k.sponge_tau - tau);
    }
    const R omg = (R)1 / tau;
    const R om1 = (R)1 - omg;
    const R usq = (R)1.5 * (ux * ux + uy * uy + uz * uz);
    const R sg = k.sigma * sp * sp;  // absorbing strength (0 outside the layers)
    const R tr = (pi[0] + pi[1] + pi[2]) * (R)(1.0 / 3.0);
    R Gx = 0, Gy = 0, Gz = 0, uG = 0, fo = 0;
    if (forcing) {
        Gx = rho * k.grav[0]; Gy = rho * k.grav[1]; Gz = rho * k.grav[2];
        uG = ux * Gx + uy * Gy + uz * Gz;
        fo = (R)1 - (R)0.5 * omg;
    }
    // The equilibrium is fe_i = even + odd with even = A cu^2 + B, odd = O cu
    // (per weight class a: 1/18, e: 1/36, all scaled by SC).  The absorbing
    // layer adds sg (ft_i - fe_i) (shader.rs:838-845), linear in the same
    // basis: with ft = feq(0, u) it is -sg rho1 w (1 - 1.5u^2 + 4.5cu^2 + 3cu);
    // with ft = feq(0, u_inf) it is sg ft_i - sg fe_i.  Folding it into the
    // coefficients leaves the per-pair cost unchanged:
    //   regularized: v = fe + (1 - omega) fneq + delta
    //   BGK:         v = (1 - omega) f + omega fe + delta
    const R wa = (R)(SC / 18.0), we = (R)(SC / 36.0), w0 = (R)(SC / 3.0);
    const R Bq = rho1 - rho * usq;
    const R lam = COLL == 1 ? omg : (R)1;
    R cA, cB, cO, dB;  // coefficient multipliers (unit weight) and the constant shift
    if (abs_u) {
        const R l2 = lam - sg;
        cA = l2 * (R)4.5 * rho;
        cB = l2 * Bq;
        cO = l2 * (R)3 * rho;
        dB = 0;
    } else {
        const R sr = sg * rho1;
        cA = (R)4.5 * (lam * rho - sr);
        cB = lam * Bq;
        dB = -sr * ((R)1 - usq);
        cO = (R)3 * (lam * rho - sr);
    }
    const R sgsc = sg * (R)SC;  // for the u_inf target, in storage units
    const R A_a = wa * cA, A_e = we * cA, B_a = wa * (cB + dB), B_e = we * (cB + dB), O_a = wa * cO, O_e = we * cO;
    // pi is in storage units: its weights carry no scale
    const R Cn_a = SC != 1 ? (R)(4.5 / 18.0) * om1 : (R)4.5 * wa * om1, Cn_e = SC != 1 ? (R)(4.5 / 36.0) * om1 : (R)4.5 * we * om1;
    // c c : Pi - tr for edges = (Pi_aa - tr/2) + (Pi_bb - tr/2) + 2 s Pi_ab
    const R ht = (R)0.5 * tr;
    const R qx = pi[0] - ht, qy = pi[1] - ht, qz = pi[2] - ht;
    // rest population
    {
        R v = w0 * (cB + dB);
        if (COLL == 1) v = v + om1 * f[0];
        else v = v - (SC != 1 ? (R)(4.5 / 3.0) * om1 : (R)4.5 * w0 * om1) * tr;
        if (abs_u) v = v + sgsc * k.ft_rest;
        if (forcing) v = v + w0 * (fo * ((R)-3 * uG));
        f[0] = v;
    }
#pragma unroll
    for (int kk = 0; kk < 9; kk++) {
        const int i = 2 * kk + 1, o = i + 1;
        const bool axis = kk < 3;
        const R cu = cdot<R>(i, ux, uy, uz);
        R even = (axis ? A_a : A_e) * (cu * cu) + (axis ? B_a : B_e);
        R odd = (axis ? O_a : O_e) * cu;
        if (abs_u) {
            even = even + sgsc * k.ft_even[kk];
            odd = odd + sgsc * k.ft_odd[kk];
        }
        R vi, vo;
        if (COLL == 1) {
            const R ei = even + om1 * f[i], eo = even + om1 * f[o];
            vi = ei + odd;
            vo = eo - odd;
        } else {
            R ccp;  // c c : Pi - tr
            if (kk == 0) ccp = pi[0] - tr;
            else if (kk == 1) ccp = pi[1] - tr;
            else if (kk == 2) ccp = pi[2] - tr;
            else {
                const R a1 = CX(i) ? qx : qy;
                const R a2 = CZ(i) ? qz : qy;
                const R pab = (CX(i) && CY(i)) ? pi[3] : ((CX(i) && CZ(i)) ? pi[4] : pi[5]);
                const int sgn = CX(i) * CY(i) + CX(i) * CZ(i) + CY(i) * CZ(i);
                ccp = (a1 + a2) + (R)(2 * sgn) * pab;
            }
            const R en = even + (axis ? Cn_a : Cn_e) * ccp;
            vi = en + odd;
            vo = en - odd;
        }
        if (forcing) {
            const R w = axis ? wa : we;
            const R cg = cdot<R>(i, Gx, Gy, Gz);
            const R fe_ = w * (fo * ((R)9 * cu * cg - (R)3 * uG));
            R fod = w * (fo * (R)3 * cg);
            if (COLL != 1) fod = fod - w * ((R)1.5 * om1 * cg);
            vi = vi + (fe_ + fod);
            vo = vo + (fe_ - fod);
        }
        f[i] = vi;
        f[o] = vo;
    }
    rho_o = rho; ux_o = ux; uy_o = uy; uz_o = uz;
}
template <class R, int COLL, int SC = 1, int FEAT = 0>
__device__ __forceinline__ void relax(const LatParams &p, const Consts<R> &k, R *f, uint32_t x, uint32_t y, uint32_t z,
                                      bool wall, uint32_t r, uint32_t mask, R pcx, R pcy, R pcz, const R *om, R &rho_o, R &ux_o,
                                      R &uy_o, R &uz_o) {
    relax_m<R, COLL, SC, FEAT>(p, k, moments<R>(f), f, x, y, z, wall, r, mask, pcx, pcy, pcz, om, rho_o, ux_o, uy_o, uz_o);
}


// ---------------------------------------------------------------- bulk
// Plain fluid cells (flag word 0): the hot loop.
template <class S, int P, int COLL>
__global__ void __launch_bounds__(BLOCK) k_bulk(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s) {
    using R = typename Pop<S>::real;
    const uint32_t n = blockIdx.x * BLOCK + threadIdx.x;
    if (n >= p.N) return;
    if ((p.flags[n] & ~FLAG_XFACE) != 0u) return;
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    const Nb nb = make_nb(p, x, y, z);
    R f[19];
    load_in<S, P>(p, n, nb, f);
    const Consts<R> &k = K<R>(p);
    R rho, ux, uy, uz;
    const R om0[3] = {0, 0, 0};
    relax<R, COLL>(p, k, f, x, y, z, false, 0, 0, 0, 0, 0, om0, rho, ux, uy, uz);
    Rng rng{sr_hash_mix(n, s.seed_mix)};
    store_out<S, P>(p, n, nb, f, rng);
}

// ---------------------------------------------------------------- faces
template <class R, int M, int I>
__device__ __forceinline__ void mirror_one(const R *g, R *f) {
    constexpr int j = DIR((M & 1) ? -CX(I) : CX(I), (M & 2) ? -CY(I) : CY(I), (M & 4) ? -CZ(I) : CZ(I));
    f[I] = g[j];
}
template <class R, int M, int... Is>
__device__ __forceinline__ void mirror_all(const R *g, R *f, std::integer_sequence<int, Is...>) {
    (mirror_one<R, M, Is>(g, f), ...);
}
template <class R, int M>
__device__ __forceinline__ void mirror(const R *g, R *f) {
    mirror_all<R, M>(g, f, std::make_integer_sequence<int, 19>{});
}

// A face cell's "previous" post-collision populations from its inner
// neighbour's post-collision populations g (shader.rs:630-687): velocity
// inlet (u = u_inf, or the far field's total pressure with u from inside),
// open face (rho = 1), both as feq + fneq(Pi) of the neighbour's state; free
// slip (no reference counterpart) as the neighbour's mirror image.  fluid:
// the inner neighbour collides (else rest at u_inf).
template <class R>
__device__ __forceinline__ void face_values(const LatParams &p, const Consts<R> &k, uint32_t info, bool fluid, const R *g, R *f) {
    if ((info & 3u) == 2u) {
        if (fluid) {
            switch ((info >> 2) & 7u) {
                case 1: mirror<R, 1>(g, f); break;
                case 2: mirror<R, 2>(g, f); break;
                case 3: mirror<R, 3>(g, f); break;
                case 4: mirror<R, 4>(g, f); break;
                case 5: mirror<R, 5>(g, f); break;
                case 6: mirror<R, 6>(g, f); break;
                case 7: mirror<R, 7>(g, f); break;
                default: mirror<R, 0>(g, f); break;
            }
        } else {
            const R usq = (R)1.5 * (k.u_inf[0] * k.u_inf[0] + k.u_inf[1] * k.u_inf[1] + k.u_inf[2] * k.u_inf[2]);
#pragma unroll
            for (int i = 0; i < 19; i++) f[i] = feq_i<R>(i, (R)0, (R)1, k.u_inf[0], k.u_inf[1], k.u_inf[2], usq);
        }
        return;
    }
    R rho = 1, ux = k.u_inf[0], uy = k.u_inf[1], uz = k.u_inf[2];
    R pi[6] = {0, 0, 0, 0, 0, 0};
    if (fluid) {
        const Moments<R> mo = moments<R>(g);
        rho = (R)1 + mo.rho1;
        ux = mo.jx / rho - (R)0.5 * k.grav[0];
        uy = mo.jy / rho - (R)0.5 * k.grav[1];
        uz = mo.jz / rho - (R)0.5 * k.grav[2];
        pi_neq<R>(mo, rho, ux, uy, uz, pi);
    }
    if ((info & 3u) == 0u) {
        if (p.total_p) {
            const R uinf2 = k.u_inf[0] * k.u_inf[0] + k.u_inf[1] * k.u_inf[1] + k.u_inf[2] * k.u_inf[2];
            rho = ((R)(1.0 / 3.0) + (R)0.5 * uinf2) / ((R)(1.0 / 3.0) + (R)0.5 * (ux * ux + uy * uy + uz * uz));
        } else {
            ux = k.u_inf[0]; uy = k.u_inf[1]; uz = k.u_inf[2];
        }
    } else {
        rho = 1;
    }
    const R rho1 = rho - (R)1;
    const R usq = (R)1.5 * (ux * ux + uy * uy + uz * uz);
    const R tr = (pi[0] + pi[1] + pi[2]) * (R)(1.0 / 3.0);
#pragma unroll
    for (int i = 0; i < 19; i++) f[i] = feq_i<R>(i, rho1, rho, ux, uy, uz, usq) + fneq_i<R>(i, pi, tr);
}

// A velocity-inlet or open face cell b of face F whose store mask is the
// planar one: its five targets and its inner neighbour's 19 sources lie
// inside the domain without wrapping when the face's two in-plane axes are
// not periodic, so every offset is a plain stride and the directions are
// known at compile time.  The same values, rounding sequence and slots as
// the general path.
template <class S, int Q, int F>
__device__ __forceinline__ void face_planar(const LatParams &p, const StepParams &s, uint32_t b, uint32_t info) {
    using R = typename Pop<S>::real;
    constexpr int A = F >> 1;
    constexpr uint32_t MASK = planar_mask(F);
    const int32_t nx = (int32_t)p.NX, nxy = (int32_t)(p.NX * p.NY);
    const Nb flat{1, -1, nx, -nx, nxy, -nxy};
    const int32_t in = (F & 1 ? -1 : 1) * (A == 0 ? 1 : (A == 1 ? nx : nxy));
    const uint32_t m = (uint32_t)((int32_t)b + in);
    const bool fluid = (p.flags[m] & 3u) == 0u;
    R g[19];
    load_prev_out<S, Q>(p, m, flat, g);
    const Consts<R> &k = K<R>(p);
    R rho = 1, ux = k.u_inf[0], uy = k.u_inf[1], uz = k.u_inf[2];
    R pi[6] = {0, 0, 0, 0, 0, 0};
    if (fluid) {
        const Moments<R> mo = moments<R>(g);
        rho = (R)1 + mo.rho1;
        ux = mo.jx / rho - (R)0.5 * k.grav[0];
        uy = mo.jy / rho - (R)0.5 * k.grav[1];
        uz = mo.jz / rho - (R)0.5 * k.grav[2];
        pi_neq<R>(mo, rho, ux, uy, uz, pi);
    }
    if ((info & 3u) == 0u) {
        if (p.total_p) {
            const R uinf2 = k.u_inf[0] * k.u_inf[0] + k.u_inf[1] * k.u_inf[1] + k.u_inf[2] * k.u_inf[2];
            rho = ((R)(1.0 / 3.0) + (R)0.5 * uinf2) / ((R)(1.0 / 3.0) + (R)0.5 * (ux * ux + uy * uy + uz * uz));
        } else {
            ux = k.u_inf[0]; uy = k.u_inf[1]; uz = k.u_inf[2];
        }
    } else {
        rho = 1;
    }
    const R rho1 = rho - (R)1;
    const R usq = (R)1.5 * (ux * ux + uy * uy + uz * uz);
    const R tr = (pi[0] + pi[1] + pi[2]) * (R)(1.0 / 3.0);
    Rng rng{sr_hash_mix(b, s.seed_mix)};
    S *pop = (S *)p.pop;
    constexpr_for<0, 19>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr ((MASK >> i) & 1u) {
            const S v = Pop<S>::enc(feq_i<R>(i, rho1, rho, ux, uy, uz, usq) + fneq_i<R>(i, pi, tr), rng);
            if (Q == 0) pop[(uint64_t)OPP(i) * p.NP + b] = v;
            else pop[(uint64_t)i * p.NP + (uint32_t)((int32_t)b + flat.off(CX(i), CY(i), CZ(i)))] = v;
        }
    });
}

template <class S, int P>
__global__ void __launch_bounds__(BLOCK) k_faces(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s) {
    using R = typename Pop<S>::real;
    constexpr int Q = 1 - P;
    // the block's group: planar cells of one face (F < 6), or the rest
    int F = 6;
#pragma unroll
    for (int g = 5; g >= 0; g--)
        if (blockIdx.x < p.fblk[g + 1]) F = g;
    const uint32_t kf = p.fplan[F] + (blockIdx.x - p.fblk[F]) * BLOCK + threadIdx.x;
    if (kf >= (F < 6 ? p.fplan[F + 1] : s.nface)) return;
    uint32_t b, info;
    if (F < 6 && p.frect[F]) {
        // the face's rectangle in cell order: the cell from its rank, no list
        // load before the neighbour's populations
        const uint32_t k = kf - p.fplan[F], v = p.frect_nu[F].div(k), u = k - v * p.frect_nu[F].d;
        b = p.frect_b0[F] + u + v * p.frect_sv[F];
        info = p.finfo[F];
    } else {
        b = p.faces[kf];
        info = p.face_info[kf];
    }
    switch (F) {
        case 0: face_planar<S, Q, 0>(p, s, b, info); return;
        case 1: face_planar<S, Q, 1>(p, s, b, info); return;
        case 2: face_planar<S, Q, 2>(p, s, b, info); return;
        case 3: face_planar<S, Q, 3>(p, s, b, info); return;
        case 4: face_planar<S, Q, 4>(p, s, b, info); return;
        case 5: face_planar<S, Q, 5>(p, s, b, info); return;
        default: break;
    }
    uint32_t x, y, z;
    coords(p, b, x, y, z);
    uint32_t cx = x, cy = y, cz = z;
    if (!p.per[0]) cx = min(max(cx, 1u), p.NX - 2);
    if (!p.per[1]) cy = min(max(cy, 1u), p.NY - 2);
    if (!p.per[2]) cz = min(max(cz, 1u), p.NZ - 2);
    const uint32_t m = (cz * p.NY + cy) * p.NX + cx;
    const bool fluid = (p.flags[m] & 3u) == 0u;
    R g[19], f[19];
    // Loaded whatever the neighbour's flag says, so that these loads and the
    // flag's go out together: the addresses depend only on m (make_nb wraps at
    // the lattice's edges), and face_values ignores g when the neighbour is
    // not fluid.
    load_prev_out<S, Q>(p, m, make_nb(p, cx, cy, cz), g);
    Rng rng{sr_hash_mix(b, s.seed_mix)};
    const Nb nb = make_nb(p, x, y, z);
    const uint32_t mask = info >> 8;
    if ((info & 3u) == 2u) {  // free slip: the mirror image
        face_values<R>(p, K<R>(p), info, fluid, g, f);
        store_prev_out<S, Q>(p, b, nb, mask, f, rng);
        return;
    }
    // velocity inlet or open face: face_values' state, then feq + fneq only in
    // the directions stored (a planar face stores 5 of the 19)
    const Consts<R> &k = K<R>(p);
    R rho = 1, ux = k.u_inf[0], uy = k.u_inf[1], uz = k.u_inf[2];
    R pi[6] = {0, 0, 0, 0, 0, 0};
    if (fluid) {
        const Moments<R> mo = moments<R>(g);
        rho = (R)1 + mo.rho1;
        ux = mo.jx / rho - (R)0.5 * k.grav[0];
        uy = mo.jy / rho - (R)0.5 * k.grav[1];
        uz = mo.jz / rho - (R)0.5 * k.grav[2];
        pi_neq<R>(mo, rho, ux, uy, uz, pi);
    }
    if ((info & 3u) == 0u) {
        if (p.total_p) {
            const R uinf2 = k.u_inf[0] * k.u_inf[0] + k.u_inf[1] * k.u_inf[1] + k.u_inf[2] * k.u_inf[2];
            rho = ((R)(1.0 / 3.0) + (R)0.5 * uinf2) / ((R)(1.0 / 3.0) + (R)0.5 * (ux * ux + uy * uy + uz * uz));
        } else {
            ux = k.u_inf[0]; uy = k.u_inf[1]; uz = k.u_inf[2];
        }
    } else {
        rho = 1;
    }
    const R rho1 = rho - (R)1;
    const R usq = (R)1.5 * (ux * ux + uy * uy + uz * uz);
    const R tr = (pi[0] + pi[1] + pi[2]) * (R)(1.0 / 3.0);
    S *pop = (S *)p.pop;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        if (!(mask & (1u << i))) continue;
        const S v = Pop<S>::enc(feq_i<R>(i, rho1, rho, ux, uy, uz, usq) + fneq_i<R>(i, pi, tr), rng);
        if (Q == 0 || i == 0) pop[(uint64_t)OPP(i) * p.NP + b] = v;
        else pop[(uint64_t)i * p.NP + (uint32_t)((int32_t)b + nb.off(CX(i), CY(i), CZ(i)))] = v;
    }
}

// ---------------------------------------------------------------- staged bulk
// The hot loop, staged through shared memory by the bulk-copy (TMA) engine.
//
// In the AA pattern a cell reads and writes the same slots: at input parity
// 0 cell n uses (n, i) for every i; at parity 1 it reads (n + c_j, j) as its
// input f[opp j] and writes its output f[j] there.  So for a tile of T
// consecutive cells, plane j's slots form one contiguous range (shifted by
// c_j at parity 1), and the tile can be updated in place: one
// cp.async.bulk per plane brings the range into shared memory, every thread
// overwrites its cell's 19 inputs with its 19 outputs at the same positions,
// and the ranges go back to HBM with bulk stores (the 16-byte-aligned
// interior; the few ragged elements at the ends with plain stores).  Cells
// the kernel skips (faces, walls, solids) keep their slots unchanged.
//
// With NX * element size a multiple of 16 bytes and 512-byte aligned planes,
// a shifted range's misalignment depends only on c_x, so each plane's first
// cell sits at a compile-time element offset lead in its slot.  Store ranges
// are clamped to real cells and real slots, so no two blocks write the same
// slot.  Requires non-periodic x and y; a periodic z wraps only at the z
// boundaries, where cells load and store their wrapped links directly.
//
// Blocks are persistent and double buffered (the next tile's copies are in
// flight while the current one is collided).  Every mbarrier wait is
// bounded; on expiry the block records ERR_COPY_WAIT, drains its copies
// (bounded) and stops.
// Warp-specialized: the first Tma<S>::cwarps warps collide, the last
// Tma<S>::pwarps warps are producers that issue the bulk loads and stores
// (producer p handles the planes j = p mod pwarps).  Per buffer a "full"
// mbarrier (one arrival per producer + transaction bytes) and an "empty"
// mbarrier (one arrival per compute thread) replace block barriers, so
// compute warps move on to the next tile while the producers write the last
// one back.
// Block shape per storage: compute warps, producer warps, cells per compute
// thread and tile, tile buffers, and the blocks per SM the register budget
// aims at.  Measured on the B200 with the 512x256x256 arm case (MLUPS FP16 /
// FP32): three blocks of 7 compute warps with 896- / 448-cell tiles 54.9 /
// 35.3 k; two blocks of 10 warps, 1280 / 640 cells 52.3 / 35.5 k; one block of
// 20 warps with three buffers of 1280 / 640 cells 46.3 / 34.6 k; one block of
// 20 warps with two buffers of 2560 / 1280 cells 56.4 / 38.9 k; the same with
// 2, 3, 4, 5 producer warps 59.8, 60.3, 60.5, 58.7 k FP16 (FP32 38.2 k with 2 or
// 3).  The copy engine takes a few hundred cycles per bulk copy (one per plane
// and tile, each way) and the copies one warp issues go one after another, so
// fewer, larger copies and several issuing warps shorten a buffer's
// turnaround.
#ifndef LBM_CWARPS_2B
#define LBM_CWARPS_2B 20  // compute warps per block for 2-byte storage
#endif
#ifndef LBM_TILE_2B
#define LBM_TILE_2B 4  // cells per compute thread and tile for 2-byte storage
#endif
#ifndef LBM_NBUF_2B
#define LBM_NBUF_2B 2  // tile buffers per block for 2-byte storage
#endif
#ifndef LBM_BLOCKS_2B
#define LBM_BLOCKS_2B 1  // blocks per SM for 2-byte storage
#endif
#ifndef LBM_PWARPS_2B
#define LBM_PWARPS_2B 4  // producer warps per block for 2-byte storage
#endif
#ifndef LBM_PWARPS_4B
#define LBM_PWARPS_4B 1
#endif
#ifndef LBM_CWARPS_4B
#define LBM_CWARPS_4B 20  // the same for 4-byte storage
#endif
#ifndef LBM_TILE_4B
#define LBM_TILE_4B 2
#endif
#ifndef LBM_NBUF_4B
#define LBM_NBUF_4B 2
#endif
#ifndef LBM_BLOCKS_4B
#define LBM_BLOCKS_4B 1
#endif
template <class S> struct Tma {
    static constexpr int cwarps = sizeof(S) == 2 ? LBM_CWARPS_2B : (sizeof(S) == 4 ? LBM_CWARPS_4B : 7);
    static constexpr int pwarps = sizeof(S) == 2 ? LBM_PWARPS_2B : (sizeof(S) == 4 ? LBM_PWARPS_4B : 1);
    static constexpr int cthreads = cwarps * 32, threads = cthreads + 32 * pwarps;  // + the producer warps
    static constexpr uint32_t cells = (uint32_t)(sizeof(S) == 2 ? LBM_TILE_2B : (sizeof(S) == 4 ? LBM_TILE_4B : 1)) * cthreads;
    static constexpr int nbuf = sizeof(S) == 2 ? LBM_NBUF_2B : (sizeof(S) == 4 ? LBM_NBUF_4B : 3);
    static constexpr int min_blocks = sizeof(S) == 2 ? LBM_BLOCKS_2B : (sizeof(S) == 4 ? LBM_BLOCKS_4B : 2);
};
template <class S> struct Tile {
    static constexpr uint32_t cells = Tma<S>::cells;
    static_assert(cells <= TILE_MAX, "the allocations' guards cover tiles up to TILE_MAX cells");
};
template <class S> constexpr uint32_t slot_bytes() { return Tile<S>::cells * (uint32_t)sizeof(S) + 16; }
template <class S> constexpr uint32_t buf_bytes() { return 19 * slot_bytes<S>() + Tile<S>::cells * 4; }
// tile buffers per block: loads run up to NBUF - 1 tiles ahead
template <class S> struct Nbuf { static constexpr int value = Tma<S>::nbuf; };
template <class S> constexpr uint32_t tma_smem() { return Nbuf<S>::value * buf_bytes<S>() + 128; }  // + alignment slack

// element offset of plane j's first tile cell in its shared-memory slot
template <class S, int P>
__host__ __device__ __forceinline__ constexpr int lead(int j) {
    return (P == 0 || j == 0) ? 0 : (CX(j) == 1 ? 1 : (CX(j) == -1 ? (int)(16 / sizeof(S)) - 1 : 0));
}

// Self-test of the bounded wait: one thread waits for a barrier phase that
// nothing completes (no arrival, no copy); the wait must give up after
// limit_ns and report it, and the context stays usable.  status[0] = 1 when
// the wait gave up, status[1] = microseconds waited.
__global__ void k_wait_selftest(uint32_t *status, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        const uint64_t t0 = global_ns();
        const bool done = mbar_wait_bounded(&bar, 0, limit_ns);
        status[0] = done ? 0u : 1u;
        const uint64_t us = (global_ns() - t0) / 1000u;
        status[1] = us > 0xffffffffull ? 0xffffffffu : (uint32_t)us;
    }
}

// signed element shift of plane j's slots relative to the cell at parity P
template <int P>
__device__ __forceinline__ int64_t plane_shift(int j, int64_t NX, int64_t NXY) {
    return (P == 0 || j == 0) ? 0 : (int64_t)CX(j) + (int64_t)CY(j) * NX + (int64_t)CZ(j) * NXY;
}

// The loads of tile n0 into a buffer by producer warp pw of NPROD: the
// planes j = pw (mod NPROD), and the flags from the last producer; each
// producer posts its own bytes on the buffer's "full" barrier.
template <class S, int P, int NPROD>
__device__ __forceinline__ void tma_load_tile(const LatParams &p, uint8_t *buf, uint64_t *bar, uint32_t n0, int pw) {
    constexpr uint32_t SLOT = slot_bytes<S>();
    constexpr uint32_t T = Tile<S>::cells;
    const S *pop = (const S *)p.pop;
    const int64_t NX = p.NX, NXY = (int64_t)p.NX * p.NY;
    const uint32_t nplanes = (uint32_t)((19 - pw + NPROD - 1) / NPROD);
    mbar_expect_tx(bar, nplanes * SLOT + (pw == NPROD - 1 ? T * 4 : 0u));
#pragma unroll
    for (int j = 0; j < 19; j++) {
        if (j % NPROD != pw) continue;
        const int64_t e = (int64_t)j * (int64_t)p.NP + n0 + plane_shift<P>(j, NX, NXY) - lead<S, P>(j);
        bulk_g2s(buf + j * SLOT, pop + e, SLOT, bar);
    }
    if (pw == NPROD - 1) bulk_g2s(buf + 19 * SLOT, p.flags + n0, T * 4, bar);
}

// The x-face cell b next to cell m (b = m - 1 when x = 1, b = m + 1 when
// x = NX - 2), on a planar x face whose inner neighbour is m: its populations
// for the next step are what the face kernel of the next step would write
// from m's post-collision state, so the thread that just collided m computes
// them from its rounded outputs and writes them into b's slots of the staged
// tile; they reach HBM with the tile.  Only the 5 directions entering the
// domain are needed (the face kernel's store mask for a planar x face).
__host__ __device__ __forceinline__ constexpr int inward_dir(bool lo, int q) {
    // c_x = +1 directions (face at x = 0) or c_x = -1 (face at x = NX - 1), ascending
    return lo ? (q == 0 ? 1 : (q == 1 ? 7 : (q == 2 ? 9 : (q == 3 ? 13 : 15)))) : (q == 0 ? 2 : (q == 1 ? 8 : (q == 2 ? 10 : (q == 3 ? 14 : 16))));
}

template <class S, int P, bool LO>
__device__ __forceinline__ void xface_side(const LatParams &p, const StepParams &s, uint8_t *buf, uint32_t c, uint32_t m, uint32_t y,
                                           uint32_t z, const S *out) {
    using R = typename Pop<S>::real;
    constexpr uint32_t SLOT = slot_bytes<S>();
    const Consts<R> &k = K<R>(p);
    const uint32_t b = LO ? m - 1 : m + 1;
    const uint32_t cb = LO ? c - 1 : c + 1;
    const uint32_t info = p.xface_info[LO ? 0 : 1];
    R g[19];
#pragma unroll
    for (int i = 0; i < 19; i++) g[i] = Pop<S>::cvt(out[i]);
    R fb[5];  // the face cell's inward populations
    if ((info & 3u) == 2u) {
        // free slip: the mirror image in x of m's populations
#pragma unroll
        for (int q = 0; q < 5; q++) {
            fb[q] = g[DIR(-CX(inward_dir(LO, q)), CY(inward_dir(LO, q)), CZ(inward_dir(LO, q)))];
        }
    } else {
        const Moments<R> mo = moments<R>(g);
        R rho = (R)1 + mo.rho1;
        R ux = mo.jx / rho - (R)0.5 * k.grav[0];
        R uy = mo.jy / rho - (R)0.5 * k.grav[1];
        R uz = mo.jz / rho - (R)0.5 * k.grav[2];
        R pi[6];
        pi_neq<R>(mo, rho, ux, uy, uz, pi);
        if ((info & 3u) == 0u) {
            if (p.total_p) {
                const R uinf2 = k.u_inf[0] * k.u_inf[0] + k.u_inf[1] * k.u_inf[1] + k.u_inf[2] * k.u_inf[2];
                rho = ((R)(1.0 / 3.0) + (R)0.5 * uinf2) / ((R)(1.0 / 3.0) + (R)0.5 * (ux * ux + uy * uy + uz * uz));
            } else {
                ux = k.u_inf[0]; uy = k.u_inf[1]; uz = k.u_inf[2];
            }
        } else {
            rho = 1;
        }
        const R rho1 = rho - (R)1;
        const R usq = (R)1.5 * (ux * ux + uy * uy + uz * uz);
        const R tr = (pi[0] + pi[1] + pi[2]) * (R)(1.0 / 3.0);
#pragma unroll
        for (int q = 0; q < 5; q++) fb[q] = feq_i<R>(inward_dir(LO, q), rho1, rho, ux, uy, uz, usq) + fneq_i<R>(inward_dir(LO, q), pi, tr);
    }
    Rng rng{sr_hash_mix(b, s.next_seed_mix)};
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int i = inward_dir(LO, q);
        // the target row must collide: not on a non-periodic y or z face
        const int64_t ty = (int64_t)y + CY(i), tz = (int64_t)z + CZ(i);
        if (!p.per[1] && (ty <= 0 || ty >= (int64_t)p.NY - 1)) continue;
        if (!p.per[2] && (tz <= 0 || tz >= (int64_t)p.NZ - 1)) continue;
        const S v = Pop<S>::enc(fb[q], rng);
        const int j = P == 0 ? OPP(i) : i;
        ((S *)(buf + j * SLOT))[lead<S, P>(j) + cb] = v;
    }
}

// The x-face cell b next to cell m (b = m - 1 when x = 1, b = m + 1 when
// x = NX - 2), on a planar x face whose inner neighbour is m: its populations
// for the next step are what the face kernel of the next step would write
// from m's post-collision state (shader.rs:630-687), so the thread that just
// collided m computes them from its rounded outputs, with the face kernel's
// arithmetic and random sequence, and writes them into b's slots of the
// staged tile; they reach HBM with the tile.  Only the 5 directions entering
// the domain are needed (the face kernel's store mask of a planar x face).
template <class S, int P>
__device__ __forceinline__ void xface_from_inner(const LatParams &p, const StepParams &s, uint8_t *buf, uint32_t c, uint32_t m, uint32_t x,
                                                 uint32_t y, uint32_t z, const S *out) {
    if (x == 1) xface_side<S, P, true>(p, s, buf, c, m, y, z, out);
    else xface_side<S, P, false>(p, s, buf, c, m, y, z, out);
}

// A cell of a periodic-z boundary plane at input parity 1: the links that
// leave the domain in z wrap to the other side, so those inputs and outputs go
// straight to HBM; the others use the staged tile like every other cell.
template <class S, int COLL>
__device__ __forceinline__ void zwrap_cell(const LatParams &p, const StepParams &s, uint8_t *buf, uint32_t c, uint32_t n, uint32_t x,
                                        uint32_t y, uint32_t z) {
    using R = typename Pop<S>::real;
    constexpr uint32_t SLOT = slot_bytes<S>();
    S *pop = (S *)p.pop;
    const int zw = z == 0 ? -1 : 1;
    const Nb nb = make_nb(p, x, y, z);
    R f[19];
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const int j = i == 0 ? 0 : OPP(i);
        if (i > 0 && CZ(i) == -zw) f[i] = Pop<S>::ld(pop + (uint64_t)j * p.NP + (uint32_t)((int32_t)n + nb.off(-CX(i), -CY(i), -CZ(i))));
        else f[i] = Pop<S>::cvt(((const S *)(buf + j * SLOT))[lead<S, 1>(j) + c]);
    }
    R rho, ux, uy, uz;
    const R om0[3] = {0, 0, 0};
    relax<R, COLL>(p, K<R>(p), f, x, y, z, false, 0, 0, 0, 0, 0, om0, rho, ux, uy, uz);
    Rng rng{sr_hash_mix(n, s.seed_mix)};
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const S v = Pop<S>::enc(f[i], rng);
        if (i > 0 && CZ(i) == zw) pop[(uint64_t)i * p.NP + (uint32_t)((int32_t)n + nb.off(CX(i), CY(i), CZ(i)))] = v;
        else ((S *)(buf + i * SLOT))[lead<S, 1>(i) + c] = v;
    }
}

template <class S, int P, int COLL, int FEAT>
__global__ void __launch_bounds__(Tma<S>::threads, Tma<S>::min_blocks) k_bulk_tma(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s) {
    using R = typename Pop<S>::real;
    constexpr int NBUF = Nbuf<S>::value;
    constexpr uint32_t T = Tile<S>::cells, SLOT = slot_bytes<S>(), BUF = buf_bytes<S>();
    constexpr int64_t E16 = 16 / sizeof(S);
    extern __shared__ __align__(128) uint8_t sm_raw[];
    // realigned with pointer arithmetic so the compiler keeps it a shared-memory pointer
    uint8_t *sm = sm_raw + ((128u - (smem_addr(sm_raw) & 127u)) & 127u);
    __shared__ __align__(8) uint64_t full[NBUF], empty[NBUF];
    __shared__ int64_t tab_sh[19];  // plane shift (elements)
    __shared__ int tab_lead[19];    // plane lead (elements)
    const uint32_t ntiles = (p.N + T - 1) / T;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NBUF; q++) {
            mbar_init(&full[q], Tma<S>::pwarps);
            mbar_init(&empty[q], Tma<S>::cthreads);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x == 32) {
#pragma unroll
        for (int j = 0; j < 19; j++) {
            tab_sh[j] = plane_shift<P>(j, (int64_t)p.NX, (int64_t)p.NX * p.NY);
            tab_lead[j] = lead<S, P>(j);
        }
    }
    __syncthreads();
    S *pop = (S *)p.pop;
    if (warp >= Tma<S>::cwarps) {
        constexpr int NPROD = Tma<S>::pwarps;
        const int pw = warp - Tma<S>::cwarps;  // this producer's planes: j = pw (mod NPROD)
        // ------------------------------------------------ producer warps
        // iteration it (0 .. K+NBUF-1 for this block's K tiles): write back
        // this producer's planes of tile it-NBUF from buffer it%NBUF once the
        // compute warps released it, then load them for tile it into the
        // same buffer (the producers' planes are disjoint slots)
        const int64_t N = p.N;
        const uint32_t G = gridDim.x;
        const uint32_t K = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;
        uint32_t it = 0;
        bool alive = true;
        for (; it < K + NBUF; ++it) {
            const int b = it % NBUF;
            if (it >= NBUF) {
                if (!mbar_wait_bounded(&empty[b], ((it - NBUF) / NBUF) & 1)) { alive = false; break; }
                if (pw + NPROD * lane < 19) {
                    // plane j's slots of the tile's cells back to HBM: cells
                    // and slots clamped to [0, N); the 16-byte-aligned interior
                    // with one bulk store, the ragged ends with plain stores
                    const int j = pw + NPROD * lane;
                    const uint32_t n0 = (blockIdx.x + (it - NBUF) * G) * T;
                    const int64_t sh = tab_sh[j];
                    const int64_t lo = max((int64_t)n0, -sh);
                    int64_t hi = min(min((int64_t)n0 + (int64_t)T, N), N - sh);
                    if (hi < lo) hi = lo;
                    int64_t a = ((lo + sh + E16 - 1) & ~(E16 - 1)) - sh;  // slots are >= 0 here
                    int64_t bb = ((hi + sh) & ~(E16 - 1)) - sh;
                    if (bb < a) { a = hi; bb = hi; }
                    S *dst = pop + (int64_t)j * (int64_t)p.NP + sh;
                    const S *src = (const S *)(sm + b * BUF + j * SLOT) + tab_lead[j] - (int64_t)n0;
                    if (bb > a) bulk_s2g(dst + a, src + a, (uint32_t)((bb - a) * (int64_t)sizeof(S)));
                    bulk_commit();
                    for (int64_t m = lo; m < min(a, hi); m++) dst[m] = src[m];
                    for (int64_t m = max(bb, lo); m < hi; m++) dst[m] = src[m];
                    bulk_wait_read_all();
                }
                __syncwarp();
            }
            if (it < K && lane == 0) {
                fence_async_smem();
                tma_load_tile<S, P, NPROD>(p, sm + b * BUF, &full[b], (blockIdx.x + it * G) * T, pw);
            }
        }
        if (!alive && lane == 0) {
            atomicOr(p.err, ERR_COPY_WAIT);
            // drain the loads still in flight (the last one into each buffer)
            for (int bq = 0; bq < NBUF; bq++) {
                int last = -1;
                for (uint32_t q = 0; q < min(it, K); q++)
                    if ((int)(q % NBUF) == bq) last = (int)q;
                if (last >= 0) mbar_wait_bounded(&full[bq], ((uint32_t)last / NBUF) & 1);
            }
        }
        if (pw + NPROD * lane < 19) bulk_wait_all();
        return;
    }
    // ---------------------------------------------------- compute warps
    const Consts<R> &k = K<R>(p);
    const bool zper = p.per[2] != 0;
    uint32_t it = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int b = it % NBUF;
        if (!mbar_wait_bounded(&full[b], (it / NBUF) & 1)) {
            atomicOr(p.err, ERR_COPY_WAIT);
            return;
        }
        uint8_t *buf = sm + b * BUF;
        const uint32_t *fl = (const uint32_t *)(buf + 19 * SLOT);
        const uint32_t n0 = t * T;
#pragma unroll 1
        for (uint32_t c = threadIdx.x; c < T; c += Tma<S>::cthreads) {
            const uint32_t n = n0 + c;
            if (n >= p.N) break;
            const uint32_t fg = fl[c];
            if ((fg & ~FLAG_XFACE) != 0u) continue;
            uint32_t x, y, z;
            coords(p, n, x, y, z);
            if (P == 1 && zper && (z == 0 || z == p.NZ - 1)) {
                zwrap_cell<S, COLL>(p, s, buf, c, n, x, y, z);
                continue;
            }
            // FP16 values stay in storage units (x 32768) through the collision
            constexpr int SC = std::is_same<S, __half>::value ? (int)FP16_SCALE : 1;
            R f[19];
#pragma unroll
            for (int i = 0; i < 19; i++) {
                const int j = (P == 0 || i == 0) ? i : OPP(i);  // plane holding input f[i]
                const S v = ((const S *)(buf + j * SLOT))[lead<S, P>(j) + c];
                if constexpr (SC != 1) f[i] = __half2float(v);
                else f[i] = Pop<S>::cvt(v);
            }
            R rho, ux, uy, uz;
            const R om0[3] = {0, 0, 0};
            relax<R, COLL, SC, FEAT>(p, k, f, x, y, z, false, 0, 0, 0, 0, 0, om0, rho, ux, uy, uz);
            Rng rng{sr_hash_mix(n, s.seed_mix)};
            S out[19];
            if constexpr (sizeof(S) == 2) {
                // two values per stochastically rounding conversion, their
                // random bits from one product of the cell's hash per pair
                const uint32_t h = rng.s;
                constexpr_for<0, 10>([&](auto kk) {
                    constexpr int K = decltype(kk)::value, i = 2 * K;
                    if constexpr (i + 1 < 19) {
                        const uint32_t h2 = Pop<S>::rs2(f[i + 1], f[i], pair_bits<K>(h));
                        out[i] = Pop<S>::bits(h2 & 0xffffu);
                        out[i + 1] = Pop<S>::bits(h2 >> 16);
                    } else {
                        out[i] = Pop<S>::bits(Pop<S>::rs2(f[i], 0.0f, pair_bits<K>(h)) >> 16);
                    }
                });
            } else {
#pragma unroll
                for (int i = 0; i < 19; i++) out[i] = Pop<S>::enc(f[i], rng);
            }
#pragma unroll
            for (int i = 0; i < 19; i++) {
                const int j = (P == 0) ? OPP(i) : i;  // plane receiving output f[i]
                ((S *)(buf + j * SLOT))[lead<S, P>(j) + c] = out[i];
            }
            if (fg & FLAG_XFACE) xface_from_inner<S, P>(p, s, buf, c, n, x, y, z, out);
        }
        fence_async_smem();  // this thread's shared-memory writes, before the bulk stores read them
        mbar_arrive(&empty[b]);
    }
}

// ---------------------------------------------------------------- walls
// One thread per wall record.  A record whose cell is a fluid wall cell is
// updated with its links (Bouzidi-Firdaouss-Lallemand interpolated
// bounce-back with the moving-wall term and Galilean-invariant momentum
// exchange, shader.rs:399-436) and its post-collision state saved to the
// record (437-441, 848-860).  Every record's F and T enter the step's sum.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

static_assert((RS * 4) % 16 == 0, "records are read with 16-byte loads");
// The record's first 32 words (mask, cell, q, post-collision populations)
// in eight 16-byte loads.
__device__ __forceinline__ void record_words32(const LatParams &p, uint32_t r, uint32_t *w) {
    const uint4 *rv = reinterpret_cast<const uint4 *>(p.recs + (uint64_t)r * RS);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const uint4 v = rv[q];
        w[4 * q] = v.x; w[4 * q + 1] = v.y; w[4 * q + 2] = v.z; w[4 * q + 3] = v.w;
    }
}

// The cut links of a wall-record cell (shader.rs:399-436): for every link i
// of the mask, Bouzidi-Firdaouss-Lallemand interpolated bounce-back with the
// moving-wall term overwrites f[opp i] (q >= 1/2 from the cell's last
// post-collision values, q < 1/2 with the opposite link open also from its
// input), and the Galilean-invariant momentum exchange (Wen et al. 2014) adds
// the link's force and moment about the centre to Fo and To.  w: the record's
// first 32 words; f: the cell's inputs; om receives the wall's angular
// velocity.
template <class R>
__device__ __forceinline__ void wall_links(const LatParams &p, const StepParams &s, uint32_t r, const uint32_t *w, R pcx, R pcy, R pcz, R *f,
                                           R *om, R *Fo, R *To) {
    const uint32_t mask = w[R_MASK];
    if (sizeof(R) == 8) { om[0] = (R)s.omega_d[0]; om[1] = (R)s.omega_d[1]; om[2] = (R)s.omega_d[2]; }
    else { om[0] = (R)s.omega[0]; om[1] = (R)s.omega[1]; om[2] = (R)s.omega[2]; }
    R fin[19];
#pragma unroll
    for (int i = 0; i < 19; i++) fin[i] = f[i];
    // post-collision population i of the last step (FP64: the double copy) and q of link i
    auto fpost = [&](int i) -> R {
        if constexpr (sizeof(R) == 8) return Rec<R>::fpost(p, r, i);
        else return __uint_as_float(w[R_FPOST + i - 1]);
    };
    auto qof = [&](int i) -> R {
        const uint32_t qw = w[R_Q + (i - 1) / 2];
        return (R)__half2float(__ushort_as_half((unsigned short)(((i - 1) & 1) ? (qw >> 16) : (qw & 0xffffu))));
    };
#pragma unroll
    for (int i = 1; i < 19; i++) {
        if (mask & (1u << i)) {
            const int o = OPP(i);
            const R wi = (R)WD(i);
            const R q = max(qof(i), (R)0.001);
            const R fpi = fpost(i) + wi;
            const R fpo = fpost(o) + wi;
            const R cx = (R)CX(i), cy = (R)CY(i), cz = (R)CZ(i);
            const R xwx = pcx + q * cx, xwy = pcy + q * cy, xwz = pcz + q * cz;
            const R uwx = om[1] * xwz - om[2] * xwy, uwy = om[2] * xwx - om[0] * xwz, uwz = om[0] * xwy - om[1] * xwx;
            const R cu = cx * uwx + cy * uwy + cz * uwz;
            R fb;
            if (q >= (R)0.5) fb = (fpi + ((R)2 * q - (R)1) * fpo - (R)6 * wi * cu) / ((R)2 * q);
            else if ((mask & (1u << o)) == 0u) fb = (R)2 * q * fpi + ((R)1 - (R)2 * q) * (fin[i] + wi) - (R)6 * wi * cu;
            else fb = fpi - (R)6 * wi * cu;
            f[o] = fb - wi;
            const R flx = (cx - uwx) * fpi + (cx + uwx) * fb;
            const R fly = (cy - uwy) * fpi + (cy + uwy) * fb;
            const R flz = (cz - uwz) * fpi + (cz + uwz) * fb;
            Fo[0] += flx; Fo[1] += fly; Fo[2] += flz;
            To[0] += xwy * flz - xwz * fly;
            To[1] += xwz * flx - xwx * flz;
            To[2] += xwx * fly - xwy * flx;
        }
    }
}

// A wall-record cell's state after its collision written to its record
// (shader.rs:437-441, 848-860): post-collision populations, rho and u, and the
// step's force and moment (plus what a spinning part's re-voxelizer booked).
template <class R>
__device__ __forceinline__ void record_after(const LatParams &p, uint32_t r, const R *f, R rho, R ux, R uy, R uz, R *Fo, R *To) {
#pragma unroll
    for (int i = 1; i < 19; i++) Rec<R>::set_fpost(p, r, i, f[i]);
    Rec<R>::set_macro(p, r, 0, rho);
    Rec<R>::set_macro(p, r, 1, ux);
    Rec<R>::set_macro(p, r, 2, uy);
    Rec<R>::set_macro(p, r, 3, uz);
    if (p.moving) {
        for (int a = 0; a < 3; a++) { Fo[a] += Rec<R>::ft(p, r, a); To[a] += Rec<R>::ft(p, r, 3 + a); }
    }
    for (int a = 0; a < 3; a++) { Rec<R>::set_ft(p, r, a, Fo[a]); Rec<R>::set_ft(p, r, 3 + a, To[a]); }
}

template <class S, int P, int COLL>
__global__ void __launch_bounds__(WBLOCK) k_walls(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s) {
    using R = typename Pop<S>::real;
    const Consts<R> &k = K<R>(p);
    const uint32_t r = blockIdx.x * WBLOCK + threadIdx.x;
    R Fo[3] = {0, 0, 0}, To[3] = {0, 0, 0};
    if (r < p.nrec) {
        // The record's first 32 words, the cell's flag and its 19 populations
        // issued together before anything waits on them: the wall kernel is
        // short and latency-bound, so one round trip to HBM instead of a chain
        // of dependent loads per cut link.
        uint32_t w[32];
        record_words32(p, r, w);
        const uint32_t cell0 = w[R_CELL];
        const bool inside = cell0 < p.N;
        const uint32_t cell = inside ? cell0 : 0u;
        const uint32_t fg = p.flags[cell];
        uint32_t x, y, z;
        coords(p, cell, x, y, z);
        const Nb nb = make_nb(p, x, y, z);
        R f[19];
        load_in<S, P>(p, cell, nb, f);
        if (inside && (fg & 3u) == 0u && (fg >> 2) == r + 1u) {
            const uint32_t mask = w[R_MASK];
            const R pcx = (R)x - k.center[0], pcy = (R)y - k.center[1], pcz = (R)z - k.center[2];
            R om[3];
            wall_links<R>(p, s, r, w, pcx, pcy, pcz, f, om, Fo, To);
            R rho, ux, uy, uz;
            relax<R, COLL>(p, k, f, x, y, z, true, r, mask, pcx, pcy, pcz, om, rho, ux, uy, uz);
            record_after<R>(p, r, f, rho, ux, uy, uz, Fo, To);
            Rng rng{sr_hash_mix(cell, s.seed_mix)};
            store_out<S, P>(p, cell, nb, f, rng);
        } else {
            for (int a = 0; a < 3; a++) { Fo[a] = Rec<R>::ft(p, r, a); To[a] = Rec<R>::ft(p, r, 3 + a); }
        }
    }
    // FP64 sum: warp shuffle -> block -> last block over all block partials
    __shared__ double sh[WBLOCK / 32][6];
    __shared__ bool last;
    double v[6] = {(double)Fo[0], (double)Fo[1], (double)Fo[2], (double)To[0], (double)To[1], (double)To[2]};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 6; j++) v[j] = warp_sum(v[j]);
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = v[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < WBLOCK / 32; w++) t += sh[w][threadIdx.x];
        p.partials[blockIdx.x * 8 + threadIdx.x] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = atomicAdd(p.ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += WBLOCK)
        for (int j = 0; j < 6; j++) acc[j] += __ldcg(&p.partials[b * 8 + j]);
#pragma unroll
    for (int j = 0; j < 6; j++) acc[j] = warp_sum(acc[j]);
    __syncthreads();
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = acc[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < WBLOCK / 32; w++) t += sh[w][threadIdx.x];
        p.hist[s.slot * 8 + threadIdx.x] = t;
    }
    if (threadIdx.x == 0) *p.ticket = 0u;
}

// ---------------------------------------------------------------- init
// shader.rs:623-628: every cell holds the equilibrium at u_init (step seed 0)
template <class S>
__global__ void __launch_bounds__(BLOCK) k_init(const __grid_constant__ LatParams p) {
    using R = typename Pop<S>::real;
    const Consts<R> &k = K<R>(p);
    const uint32_t n = blockIdx.x * BLOCK + threadIdx.x;
    if (n >= p.N) return;
    S *pop = (S *)p.pop;
    const R usq = (R)1.5 * (k.u_init[0] * k.u_init[0] + k.u_init[1] * k.u_init[1] + k.u_init[2] * k.u_init[2]);
    Rng rng{sr_hash(n, 0u)};
#pragma unroll
    for (int i = 0; i < 19; i++) pop[(uint64_t)i * p.NP + n] = Pop<S>::enc(feq_i<R>(i, (R)0, (R)1, k.u_init[0], k.u_init[1], k.u_init[2], usq), rng);
}

// ---------------------------------------------------------------- dump
// shader.rs:599-621, 786-792: (rho, u) between steps; NaN off the fluid
template <class S, int Q>
__global__ void __launch_bounds__(BLOCK) k_dump(const __grid_constant__ LatParams p) {
    using R = typename Pop<S>::real;
    const Consts<R> &k = K<R>(p);
    const uint32_t n = blockIdx.x * BLOCK + threadIdx.x;
    if (n >= p.N) return;
    const uint32_t fg = p.flags[n] & ~FLAG_XFACE;
    if (fg & 3u) { p.dump[n] = make_float4(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000), __int_as_float(0x7fc00000), __int_as_float(0x7fc00000)); return; }
    const uint32_t rec = fg >> 2;
    if (rec) {
        p.dump[n] = make_float4((float)Rec<R>::macro(p, rec - 1, 0), (float)Rec<R>::macro(p, rec - 1, 1), (float)Rec<R>::macro(p, rec - 1, 2),
                                (float)Rec<R>::macro(p, rec - 1, 3));
        return;
    }
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    const Nb nb = make_nb(p, x, y, z);
    R f[19];
    load_prev_out<S, Q>(p, n, nb, f);
    const Moments<R> mo = moments<R>(f);
    const R rho = (R)1 + mo.rho1;
    p.dump[n] = make_float4((float)rho, (float)(mo.jx / rho - (R)0.5 * k.grav[0]), (float)(mo.jy / rho - (R)0.5 * k.grav[1]),
                            (float)(mo.jz / rho - (R)0.5 * k.grav[2]));
}

// ---------------------------------------------------------------- sampling
// Density and velocity of a cell between steps (shader.rs:599-621): wall
// cells from their records, fluid cells from their last post-collision
// populations, nothing for solid and face cells.
template <class S, int Q>
__device__ __forceinline__ bool cell_macro(const LatParams &p, uint32_t m, float &rho, float &ux, float &uy, float &uz) {
    using R = typename Pop<S>::real;
    const Consts<R> &k = K<R>(p);
    const uint32_t fg = p.flags[m] & ~FLAG_XFACE;
    if (fg & 3u) return false;
    const uint32_t rec = fg >> 2;
    if (rec) {
        rho = (float)Rec<R>::macro(p, rec - 1, 0);
        ux = (float)Rec<R>::macro(p, rec - 1, 1);
        uy = (float)Rec<R>::macro(p, rec - 1, 2);
        uz = (float)Rec<R>::macro(p, rec - 1, 3);
        return true;
    }
    uint32_t x, y, z;
    coords(p, m, x, y, z);
    const Nb nb = make_nb(p, x, y, z);
    R f[19];
    load_prev_out<S, Q>(p, m, nb, f);
    const Moments<R> mo = moments<R>(f);
    const R r = (R)1 + mo.rho1;
    rho = (float)r;
    ux = (float)(mo.jx / r - (R)0.5 * k.grav[0]);
    uy = (float)(mo.jy / r - (R)0.5 * k.grav[1]);
    uz = (float)(mo.jz / r - (R)0.5 * k.grav[2]);
    return true;
}

// shader.rs:736-759: trilinear density at rotated surface points
template <class S, int Q>
__global__ void __launch_bounds__(BLOCK) k_sample_verts(const __grid_constant__ LatParams p, const __grid_constant__ StepParams s,
                                                        const float *verts, uint32_t nvert, float voff, double *vacc) {
    const uint32_t v = blockIdx.x * BLOCK + threadIdx.x;
    if (v >= nvert) return;
    const float bx = verts[8 * v] + voff * verts[8 * v + 4];
    const float by = verts[8 * v + 1] + voff * verts[8 * v + 5];
    const float bz = verts[8 * v + 2] + voff * verts[8 * v + 6];
    float sp[3];
    for (int a = 0; a < 3; a++) sp[a] = p.kf.center[a] + (s.rot[a * 3] * bx + s.rot[a * 3 + 1] * by + s.rot[a * 3 + 2] * bz);
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
        if (cell_macro<S, Q>(p, m, rho, ux, uy, uz) && w > 0.f) { acc += w * rho; wsum += w; }
    }
    if (wsum > 1e-6f) {
        vacc[2 * v] += (double)(acc / wsum);
        vacc[2 * v + 1] += 1.0;
    }
}

// shader.rs:761-784: running sums of (rho, u) at slice pixels
template <class S, int Q>
__global__ void __launch_bounds__(BLOCK) k_sample_slices(const __grid_constant__ LatParams p, const int32_t *sd, uint32_t nslices,
                                                         uint32_t npix, double *sacc) {
    const uint32_t k = blockIdx.x * BLOCK + threadIdx.x;
    if (k >= npix) return;
    uint32_t acc = 0;
    for (uint32_t sl = 0; sl < nslices; sl++) {
        const int32_t *o = sd + 4 + 12 * sl;
        const uint32_t nu = (uint32_t)o[3], nv = (uint32_t)o[7];
        if (k < acc + nu * nv) {
            const uint32_t l = k - acc, iv = l / nu, iu = l - iv * nu;
            const long long c[3] = {(long long)o[0] + (long long)iu * o[4] + (long long)iv * o[8],
                                    (long long)o[1] + (long long)iu * o[5] + (long long)iv * o[9],
                                    (long long)o[2] + (long long)iu * o[6] + (long long)iv * o[10]};
            if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= p.NX || c[1] >= p.NY || c[2] >= p.NZ) return;
            float rho, ux, uy, uz;
            if (cell_macro<S, Q>(p, ((uint32_t)c[2] * p.NY + (uint32_t)c[1]) * p.NX + (uint32_t)c[0], rho, ux, uy, uz)) {
                double *b = sacc + 5ull * k;
                b[0] += rho; b[1] += ux; b[2] += uy; b[3] += uz; b[4] += 1.0;
            }
            return;
        }
        acc += nu * nv;
    }
}

// ---------------------------------------------------------------- mass
// FP64 sum of rho over fluid cells (wall cells included) from the
// post-collision populations of the last step, and a count of non-finite
// densities.
// Grid-stride over the cells (a few blocks per SM), each thread summing its
// cells in order, then the deterministic grid sum of reduce.cuh: the same
// result on every run, one atomic per block.  out[0] = mass, out[1] = the
// count of non-finite densities.
template <class S, int Q>
__global__ void __launch_bounds__(BLOCK) k_mass(const __grid_constant__ LatParams p, double *scratch, double *out) {
    using R = typename Pop<S>::real;
    double v = 0, nbad = 0;
    const uint32_t stride = gridDim.x * BLOCK;
#pragma unroll 1
    for (uint32_t n = blockIdx.x * BLOCK + threadIdx.x; n < p.N; n += stride) {
        const uint32_t fg = p.flags[n];
        if ((fg & 3u) != 0u) continue;
        uint32_t x, y, z;
        coords(p, n, x, y, z);
        const Nb nb = make_nb(p, x, y, z);
        R f[19];
        load_prev_out<S, Q>(p, n, nb, f);
        double sum = 0;
#pragma unroll
        for (int i = 0; i < 19; i++) sum += (double)f[i];
        const double rho = 1.0 + sum;
        if (isfinite(rho)) v += rho;
        else nbad += 1.0;
    }
    grid_sum2<BLOCK>(v, nbad, scratch, out);
}

// ---------------------------------------------------------------- launchers
static inline unsigned blocks_for(uint64_t n) { return (unsigned)((n + BLOCK - 1) / BLOCK); }

static int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return n;
}

// persistent grid of the staged kernel: resident blocks per SM x SMs
template <class S, int P, int COLL, int FEAT>
static unsigned tma_grid() {
    static unsigned g = 0;
    if (!g) {
        auto kern = k_bulk_tma<S, P, COLL, FEAT>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem<S>());
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Tma<S>::threads, tma_smem<S>());
        g = (unsigned)(std::max(per_sm, 1) * num_sms());
    }
    return g;
}

template <class S, int P, int COLL, int FEAT>
static void launch_tma(const LatParams &p, const StepParams &s, cudaStream_t st) {
    const unsigned ntiles = (unsigned)((p.N + Tile<S>::cells - 1) / Tile<S>::cells);
    k_bulk_tma<S, P, COLL, FEAT><<<std::min(ntiles, tma_grid<S, P, COLL, FEAT>()), Tma<S>::threads, tma_smem<S>(), st>>>(p, s);
}

// one step: faces, wall cells (on the side stream `side` when they cannot
// touch the faces' slots, overlapping the face kernel), then the bulk
template <class S, int P, int COLL>
static cudaError_t step_t(const LatParams &p, const StepParams &s, cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join,
                          cudaEvent_t *ev) {
    if (ev && ev[0]) cudaEventRecord(ev[0], st);
    if (p.moving) {
        // re-voxelize the spinning part's swept box for this step's rotation
        // (lattice.rs:719-723): triangles -> link scratch, cells, scratch reset
        if (p.ntri) k_tri_scatter<<<blocks_for((uint64_t)p.ntri * 32u), BLOCK, 0, st>>>(p, s);
        k_voxelize<S, 1 - P><<<blocks_for(p.nrec), BLOCK, 0, st>>>(p, s);
        k_qclear<<<blocks_for((uint64_t)p.nrec * 9u), BLOCK, 0, st>>>(p);
    }
    const bool overlap = side && p.nrec && s.nface && !p.moving;
    if (overlap) {
        cudaEventRecord(fork, st);
        cudaStreamWaitEvent(side, fork, 0);
        k_walls<S, P, COLL><<<(unsigned)((p.nrec + WBLOCK - 1) / WBLOCK), WBLOCK, 0, side>>>(p, s);
        cudaEventRecord(join, side);
    }
    if (s.nface) k_faces<S, P><<<p.fblk[6] + blocks_for(s.nface - p.fplan[6]), BLOCK, 0, st>>>(p, s);
    if (ev && ev[1]) cudaEventRecord(ev[1], st);
    if (overlap) cudaStreamWaitEvent(st, join, 0);
    else if (p.nrec) k_walls<S, P, COLL><<<(unsigned)((p.nrec + WBLOCK - 1) / WBLOCK), WBLOCK, 0, st>>>(p, s);
    if (ev && ev[2]) cudaEventRecord(ev[2], st);
    if (p.tma) {
        if (!p.forcing && !p.abs_u) {
            if (p.les_on) launch_tma<S, P, COLL, 3>(p, s, st);
            else launch_tma<S, P, COLL, 1>(p, s, st);
        } else {
            launch_tma<S, P, COLL, 0>(p, s, st);
        }
    } else {
        k_bulk<S, P, COLL><<<blocks_for(p.N), BLOCK, 0, st>>>(p, s);
    }
    if (ev && ev[3]) cudaEventRecord(ev[3], st);
    return cudaGetLastError();
}

template <class S>
static cudaError_t step_s(const LatParams &p, const StepParams &s, int parity, int coll, cudaStream_t st, cudaStream_t side, cudaEvent_t fork,
                          cudaEvent_t join, cudaEvent_t *ev) {
    if (parity == 0) return coll == 1 ? step_t<S, 0, 1>(p, s, st, side, fork, join, ev) : step_t<S, 0, 0>(p, s, st, side, fork, join, ev);
    return coll == 1 ? step_t<S, 1, 1>(p, s, st, side, fork, join, ev) : step_t<S, 1, 0>(p, s, st, side, fork, join, ev);
}

cudaError_t launch_step(int storage, const LatParams &p, const StepParams &s, int parity, int coll, cudaStream_t st, cudaStream_t side,
                        cudaEvent_t fork, cudaEvent_t join, cudaEvent_t *ev) {
    switch (storage) {
        case 0: return step_s<float>(p, s, parity, coll, st, side, fork, join, ev);
        case 1: return step_s<__half>(p, s, parity, coll, st, side, fork, join, ev);
        case 2: return step_s<__nv_bfloat16>(p, s, parity, coll, st, side, fork, join, ev);
        case 3: return step_s<double>(p, s, parity, coll, st, side, fork, join, ev);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_init(int storage, const LatParams &p, cudaStream_t st) {
    const unsigned g = blocks_for(p.N);
    switch (storage) {
        case 0: k_init<float><<<g, BLOCK, 0, st>>>(p); break;
        case 1: k_init<__half><<<g, BLOCK, 0, st>>>(p); break;
        case 2: k_init<__nv_bfloat16><<<g, BLOCK, 0, st>>>(p); break;
        case 3: k_init<double><<<g, BLOCK, 0, st>>>(p); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class S>
static void dump_s(const LatParams &p, int q, cudaStream_t st) {
    const unsigned g = blocks_for(p.N);
    if (q == 0) k_dump<S, 0><<<g, BLOCK, 0, st>>>(p);
    else k_dump<S, 1><<<g, BLOCK, 0, st>>>(p);
}

cudaError_t launch_dump(int storage, const LatParams &p, int q, cudaStream_t st) {
    switch (storage) {
        case 0: dump_s<float>(p, q, st); break;
        case 1: dump_s<__half>(p, q, st); break;
        case 2: dump_s<__nv_bfloat16>(p, q, st); break;
        case 3: dump_s<double>(p, q, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

uint32_t mass_blocks() { return (uint32_t)(4 * num_sms()); }

template <class S>
static void mass_s(const LatParams &p, int q, double *scratch, double *out, cudaStream_t st) {
    const unsigned g = std::min<unsigned>(mass_blocks(), blocks_for(p.N));
    if (q == 0) k_mass<S, 0><<<g, BLOCK, 0, st>>>(p, scratch, out);
    else k_mass<S, 1><<<g, BLOCK, 0, st>>>(p, scratch, out);
}

cudaError_t launch_mass(int storage, const LatParams &p, int q, double *scratch, double *out, cudaStream_t st) {
    switch (storage) {
        case 0: mass_s<float>(p, q, scratch, out, st); break;
        case 1: mass_s<__half>(p, q, scratch, out, st); break;
        case 2: mass_s<__nv_bfloat16>(p, q, scratch, out, st); break;
        case 3: mass_s<double>(p, q, scratch, out, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class S>
static void sample_s(const LatParams &p, const StepParams &s, int q, const float *verts, uint32_t nvert, float voff, double *vacc,
                     const int32_t *sd, uint32_t nslices, uint32_t npix, double *sacc, cudaStream_t st) {
    if (nvert) {
        if (q == 0) k_sample_verts<S, 0><<<blocks_for(nvert), BLOCK, 0, st>>>(p, s, verts, nvert, voff, vacc);
        else k_sample_verts<S, 1><<<blocks_for(nvert), BLOCK, 0, st>>>(p, s, verts, nvert, voff, vacc);
    }
    if (npix) {
        if (q == 0) k_sample_slices<S, 0><<<blocks_for(npix), BLOCK, 0, st>>>(p, sd, nslices, npix, sacc);
        else k_sample_slices<S, 1><<<blocks_for(npix), BLOCK, 0, st>>>(p, sd, nslices, npix, sacc);
    }
}

cudaError_t launch_sample(int storage, const LatParams &p, const StepParams &s, int q, const float *verts, uint32_t nvert, float voff,
                          double *vacc, const int32_t *sd, uint32_t nslices, uint32_t npix, double *sacc, cudaStream_t st) {
    switch (storage) {
        case 0: sample_s<float>(p, s, q, verts, nvert, voff, vacc, sd, nslices, npix, sacc, st); break;
        case 1: sample_s<__half>(p, s, q, verts, nvert, voff, vacc, sd, nslices, npix, sacc, st); break;
        case 2: sample_s<__nv_bfloat16>(p, s, q, verts, nvert, voff, vacc, sd, nslices, npix, sacc, st); break;
        case 3: sample_s<double>(p, s, q, verts, nvert, voff, vacc, sd, nslices, npix, sacc, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_wait_selftest(uint32_t *status, uint64_t limit_ns, cudaStream_t st) {
    k_wait_selftest<<<1, 32, 0, st>>>(status, limit_ns);
    return cudaGetLastError();
}

}  // namespace lbm
