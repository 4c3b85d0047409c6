// TEST INFRASTRUCTURE -- the CPU oracle for the gray-level lattice and its
// discrete adjoint.
//
// Nothing in the reference corresponds to this path (it has no gray level and
// no adjoint), so it has no reference file to follow and its parity is
// unpinned by the reference: the forward model is written out here from its
// definition, and the adjoint is checked against central finite differences of
// this forward model (tests/test_oracle_gray.py).
//
// Forward model (one step, state P = post-collision populations, shifted by
// the weights):
//   faces:   x = 0 cells hold feq(1, u_in); x = NX-1 cells copy the cell at x-1
//   stream:  g_i(n) = P_i(n - c_i) (periodic in y and z)
//   collide: BGK with the Brinkman drag of the exact-difference method
//            (Kupershtokh 2004): P_i = g_i - omega (g_i - feq_i(rho, u))
//                                      + feq_i(rho, (1 - a) u) - feq_i(rho, u),
//            a = alpha * gamma, which removes a * j of momentum and no mass
//   force:   F = sum over cells of a * j(g), moment M = sum a * (x - center) x j
// Adjoint: the reverse sweep stores every step's pre-collision populations and
// builds each cell's 19x19 Jacobian of the collision explicitly (the engine
// uses a contracted form that needs only the moments; the two are checked
// against each other and against finite differences).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "../include/simlab_lbm.h"
#include "d3q19_oracle.hpp"

namespace oracle {

template <class Real>
struct Gray {
    uint32_t NX = 0, NY = 0, NZ = 0;
    uint64_t N = 0;
    Real omega = 0, alpha = 0;
    Real u_in[3] = {0, 0, 0}, center[3] = {0, 0, 0};
    uint32_t box_lo[3] = {0, 0, 0}, box_n[3] = {0, 0, 0};
    std::vector<Real> P;   // 19 x N, shifted
    std::vector<Real> a;   // per cell
    Real W[19];
    uint64_t steps_done = 0;

    void create(const lbm_gray_setup &s) {
        NX = s.dims[0]; NY = s.dims[1]; NZ = s.dims[2];
        N = (uint64_t)NX * NY * NZ;
        if (NX < 4 || NY < 1 || NZ < 1) throw std::runtime_error("grid must be at least 4 cells along x");
        omega = (Real)(1.0 / (0.5 + 3.0 * s.nu));
        alpha = (Real)s.alpha;
        for (int k = 0; k < 3; k++) {
            u_in[k] = (Real)s.u_in[k];
            center[k] = (Real)s.center[k];
            box_lo[k] = s.box_lo[k];
            box_n[k] = s.box_n[k];
        }
        for (int i = 0; i < 19; i++) W[i] = (Real)weight19(i);
        a.assign(N, (Real)0);
        reset();
    }
    uint64_t nbox() const { return (uint64_t)box_n[0] * box_n[1] * box_n[2]; }
    void set_field(const double *gamma) {
        std::fill(a.begin(), a.end(), (Real)0);
        for (uint32_t z = 0; z < box_n[2]; z++)
            for (uint32_t y = 0; y < box_n[1]; y++)
                for (uint32_t x = 0; x < box_n[0]; x++) {
                    const uint64_t b = ((uint64_t)z * box_n[1] + y) * box_n[0] + x;
                    a[cell(box_lo[0] + x, box_lo[1] + y, box_lo[2] + z)] = alpha * (Real)gamma[b];
                }
    }
    uint64_t cell(uint32_t x, uint32_t y, uint32_t z) const { return ((uint64_t)z * NY + y) * NX + x; }
    void feqs(Real rho1, const Real *u, Real *f) const {
        const Real rho = 1 + rho1, usq = (Real)1.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        for (int i = 0; i < 19; i++) {
            const Real cu = C19[i][0] * u[0] + C19[i][1] * u[1] + C19[i][2] * u[2];
            f[i] = W[i] * (rho1 + rho * (3 * cu + (Real)4.5 * cu * cu - usq));
        }
    }
    void reset() {
        P.assign(19 * N, (Real)0);
        Real f[19];
        feqs(0, u_in, f);
        for (int i = 0; i < 19; i++)
            for (uint64_t n = 0; n < N; n++) P[i * N + n] = f[i];
        steps_done = 0;
    }
    void faces(std::vector<Real> &S) const {
        Real f[19];
        feqs(0, u_in, f);
        for (uint32_t z = 0; z < NZ; z++)
            for (uint32_t y = 0; y < NY; y++) {
                const uint64_t b0 = cell(0, y, z), b1 = cell(NX - 1, y, z);
                for (int i = 0; i < 19; i++) {
                    S[i * N + b0] = f[i];
                    S[i * N + b1] = S[i * N + b1 - 1];
                }
            }
    }
    // g_i(n) = S_i(n - c_i)
    void pull(const std::vector<Real> &S, uint32_t x, uint32_t y, uint32_t z, Real *g) const {
        for (int i = 0; i < 19; i++) {
            const uint32_t xx = x - C19[i][0];
            const uint32_t yy = (y + NY - C19[i][1]) % NY, zz = (z + NZ - C19[i][2]) % NZ;
            g[i] = S[i * N + cell(xx, yy, zz)];
        }
    }
    static void mom(const Real *g, Real &rho1, Real *j) {
        rho1 = 0;
        j[0] = j[1] = j[2] = 0;
        for (int i = 0; i < 19; i++) {
            rho1 += g[i];
            for (int k = 0; k < 3; k++) j[k] += C19[i][k] * g[i];
        }
    }
    void collide(const Real *g, Real an, Real *out) const {
        Real rho1, j[3];
        mom(g, rho1, j);
        const Real rho = 1 + rho1, jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
        const Real B = omega - 1 + (1 - an) * (1 - an);
        for (int i = 0; i < 19; i++) {
            const Real cj = C19[i][0] * j[0] + C19[i][1] * j[1] + C19[i][2] * j[2];
            const Real Q = (Real)4.5 * cj * cj - (Real)1.5 * jj;
            out[i] = (1 - omega) * g[i] + W[i] * (omega * rho1 + 3 * (omega - an) * cj + B * Q / rho);
        }
    }
    void weight_vec(int objective, const double *dir, uint32_t x, uint32_t y, uint32_t z, Real *e) const {
        if (objective == 0) { for (int k = 0; k < 3; k++) e[k] = (Real)dir[k]; return; }
        const Real r[3] = {(Real)x - center[0], (Real)y - center[1], (Real)z - center[2]};
        // dir . (r x j) = j . (dir x r)
        e[0] = (Real)dir[1] * r[2] - (Real)dir[2] * r[1];
        e[1] = (Real)dir[2] * r[0] - (Real)dir[0] * r[2];
        e[2] = (Real)dir[0] * r[1] - (Real)dir[1] * r[0];
    }
    // one step; returns force and moment on the gray body
    std::array<double, 6> step() {
        faces(P);
        std::vector<Real> Pn(P);
        std::array<double, 6> fm{};
        for (uint32_t z = 0; z < NZ; z++)
            for (uint32_t y = 0; y < NY; y++)
                for (uint32_t x = 1; x + 1 < NX; x++) {
                    const uint64_t n = cell(x, y, z);
                    Real g[19], o[19];
                    pull(P, x, y, z, g);
                    collide(g, a[n], o);
                    for (int i = 0; i < 19; i++) Pn[i * N + n] = o[i];
                    if (a[n] != 0) {
                        Real rho1, j[3];
                        mom(g, rho1, j);
                        const Real r[3] = {(Real)x - center[0], (Real)y - center[1], (Real)z - center[2]};
                        const Real F[3] = {a[n] * j[0], a[n] * j[1], a[n] * j[2]};
                        for (int k = 0; k < 3; k++) fm[k] += (double)F[k];
                        fm[3] += (double)(r[1] * F[2] - r[2] * F[1]);
                        fm[4] += (double)(r[2] * F[0] - r[0] * F[2]);
                        fm[5] += (double)(r[0] * F[1] - r[1] * F[0]);
                    }
                }
        P.swap(Pn);
        steps_done++;
        return fm;
    }

    // objective and its gradient with respect to gamma of every box cell
    double backward(const lbm_adjoint_spec &sp, double *grad_box) {
        reset();
        const uint64_t T = sp.steps;
        const Real wt = (Real)(1.0 / (double)(sp.t1 - sp.t0 + 1));
        // forward, keeping every step's pre-collision populations of the bulk
        std::vector<std::vector<Real>> G(T + 1);
        double J = 0;
        for (uint64_t t = 1; t <= T; t++) {
            faces(P);
            G[t].assign(19 * N, (Real)0);
            for (uint32_t z = 0; z < NZ; z++)
                for (uint32_t y = 0; y < NY; y++)
                    for (uint32_t x = 1; x + 1 < NX; x++) {
                        Real g[19];
                        pull(P, x, y, z, g);
                        for (int i = 0; i < 19; i++) G[t][i * N + cell(x, y, z)] = g[i];
                    }
            std::vector<Real> Pn(P);
            for (uint32_t z = 0; z < NZ; z++)
                for (uint32_t y = 0; y < NY; y++)
                    for (uint32_t x = 1; x + 1 < NX; x++) {
                        const uint64_t n = cell(x, y, z);
                        Real g[19], o[19];
                        for (int i = 0; i < 19; i++) g[i] = G[t][i * N + n];
                        collide(g, a[n], o);
                        for (int i = 0; i < 19; i++) Pn[i * N + n] = o[i];
                        if (t >= sp.t0 && t <= sp.t1 && a[n] != 0) {
                            Real rho1, j[3], e[3];
                            mom(g, rho1, j);
                            weight_vec(sp.objective, sp.dir, x, y, z, e);
                            J += (double)(wt * a[n] * (e[0] * j[0] + e[1] * j[1] + e[2] * j[2]));
                        }
                    }
            P.swap(Pn);
        }
        steps_done = T;
        // reverse sweep; L = adjoint of the pre-collision populations of step t+1
        std::vector<Real> L(19 * N, (Real)0), Ln(19 * N, (Real)0), gradc(N, (Real)0);
        auto bulk = [&](int64_t x) { return x >= 1 && x <= (int64_t)NX - 2; };
        for (uint64_t t = T; t >= 1; t--) {
            std::fill(Ln.begin(), Ln.end(), (Real)0);
            const Real wstep = (t >= sp.t0 && t <= sp.t1) ? wt : (Real)0;
            for (uint32_t z = 0; z < NZ; z++)
                for (uint32_t y = 0; y < NY; y++)
                    for (uint32_t x = 1; x + 1 < NX; x++) {
                        const uint64_t n = cell(x, y, z);
                        // adjoint of P_t(n): through the next step's pull and the outlet copy
                        Real mu[19];
                        for (int i = 0; i < 19; i++) {
                            mu[i] = 0;
                            const uint32_t yy = (y + NY + C19[i][1]) % NY, zz = (z + NZ + C19[i][2]) % NZ;
                            if (bulk((int64_t)x + C19[i][0])) mu[i] += L[i * N + cell(x + C19[i][0], yy, zz)];
                            if (x == NX - 2 && C19[i][0] == -1) mu[i] += L[i * N + cell(x + 1 + C19[i][0], yy, zz)];
                        }
                        Real g[19];
                        for (int i = 0; i < 19; i++) g[i] = G[t][i * N + n];
                        Real rho1, j[3];
                        mom(g, rho1, j);
                        const Real rho = 1 + rho1, jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
                        const Real an = a[n];
                        const Real B = omega - 1 + (1 - an) * (1 - an);
                        // dense Jacobian dP_i/dg_k and dP_i/da
                        Real e[3];
                        weight_vec(sp.objective, sp.dir, x, y, z, e);
                        Real ga = 0;
                        for (int k = 0; k < 19; k++) {
                            Real s = 0;
                            for (int i = 0; i < 19; i++) {
                                const Real ci_ck = C19[i][0] * C19[k][0] + C19[i][1] * C19[k][1] + C19[i][2] * C19[k][2];
                                const Real cj = C19[i][0] * j[0] + C19[i][1] * j[1] + C19[i][2] * j[2];
                                const Real Q = (Real)4.5 * cj * cj - (Real)1.5 * jj;
                                Real dQ = 0;  // dQ_i/dj . c_k
                                for (int q = 0; q < 3; q++) dQ += (9 * cj * C19[i][q] - 3 * j[q]) * C19[k][q];
                                const Real jac = (i == k ? 1 - omega : (Real)0) +
                                                 W[i] * (omega + 3 * (omega - an) * ci_ck + B * dQ / rho - B * Q / (rho * rho));
                                s += mu[i] * jac;
                            }
                            const Real ec = e[0] * C19[k][0] + e[1] * C19[k][1] + e[2] * C19[k][2];
                            Ln[k * N + n] = s + wstep * an * ec;
                        }
                        for (int i = 0; i < 19; i++) {
                            const Real cj = C19[i][0] * j[0] + C19[i][1] * j[1] + C19[i][2] * j[2];
                            const Real Q = (Real)4.5 * cj * cj - (Real)1.5 * jj;
                            ga += mu[i] * W[i] * (-3 * cj - 2 * (1 - an) * Q / rho);
                        }
                        ga += wstep * (e[0] * j[0] + e[1] * j[1] + e[2] * j[2]);
                        gradc[n] += ga;
                    }
            L.swap(Ln);
        }
        for (uint32_t z = 0; z < box_n[2]; z++)
            for (uint32_t y = 0; y < box_n[1]; y++)
                for (uint32_t x = 0; x < box_n[0]; x++) {
                    const uint64_t b = ((uint64_t)z * box_n[1] + y) * box_n[0] + x;
                    grad_box[b] = (double)(alpha * gradc[cell(box_lo[0] + x, box_lo[1] + y, box_lo[2] + z)]);
                }
        return J;
    }
};

}  // namespace oracle
