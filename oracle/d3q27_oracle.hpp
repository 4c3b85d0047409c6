// TEST INFRASTRUCTURE -- the CPU oracle for the multi-level D3Q27 time step.
//
// A restatement of SimLab's WGSL D3Q27 level kernels (crates/cfd/src/mshader.rs)
// and their host driver (crates/cfd/src/mlattice.rs): per-level setup, cell
// types and lists, pull streaming over two population sets, Bouzidi walls
// with momentum exchange, the cumulant-type collision (`gauss`), domain faces,
// ghost interpolation, restriction and the recursive sub-cycling schedule.
// Only the tests, the smoke check and the bench's CPU baseline use it; the
// engine never links or calls it.
//
// Parity pin: the reference ships no golden vectors and cannot run here, so
// this restatement is pinned by the reference's own known-answer tests for
// the refined solver, re-run against it (crates/cfd/tests/refined.rs):
// D3Q27 Poiseuille flow with second-order convergence and force balance
// (34-81), momentum lost by the fluid = impulse on the body (83-98) and a
// uniform stream crossing two refinement levels unchanged (100-119).
//
// Templated on the arithmetic type: float follows the reference's FP32
// operations in order (compile with -ffp-contract=off); double is the FP64
// oracle.  Storage: FP32, FP64, FP16 (scaled by 32768, stochastic rounding
// with the reference's hash and seeds, mshader.rs:171-177, 468-476,
// mlattice.rs:694-703) and BF16 (no reference counterpart).  Forces are
// summed in double (the reference sums in f32, mshader.rs:519-562).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/simlab_lbm.h"
#include "d3q19_oracle.hpp"

namespace oracle {
namespace q27 {

// d3q27.rs:1-29: direction i has velocity (i%3-1, (i/3)%3-1, i/9-1)
constexpr int Q = 27, REST = 13;
inline int cx(int i) { return i % 3 - 1; }
inline int cy(int i) { return (i / 3) % 3 - 1; }
inline int cz(int i) { return i / 9 - 1; }
inline int opp(int i) { return 26 - i; }
inline int slot(int i) { return i < REST ? i : i - 1; }
inline double weight(int i) {
    switch (std::abs(cx(i)) + std::abs(cy(i)) + std::abs(cz(i))) {
        case 0: return 8.0 / 27.0;
        case 1: return 2.0 / 27.0;
        case 2: return 1.0 / 54.0;
        default: return 1.0 / 216.0;
    }
}

// mshader.rs:32-48
constexpr uint32_t RS = 24, R_MASK = 0, R_CELL = 1, R_Q = 2, R_FT = 15, MW = 12;
constexpr uint32_t T_FLUID = 0, T_SOLID = 1, T_FACE = 2, T_GHOST = 3, T_RESTRICT = 4;
constexpr size_t HIST_CAP = 1024;  // mlattice.rs:283
constexpr uint32_t SEED_SRC_MUL = 7919u, SEED_MW_MUL = 104729u;  // mlattice.rs:704

}  // namespace q27

template <class Real>
struct Multi27 {
    using F = std::array<Real, 27>;
    using Set = lbm_multi_setup;
    struct Mom { Real rho1; Real j[3]; Real s[6]; };

    struct Level {
        uint32_t NX = 0, NY = 0, NZ = 0;
        uint64_t N = 0;
        bool per[3] = {false, false, false};
        Real TAU0{}, SMAG2{}, SPONGE_TAU{}, SIGMA{};
        Real SP_LO[3]{}, SP_HI[3]{}, U_INF[3]{}, U_INIT[3]{}, GRAV[3]{}, CENTER[3]{};
        bool N_SPONGE = false, forcing = false;
        bool has_child = false, has_parent = false;
        int32_t ch_lo[3] = {0, 0, 0};
        uint32_t ch_n[3] = {1, 1, 1};
        uint64_t ch_nodes = 1;
        uint32_t pn[3] = {0, 0, 0};
        uint64_t pnodes = 0;
        std::vector<float> p32[2];
        std::vector<double> p64[2];
        std::vector<uint16_t> p16[2];
        std::vector<uint32_t> flags, faces, ghosts, restricted;
        std::vector<Real> mom_child, mom_up;
        uint32_t src = 0, mslot = 1;
        uint64_t steps = 0;
        bool finest = false;
    };

    // per-dispatch parameters (mlattice.rs:97-112)
    struct Par {
        uint32_t src = 0, mw = 0, mold = 0, mnew = 0, seed = 0;
        Real blend = 0;
        Real omega[3] = {0, 0, 0};
        float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, rot_prev[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    };
    // spinning part on the finest level (no reference counterpart): the D3Q19
    // re-voxelizer of shader.rs:865-1104 carried to 27 directions, links kept
    // at the cell they leave along i = 14..26
    bool moving = false;
    std::vector<uint32_t> occ;
    float occ_lo[3] = {0, 0, 0}, occ_invh = 1.f, CENTERF[3] = {0, 0, 0};
    int32_t occ_n[3] = {0, 0, 0}, box_lo[3] = {0, 0, 0};
    uint32_t box_n[3] = {0, 0, 0};
    std::vector<std::array<float, 12>> tris;
    std::vector<uint32_t> qscr;

    int storage = LBM_STORAGE_FP32;
    bool ABS_U = false, TOTAL_P = false;
    std::vector<Level> lv;
    std::vector<uint32_t> rec_words;   // RS words per record
    std::vector<Real> rec_q;           // 26 per record (slot order), decoded from f16
    std::vector<Real> rec_ft;          // 6 per record
    uint32_t nrec = 0;
    uint64_t fine_steps = 0;
    Real W[27]{}, W45[27]{};
    // probes (mlattice.rs:79-84, 243-305): surface vertices on the finest
    // level, each slice pixel on the finest level whose interior holds it
    std::vector<std::array<float, 8>> pverts;  // position, 0, normal, 0 (body coordinates)
    float VOFF = 0.f;
    std::vector<double> vacc;                  // 2 per vertex: sum of rho, count
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> pix;  // per level: (pixel, cell)
    uint32_t npix = 0;
    std::vector<double> sacc;                  // 5 per pixel

    // ------------------------------------------------------------ storage
    inline Real L(const Level &l, uint32_t set, int d, uint64_t cell) const {
        uint64_t k = (uint64_t)d * l.N + cell;
        switch (storage) {
            case LBM_STORAGE_FP32: return (Real)l.p32[set][k];
            case LBM_STORAGE_FP64: return (Real)l.p64[set][k];
            case LBM_STORAGE_FP16: return (Real)(f16_to_f32(l.p16[set][k]) * (1.0f / FP16_SCALE));
            default: return (Real)bf16_to_f32(l.p16[set][k]);
        }
    }
    inline void S(Level &l, uint32_t set, int d, uint64_t cell, Real v, uint32_t seed) {
        uint64_t k = (uint64_t)d * l.N + cell;
        const uint32_t key = (uint32_t)cell * 27u + (uint32_t)d;
        switch (storage) {
            case LBM_STORAGE_FP32: l.p32[set][k] = (float)v; break;
            case LBM_STORAGE_FP64: l.p64[set][k] = (double)v; break;
            case LBM_STORAGE_FP16: l.p16[set][k] = f32_to_f16(sround16((float)v * FP16_SCALE, key, seed)); break;
            default: l.p16[set][k] = f32_to_bf16(sround_bf16((float)v, key, seed)); break;
        }
    }
    F own(const Level &l, uint32_t set, uint64_t n) const {  // mshader.rs:201-206
        F f;
        for (int i = 0; i < 27; i++) f[i] = L(l, set, i, n);
        return f;
    }
    void put(Level &l, uint32_t set, uint64_t n, const F &f, uint32_t seed) {  // mshader.rs:207-217
        for (int i = 0; i < 27; i++) S(l, set, i, n, f[i], seed);
    }
    static void coords(const Level &l, uint64_t n, uint32_t &x, uint32_t &y, uint32_t &z) {
        z = (uint32_t)(n / ((uint64_t)l.NX * l.NY));
        uint64_t r = n - (uint64_t)z * l.NX * l.NY;
        y = (uint32_t)(r / l.NX);
        x = (uint32_t)(r - (uint64_t)y * l.NX);
    }
    static uint64_t cidx(const Level &l, uint32_t x, uint32_t y, uint32_t z) { return ((uint64_t)z * l.NY + y) * l.NX + x; }
    // mshader.rs:218-227 with the neighbour prelude of mshader.rs:135-138
    F pull(const Level &l, uint32_t set, uint64_t n) const {
        uint32_t x, y, z;
        coords(l, n, x, y, z);
        const uint32_t xp = x == l.NX - 1 ? 0 : x + 1, xm = x == 0 ? l.NX - 1 : x - 1;
        const uint32_t yp = y == l.NY - 1 ? 0 : y + 1, ym = y == 0 ? l.NY - 1 : y - 1;
        const uint32_t zp = z == l.NZ - 1 ? 0 : z + 1, zm = z == 0 ? l.NZ - 1 : z - 1;
        F f;
        for (int i = 0; i < 27; i++) {
            if (i == q27::REST) { f[i] = L(l, set, i, n); continue; }
            const int dx = -q27::cx(i), dy = -q27::cy(i), dz = -q27::cz(i);
            const uint32_t xx = dx == 1 ? xp : (dx == -1 ? xm : x);
            const uint32_t yy = dy == 1 ? yp : (dy == -1 ? ym : y);
            const uint32_t zz = dz == 1 ? zp : (dz == -1 ? zm : z);
            f[i] = L(l, set, i, cidx(l, xx, yy, zz));
        }
        return f;
    }

    // ------------------------------------------------------------ math
    // mshader.rs:236-255: sums in direction order starting from 0.0
    static Mom moments(const F &f) {
        Mom m;
        Real r = 0;
        for (int i = 0; i < 27; i++) r = r + f[i];
        m.rho1 = r;
        for (int a = 0; a < 3; a++) {
            Real t = 0;
            for (int i = 0; i < 27; i++) {
                const int c = a == 0 ? q27::cx(i) : (a == 1 ? q27::cy(i) : q27::cz(i));
                if (c == 1) t = t + f[i]; else if (c == -1) t = t - f[i];
            }
            m.j[a] = t;
        }
        static const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
        for (int q = 0; q < 6; q++) {
            Real t = 0;
            for (int i = 0; i < 27; i++) {
                const int v[3] = {q27::cx(i), q27::cy(i), q27::cz(i)};
                const int k = v[pa[q]] * v[pb[q]];
                if (k == 1) t = t + f[i]; else if (k == -1) t = t - f[i];
            }
            m.s[q] = t;
        }
        return m;
    }
    // mshader.rs:257-266: product-form equilibrium, shifted
    F feq(Real rho, const Real *u) const {
        const Real third = (Real)1 / (Real)3, two3 = (Real)2 / (Real)3, h = (Real)0.5;
        Real a[3][3];
        for (int k = 0; k < 3; k++) {
            a[k][0] = h * (third + u[k] * u[k] - u[k]);
            a[k][1] = two3 - u[k] * u[k];
            a[k][2] = h * (third + u[k] * u[k] + u[k]);
        }
        F f;
        for (int i = 0; i < 27; i++) f[i] = rho * a[0][q27::cx(i) + 1] * a[1][q27::cy(i) + 1] * a[2][q27::cz(i) + 1] - W[i];
        return f;
    }
    // mshader.rs:268-280: second-order Hermite non-equilibrium of a stress
    F fneq(const Real *p) const {
        F f;
        const Real tr = (p[0] + p[1] + p[2]) * ((Real)1 / (Real)3);
        static const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
        for (int i = 0; i < 27; i++) {
            const int v[3] = {q27::cx(i), q27::cy(i), q27::cz(i)};
            Real t = -tr;
            for (int q = 0; q < 6; q++) {
                const int m = v[pa[q]] * v[pb[q]] * (pa[q] == pb[q] ? 1 : 2);
                if (m != 0) t = t + (Real)m * p[q];
            }
            f[i] = W45[i] * t;
        }
        return f;
    }
    // mshader.rs:486-495 (division by 3, not multiplication by 1/3)
    static void stress(const Mom &mo, Real rho, const Real *u, Real *p) {
        p[0] = mo.s[0] - rho * u[0] * u[0] - mo.rho1 / (Real)3;
        p[1] = mo.s[1] - rho * u[1] * u[1] - mo.rho1 / (Real)3;
        p[2] = mo.s[2] - rho * u[2] * u[2] - mo.rho1 / (Real)3;
        p[3] = mo.s[3] - rho * u[0] * u[1];
        p[4] = mo.s[4] - rho * u[0] * u[2];
        p[5] = mo.s[5] - rho * u[1] * u[2];
    }
    static void deviator(const Real *p, Real *d) {  // mshader.rs:496-501
        for (int k = 0; k < 6; k++) d[k] = p[k];
        const Real tr = (p[0] + p[1] + p[2]) / (Real)3;
        d[0] -= tr; d[1] -= tr; d[2] -= tr;
    }
    F rebuild(Real rho, const Real *u, const Real *pp) const {  // mshader.rs:503-509
        const F fe = feq(rho, u);
        Real d[6];
        deviator(pp, d);
        const F fn = fneq(d);
        F f;
        for (int i = 0; i < 27; i++) f[i] = fe[i] + fn[i];
        return f;
    }
    // mshader.rs:286-362: populations of a Gaussian with covariance sg and first
    // central moments m1 (all higher cumulants zero), via backward central-moment
    // transforms along z, then y, then x
    F gauss(Real rho, const Real *u, const Real *sg, const Real *m1) const {
        const Real a = sg[0], b = sg[1], cc = sg[2], d = sg[3], e = sg[4], g = sg[5];
        const Real two = 2, eight = 8, h = (Real)0.5;
        Real K[3][3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++) {
                    Real m = 0;
                    const int key = i * 100 + j * 10 + k;
                    switch (key) {
                        case 0: m = 1; break;
                        case 100: m = m1[0]; break;
                        case 10: m = m1[1]; break;
                        case 1: m = m1[2]; break;
                        case 200: m = a; break;
                        case 20: m = b; break;
                        case 2: m = cc; break;
                        case 110: m = d; break;
                        case 101: m = e; break;
                        case 11: m = g; break;
                        case 220: m = a * b + two * d * d; break;
                        case 202: m = a * cc + two * e * e; break;
                        case 22: m = b * cc + two * g * g; break;
                        case 211: m = a * g + two * d * e; break;
                        case 121: m = b * e + two * d * g; break;
                        case 112: m = cc * d + two * e * g; break;
                        case 222: m = a * b * cc + two * (a * g * g + b * e * e + cc * d * d) + eight * d * e * g; break;
                        default: m = 0; break;
                    }
                    K[i][j][k] = rho * m;
                }
        auto back = [&](Real k0, Real k1, Real k2, Real w, Real *out) {
            const Real r1 = k1 + w * k0;
            const Real r2 = k2 + two * w * k1 + w * w * k0;
            out[0] = h * (r2 - r1);
            out[1] = k0 - r2;
            out[2] = h * (r2 + r1);
        };
        Real Z[3][3][3], Y[3][3][3], X[3][3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) back(K[i][j][0], K[i][j][1], K[i][j][2], u[2], Z[i][j]);
        for (int i = 0; i < 3; i++)
            for (int c = 0; c < 3; c++) {
                Real o[3];
                back(Z[i][0][c], Z[i][1][c], Z[i][2][c], u[1], o);
                for (int t = 0; t < 3; t++) Y[i][c][t] = o[t];  // Y[i][cz][cy]
            }
        for (int cyi = 0; cyi < 3; cyi++)
            for (int czi = 0; czi < 3; czi++) back(Y[0][czi][cyi], Y[1][czi][cyi], Y[2][czi][cyi], u[0], X[cyi][czi]);
        F f;
        for (int i = 0; i < 27; i++) f[i] = X[q27::cy(i) + 1][q27::cz(i) + 1][q27::cx(i) + 1] - W[i];
        return f;
    }
    // mshader.rs:480-490
    Real sponge(const Level &l, uint32_t x, uint32_t y, uint32_t z) const {
        const Real p[3] = {(Real)(float)x, (Real)(float)y, (Real)(float)z};
        const Real hi[3] = {(Real)(float)(l.NX - 1) - p[0], (Real)(float)(l.NY - 1) - p[1], (Real)(float)(l.NZ - 1) - p[2]};
        Real s = 0;
        for (int k = 0; k < 3; k++) {
            if (l.SP_LO[k] > 0) s = std::max(s, (Real)1 - p[k] / l.SP_LO[k]);
            if (l.SP_HI[k] > 0) s = std::max(s, (Real)1 - hi[k] / l.SP_HI[k]);
        }
        return std::min(std::max(s, (Real)0), (Real)1);
    }

    // ------------------------------------------------------------ setup
    // mlattice.rs:195-548 (host side of MultiLattice::new)
    void create(const Set &s, const lbm_geometry *geom, const lbm_probes *probes = nullptr) {
        storage = s.storage;
        ABS_U = s.absorb_velocity != 0;
        TOTAL_P = s.total_pressure_inlet != 0;
        for (int i = 0; i < 27; i++) {
            W[i] = (Real)(float)q27::weight(i);
            W45[i] = (Real)(float)(4.5 * q27::weight(i));
            if (sizeof(Real) == 8) { W[i] = (Real)q27::weight(i); W45[i] = (Real)(4.5 * q27::weight(i)); }
        }
        const size_t nl = (size_t)s.nboxes + 1;
        const size_t finest = nl - 1;
        const bool periodic0[3] = {s.faces[0] == LBM_FACE_PERIODIC, s.faces[2] == LBM_FACE_PERIODIC, s.faces[4] == LBM_FACE_PERIODIC};
        auto dims = [&](size_t l) -> std::array<uint32_t, 3> {
            if (l == 0) return {s.dims0[0], s.dims0[1], s.dims0[2]};
            const lbm_level_box &b = s.boxes[l - 1];
            return {2 * (b.n[0] - 1) + 1, 2 * (b.n[1] - 1) + 1, 2 * (b.n[2] - 1) + 1};
        };
        if (nl > 1 && (periodic0[0] || periodic0[1] || periodic0[2])) throw std::runtime_error("periodic faces only work without refinement");
        for (size_t l = 1; l < nl; l++) {
            const lbm_level_box &b = s.boxes[l - 1];
            const auto pd = dims(l - 1);
            for (int k = 0; k < 3; k++) {
                const int64_t hi = (int64_t)b.lo[k] + (int64_t)b.n[k] - 1;
                const int margin = l == 1 ? 2 : 3;
                if (b.lo[k] < margin || hi > (int64_t)pd[k] - 1 - margin || b.n[k] < 8)
                    throw std::runtime_error("refinement box " + std::to_string(l) + " does not fit inside its parent");
            }
        }
        // origins and scales of the levels in finest-level node coordinates
        std::vector<std::array<double, 3>> org(nl, {0, 0, 0});
        std::vector<double> scale(nl, 1.0);
        scale[0] = (double)(1ull << finest);
        for (size_t l = 1; l < nl; l++) {
            scale[l] = scale[l - 1] / 2.0;
            for (int k = 0; k < 3; k++) org[l][k] = org[l - 1][k] + s.boxes[l - 1].lo[k] * scale[l - 1];
        }
        // probes (mlattice.rs:243-305): a slice pixel belongs to the finest
        // level whose interior without the ghost layer (x in [1, d-2] on the
        // coarsest level, [2, d-3] on the others) holds its nearest node
        pix.assign(nl, {});
        if (probes) {
            for (uint64_t v = 0; v < probes->nvert; v++) {
                const double *q = probes->verts + 6 * v;
                pverts.push_back({(float)q[0], (float)q[1], (float)q[2], 0.f, (float)q[3], (float)q[4], (float)q[5], 0.f});
            }
            VOFF = (float)probes->vertex_offset;
            uint32_t base = 0;
            for (uint64_t sl = 0; sl < probes->nslices; sl++) {
                const lbm_slice_def &d = probes->slices[sl];
                for (uint32_t iv = 0; iv < d.nv; iv++)
                    for (uint32_t iu = 0; iu < d.nu; iu++) {
                        const double p[3] = {(double)(d.origin[0] + (int32_t)iu * d.u[0] + (int32_t)iv * d.v[0]),
                                             (double)(d.origin[1] + (int32_t)iu * d.u[1] + (int32_t)iv * d.v[1]),
                                             (double)(d.origin[2] + (int32_t)iu * d.u[2] + (int32_t)iv * d.v[2])};
                        for (size_t l = nl; l-- > 0;) {
                            const auto dl = dims(l);
                            const double lo = l == 0 ? 1.0 : 2.0;
                            bool ok = true;
                            uint32_t cell[3] = {0, 0, 0};
                            for (int k = 0; k < 3; k++) {
                                const double x = std::round((p[k] - org[l][k]) / scale[l]);
                                if (x < lo || x > (double)dl[k] - 1.0 - lo) { ok = false; break; }
                                cell[k] = (uint32_t)x;
                            }
                            if (ok) {
                                pix[l].push_back({base + iv * d.nu + iu, (cell[2] * dl[1] + cell[1]) * dl[0] + cell[0]});
                                break;
                            }
                        }
                    }
                base += d.nu * d.nv;
            }
            npix = base;
        }
        vacc.assign(2 * pverts.size(), 0.0);
        sacc.assign(5 * (size_t)npix, 0.0);
        // records (mlattice.rs:178-192, 345-354); a spinning part makes every
        // swept-box cell of the finest level a record without links
        std::vector<std::pair<uint32_t, uint32_t>> rec_of;
        std::vector<uint32_t> solid;
        std::vector<lbm_wall_cell> boxwalls;
        lbm_geometry boxgeom{};
        for (int k = 0; k < 3; k++) CENTERF[k] = (float)s.center[k];
        if (geom && geom->kind == 2) {
            const auto fd = dims(finest);
            moving = true;
            for (int k = 0; k < 3; k++) {
                box_lo[k] = geom->box_lo[k];
                box_n[k] = geom->box_n[k];
                occ_lo[k] = (float)geom->occ_lo[k];
                occ_n[k] = (int32_t)geom->occ_dims[k];
                if (box_lo[k] < 1 || (int64_t)box_lo[k] + box_n[k] > (int64_t)fd[k] - 1)
                    throw std::runtime_error("the spinning part's swept box leaves the finest level");
            }
            occ_invh = (float)(1.0 / geom->occ_h);
            const uint64_t nocc = (uint64_t)occ_n[0] * occ_n[1] * occ_n[2];
            occ.assign(geom->occ_bits, geom->occ_bits + (nocc + 31) / 32);
            tris.resize(geom->ntri);
            for (uint64_t t = 0; t < geom->ntri; t++)
                for (int j = 0; j < 12; j++) tris[t][j] = geom->tris[12 * t + j];
            const uint64_t nb = (uint64_t)box_n[0] * box_n[1] * box_n[2];
            boxwalls.resize(nb);
            uint64_t k = 0;
            for (uint32_t z = 0; z < box_n[2]; z++)
                for (uint32_t y = 0; y < box_n[1]; y++)
                    for (uint32_t x = 0; x < box_n[0]; x++, k++) {
                        boxwalls[k].cell = (uint32_t)((((uint64_t)z + box_lo[2]) * fd[1] + y + box_lo[1]) * fd[0] + x + box_lo[0]);
                        boxwalls[k].mask = 0;
                        for (int i = 0; i < 27; i++) boxwalls[k].q[i] = 1.0f;
                    }
            boxgeom.kind = 1;
            boxgeom.walls = boxwalls.data();
            boxgeom.nwalls = nb;
            geom = &boxgeom;
            qscr.assign(nb * 39, 0u);
            for (size_t j = 0; j < qscr.size(); j += 3) qscr[j] = 0x7f7fffffu;
        }
        if (geom && geom->kind == 1) {
            nrec = (uint32_t)geom->nwalls;
            rec_words.assign((size_t)nrec * q27::RS, 0u);
            rec_q.assign((size_t)nrec * 26, (Real)1);
            rec_ft.assign((size_t)nrec * 6, (Real)0);
            for (uint32_t r = 0; r < nrec; r++) {
                const lbm_wall_cell &w = geom->walls[r];
                uint32_t *wd = &rec_words[(size_t)r * q27::RS];
                wd[q27::R_MASK] = w.mask;
                wd[q27::R_CELL] = w.cell;
                float qs[26];
                for (int k = 0; k < 26; k++) qs[k] = 1.0f;
                for (int i = 0; i < 27; i++)
                    if (i != q27::REST) qs[q27::slot(i)] = w.q[i];
                for (int k = 0; k < 13; k++) {
                    const uint16_t lo = f16_bits_ref(qs[2 * k]), hi = f16_bits_ref(qs[2 * k + 1]);
                    wd[q27::R_Q + k] = (uint32_t)lo | ((uint32_t)hi << 16);
                    rec_q[(size_t)r * 26 + 2 * k] = (Real)f16_to_f32(lo);
                    rec_q[(size_t)r * 26 + 2 * k + 1] = (Real)f16_to_f32(hi);
                }
                rec_of.push_back({w.cell, r + 1});
            }
            solid.assign(geom->solid, geom->solid + geom->nsolid);
        }
        std::sort(rec_of.begin(), rec_of.end());
        std::sort(solid.begin(), solid.end());

        lv.assign(nl, Level());
        for (size_t l = 0; l < nl; l++) {
            Level &L_ = lv[l];
            const auto d = dims(l);
            L_.NX = d[0]; L_.NY = d[1]; L_.NZ = d[2];
            L_.N = (uint64_t)d[0] * d[1] * d[2];
            if (L_.N >= 0xffffffffull) throw std::runtime_error("level " + std::to_string(l) + " has too many cells");
            L_.finest = l == finest;
            for (int k = 0; k < 3; k++) L_.per[k] = l == 0 ? periodic0[k] : false;
            L_.has_child = l + 1 < nl;
            L_.has_parent = l > 0;
            if (L_.has_child) {
                for (int k = 0; k < 3; k++) { L_.ch_lo[k] = s.boxes[l].lo[k]; L_.ch_n[k] = s.boxes[l].n[k]; }
                L_.ch_nodes = (uint64_t)L_.ch_n[0] * L_.ch_n[1] * L_.ch_n[2];
            }
            for (int k = 0; k < 3; k++) L_.pn[k] = (d[k] - 1) / 2 + 1;
            L_.pnodes = l > 0 ? (uint64_t)L_.pn[0] * L_.pn[1] * L_.pn[2] : 0;
            const double tau_l = 0.5 + 3.0 * s.nu0 * (double)(1ull << l);
            auto R = [](double v) { return sizeof(Real) == 8 ? (Real)v : (Real)(float)v; };
            L_.TAU0 = R(tau_l);
            L_.SMAG2 = R(s.smagorinsky * s.smagorinsky);
            const double sp[6] = {l == 0 ? (double)s.sponge[0] : 0.0, l == 0 ? (double)s.sponge[1] : 0.0, l == 0 ? (double)s.sponge[2] : 0.0,
                                  l == 0 ? (double)s.sponge[3] : 0.0, l == 0 ? (double)s.sponge[4] : 0.0, l == 0 ? (double)s.sponge[5] : 0.0};
            for (int k = 0; k < 3; k++) { L_.SP_LO[k] = R(sp[2 * k]); L_.SP_HI[k] = R(sp[2 * k + 1]); }
            L_.N_SPONGE = false;
            for (int k = 0; k < 6; k++) L_.N_SPONGE = L_.N_SPONGE || sp[k] > 0;
            L_.SPONGE_TAU = R(l == 0 ? s.sponge_tau : 0.0);
            L_.SIGMA = R(l == 0 ? s.sponge_sigma : 0.0);
            const double sc_l = (double)(1ull << (finest - l));
            for (int k = 0; k < 3; k++) {
                L_.U_INF[k] = R(s.u_inf[k]);
                L_.U_INIT[k] = R(s.u_init[k]);
                L_.GRAV[k] = R(s.body_force0[k] / (double)(1ull << l));
                L_.CENTER[k] = R(l == finest ? s.center[k] : (s.center[k] - org[l][k]) / sc_l);
            }
            L_.forcing = s.body_force0[0] != 0.0 || s.body_force0[1] != 0.0 || s.body_force0[2] != 0.0;
            // cell types and lists (mlattice.rs:404-478)
            const uint32_t nx = d[0], ny = d[1], nz = d[2];
            L_.flags.assign(L_.N, 0u);
            size_t fi = 0, si = 0;
            for (uint64_t cc = 0; cc < L_.N; cc++) {
                const uint32_t x = (uint32_t)(cc % nx), y = (uint32_t)((cc / nx) % ny), z = (uint32_t)(cc / ((uint64_t)nx * ny));
                int ty = 0;  // face type, 0 = none
                if (l == 0) {
                    const bool on[6] = {x == 0, x == nx - 1, y == 0, y == ny - 1, z == 0, z == nz - 1};
                    for (int f = 0; f < 6; f++)
                        if (on[f] && s.faces[f] != LBM_FACE_PERIODIC) {
                            const int t = s.faces[f] == LBM_FACE_VELOCITY ? 1 : 2;
                            ty = ty == 1 ? 1 : t;
                        }
                }
                const bool ghost = l > 0 && (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1);
                bool restr = false;
                if (L_.has_child) {
                    const int p[3] = {(int)x, (int)y, (int)z};
                    restr = true;
                    for (int k = 0; k < 3; k++) restr = restr && p[k] >= L_.ch_lo[k] + 2 && p[k] <= L_.ch_lo[k] + (int)L_.ch_n[k] - 3;
                }
                uint32_t v = 0;
                if (ty) { v = q27::T_FACE | ((uint32_t)ty << 3); L_.faces.push_back((uint32_t)cc); }
                else if (ghost) { v = q27::T_GHOST; L_.ghosts.push_back((uint32_t)cc); }
                else if (restr) { v = q27::T_RESTRICT; L_.restricted.push_back((uint32_t)cc); }
                if (L_.finest) {
                    while (si < solid.size() && solid[si] < cc) si++;
                    while (si < solid.size() && solid[si] == cc) { if (v == 0) v = q27::T_SOLID; si++; }
                    while (fi < rec_of.size() && rec_of[fi].first < cc) fi++;
                    while (fi < rec_of.size() && rec_of[fi].first == cc) {
                        if ((v & 7u) == 0 || (v & 7u) == q27::T_SOLID) v = (v & 7u) | (rec_of[fi].second << 3);
                        fi++;
                    }
                }
                L_.flags[cc] = v;
            }
            // initial moments: rest at the initial velocity (mlattice.rs:484-501)
            auto init_m = [&](std::vector<Real> &m, uint64_t nodes) {
                m.assign(nodes * q27::MW, (Real)0);
                for (uint64_t k = 0; k < nodes; k++) {
                    Real *c = &m[k * q27::MW];
                    c[0] = 1;
                    c[1] = L_.U_INIT[0]; c[2] = L_.U_INIT[1]; c[3] = L_.U_INIT[2];
                    c[10] = R(tau_l);
                }
            };
            init_m(L_.mom_child, L_.has_child ? 2 * L_.ch_nodes : 0);
            init_m(L_.mom_up, L_.pnodes);
            for (int set = 0; set < 2; set++) {
                if (storage == LBM_STORAGE_FP32) L_.p32[set].assign(27 * L_.N, 0.f);
                else if (storage == LBM_STORAGE_FP64) L_.p64[set].assign(27 * L_.N, 0.0);
                else L_.p16[set].assign(27 * L_.N, 0);
            }
        }
        // initial state: feq(1, u_init) in both sets (mshader.rs:520-527), seed 0
        for (size_t l = 0; l < nl; l++) {
            Level &L_ = lv[l];
            const F f = feq((Real)1, L_.U_INIT);
            for (uint64_t n = 0; n < L_.N; n++) { put(L_, 0, n, f, 0u); put(L_, 1, n, f, 0u); }
            L_.src = 0;
            L_.mslot = 1;
        }
    }

    size_t levels() const { return lv.size(); }
    size_t sub_steps() const { return (size_t)1 << (lv.size() - 1); }

    // mlattice.rs:692-703
    uint32_t seed_of(uint32_t hslot, uint32_t src, uint32_t mw) const {
        return ((uint32_t)fine_steps + hslot) * STEP_SEED_MUL + (src * q27::SEED_SRC_MUL + mw * q27::SEED_MW_MUL);
    }

    // ------------------------------------------------------------ kernels
    // mshader.rs:702-733
    void face_bc(Level &l, const Par &st) {
#pragma omp parallel for schedule(static)
        for (size_t fi = 0; fi < l.faces.size(); fi++) {
            const uint32_t b = l.faces[fi];
            uint32_t x, y, z;
            coords(l, b, x, y, z);
            if (!l.per[0]) x = std::min(std::max(x, 1u), l.NX - 2);
            if (!l.per[1]) y = std::min(std::max(y, 1u), l.NY - 2);
            if (!l.per[2]) z = std::min(std::max(z, 1u), l.NZ - 2);
            const uint64_t m = cidx(l, x, y, z);
            Real rho = 1, u[3] = {l.U_INF[0], l.U_INF[1], l.U_INF[2]}, pp[6] = {0, 0, 0, 0, 0, 0};
            if ((l.flags[m] & 7u) == 0) {
                const Mom mo = moments(own(l, st.src, m));
                rho = (Real)1 + mo.rho1;
                for (int k = 0; k < 3; k++) u[k] = mo.j[k] / rho;
                stress(mo, rho, u, pp);
            }
            const uint32_t ty = (l.flags[b] >> 3) & 3u;
            if (ty == 1) {
                if (TOTAL_P) {
                    const Real third = (Real)1 / (Real)3, h = (Real)0.5;
                    const Real uinf2 = l.U_INF[0] * l.U_INF[0] + l.U_INF[1] * l.U_INF[1] + l.U_INF[2] * l.U_INF[2];
                    const Real u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
                    rho = (third + h * uinf2) / (third + h * u2);
                } else {
                    for (int k = 0; k < 3; k++) u[k] = l.U_INF[k];
                }
            } else {
                rho = 1;
            }
            put(l, st.src, b, rebuild(rho, u, pp), st.seed);
        }
    }

    // mshader.rs:612-699 plus the walls of mshader.rs:364-403
    void step(size_t li, const Par &st) {
        Level &l = lv[li];
        const uint32_t dst = 1u - st.src;
#pragma omp parallel for schedule(static)
        for (uint64_t n = 0; n < l.N; n++) {
            const uint32_t fg = l.flags[n];
            if ((fg & 7u) != 0) continue;
            uint32_t x, y, z;
            coords(l, n, x, y, z);
            F f = pull(l, st.src, n);
            const uint32_t rec = fg >> 3;
            Real Fv[3] = {0, 0, 0}, Tv[3] = {0, 0, 0};
            if (rec != 0) {
                const uint32_t r = rec - 1;
                const uint32_t mask = rec_words[(size_t)r * q27::RS + q27::R_MASK];
                const F fin = f;
                const Real pc[3] = {(Real)(float)x - l.CENTER[0], (Real)(float)y - l.CENTER[1], (Real)(float)z - l.CENTER[2]};
                for (int i = 0; i < 27; i++) {
                    if (i == q27::REST || !(mask & (1u << i))) continue;
                    const int o = q27::opp(i);
                    const Real q = std::max(rec_q[(size_t)r * 26 + q27::slot(i)], (Real)0.001f);
                    const Real fpi = L(l, st.src, i, n) + W[i];
                    const Real fpo = L(l, st.src, o, n) + W[i];
                    const Real ci[3] = {(Real)q27::cx(i), (Real)q27::cy(i), (Real)q27::cz(i)};
                    const Real xw[3] = {pc[0] + q * ci[0], pc[1] + q * ci[1], pc[2] + q * ci[2]};
                    const Real uw[3] = {st.omega[1] * xw[2] - st.omega[2] * xw[1], st.omega[2] * xw[0] - st.omega[0] * xw[2],
                                        st.omega[0] * xw[1] - st.omega[1] * xw[0]};
                    const Real cu = ci[0] * uw[0] + ci[1] * uw[1] + ci[2] * uw[2];
                    const Real w6 = (Real)6 * W[i];
                    Real fb;
                    if (q >= (Real)0.5) fb = (fpi + ((Real)2 * q - (Real)1) * fpo - w6 * cu) / ((Real)2 * q);
                    else if (!(mask & (1u << o))) fb = (Real)2 * q * fpi + ((Real)1 - (Real)2 * q) * (fin[i] + W[i]) - w6 * cu;
                    else fb = fpi - w6 * cu;
                    f[o] = fb - W[i];
                    Real flk[3];
                    for (int k = 0; k < 3; k++) flk[k] = (ci[k] - uw[k]) * fpi + (ci[k] + uw[k]) * fb;
                    for (int k = 0; k < 3; k++) Fv[k] += flk[k];
                    Tv[0] += xw[1] * flk[2] - xw[2] * flk[1];
                    Tv[1] += xw[2] * flk[0] - xw[0] * flk[2];
                    Tv[2] += xw[0] * flk[1] - xw[1] * flk[0];
                }
            }
            const Mom mo = moments(f);
            const Real rho = (Real)1 + mo.rho1;
            Real G[3], u[3];
            for (int k = 0; k < 3; k++) G[k] = rho * l.GRAV[k];
            for (int k = 0; k < 3; k++) u[k] = (mo.j[k] + (Real)0.5 * G[k]) / rho;
            Real p[6];
            stress(mo, rho, u, p);
            Real tau = l.TAU0;
            if (l.SMAG2 > 0) {
                Real dv[6];
                deviator(p, dv);
                const Real pp = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2] + (Real)2 * (dv[3] * dv[3] + dv[4] * dv[4] + dv[5] * dv[5]);
                tau = (Real)0.5 * (l.TAU0 + std::sqrt(l.TAU0 * l.TAU0 + (Real)18 * l.SMAG2 * std::sqrt((Real)2 * pp) / rho));
            }
            Real sp = 0;
            if (l.N_SPONGE) {
                sp = sponge(l, x, y, z);
                if (sp > 0 && l.SPONGE_TAU > tau) tau += sp * sp * (l.SPONGE_TAU - tau);
            }
            const Real om = (Real)1 / tau;
            Real dv[6], sg[6];
            deviator(p, dv);
            const Real third = (Real)1 / (Real)3;
            for (int k = 0; k < 3; k++) sg[k] = third + ((Real)1 - om) * dv[k] / rho;
            for (int k = 3; k < 6; k++) sg[k] = ((Real)1 - om) * dv[k] / rho;
            Real m1[3] = {0, 0, 0};
            if (l.forcing)
                for (int k = 0; k < 3; k++) m1[k] = (Real)0.5 * G[k] / rho;
            F fo = gauss(rho, u, sg, m1);
            if (l.N_SPONGE && l.SIGMA > 0 && sp > 0) {
                const Real *ut = ABS_U ? l.U_INF : u;
                const F ft = feq((Real)1, ut);
                const F fc = feq(rho, u);
                const Real sgm = l.SIGMA * sp * sp;
                for (int i = 0; i < 27; i++) fo[i] += sgm * (ft[i] - fc[i]);
            }
            if (rec != 0) {
                const uint32_t r = rec - 1;
                if (moving)
                    for (int k = 0; k < 3; k++) { Fv[k] += rec_ft[(size_t)r * 6 + k]; Tv[k] += rec_ft[(size_t)r * 6 + 3 + k]; }
                for (int k = 0; k < 3; k++) { rec_ft[(size_t)r * 6 + k] = Fv[k]; rec_ft[(size_t)r * 6 + 3 + k] = Tv[k]; }
                for (int k = 0; k < 6; k++) rec_words[(size_t)r * q27::RS + q27::R_FT + k] = fbits((float)rec_ft[(size_t)r * 6 + k]);
            }
            put(l, dst, n, fo, st.seed);
            auto exportm = [&](Real *o) {
                o[0] = rho; o[1] = u[0]; o[2] = u[1]; o[3] = u[2];
                for (int k = 0; k < 6; k++) o[4 + k] = p[k];
                o[10] = tau;
            };
            if (l.has_child) {
                const int lx = (int)x - l.ch_lo[0], ly = (int)y - l.ch_lo[1], lz = (int)z - l.ch_lo[2];
                if (lx >= 0 && ly >= 0 && lz >= 0 && lx < (int)l.ch_n[0] && ly < (int)l.ch_n[1] && lz < (int)l.ch_n[2]) {
                    const bool surf = lx == 0 || ly == 0 || lz == 0 || lx == (int)l.ch_n[0] - 1 || ly == (int)l.ch_n[1] - 1 || lz == (int)l.ch_n[2] - 1;
                    if (surf) exportm(&l.mom_child[(st.mw * l.ch_nodes + ((uint64_t)lz * l.ch_n[1] + ly) * l.ch_n[0] + lx) * q27::MW]);
                }
            }
            if (l.has_parent && (x & 1u) == 0 && (y & 1u) == 0 && (z & 1u) == 0)
                exportm(&l.mom_up[(((uint64_t)(z / 2) * l.pn[1] + y / 2) * l.pn[0] + x / 2) * q27::MW]);
        }
    }

    // mshader.rs:742-775
    void ghost_fill(size_t ci, const Par &st) {
        Level &c = lv[ci];
        const Level &p = lv[ci - 1];
#pragma omp parallel for schedule(static)
        for (size_t gi = 0; gi < c.ghosts.size(); gi++) {
            const uint32_t n = c.ghosts[gi];
            uint32_t xyz[3];
            coords(c, n, xyz[0], xyz[1], xyz[2]);
            const uint32_t h0[3] = {xyz[0] / 2, xyz[1] / 2, xyz[2] / 2};
            const uint32_t odd[3] = {xyz[0] & 1u, xyz[1] & 1u, xyz[2] & 1u};
            Real acc[11];
            for (int j = 0; j < 11; j++) acc[j] = 0;
            Real wsum = 0;
            for (uint32_t k = 0; k < 8; k++) {
                const uint32_t o[3] = {k & 1u, (k >> 1) & 1u, (k >> 2) & 1u};
                if ((o[0] == 1 && odd[0] == 0) || (o[1] == 1 && odd[1] == 0) || (o[2] == 1 && odd[2] == 0)) continue;
                const uint32_t node[3] = {h0[0] + o[0], h0[1] + o[1], h0[2] + o[2]};
                const Real w = (odd[0] == 1 ? (Real)0.5 : (Real)1) * (odd[1] == 1 ? (Real)0.5 : (Real)1) * (odd[2] == 1 ? (Real)0.5 : (Real)1);
                const uint64_t nd = ((uint64_t)node[2] * c.pn[1] + node[1]) * c.pn[0] + node[0];
                const Real *a = &p.mom_child[(st.mold * p.ch_nodes + nd) * q27::MW];
                const Real *b = &p.mom_child[(st.mnew * p.ch_nodes + nd) * q27::MW];
                for (int j = 0; j < 11; j++) acc[j] += w * (((Real)1 - st.blend) * a[j] + st.blend * b[j]);
                wsum += w;
            }
            const Real rho = acc[0] / wsum;
            const Real u[3] = {acc[1] / wsum, acc[2] / wsum, acc[3] / wsum};
            const Real tc = acc[10] / wsum;
            const Real tf = (Real)0.5 + (Real)2 * (tc - (Real)0.5);
            const Real sc = tf / ((Real)2 * tc) * ((Real)1 - (Real)1 / tf);
            Real pp[6];
            for (int j = 0; j < 6; j++) pp[j] = acc[4 + j] / wsum * sc;
            put(c, st.src, n, rebuild(rho, u, pp), st.seed);
        }
    }

    // mshader.rs:777-793
    void restrict_fill(size_t li, const Par &st) {
        Level &l = lv[li];
        const Level &c = lv[li + 1];
#pragma omp parallel for schedule(static)
        for (size_t ri = 0; ri < l.restricted.size(); ri++) {
            const uint32_t n = l.restricted[ri];
            uint32_t x, y, z;
            coords(l, n, x, y, z);
            const uint32_t lx = (uint32_t)((int)x - l.ch_lo[0]), ly = (uint32_t)((int)y - l.ch_lo[1]), lz = (uint32_t)((int)z - l.ch_lo[2]);
            const Real *m = &c.mom_up[(((uint64_t)lz * l.ch_n[1] + ly) * l.ch_n[0] + lx) * q27::MW];
            const Real rho = m[0];
            const Real u[3] = {m[1], m[2], m[3]};
            const Real tf = m[10];
            const Real tc = (Real)0.5 + (Real)0.5 * (tf - (Real)0.5);
            const Real sc = (Real)2 * tc / tf * ((Real)1 - (Real)1 / tc);
            Real pp[6];
            for (int j = 0; j < 6; j++) pp[j] = m[4 + j] * sc;
            put(l, st.src, n, rebuild(rho, u, pp), st.seed);
        }
    }

    // ------------------------------------------------------------ spinning part
    // f32 geometry, one rounding per operation (compiled without contraction)
    struct V3f { float x, y, z; };
    static float dotf(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    static V3f crossf(V3f a, V3f b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
    static V3f colf(const float *r, int k) { return {r[k], r[3 + k], r[6 + k]}; }
    static V3f to_body(const float *r, V3f v) { return {dotf(colf(r, 0), v), dotf(colf(r, 1), v), dotf(colf(r, 2), v)}; }
    static V3f from_body(const float *r, V3f b) {
        const V3f c0 = colf(r, 0), c1 = colf(r, 1), c2 = colf(r, 2);
        return {c0.x * b.x + c1.x * b.y + c2.x * b.z, c0.y * b.x + c1.y * b.y + c2.y * b.z, c0.z * b.x + c1.z * b.y + c2.z * b.z};
    }
    bool solid_at(const float *rot, int x, int y, int z) const {
        const V3f b = to_body(rot, {(float)x - CENTERF[0], (float)y - CENTERF[1], (float)z - CENTERF[2]});
        const float gx = std::nearbyint((b.x - occ_lo[0]) * occ_invh), gy = std::nearbyint((b.y - occ_lo[1]) * occ_invh),
                    gz = std::nearbyint((b.z - occ_lo[2]) * occ_invh);
        if (!(gx >= 0.f && gy >= 0.f && gz >= 0.f) || gx >= (float)occ_n[0] || gy >= (float)occ_n[1] || gz >= (float)occ_n[2]) return false;
        const uint64_t li = ((uint64_t)gz * (uint64_t)occ_n[1] + (uint64_t)gy) * (uint64_t)occ_n[0] + (uint64_t)gx;
        return ((occ[li >> 5] >> (li & 31u)) & 1u) != 0u;
    }
    static float ray_tri(V3f o, V3f d, V3f v0, V3f e1, V3f e2) {
        const V3f pv = crossf(d, e2);
        const float det = dotf(e1, pv);
        if (std::fabs(det) < 1e-12f) return 9.0f;
        const float inv = 1.0f / det;
        const V3f tv = {o.x - v0.x, o.y - v0.y, o.z - v0.z};
        const float a = dotf(tv, pv) * inv;
        if (a < 0.0f || a > 1.0f) return 9.0f;
        const V3f qv = crossf(tv, e1);
        const float b = dotf(d, qv) * inv;
        if (b < 0.0f || a + b > 1.0f) return 9.0f;
        const float t = dotf(e2, qv) * inv;
        if (t < -1e-4f || t > 1.0f) return 9.0f;
        return t > 0.0f ? t : 0.0f;
    }
    bool in_box(int lx, int ly, int lz) const {
        return lx >= 0 && ly >= 0 && lz >= 0 && lx < (int)box_n[0] && ly < (int)box_n[1] && lz < (int)box_n[2];
    }
    void revoxel(Level &l, const Par &st) {
        // links: triangles rotated to this step's angle against the links around them
        const float REACH = 1.733f;
        for (const auto &tr : tris) {
            const V3f v0 = from_body(st.rot, {tr[0], tr[1], tr[2]});
            const V3f a = {CENTERF[0] + v0.x, CENTERF[1] + v0.y, CENTERF[2] + v0.z};
            const V3f e1 = from_body(st.rot, {tr[4], tr[5], tr[6]}), e2 = from_body(st.rot, {tr[8], tr[9], tr[10]});
            const V3f nrm = crossf(e1, e2);
            const float nl = std::sqrt(dotf(nrm, nrm));
            if (nl < 1e-12f) continue;
            const V3f nn = {nrm.x / nl, nrm.y / nl, nrm.z / nl};
            const V3f b = {a.x + e1.x, a.y + e1.y, a.z + e1.z}, c = {a.x + e2.x, a.y + e2.y, a.z + e2.z};
            const float mn[3] = {std::min(std::min(a.x, b.x), c.x), std::min(std::min(a.y, b.y), c.y), std::min(std::min(a.z, b.z), c.z)};
            const float mx[3] = {std::max(std::max(a.x, b.x), c.x), std::max(std::max(a.y, b.y), c.y), std::max(std::max(a.z, b.z), c.z)};
            int lo[3], hi[3];
            for (int k = 0; k < 3; k++) {
                lo[k] = std::max((int)std::ceil(mn[k] - REACH), box_lo[k]);
                hi[k] = std::min((int)std::floor(mx[k] + REACH), box_lo[k] + (int)box_n[k] - 1);
            }
            for (int z = lo[2]; z <= hi[2]; z++)
                for (int y = lo[1]; y <= hi[1]; y++)
                    for (int x = lo[0]; x <= hi[0]; x++) {
                        const V3f pt = {(float)x, (float)y, (float)z};
                        const float d0 = dotf(nn, {pt.x - a.x, pt.y - a.y, pt.z - a.z});
                        if (std::fabs(d0) > REACH) continue;
                        const uint32_t k = ((uint32_t)(z - box_lo[2]) * box_n[1] + (uint32_t)(y - box_lo[1])) * box_n[0] + (uint32_t)(x - box_lo[0]);
                        for (int i = 14; i < 27; i++) {
                            const V3f cv = {(float)q27::cx(i), (float)q27::cy(i), (float)q27::cz(i)};
                            const float d1 = d0 + dotf(nn, cv);
                            if (d0 * d1 > 0.0f && std::fabs(d0) > 1e-6f) continue;
                            const float tt = ray_tri(pt, cv, a, e1, e2);
                            if (tt <= 1.0f) {
                                const uint64_t o = ((uint64_t)k * 13u + (uint32_t)(i - 14)) * 3u;
                                const uint32_t tb = fbits(tt > 0.0f ? tt : 0.0f);
                                qscr[o] = std::min(qscr[o], tb);
                                qscr[o + 1] = std::max(qscr[o + 1], tb);
                                qscr[o + 2] += 1u;
                            }
                        }
                    }
        }
        // cells: solid or fluid, links and q, refill, cover / uncover momentum
        for (uint32_t k = 0; k < nrec; k++) {
            const int lx = (int)(k % box_n[0]), ly = (int)((k / box_n[0]) % box_n[1]), lz = (int)(k / (box_n[0] * box_n[1]));
            const int px = lx + box_lo[0], py = ly + box_lo[1], pz = lz + box_lo[2];
            const uint64_t n = cidx(l, (uint32_t)px, (uint32_t)py, (uint32_t)pz);
            uint32_t *w = &rec_words[(size_t)k * q27::RS];
            const Real pc[3] = {(Real)px - l.CENTER[0], (Real)py - l.CENTER[1], (Real)pz - l.CENTER[2]};
            const bool solid_now = solid_at(st.rot, px, py, pz), solid_before = solid_at(st.rot_prev, px, py, pz);
            Real Fv[3] = {0, 0, 0};
            if (solid_now) {
                l.flags[n] = q27::T_SOLID | ((k + 1u) << 3);
                w[q27::R_MASK] = 0;
                if (!solid_before) {
                    const Mom mo = moments(own(l, st.src, n));
                    for (int c = 0; c < 3; c++) Fv[c] = mo.j[c];
                }
            } else {
                float qv[27], qx[27];
                uint32_t nh[27];
                for (int i = 0; i < 27; i++) {
                    qv[i] = 9.0f; qx[i] = -1.0f; nh[i] = 0;
                    if (i == q27::REST) continue;
                    if (i > q27::REST) {
                        const uint64_t o = ((uint64_t)k * 13u + (uint32_t)(i - 14)) * 3u;
                        if (qscr[o + 2]) { qv[i] = bitsf(qscr[o]); qx[i] = bitsf(qscr[o + 1]); nh[i] = qscr[o + 2]; }
                    } else if (in_box(lx + q27::cx(i), ly + q27::cy(i), lz + q27::cz(i))) {
                        const uint32_t k2 = ((uint32_t)(lz + q27::cz(i)) * box_n[1] + (uint32_t)(ly + q27::cy(i))) * box_n[0] + (uint32_t)(lx + q27::cx(i));
                        const uint64_t o = ((uint64_t)k2 * 13u + (uint32_t)(26 - i - 14)) * 3u;
                        if (qscr[o + 2]) { qv[i] = 1.0f - bitsf(qscr[o + 1]); qx[i] = 1.0f - bitsf(qscr[o]); nh[i] = qscr[o + 2]; }
                    }
                }
                uint32_t mask = 0;
                for (int i = 0; i < 27; i++) {
                    if (i == q27::REST) continue;
                    if (solid_at(st.rot, px + q27::cx(i), py + q27::cy(i), pz + q27::cz(i))) {
                        if (nh[i] == 0) qv[i] = 1.0f;
                        mask |= 1u << i;
                    } else if (nh[i] >= 2 && qx[i] - qv[i] > 1e-5f) {
                        mask |= 1u << i;
                    } else {
                        qv[i] = 1.0f;
                    }
                }
                for (int wd = 0; wd < 13; wd++) {
                    const int i0 = 2 * wd < 13 ? 2 * wd : 2 * wd + 1, i1 = 2 * wd + 1 < 13 ? 2 * wd + 1 : 2 * wd + 2;
                    const uint16_t lo = f32_to_f16(std::min(qv[i0], 1.0f)), hi = f32_to_f16(std::min(qv[i1], 1.0f));
                    w[q27::R_Q + wd] = (uint32_t)lo | ((uint32_t)hi << 16);
                    rec_q[(size_t)k * 26 + 2 * wd] = (Real)f16_to_f32(lo);
                    rec_q[(size_t)k * 26 + 2 * wd + 1] = (Real)f16_to_f32(hi);
                }
                w[q27::R_MASK] = mask;
                if (solid_before) {
                    Real rs = 0, cnt = 0, pis[6] = {0, 0, 0, 0, 0, 0};
                    for (int i = 0; i < 27; i++) {
                        if (i == q27::REST) continue;
                        const int x2 = px + q27::cx(i), y2 = py + q27::cy(i), z2 = pz + q27::cz(i);
                        if (solid_at(st.rot, x2, y2, z2) || solid_at(st.rot_prev, x2, y2, z2)) continue;
                        const Mom mo = moments(own(l, st.src, cidx(l, (uint32_t)x2, (uint32_t)y2, (uint32_t)z2)));
                        const Real r2 = (Real)1 + mo.rho1;
                        const Real u2[3] = {mo.j[0] / r2, mo.j[1] / r2, mo.j[2] / r2};
                        Real ps[6];
                        stress(mo, r2, u2, ps);
                        for (int c = 0; c < 6; c++) pis[c] += ps[c];
                        rs += r2;
                        cnt += 1;
                    }
                    const Real rho = cnt > 0 ? rs / cnt : (Real)1;
                    if (cnt > 0)
                        for (int c = 0; c < 6; c++) pis[c] /= cnt;
                    const Real uw[3] = {st.omega[1] * pc[2] - st.omega[2] * pc[1], st.omega[2] * pc[0] - st.omega[0] * pc[2],
                                        st.omega[0] * pc[1] - st.omega[1] * pc[0]};
                    put(l, st.src, n, rebuild(rho, uw, pis), st.seed);
                    for (int c = 0; c < 3; c++) Fv[c] = -rho * uw[c];
                }
                l.flags[n] = (k + 1u) << 3;
            }
            Real *ft = &rec_ft[(size_t)k * 6];
            for (int c = 0; c < 3; c++) ft[c] = Fv[c];
            ft[3] = pc[1] * Fv[2] - pc[2] * Fv[1];
            ft[4] = pc[2] * Fv[0] - pc[0] * Fv[2];
            ft[5] = pc[0] * Fv[1] - pc[1] * Fv[0];
            for (int c = 0; c < 6; c++) w[q27::R_FT + c] = fbits((float)ft[c]);
        }
        for (size_t j = 0; j < qscr.size(); j += 3) { qscr[j] = 0x7f7fffffu; qscr[j + 1] = 0; qscr[j + 2] = 0; }
    }

    std::array<double, 6> reduce() const {
        std::array<double, 6> v{};
        for (uint32_t r = 0; r < nrec; r++)
            for (int k = 0; k < 6; k++) v[k] += (double)rec_ft[(size_t)r * 6 + k];
        return v;
    }

    // ------------------------------------------------------------ schedule
    // mlattice.rs:786-842: one step of level l and, below it, two of each finer level
    void schedule(size_t l, const lbm_step_in *fine, size_t &fine_i, std::vector<std::array<double, 6>> &out) {
        const size_t nl = lv.size(), finest = nl - 1;
        const lbm_step_in *sin = l == finest ? &fine[fine_i] : nullptr;
        const uint32_t lsrc = lv[l].src;
        const uint32_t lmw = 1u - lv[l].mslot;
        const uint32_t hslot = (uint32_t)(fine_i % q27::HIST_CAP);
        Par base;
        base.src = lsrc;
        base.mw = lmw;
        base.seed = seed_of(hslot, lsrc, lmw);
        if (sin)
            for (int k = 0; k < 3; k++) base.omega[k] = sizeof(Real) == 8 ? (Real)sin->omega[k] : (Real)(float)sin->omega[k];
        if (sin)
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) { base.rot[3 * r + c] = (float)sin->rot[r][c]; base.rot_prev[3 * r + c] = (float)sin->rot_prev[r][c]; }
        if (l == 0 && !lv[0].faces.empty()) face_bc(lv[0], base);
        if (moving && l == finest) revoxel(lv[l], base);
        step(l, base);
        lv[l].src = 1u - lsrc;
        lv[l].mslot = lmw;
        lv[l].steps++;
        if (l == finest) {
            out.push_back(reduce());
            if (sin->sample) sample(base);  // mlattice.rs:812-824
            fine_i++;
        }
        if (l + 1 < nl) {
            const uint32_t mold = 1u - lmw;
            for (int sub = 0; sub < 2; sub++) {
                const size_t c = l + 1;
                Par g;
                g.src = lv[c].src;
                g.mold = mold;
                g.mnew = lmw;
                g.blend = (Real)0.5 * (Real)sub;
                g.seed = seed_of(0, g.src, 0);
                ghost_fill(c, g);
                schedule(c, fine, fine_i, out);
            }
            Par r;
            r.src = lv[l].src;
            r.seed = seed_of(0, r.src, 0);
            restrict_fill(l, r);
        }
    }

    // mshader.rs:495-505: density and velocity of any cell but a solid one,
    // from the level's current source set
    bool cell_macro(const Level &l, uint32_t m, float &rho, float &ux, float &uy, float &uz) const {
        if ((l.flags[m] & 7u) == q27::T_SOLID) return false;
        const Mom mo = moments(own(l, l.src, m));
        const Real r = (Real)1 + mo.rho1;
        rho = (float)r;
        ux = (float)(mo.j[0] / r - (Real)0.5 * l.GRAV[0]);
        uy = (float)(mo.j[1] / r - (Real)0.5 * l.GRAV[1]);
        uz = (float)(mo.j[2] / r - (Real)0.5 * l.GRAV[2]);
        return true;
    }

    // mshader.rs:563-602, after a finest step that asked for samples: the
    // vertices on the finest level with the step's rotation (trilinear
    // density over the usable cells around each), then every level's pixels
    void sample(const Par &par) {
        const Level &f = lv.back();
        for (size_t v = 0; v < pverts.size(); v++) {
            const auto &q = pverts[v];
            const float b[3] = {q[0] + VOFF * q[4], q[1] + VOFF * q[5], q[2] + VOFF * q[6]};
            float sp[3], b0[3], fr[3];
            for (int c = 0; c < 3; c++) {
                sp[c] = (float)f.CENTER[c] + (par.rot[3 * c] * b[0] + par.rot[3 * c + 1] * b[1] + par.rot[3 * c + 2] * b[2]);
                b0[c] = std::floor(sp[c]);
                fr[c] = sp[c] - b0[c];
            }
            float acc = 0.f, wsum = 0.f;
            for (int k = 0; k < 8; k++) {
                const int o[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
                const int ci[3] = {(int)b0[0] + o[0], (int)b0[1] + o[1], (int)b0[2] + o[2]};
                if (ci[0] < 1 || ci[1] < 1 || ci[2] < 1 || ci[0] >= (int)f.NX - 1 || ci[1] >= (int)f.NY - 1 || ci[2] >= (int)f.NZ - 1) continue;
                const float w = (o[0] ? fr[0] : 1.f - fr[0]) * (o[1] ? fr[1] : 1.f - fr[1]) * (o[2] ? fr[2] : 1.f - fr[2]);
                float rho, ux, uy, uz;
                if (cell_macro(f, ((uint32_t)ci[2] * f.NY + (uint32_t)ci[1]) * f.NX + (uint32_t)ci[0], rho, ux, uy, uz) && w > 0.f) {
                    acc += w * rho;
                    wsum += w;
                }
            }
            if (wsum > 1e-6f) {
                vacc[2 * v] += (double)(acc / wsum);
                vacc[2 * v + 1] += 1.0;
            }
        }
        for (size_t li = 0; li < lv.size(); li++)
            for (const auto &pc : pix[li]) {
                float rho, ux, uy, uz;
                if (cell_macro(lv[li], pc.second, rho, ux, uy, uz)) {
                    double *a = &sacc[5 * (size_t)pc.first];
                    a[0] += rho; a[1] += ux; a[2] += uy; a[3] += uz; a[4] += 1.0;
                }
            }
    }
    void reset_samples() {
        std::fill(vacc.begin(), vacc.end(), 0.0);
        std::fill(sacc.begin(), sacc.end(), 0.0);
    }
    void vertex_means(float *out) const {
        for (size_t v = 0; v < pverts.size(); v++) out[v] = vacc[2 * v + 1] > 0 ? (float)(vacc[2 * v] / vacc[2 * v + 1]) : std::nanf("");
    }
    void slice_means(float *out) const {
        for (uint32_t i = 0; i < npix; i++) {
            const double c = sacc[5 * (size_t)i + 4];
            for (int a = 0; a < 4; a++) out[4 * i + a] = c > 0 ? (float)(sacc[5 * (size_t)i + a] / c) : std::nanf("");
        }
    }

    // mlattice.rs:723-784 (readback chunks of HIST_CAP finest steps)
    std::vector<std::array<double, 6>> run(const lbm_step_in *fine, size_t n) {
        const size_t ss = sub_steps();
        if (n % ss != 0) throw std::runtime_error("step count must be a multiple of " + std::to_string(ss));
        std::vector<std::array<double, 6>> out;
        const size_t max_coarse = std::max<size_t>(q27::HIST_CAP / ss, 1);
        size_t done = 0;
        while (done < n) {
            const size_t nc = std::min((n - done) / ss, max_coarse);
            size_t fine_i = 0;
            for (size_t k = 0; k < nc; k++) schedule(0, fine + done, fine_i, out);
            fine_steps += nc * ss;
            done += nc * ss;
        }
        return out;
    }

    // mshader.rs:495-505, 602-610: (rho, u) of plain fluid cells, NaN elsewhere
    void macros(size_t li, float *out) const {
        const Level &l = lv[li];
        const float nan = std::nanf("");
        for (uint64_t n = 0; n < l.N; n++) {
            float *o = &out[4 * n];
            if ((l.flags[n] & 7u) != 0) { o[0] = o[1] = o[2] = o[3] = nan; continue; }
            const Mom mo = moments(own(l, l.src, n));
            const Real rho = (Real)1 + mo.rho1;
            o[0] = (float)rho;
            for (int k = 0; k < 3; k++) o[1 + k] = (float)(mo.j[k] / rho - (Real)0.5 * l.GRAV[k]);
        }
    }
};

}  // namespace oracle
