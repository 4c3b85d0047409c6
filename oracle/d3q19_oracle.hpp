// TEST INFRASTRUCTURE -- the CPU oracle for the D3Q19 lattice time step.
//
// This is a restatement of SimLab's WGSL D3Q19 update (crates/cfd/src/shader.rs)
// and its host driver (crates/cfd/src/lattice.rs), written to check the CUDA
// engine against.  Only the tests, the smoke check and the bench's CPU
// baseline use it; the engine never links or calls it.
//
// Parity pin: the reference ships no golden vectors and cannot run here (Rust
// and wgpu/Metal are absent), so this restatement is pinned by the reference's
// own known-answer tests, re-run against it: Poiseuille flow between off-grid
// Bouzidi walls with its second-order convergence and force balance
// (crates/cfd/tests/channel.rs:40-89), FP16 stochastic-rounding storage
// (channel.rs:91-101), momentum lost by the fluid = impulse on the body
// (crates/cfd/tests/momentum.rs:39-51) and zero force in a uniform state
// (momentum.rs:73-85).
//
// Templated on the arithmetic type: float reproduces the reference's FP32
// update operation by operation (compile with -ffp-contract=off); double is
// the FP64 oracle.  Storage: FP32, FP64, FP16 (scaled by 32768, stochastic
// rounding, shader.rs:153-162, 507-517) and BF16 (no reference counterpart).
//
// Everything listed as "no counterpart" (plain BGK, free-slip faces, BF16) is
// new and has only this oracle and analytic checks behind it.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/simlab_lbm.h"

namespace oracle {

// shader.rs:22-60 -- D3Q19 velocities: rest, +-x, +-y, +-z, then 12 edges.
static const int C19[19][3] = {
    {0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
    {1, 1, 0},  {-1, -1, 0}, {1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, -1}, {1, -1, 0},
    {-1, 1, 0}, {1, 0, -1}, {-1, 0, 1}, {0, 1, -1}, {0, -1, 1}};

inline int opp19(int i) { return i == 0 ? 0 : (i % 2 == 1 ? i + 1 : i - 1); }  // shader.rs:44-52
inline double weight19(int i) { return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }

// record layout, shader.rs:62-69
constexpr uint32_t RS = 40, R_MASK = 0, R_CELL = 1, R_Q = 2, R_FPOST = 11, R_MACRO = 29, R_FT = 33;
constexpr float FP16_SCALE = 32768.0f;          // shader.rs:73
constexpr uint32_t STEP_SEED_MUL = 2654435761u;  // lattice.rs:676

// ---------------------------------------------------------------- bit helpers
inline uint32_t fbits(float x) { uint32_t b; std::memcpy(&b, &x, 4); return b; }
inline float bitsf(uint32_t b) { float x; std::memcpy(&x, &b, 4); return x; }

// IEEE binary16, round to nearest even (WGSL f16(x) conversion).
inline uint16_t f32_to_f16(float x) {
    uint32_t b = fbits(x);
    uint32_t sign = (b >> 16) & 0x8000u;
    uint32_t ax = b & 0x7fffffffu;
    if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
    int e = (int)(ax >> 23) - 127;
    if (e > 15) return (uint16_t)(sign | 0x7c00u);
    if (e >= -14) {
        uint32_t man = ax & 0x7fffffu;
        uint32_t h = ((uint32_t)(e + 15) << 10) | (man >> 13);
        uint32_t rem = man & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;  // may carry into exponent: correct
        return (uint16_t)(sign | h);
    }
    // subnormal or zero: value = m * 2^-24
    if (e < -25) return (uint16_t)sign;
    uint32_t man = (ax & 0x7fffffu) | 0x800000u;  // 24 bits, value man * 2^(e-23)
    int shift = -e - 1;                           // (e - 23) -> -24 means shift by (-24 - (e-23)) = -e - 1
    uint32_t h = man >> shift;
    uint32_t rem = man & ((1u << shift) - 1u);
    uint32_t half = 1u << (shift - 1);
    if (rem > half || (rem == half && (h & 1u))) h += 1;
    return (uint16_t)(sign | h);
}

inline float f16_to_f32(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    if (e == 0) {
        float v = std::ldexp((float)m, -24);
        return sign ? -v : v;
    }
    if (e == 31) return bitsf(sign | 0x7f800000u | (m << 13));
    return bitsf(sign | ((e + 112u) << 23) | (m << 13));
}

// lattice.rs:172-189: the host's f16 packing of wall distances q (round half
// up on the magnitude, flush below the normal range to zero).
inline uint16_t f16_bits_ref(float x) {
    uint32_t b = fbits(x);
    uint16_t sign = (uint16_t)((b >> 16) & 0x8000u);
    int exp = (int)((b >> 23) & 0xffu) - 127 + 15;
    uint32_t man = b & 0x7fffffu;
    if (exp <= 0) return sign;
    if (exp >= 31) return (uint16_t)(sign | 0x7c00u);
    uint32_t h = (uint32_t)sign | ((uint32_t)exp << 10) | (man >> 13);
    if (man & 0x1000u) h += 1;
    return (uint16_t)h;
}

// bfloat16, round to nearest even (no reference counterpart).
inline uint16_t f32_to_bf16(float x) {
    uint32_t b = fbits(x);
    if ((b & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((b >> 16) | 0x40u);
    uint32_t r = 0x7fffu + ((b >> 16) & 1u);
    return (uint16_t)((b + r) >> 16);
}
inline float bf16_to_f32(uint16_t h) { return bitsf((uint32_t)h << 16); }

// shader.rs:510-517: stochastic rounding noise for FP16 storage.  r is uniform
// in [-1/2, 1/2) from an integer hash of the slot key and the step seed, and
// is scaled by one binary16 unit in the last place of x.
inline uint32_t sr_hash(uint32_t key, uint32_t seed) {
    uint32_t h = (key * 0x9E3779B1u) ^ (seed * 0x85EBCA77u + 0x632BE5ABu);
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    return h;
}
inline float sround16(float x, uint32_t key, uint32_t seed) {
    float r = (float)(sr_hash(key, seed) >> 8) * (1.0f / 16777216.0f) - 0.5f;
    int e = (int)((fbits(x) >> 23) & 0xffu) - 127;
    float ulp = std::ldexp(1.0f, std::max(e, -14) - 10);  // exact power of two
    float v = x + r * ulp;
    return std::min(std::max(v, -65000.0f), 65000.0f);
}
// BF16 variant: one bfloat16 ulp (8 significant bits), exponent floored at
// -119 so the ulp is a normal float; no scaling, no clamp.
inline float sround_bf16(float x, uint32_t key, uint32_t seed) {
    float r = (float)(sr_hash(key, seed) >> 8) * (1.0f / 16777216.0f) - 0.5f;
    int e = (int)((fbits(x) >> 23) & 0xffu) - 127;
    float ulp = std::ldexp(1.0f, std::max(e, -119) - 7);
    return x + r * ulp;
}

// ---------------------------------------------------------------- the lattice
template <class Real>
struct D3Q19 {
    using F = std::array<Real, 19>;
    struct Mom { Real rho1; Real j[3]; Real s[6]; };
    struct Rec {  // one wall record (shader.rs:62-69), float fields kept in Real
        uint32_t mask = 0, cell = 0;
        uint16_t qh[18] = {};  // f16 bits of q, directions 1..18
        Real fpost[19] = {};   // index 1..18 used
        Real macro[4] = {};
        Real ft[6] = {};
    };

    // configuration
    uint32_t NX = 0, NY = 0, NZ = 0;
    uint64_t N = 0;
    bool per[3] = {false, false, false};
    int storage = LBM_STORAGE_FP32;
    int collision = LBM_COLLISION_REGULARIZED;
    Real TAU0{}, SMAG2{}, SPONGE_TAU{}, SIGMA{};
    Real SP_LO[3]{}, SP_HI[3]{}, U_INF[3]{}, U_INIT[3]{}, GRAV[3]{}, CENTER[3]{};
    bool ABS_U = false, TOTAL_P = false, WALL_MODEL = false, forcing = false;
    Real W[19]{}, W45[19]{};

    // state
    std::vector<float> p32;
    std::vector<double> p64;
    std::vector<uint16_t> p16;  // FP16 or BF16 bits
    std::vector<uint32_t> flags;
    std::vector<Rec> recs;
    std::vector<uint32_t> faces;
    std::vector<uint8_t> face_kind;   // 0 velocity, 1 open, 2 free slip
    std::vector<uint8_t> face_mirror; // free slip: bit a = mirror axis a
    uint64_t steps_done = 0;
    uint32_t seed = 0;  // StepParams.seed of the step being run
    // spinning part (Geometry::Spin): body-frame occupancy, triangles, swept
    // box, per-link hit scratch (shader.rs:865-1104)
    bool moving = false;
    std::vector<uint32_t> occ;
    float occ_lo[3] = {0, 0, 0}, occ_invh = 1.f, CENTERF[3] = {0, 0, 0};
    int32_t occ_n[3] = {0, 0, 0}, box_lo[3] = {0, 0, 0};
    uint32_t box_n[3] = {0, 0, 0};
    std::vector<std::array<float, 12>> tris;
    std::vector<uint32_t> qscr;

    // ------------------------------------------------------------ storage
    inline Real L(int d, uint64_t cell) const {
        uint64_t k = (uint64_t)d * N + cell;
        switch (storage) {
            case LBM_STORAGE_FP32: return (Real)p32[k];
            case LBM_STORAGE_FP64: return (Real)p64[k];
            case LBM_STORAGE_FP16: return (Real)(f16_to_f32(p16[k]) * (1.0f / FP16_SCALE));
            default: return (Real)bf16_to_f32(p16[k]);
        }
    }
    inline void S(int d, uint64_t cell, Real v, uint32_t key) {
        uint64_t k = (uint64_t)d * N + cell;
        switch (storage) {
            case LBM_STORAGE_FP32: p32[k] = (float)v; break;
            case LBM_STORAGE_FP64: p64[k] = (double)v; break;
            case LBM_STORAGE_FP16: p16[k] = f32_to_f16(sround16((float)v * FP16_SCALE, key, seed)); break;
            default: p16[k] = f32_to_bf16(sround_bf16((float)v, key, seed)); break;
        }
    }

    // ------------------------------------------------------------ indexing
    struct Nb { uint32_t x, y, z, xp, xm, yp, ym, zp, zm; };
    inline Nb neigh(uint64_t n) const {  // shader.rs:240-252
        Nb b;
        b.z = (uint32_t)(n / ((uint64_t)NX * NY));
        uint64_t r = n - (uint64_t)b.z * NX * NY;
        b.y = (uint32_t)(r / NX);
        b.x = (uint32_t)(r - (uint64_t)b.y * NX);
        b.xp = b.x == NX - 1 ? 0 : b.x + 1; b.xm = b.x == 0 ? NX - 1 : b.x - 1;
        b.yp = b.y == NY - 1 ? 0 : b.y + 1; b.ym = b.y == 0 ? NY - 1 : b.y - 1;
        b.zp = b.z == NZ - 1 ? 0 : b.z + 1; b.zm = b.z == 0 ? NZ - 1 : b.z - 1;
        return b;
    }
    inline uint64_t nb(const Nb &b, int dx, int dy, int dz) const {
        uint32_t xx = dx == 1 ? b.xp : (dx == -1 ? b.xm : b.x);
        uint32_t yy = dy == 1 ? b.yp : (dy == -1 ? b.ym : b.y);
        uint32_t zz = dz == 1 ? b.zp : (dz == -1 ? b.zm : b.z);
        return ((uint64_t)zz * NY + yy) * NX + xx;
    }

    // ------------------------------------------------------------ AA access
    // shader.rs:254-271
    F load_in(uint64_t n, int p) const {
        F f;
        if (p == 0) { for (int i = 0; i < 19; i++) f[i] = L(i, n); return f; }
        Nb b = neigh(n);
        f[0] = L(0, n);
        for (int i = 1; i < 19; i++) f[i] = L(opp19(i), nb(b, -C19[i][0], -C19[i][1], -C19[i][2]));
        return f;
    }
    // shader.rs:275-305 (guard: skip targets that leave a non-periodic domain)
    void store_out(uint64_t n, int p, const F &f, bool guard) {
        uint32_t key0 = (uint32_t)n * 19u;
        if (p == 0) { for (int i = 0; i < 19; i++) S(opp19(i), n, f[i], key0 + (uint32_t)opp19(i)); return; }
        Nb b = neigh(n);
        S(0, n, f[0], key0);
        for (int i = 1; i < 19; i++) {
            if (guard) {
                bool ok = true;
                const uint32_t xyz[3] = {b.x, b.y, b.z}, lim[3] = {NX, NY, NZ};
                for (int k = 0; k < 3; k++) {
                    if (C19[i][k] == 1) ok = ok && (per[k] || xyz[k] < lim[k] - 1);
                    else if (C19[i][k] == -1) ok = ok && (per[k] || xyz[k] > 0);
                }
                if (!ok) continue;
            }
            S(i, nb(b, C19[i][0], C19[i][1], C19[i][2]), f[i], key0 + (uint32_t)i);
        }
    }
    // shader.rs:310-321
    F load_prev_out(uint64_t n, int p) const {
        F f;
        if (p == 0) { for (int i = 0; i < 19; i++) f[i] = L(opp19(i), n); return f; }
        Nb b = neigh(n);
        f[0] = L(0, n);
        for (int i = 1; i < 19; i++) f[i] = L(i, nb(b, C19[i][0], C19[i][1], C19[i][2]));
        return f;
    }
    // shader.rs:323-339 (only parity 0 is used: init)
    void store_in0(uint64_t n, const F &f) {
        uint32_t key0 = (uint32_t)n * 19u;
        for (int i = 0; i < 19; i++) S(i, n, f[i], key0 + (uint32_t)i);
    }

    // ------------------------------------------------------------ moments
    // shader.rs:341-365; sums in direction order starting from 0.0
    static Mom moments(const F &f) {
        Mom m;
        Real r = 0;
        for (int i = 0; i < 19; i++) r = r + f[i];
        m.rho1 = r;
        for (int a = 0; a < 3; a++) {
            Real t = 0;
            for (int i = 0; i < 19; i++) {
                int k = C19[i][a];
                if (k == 1) t = t + f[i]; else if (k == -1) t = t - f[i];
            }
            m.j[a] = t;
        }
        static const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
        for (int q = 0; q < 6; q++) {
            Real t = 0;
            for (int i = 0; i < 19; i++) {
                int k = C19[i][pa[q]] * C19[i][pb[q]];
                if (k == 1) t = t + f[i]; else if (k == -1) t = t - f[i];
            }
            m.s[q] = t;
        }
        return m;
    }
    static Real cdot(int i, const Real *v) {  // shader.rs:465-475
        Real t = 0;
        for (int k = 0; k < 3; k++) {
            if (C19[i][k] == 1) t = t + v[k]; else if (C19[i][k] == -1) t = t - v[k];
        }
        return t;
    }
    static Real dot3(const Real *a, const Real *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
    // shader.rs:367-377
    F feq(Real rho1, const Real *u) const {
        F f;
        Real rho = (Real)1 + rho1;
        Real usq = (Real)1.5 * dot3(u, u);
        for (int i = 0; i < 19; i++) {
            Real cu = cdot(i, u);
            f[i] = W[i] * (rho1 + rho * ((Real)3 * cu + (Real)4.5 * cu * cu - usq));
        }
        return f;
    }
    // shader.rs:379-396
    F fneq(const Real *p) const {
        F f;
        Real tr = (p[0] + p[1] + p[2]) * (Real)(1.0 / 3.0);
        static const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
        for (int i = 0; i < 19; i++) {
            Real t = -tr;
            for (int q = 0; q < 6; q++) {
                int v = C19[i][pa[q]] * C19[i][pb[q]] * (pa[q] == pb[q] ? 1 : 2);
                if (v != 0) t = t + (Real)v * p[q];
            }
            f[i] = W45[i] * t;
        }
        return f;
    }
    // the non-equilibrium stress of shader.rs:818-824 / 648-653
    static void pi_neq(const Mom &mo, Real rho, const Real *u, Real *pi) {
        pi[0] = mo.s[0] - rho * u[0] * u[0] - mo.rho1 / (Real)3;
        pi[1] = mo.s[1] - rho * u[1] * u[1] - mo.rho1 / (Real)3;
        pi[2] = mo.s[2] - rho * u[2] * u[2] - mo.rho1 / (Real)3;
        pi[3] = mo.s[3] - rho * u[0] * u[1];
        pi[4] = mo.s[4] - rho * u[0] * u[2];
        pi[5] = mo.s[5] - rho * u[1] * u[2];
    }

    // shader.rs:528-538
    Real sponge(uint32_t x, uint32_t y, uint32_t z) const {
        Real p[3] = {(Real)x, (Real)y, (Real)z};
        Real hi[3] = {(Real)(NX - 1) - p[0], (Real)(NY - 1) - p[1], (Real)(NZ - 1) - p[2]};
        Real s = 0;
        for (int k = 0; k < 3; k++) {
            if (SP_LO[k] > 0) s = std::max(s, (Real)1 - p[k] / SP_LO[k]);
            if (SP_HI[k] > 0) s = std::max(s, (Real)1 - hi[k] / SP_HI[k]);
        }
        return std::min(std::max(s, (Real)0), (Real)1);
    }

    Real q_of(const Rec &r, int i) const { return (Real)f16_to_f32(r.qh[i - 1]); }

    // shader.rs:546-597 (Spalding wall model)
    Real wall_tau(const Rec &rc, uint32_t mask, const Real *pc, const Real *u, Real tau_les, const Real *omega) const {
        Real nsum[3] = {0, 0, 0};
        for (int i = 1; i < 19; i++) {
            if (mask & (1u << i)) {
                Real q = q_of(rc, i);
                Real w = i < 7 ? (Real)(1.0 / 18.0) : (Real)(1.0 / 36.0);
                for (int k = 0; k < 3; k++) nsum[k] = nsum[k] + (Real)C19[i][k] * w * ((Real)1.5 - q);
            }
        }
        Real nl = std::sqrt(dot3(nsum, nsum));
        if (nl < (Real)1e-6) return tau_les;
        Real nw[3] = {nsum[0] / nl, nsum[1] / nl, nsum[2] / nl};
        Real y = 2;
        for (int i = 1; i < 19; i++) {
            if (mask & (1u << i)) {
                Real cv[3] = {(Real)C19[i][0], (Real)C19[i][1], (Real)C19[i][2]};
                Real cn = dot3(cv, nw);
                if (cn > (Real)0.3) {
                    Real q = q_of(rc, i);
                    y = std::min(y, std::max(q, (Real)0.02) * cn);
                }
            }
        }
        if (y > (Real)1.9) return tau_les;
        Real xw[3] = {pc[0] + y * nw[0], pc[1] + y * nw[1], pc[2] + y * nw[2]};
        Real uwall[3] = {omega[1] * xw[2] - omega[2] * xw[1], omega[2] * xw[0] - omega[0] * xw[2], omega[0] * xw[1] - omega[1] * xw[0]};
        Real ur[3] = {u[0] - uwall[0], u[1] - uwall[1], u[2] - uwall[2]};
        Real un = dot3(ur, nw);
        Real tv[3] = {ur[0] - un * nw[0], ur[1] - un * nw[1], ur[2] - un * nw[2]};
        Real ut = std::sqrt(dot3(tv, tv));
        Real nu0 = (TAU0 - (Real)0.5) / (Real)3;
        if (ut < (Real)1e-7) return tau_les;
        Real kap = (Real)0.41;
        Real eb = std::exp(-kap * (Real)5.2);
        Real ust = std::sqrt(nu0 * ut / y);
        for (int it = 0; it < 12; it++) {
            Real up = ut / ust;
            Real yp = y * ust / nu0;
            Real ku = std::min(kap * up, (Real)30);
            Real g = up + eb * (std::exp(ku) - (Real)1 - ku - (Real)0.5 * ku * ku - ku * ku * ku / (Real)6) - yp;
            Real dgdup = (Real)1 + eb * kap * (std::exp(ku) - (Real)1 - ku - (Real)0.5 * ku * ku);
            Real dg = dgdup * (-up / ust) - y / nu0;
            Real step = g / dg;
            ust = std::min(std::max(ust - step, (Real)0.1 * ust), (Real)10 * ust);
            if (std::abs(step) < (Real)1e-5 * ust) break;
        }
        Real nuw = ust * ust * y / ut;
        return std::max((Real)0.5 + (Real)3 * std::max(nuw, nu0), tau_les);
    }

    // ------------------------------------------------------------ setup
    // lattice.rs:229-526 (validation, face list, records, flags) and 661-671 (init)
    void create(const lbm_setup &st, const lbm_geometry *geom) {
        NX = st.dims[0]; NY = st.dims[1]; NZ = st.dims[2];
        N = (uint64_t)NX * NY * NZ;
        if (N == 0 || N >= 0xffffffffull) throw std::runtime_error("grid out of range");
        if (NX < 3 || NY < 3 || NZ < 3) throw std::runtime_error("grid must be at least 3 cells in every direction");
        for (int a = 0; a < 3; a++) {
            bool p0 = st.faces[2 * a] == LBM_FACE_PERIODIC, p1 = st.faces[2 * a + 1] == LBM_FACE_PERIODIC;
            if (p0 != p1) throw std::runtime_error("periodic faces must come in pairs");
            per[a] = p0;
        }
        storage = st.storage;
        collision = st.collision;
        TAU0 = (Real)(0.5 + 3.0 * st.nu);
        SMAG2 = (Real)(st.smagorinsky * st.smagorinsky);
        SPONGE_TAU = (Real)st.sponge_tau;
        SIGMA = (Real)st.sponge_sigma;
        ABS_U = st.absorb_velocity != 0;
        TOTAL_P = st.total_pressure_inlet != 0;
        WALL_MODEL = st.wall_model != 0;
        for (int k = 0; k < 3; k++) {
            SP_LO[k] = (Real)st.sponge[2 * k];
            SP_HI[k] = (Real)st.sponge[2 * k + 1];
            U_INF[k] = (Real)st.u_inf[k];
            U_INIT[k] = (Real)st.u_init[k];
            GRAV[k] = (Real)st.body_force[k];
            CENTER[k] = (Real)st.center[k];
        }
        forcing = st.body_force[0] != 0.0 || st.body_force[1] != 0.0 || st.body_force[2] != 0.0;
        for (int i = 0; i < 19; i++) { W[i] = (Real)weight19(i); W45[i] = (Real)(4.5 * weight19(i)); }

        switch (storage) {
            case LBM_STORAGE_FP32: p32.assign(19 * N, 0.0f); break;
            case LBM_STORAGE_FP64: p64.assign(19 * N, 0.0); break;
            case LBM_STORAGE_FP16: case LBM_STORAGE_BF16: p16.assign(19 * N, 0); break;
            default: throw std::runtime_error("unknown storage");
        }

        // face cells (lattice.rs:283-324), with free slip added: velocity
        // sticks, otherwise the later face in -x,+x,-y,+y,-z,+z order wins.
        auto face_type = [&](uint32_t x, uint32_t y, uint32_t z, uint8_t *mirror) -> int {
            bool on[6] = {x == 0, x == NX - 1, y == 0, y == NY - 1, z == 0, z == NZ - 1};
            int ty = -1;
            uint8_t mir = 0;
            for (int f = 0; f < 6; f++) {
                if (on[f] && st.faces[f] != LBM_FACE_PERIODIC) {
                    int t = st.faces[f] == LBM_FACE_VELOCITY ? 0 : (st.faces[f] == LBM_FACE_OPEN ? 1 : 2);
                    if (st.faces[f] == LBM_FACE_FREE_SLIP) mir |= (uint8_t)(1u << (f / 2));
                    ty = (ty == 0) ? 0 : t;
                }
            }
            if (mirror) *mirror = mir;
            return ty;
        };
        faces.clear(); face_kind.clear(); face_mirror.clear();
        for (uint32_t z = 0; z < NZ; z++)
            for (uint32_t y = 0; y < NY; y++) {
                bool edge = y == 0 || y == NY - 1 || z == 0 || z == NZ - 1;
                auto visit = [&](uint32_t x) {
                    uint8_t mir;
                    int t = face_type(x, y, z, &mir);
                    if (t >= 0) { faces.push_back((z * NY + y) * NX + x); face_kind.push_back((uint8_t)t); face_mirror.push_back(mir); }
                };
                if (edge) { for (uint32_t x = 0; x < NX; x++) visit(x); }
                else { visit(0); if (NX - 1 != 0) visit(NX - 1); }
            }

        // records (lattice.rs:454-482, record_words 202-218); a spinning part
        // makes every swept-box cell a record without links (465-480)
        recs.clear();
        std::vector<std::pair<uint32_t, uint32_t>> rec_of;
        std::vector<lbm_wall_cell> boxwalls;
        lbm_geometry boxgeom{};
        for (int k = 0; k < 3; k++) CENTERF[k] = (float)st.center[k];
        if (geom && geom->kind == 2) {
            moving = true;
            for (int k = 0; k < 3; k++) {
                box_lo[k] = geom->box_lo[k];
                box_n[k] = geom->box_n[k];
                occ_lo[k] = (float)geom->occ_lo[k];
                occ_n[k] = (int32_t)geom->occ_dims[k];
                if (box_lo[k] < 1 || (int64_t)box_lo[k] + box_n[k] > (int64_t)st.dims[k] - 1)
                    throw std::runtime_error("the spinning part's swept box leaves the domain");
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
                        boxwalls[k].cell = (uint32_t)((((uint64_t)z + box_lo[2]) * NY + y + box_lo[1]) * NX + x + box_lo[0]);
                        boxwalls[k].mask = 0;
                        for (int i = 0; i < 27; i++) boxwalls[k].q[i] = 1.0f;
                    }
            boxgeom.kind = 1;
            boxgeom.walls = boxwalls.data();
            boxgeom.nwalls = nb;
            geom = &boxgeom;
            qscr.assign(nb * 27, 0u);
            for (size_t j = 0; j < qscr.size(); j += 3) qscr[j] = 0x7f7fffffu;
        }
        if (geom && geom->kind == 1) {
            for (uint64_t r = 0; r < geom->nwalls; r++) {
                const lbm_wall_cell &w = geom->walls[r];
                Rec rc;
                rc.mask = w.mask; rc.cell = w.cell;
                for (int i = 1; i < 19; i++) rc.qh[i - 1] = f16_bits_ref(w.q[i]);
                // feq_shifted (lattice.rs:191-200): computed in f64, stored as f32
                double usq = 1.5 * (st.u_init[0] * st.u_init[0] + st.u_init[1] * st.u_init[1] + st.u_init[2] * st.u_init[2]);
                for (int i = 1; i < 19; i++) {
                    double cu = C19[i][0] * st.u_init[0] + C19[i][1] * st.u_init[1] + C19[i][2] * st.u_init[2];
                    rc.fpost[i] = (Real)(weight19(i) * (3.0 * cu + 4.5 * cu * cu - usq));  // f32 record word in FP32
                }
                rc.macro[0] = (Real)1.0;
                for (int k = 0; k < 3; k++) rc.macro[1 + k] = (Real)st.u_init[k];
                recs.push_back(rc);
                rec_of.push_back({w.cell, (uint32_t)r + 1});
            }
        }
        // flags (lattice.rs:489-526): 0 fluid, 1 solid, 2 velocity face,
        // 3 other face, (rec+1)<<2 wall cell
        flags.assign(N, 0);
        for (size_t k = 0; k < faces.size(); k++) flags[faces[k]] = face_kind[k] == 0 ? 2u : 3u;
        if (geom && geom->kind == 1) {
            for (uint64_t s = 0; s < geom->nsolid; s++) {
                uint32_t c = geom->solid[s];
                if (c < N && flags[c] == 0) flags[c] = 1;
            }
        }
        for (auto &ro : rec_of)
            if (ro.first < N && (flags[ro.first] & 3u) == 0) flags[ro.first] = ro.second << 2;

        // initial state (shader.rs:623-628), step seed 0
        steps_done = 0;
        seed = 0;
        Real zero[3] = {0, 0, 0};
        (void)zero;
        F fe = feq((Real)0, U_INIT);
        for (uint64_t n = 0; n < N; n++) store_in0(n, fe);
    }

    // ------------------------------------------------------------ faces
    // shader.rs:630-687, plus free slip (mirror image of the inner
    // neighbour's post-collision populations; no reference counterpart).
    void faces_step(int p) {
        const int q = 1 - p;
        const size_t nf = faces.size();
        std::vector<F> buf(nf);
#pragma omp parallel for schedule(static)
        for (long long k = 0; k < (long long)nf; k++) {
            uint32_t b = faces[k];
            Nb c = neigh(b);
            uint32_t cx = c.x, cy = c.y, cz = c.z;
            if (!per[0]) cx = std::min(std::max(cx, 1u), NX - 2);
            if (!per[1]) cy = std::min(std::max(cy, 1u), NY - 2);
            if (!per[2]) cz = std::min(std::max(cz, 1u), NZ - 2);
            uint64_t m = ((uint64_t)cz * NY + cy) * NX + cx;
            uint32_t fg = flags[m];
            if (face_kind[k] == 2) {
                if ((fg & 3u) == 0) {
                    F g = load_prev_out(m, q);
                    F f;
                    for (int i = 0; i < 19; i++) {
                        int d[3] = {C19[i][0], C19[i][1], C19[i][2]};
                        for (int a = 0; a < 3; a++) if (face_mirror[k] & (1u << a)) d[a] = -d[a];
                        int j = 0;
                        for (int t = 0; t < 19; t++) if (C19[t][0] == d[0] && C19[t][1] == d[1] && C19[t][2] == d[2]) j = t;
                        f[i] = g[j];
                    }
                    buf[k] = f;
                } else {
                    buf[k] = feq((Real)0, U_INF);
                }
                continue;
            }
            Real rho = 1, u[3] = {U_INF[0], U_INF[1], U_INF[2]}, pi[6] = {0, 0, 0, 0, 0, 0};
            if ((fg & 3u) == 0) {
                Mom mo = moments(load_prev_out(m, q));
                rho = (Real)1 + mo.rho1;
                for (int a = 0; a < 3; a++) u[a] = mo.j[a] / rho - (Real)0.5 * GRAV[a];
                pi_neq(mo, rho, u, pi);
            }
            if (face_kind[k] == 0) {
                if (TOTAL_P) rho = ((Real)(1.0 / 3.0) + (Real)0.5 * dot3(U_INF, U_INF)) / ((Real)(1.0 / 3.0) + (Real)0.5 * dot3(u, u));
                else { u[0] = U_INF[0]; u[1] = U_INF[1]; u[2] = U_INF[2]; }
            } else {
                rho = 1;
            }
            F fe = feq(rho - (Real)1, u), fq = fneq(pi), f;
            for (int i = 0; i < 19; i++) f[i] = fe[i] + fq[i];
            buf[k] = f;
        }
        for (size_t k = 0; k < nf; k++) store_out(faces[k], q, buf[k], true);
    }

    // ------------------------------------------------------------ main step
    // shader.rs:795-862 with the $WALLS$ (399-436), $FORCING$ (442-455) and
    // $SAVE$ (437-441) expansions.  Plain BGK (no counterpart) relaxes f
    // itself and omits the regularization correction of the forcing.
    void main_cell(uint64_t n, int p, const Real *omega) {
        uint32_t fg = flags[n];
        if ((fg & 3u) != 0) return;
        Nb xyz = neigh(n);
        F f = load_in(n, p);
        uint32_t rec = fg >> 2;
        Real Fo[3] = {0, 0, 0}, To[3] = {0, 0, 0};
        uint32_t mask = 0;
        Rec *rc = nullptr;
        Real pc[3] = {(Real)xyz.x - CENTER[0], (Real)xyz.y - CENTER[1], (Real)xyz.z - CENTER[2]};
        if (rec != 0) {
            rc = &recs[rec - 1];
            mask = rc->mask;
            F fin = f;
            for (int i = 1; i < 19; i++) {
                if (!(mask & (1u << i))) continue;
                int o = opp19(i);
                Real w = W[i];
                Real q = std::max(q_of(*rc, i), (Real)0.001);
                Real fpi = rc->fpost[i] + w;
                Real fpo = rc->fpost[o] + w;
                Real ci[3] = {(Real)C19[i][0], (Real)C19[i][1], (Real)C19[i][2]};
                Real xw[3] = {pc[0] + q * ci[0], pc[1] + q * ci[1], pc[2] + q * ci[2]};
                Real uw[3] = {omega[1] * xw[2] - omega[2] * xw[1], omega[2] * xw[0] - omega[0] * xw[2], omega[0] * xw[1] - omega[1] * xw[0]};
                Real cu = dot3(ci, uw);
                Real fb;
                if (q >= (Real)0.5) fb = (fpi + ((Real)2 * q - (Real)1) * fpo - (Real)6 * w * cu) / ((Real)2 * q);
                else if ((mask & (1u << o)) == 0) fb = (Real)2 * q * fpi + ((Real)1 - (Real)2 * q) * (fin[i] + w) - (Real)6 * w * cu;
                else fb = fpi - (Real)6 * w * cu;
                f[o] = fb - w;
                Real fl[3];
                for (int k = 0; k < 3; k++) fl[k] = (ci[k] - uw[k]) * fpi + (ci[k] + uw[k]) * fb;
                for (int k = 0; k < 3; k++) Fo[k] = Fo[k] + fl[k];
                Real tq[3] = {xw[1] * fl[2] - xw[2] * fl[1], xw[2] * fl[0] - xw[0] * fl[2], xw[0] * fl[1] - xw[1] * fl[0]};
                for (int k = 0; k < 3; k++) To[k] = To[k] + tq[k];
            }
        }
        Mom mo = moments(f);
        Real rho = (Real)1 + mo.rho1;
        Real u[3];
        for (int a = 0; a < 3; a++) u[a] = mo.j[a] / rho + (Real)0.5 * GRAV[a];
        Real pi[6];
        pi_neq(mo, rho, u, pi);
        Real pp = pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] + (Real)2 * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]);
        Real qn = std::sqrt((Real)2 * pp);
        Real tau = (Real)0.5 * (TAU0 + std::sqrt(TAU0 * TAU0 + (Real)18 * SMAG2 * qn / rho));
        if (WALL_MODEL && mask != 0) tau = wall_tau(*rc, mask, pc, u, tau, omega);
        Real sp = sponge(xyz.x, xyz.y, xyz.z);
        if (sp > 0 && SPONGE_TAU > tau) tau = tau + sp * sp * (SPONGE_TAU - tau);
        Real om = (Real)1 / tau;
        F fe = feq(mo.rho1, u);
        if (collision == LBM_COLLISION_BGK) {
            for (int i = 0; i < 19; i++) f[i] = f[i] - om * (f[i] - fe[i]);
        } else {
            F fq = fneq(pi);
            for (int i = 0; i < 19; i++) f[i] = fe[i] + ((Real)1 - om) * fq[i];
        }
        if (sp > 0 && SIGMA > 0) {
            Real ut[3] = {ABS_U ? U_INF[0] : u[0], ABS_U ? U_INF[1] : u[1], ABS_U ? U_INF[2] : u[2]};
            F ft = feq((Real)0, ut);
            Real sg = SIGMA * sp * sp;
            for (int i = 0; i < 19; i++) f[i] = f[i] + sg * (ft[i] - fe[i]);
        }
        if (forcing) {
            Real G[3] = {rho * GRAV[0], rho * GRAV[1], rho * GRAV[2]};
            Real uG = dot3(u, G);
            Real fo = (Real)1 - (Real)0.5 * om;
            for (int i = 0; i < 19; i++) {
                Real cu = cdot(i, u), cg = cdot(i, G);
                Real t = fo * ((Real)3 * (cg - uG) + (Real)9 * cu * cg);
                if (collision != LBM_COLLISION_BGK) t = t - (Real)1.5 * ((Real)1 - om) * cg;
                f[i] = f[i] + W[i] * t;
            }
        }
        if (rc) {
            for (int i = 1; i < 19; i++) rc->fpost[i] = f[i];
            rc->macro[0] = rho;
            for (int a = 0; a < 3; a++) rc->macro[1 + a] = u[a];
            if (moving)
                for (int a = 0; a < 3; a++) { Fo[a] = Fo[a] + rc->ft[a]; To[a] = To[a] + rc->ft[3 + a]; }
            for (int a = 0; a < 3; a++) { rc->ft[a] = Fo[a]; rc->ft[3 + a] = To[a]; }
        }
        store_out(n, p, f, false);
    }

    // ------------------------------------------------------------ spinning part
    // shader.rs:865-1104 in f32, one rounding per operation (compiled without
    // contraction), rot row-major with the body axes as columns
    struct V3f { float x, y, z; };
    static float dotf(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    static V3f crossf(V3f a, V3f b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
    static V3f colf(const float *r, int k) { return {r[k], r[3 + k], r[6 + k]}; }
    static V3f to_body(const float *r, V3f v) { return {dotf(colf(r, 0), v), dotf(colf(r, 1), v), dotf(colf(r, 2), v)}; }
    static V3f from_body(const float *r, V3f b) {
        const V3f c0 = colf(r, 0), c1 = colf(r, 1), c2 = colf(r, 2);
        return {c0.x * b.x + c1.x * b.y + c2.x * b.z, c0.y * b.x + c1.y * b.y + c2.y * b.z, c0.z * b.x + c1.z * b.y + c2.z * b.z};
    }
    bool occ_at(V3f b) const {
        const float gx = std::nearbyint((b.x - occ_lo[0]) * occ_invh), gy = std::nearbyint((b.y - occ_lo[1]) * occ_invh),
                    gz = std::nearbyint((b.z - occ_lo[2]) * occ_invh);
        if (!(gx >= 0.f && gy >= 0.f && gz >= 0.f) || gx >= (float)occ_n[0] || gy >= (float)occ_n[1] || gz >= (float)occ_n[2]) return false;
        const uint64_t l = ((uint64_t)gz * (uint64_t)occ_n[1] + (uint64_t)gy) * (uint64_t)occ_n[0] + (uint64_t)gx;
        return ((occ[l >> 5] >> (l & 31u)) & 1u) != 0u;
    }
    bool solid_at(const float *rot, int x, int y, int z) const {
        return occ_at(to_body(rot, {(float)x - CENTERF[0], (float)y - CENTERF[1], (float)z - CENTERF[2]}));
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
        return t > 0.0f ? t : 0.0f;  // +0 for -0 too: the hit bits are compared as integers
    }
    uint32_t box_index(int x, int y, int z) const {
        return ((uint32_t)(z - box_lo[2]) * box_n[1] + (uint32_t)(y - box_lo[1])) * box_n[0] + (uint32_t)(x - box_lo[0]);
    }
    // shader.rs:902-940
    void tri_scatter(const float *rot) {
        for (const auto &tr : tris) {
            const V3f v0 = from_body(rot, {tr[0], tr[1], tr[2]});
            const V3f a = {CENTERF[0] + v0.x, CENTERF[1] + v0.y, CENTERF[2] + v0.z};
            const V3f e1 = from_body(rot, {tr[4], tr[5], tr[6]}), e2 = from_body(rot, {tr[8], tr[9], tr[10]});
            const V3f nrm = crossf(e1, e2);
            const float nl = std::sqrt(dotf(nrm, nrm));
            if (nl < 1e-12f) continue;
            const V3f nn = {nrm.x / nl, nrm.y / nl, nrm.z / nl};
            const V3f b = {a.x + e1.x, a.y + e1.y, a.z + e1.z}, c = {a.x + e2.x, a.y + e2.y, a.z + e2.z};
            const float mn[3] = {std::min(std::min(a.x, b.x), c.x), std::min(std::min(a.y, b.y), c.y), std::min(std::min(a.z, b.z), c.z)};
            const float mx[3] = {std::max(std::max(a.x, b.x), c.x), std::max(std::max(a.y, b.y), c.y), std::max(std::max(a.z, b.z), c.z)};
            int lo[3], hi[3];
            for (int k = 0; k < 3; k++) {
                lo[k] = std::max((int)std::ceil(mn[k] - 1.415f), box_lo[k]);
                hi[k] = std::min((int)std::floor(mx[k] + 1.415f), box_lo[k] + (int)box_n[k] - 1);
            }
            for (int z = lo[2]; z <= hi[2]; z++)
                for (int y = lo[1]; y <= hi[1]; y++)
                    for (int x = lo[0]; x <= hi[0]; x++) {
                        const V3f pt = {(float)x, (float)y, (float)z};
                        const float d0 = dotf(nn, {pt.x - a.x, pt.y - a.y, pt.z - a.z});
                        if (std::fabs(d0) > 1.415f) continue;
                        const uint32_t k = box_index(x, y, z);
                        for (int i = 1; i < 19; i += 2) {
                            const V3f cv = {(float)C19[i][0], (float)C19[i][1], (float)C19[i][2]};
                            const float d1 = d0 + dotf(nn, cv);
                            if (d0 * d1 > 0.0f && std::fabs(d0) > 1e-6f) continue;
                            const float tt = ray_tri(pt, cv, a, e1, e2);
                            if (tt <= 1.0f) {
                                const uint64_t o = ((uint64_t)k * 9u + (uint32_t)(i - 1) / 2u) * 3u;
                                const uint32_t tb = fbits(tt > 0.0f ? tt : 0.0f);
                                qscr[o] = std::min(qscr[o], tb);
                                qscr[o + 1] = std::max(qscr[o + 1], tb);
                                qscr[o + 2] += 1u;
                            }
                        }
                    }
        }
    }
    // shader.rs:953-1104 for every swept-box cell; Q = the previous step's parity
    void voxelize(const float *rot, const float *rotp, const Real *omega, int Q) {
        const uint64_t nb = (uint64_t)box_n[0] * box_n[1] * box_n[2];
        // classification first (reads only the scratch and occupancy), then the
        // refill (reads neighbours' records of cells that were fluid before,
        // which nobody writes here)
#pragma omp parallel for schedule(static)
        for (long long kk = 0; kk < (long long)nb; kk++) {
            const uint32_t k = (uint32_t)kk;
            const int lx = (int)(k % box_n[0]), ly = (int)((k / box_n[0]) % box_n[1]), lz = (int)(k / (box_n[0] * box_n[1]));
            const int px = lx + box_lo[0], py = ly + box_lo[1], pz = lz + box_lo[2];
            const uint64_t n = ((uint64_t)pz * NY + py) * NX + px;
            Rec &rc = recs[k];
            const Real pc[3] = {(Real)px - CENTER[0], (Real)py - CENTER[1], (Real)pz - CENTER[2]};
            const bool solid_now = solid_at(rot, px, py, pz), solid_before = solid_at(rotp, px, py, pz);
            Real Fv[3] = {0, 0, 0};
            if (solid_now) {
                flags[n] = 1u | ((k + 1u) << 2);
                rc.mask = 0;
                if (!solid_before)
                    for (int a = 0; a < 3; a++) Fv[a] = rc.macro[0] * rc.macro[1 + a];
            } else {
                float qv[19], qx[19];
                uint32_t nh[19];
                for (int i = 1; i < 19; i++) {
                    qv[i] = 9.0f; qx[i] = -1.0f; nh[i] = 0;
                    if (i & 1) {
                        const uint64_t o = ((uint64_t)k * 9u + (uint32_t)(i - 1) / 2u) * 3u;
                        if (qscr[o + 2]) { qv[i] = bitsf(qscr[o]); qx[i] = bitsf(qscr[o + 1]); nh[i] = qscr[o + 2]; }
                    } else {
                        const int qx_ = lx + C19[i][0], qy_ = ly + C19[i][1], qz_ = lz + C19[i][2];
                        if (qx_ >= 0 && qy_ >= 0 && qz_ >= 0 && qx_ < (int)box_n[0] && qy_ < (int)box_n[1] && qz_ < (int)box_n[2]) {
                            const uint32_t k2 = ((uint32_t)qz_ * box_n[1] + (uint32_t)qy_) * box_n[0] + (uint32_t)qx_;
                            const uint64_t o = ((uint64_t)k2 * 9u + (uint32_t)(i - 2) / 2u) * 3u;
                            if (qscr[o + 2]) { qv[i] = 1.0f - bitsf(qscr[o + 1]); qx[i] = 1.0f - bitsf(qscr[o]); nh[i] = qscr[o + 2]; }
                        }
                    }
                }
                uint32_t mask = 0;
                for (int i = 1; i < 19; i++) {
                    if (solid_at(rot, px + C19[i][0], py + C19[i][1], pz + C19[i][2])) {
                        if (nh[i] == 0) qv[i] = 1.0f;
                        mask |= 1u << i;
                    } else if (nh[i] >= 2 && qx[i] - qv[i] > 1e-5f) {
                        mask |= 1u << i;
                    } else {
                        qv[i] = 1.0f;
                    }
                }
                for (int i = 1; i < 19; i++) rc.qh[i - 1] = f32_to_f16(std::min(qv[i], 1.0f));
                rc.mask = mask;
            }
            for (int a = 0; a < 3; a++) { rc.ft[a] = Fv[a]; rc.ft[3 + a] = 0; }
            if (solid_now) {
                rc.ft[3] = pc[1] * Fv[2] - pc[2] * Fv[1];
                rc.ft[4] = pc[2] * Fv[0] - pc[0] * Fv[2];
                rc.ft[5] = pc[0] * Fv[1] - pc[1] * Fv[0];
            }
        }
        // refill of the cells the part uncovered
        for (uint32_t k = 0; k < (uint32_t)nb; k++) {
            const int lx = (int)(k % box_n[0]), ly = (int)((k / box_n[0]) % box_n[1]), lz = (int)(k / (box_n[0] * box_n[1]));
            const int px = lx + box_lo[0], py = ly + box_lo[1], pz = lz + box_lo[2];
            const uint64_t n = ((uint64_t)pz * NY + py) * NX + px;
            if (solid_at(rot, px, py, pz)) continue;
            Rec &rc = recs[k];
            const Real pc[3] = {(Real)px - CENTER[0], (Real)py - CENTER[1], (Real)pz - CENTER[2]};
            Real Fv[3] = {0, 0, 0};
            if (solid_at(rotp, px, py, pz)) {
                Real rs = 0, cnt = 0, pis[6] = {0, 0, 0, 0, 0, 0};
                for (int i = 1; i < 19; i++) {
                    const int nx_ = px + C19[i][0], ny_ = py + C19[i][1], nz_ = pz + C19[i][2];
                    if (solid_at(rot, nx_, ny_, nz_) || solid_at(rotp, nx_, ny_, nz_)) continue;
                    const int qx_ = lx + C19[i][0], qy_ = ly + C19[i][1], qz_ = lz + C19[i][2];
                    if (!(qx_ >= 0 && qy_ >= 0 && qz_ >= 0 && qx_ < (int)box_n[0] && qy_ < (int)box_n[1] && qz_ < (int)box_n[2])) continue;
                    const Rec &r2c = recs[((uint32_t)qz_ * box_n[1] + (uint32_t)qy_) * box_n[0] + (uint32_t)qx_];
                    rs = rs + r2c.macro[0];
                    cnt = cnt + 1;
                    F fp;
                    fp[0] = 0;
                    for (int j = 1; j < 19; j++) fp[j] = r2c.fpost[j];
                    const Mom mo2 = moments(fp);
                    const Real r2 = r2c.macro[0], u2[3] = {r2c.macro[1], r2c.macro[2], r2c.macro[3]};
                    pis[3] = pis[3] + (mo2.s[3] - r2 * u2[0] * u2[1]);
                    pis[4] = pis[4] + (mo2.s[4] - r2 * u2[0] * u2[2]);
                    pis[5] = pis[5] + (mo2.s[5] - r2 * u2[1] * u2[2]);
                    const Real tr = (mo2.s[0] + mo2.s[1] + mo2.s[2]) / (Real)3;
                    const Real uu = dot3(u2, u2);
                    for (int a = 0; a < 3; a++) pis[a] = pis[a] + (mo2.s[a] - tr - r2 * (u2[a] * u2[a] - uu / (Real)3));
                }
                const Real rho = cnt > 0 ? rs / cnt : (Real)1;
                const Real uw[3] = {omega[1] * pc[2] - omega[2] * pc[1], omega[2] * pc[0] - omega[0] * pc[2], omega[0] * pc[1] - omega[1] * pc[0]};
                F fe = feq(rho - (Real)1, uw);
                if (cnt > 0) {
                    for (int j = 0; j < 6; j++) pis[j] = pis[j] / cnt;
                    const F fq = fneq(pis);
                    for (int i = 0; i < 19; i++) fe[i] = fe[i] + fq[i];
                }
                store_out(n, Q, fe, true);
                for (int a = 0; a < 3; a++) Fv[a] = -rho * uw[a];
                for (int i = 1; i < 19; i++) rc.fpost[i] = fe[i];
                rc.macro[0] = rho;
                for (int a = 0; a < 3; a++) rc.macro[1 + a] = uw[a];
            }
            for (int a = 0; a < 3; a++) rc.ft[a] = Fv[a];
            rc.ft[3] = pc[1] * Fv[2] - pc[2] * Fv[1];
            rc.ft[4] = pc[2] * Fv[0] - pc[0] * Fv[2];
            rc.ft[5] = pc[0] * Fv[1] - pc[1] * Fv[0];
            flags[n] = (k + 1u) << 2;
        }
        for (size_t j = 0; j < qscr.size(); j += 3) { qscr[j] = 0x7f7fffffu; qscr[j + 1] = 0; qscr[j + 2] = 0; }
    }

    // one time step (lattice.rs:715-737 for a still geometry); returns the
    // force and moment summed over all records (FP64, record order)
    std::array<double, 6> step(const lbm_step_in &sin) {
        int p = (int)(steps_done % 2);
        seed = (uint32_t)steps_done * STEP_SEED_MUL;  // lattice.rs:676
        Real omega[3] = {(Real)sin.omega[0], (Real)sin.omega[1], (Real)sin.omega[2]};
        if (moving) {
            float rot[9], rotp[9];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) { rot[3 * r + c] = (float)sin.rot[r][c]; rotp[3 * r + c] = (float)sin.rot_prev[r][c]; }
            tri_scatter(rot);
            voxelize(rot, rotp, omega, 1 - p);
        }
        if (!faces.empty()) faces_step(p);
#pragma omp parallel for schedule(static)
        for (long long n = 0; n < (long long)N; n++) main_cell((uint64_t)n, p, omega);
        std::array<double, 6> out{};
        for (auto &r : recs)
            for (int j = 0; j < 6; j++) out[j] += (double)r.ft[j];
        steps_done++;
        return out;
    }

    // CPU-baseline timing only: the collide-stream of one step restricted to
    // the z-planes [z0, z1) (no faces, the step counter is not advanced)
    void step_slab(uint32_t z0, uint32_t z1) {
        int p = (int)(steps_done % 2);
        seed = (uint32_t)steps_done * STEP_SEED_MUL;
        Real omega[3] = {0, 0, 0};
        uint64_t a = (uint64_t)z0 * NX * NY, b = (uint64_t)std::min(z1, NZ) * NX * NY;
#pragma omp parallel for schedule(static)
        for (long long n = (long long)a; n < (long long)b; n++) main_cell((uint64_t)n, p, omega);
    }

    // shader.rs:599-621 / 786-792: (rho, u) between steps, NaN off fluid
    void macros(double *out) const {
        int q = 1 - (int)(steps_done % 2);
#pragma omp parallel for schedule(static)
        for (long long nn = 0; nn < (long long)N; nn++) {
            uint64_t n = (uint64_t)nn;
            uint32_t fg = flags[n];
            double *o = out + 4 * n;
            if (fg & 3u) { o[0] = o[1] = o[2] = o[3] = std::numeric_limits<double>::quiet_NaN(); continue; }
            uint32_t rec = fg >> 2;
            if (rec) { for (int a = 0; a < 4; a++) o[a] = (double)recs[rec - 1].macro[a]; continue; }
            Mom mo = moments(load_prev_out(n, q));
            Real rho = (Real)1 + mo.rho1;
            o[0] = (double)rho;
            for (int a = 0; a < 3; a++) o[1 + a] = (double)(mo.j[a] / rho - (Real)0.5 * GRAV[a]);
        }
    }

    // records in the reference's 40-word layout
    void record_words(uint32_t *out) const {
        for (size_t r = 0; r < recs.size(); r++) {
            uint32_t *w = out + r * RS;
            std::memset(w, 0, RS * 4);
            const Rec &rc = recs[r];
            w[R_MASK] = rc.mask; w[R_CELL] = rc.cell;
            for (int k = 0; k < 9; k++) w[R_Q + k] = (uint32_t)rc.qh[2 * k] | ((uint32_t)rc.qh[2 * k + 1] << 16);
            for (int i = 1; i < 19; i++) w[R_FPOST + i - 1] = fbits((float)rc.fpost[i]);
            for (int a = 0; a < 4; a++) w[R_MACRO + a] = fbits((float)rc.macro[a]);
            for (int a = 0; a < 6; a++) w[R_FT + a] = fbits((float)rc.ft[a]);
        }
    }

    // raw populations as double, slot-major (d * N + cell), unshifted values
    // are f + w; this returns the stored (shifted) values
    void raw(double *out) const {
        for (int d = 0; d < 19; d++)
            for (uint64_t n = 0; n < N; n++) out[(uint64_t)d * N + n] = (double)L(d, n);
    }
};

}  // namespace oracle
