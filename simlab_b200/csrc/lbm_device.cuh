// Device-side building blocks of the D3Q19 time step: the velocity set,
// population storage formats (FP32 / FP64 / FP16 / BF16 deviations from the
// weights), stochastic rounding, launch parameters, record access and the
// AA-pattern access functions.
//
// Reference semantics: crates/cfd/src/shader.rs (velocity set 22-60, record
// layout 62-69, storage 147-162, stochastic rounding 507-517, AA access
// 254-339).
//
// HBM layout: the 19 population planes are stored slot-major like the
// reference (direction d of cell n at d * NP + n), with the plane stride NP
// rounded up to 256 cells so every plane starts 512-byte aligned, and guard
// zones before the first and after the last plane so the shifted ranges the
// bulk copies fetch for a tile never leave the allocation.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbm {

// ------------------------------------------------------------ velocity set
// D3Q19 in the reference's order: rest, +-x, +-y, +-z, then the 12 edges
// (shader.rs:22-42); opposite directions are neighbours (shader.rs:44-52), so
// the 9 pairs (2k+1, 2k+2) each hold a velocity and its opposite.
__host__ __device__ __forceinline__ constexpr int CX(int i) {
    return (i == 1 || i == 7 || i == 9 || i == 13 || i == 15) ? 1 : ((i == 2 || i == 8 || i == 10 || i == 14 || i == 16) ? -1 : 0);
}
__host__ __device__ __forceinline__ constexpr int CY(int i) {
    return (i == 3 || i == 7 || i == 11 || i == 14 || i == 17) ? 1 : ((i == 4 || i == 8 || i == 12 || i == 13 || i == 18) ? -1 : 0);
}
__host__ __device__ __forceinline__ constexpr int CZ(int i) {
    return (i == 5 || i == 9 || i == 11 || i == 16 || i == 18) ? 1 : ((i == 6 || i == 10 || i == 12 || i == 15 || i == 17) ? -1 : 0);
}
__host__ __device__ __forceinline__ constexpr int OPP(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
__host__ __device__ __forceinline__ constexpr double WD(int i) { return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }
// The store mask of a planar cell of face F (0..5: -x, +x, -y, +y, -z, +z)
// away from the face's edges: the five directions pointing into the domain.
__host__ __device__ __forceinline__ constexpr uint32_t planar_mask(int F) {
    uint32_t m = 0;
    for (int i = 0; i < 19; i++) {
        const int c = (F >> 1) == 0 ? CX(i) : ((F >> 1) == 1 ? CY(i) : CZ(i));
        if (c == ((F & 1) ? -1 : 1)) m |= 1u << i;
    }
    return m;
}
__host__ __device__ __forceinline__ constexpr int DIR(int x, int y, int z) {
    int r = 0;
    for (int i = 0; i < 19; i++)
        if (CX(i) == x && CY(i) == y && CZ(i) == z) r = i;
    return r;
}

// FP16 storage scale (shader.rs:73) and the step seed multiplier of the
// stochastic rounding (lattice.rs:676: seed = step * 2654435761)
constexpr float FP16_SCALE = 32768.0f;
constexpr uint32_t STEP_SEED_MUL = 2654435761u;

// record layout (u32 words per wall record), shader.rs:62-69
constexpr uint32_t RS = 40, R_MASK = 0, R_CELL = 1, R_Q = 2, R_FPOST = 11, R_MACRO = 29, R_FT = 33;
// FP64 engine keeps the float fields of a record in doubles: 18 fpost, 4 macro, 6 ft
constexpr uint32_t RD = 28, RD_FPOST = 0, RD_MACRO = 18, RD_FT = 22;

constexpr int BLOCK = 256;
#ifndef LBM_WBLOCK
#define LBM_WBLOCK 64
#endif
constexpr int WBLOCK = LBM_WBLOCK;  // threads per block of the wall-cell kernel
// flag bit of a fluid cell whose x neighbour is a planar x-face cell it feeds
constexpr uint32_t FLAG_XFACE = 0x80000000u;
// wall-record indices stay below 2^29, so the record field ((r + 1) << 2)
// never reaches FLAG_XFACE
constexpr uint32_t MAX_RECORDS = (1u << 29) - 2;
constexpr uint32_t PLANE_ALIGN = 256;  // cells
constexpr uint32_t TILE_MAX = 4096;    // cells of the staged kernel's largest tile (allocation guards)

// error bits set by kernels (read by the host after each chunk)
constexpr uint32_t ERR_COPY_WAIT = 1u;  // a bulk-copy wait passed its iteration limit

// ------------------------------------------------------------ fast division
// Unsigned 32-bit division by a run-time constant with a multiply-high
// (Granlund & Montgomery 1994, round-up multiplier with a 33-bit add):
// q = (umulhi(n, m) + n) >> s, exact for every 32-bit n.
struct FastDiv {
    uint32_t d, m, s;
    __host__ void init(uint32_t div) {
        d = div;
        s = 0;
        while ((1ull << s) < div) s++;
        m = (uint32_t)((((1ull << s) - div) << 32) / div + 1);
        if (div == 1) { m = 0; s = 0; }
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
        const uint32_t hi = __umulhi(n, m);
#else
        const uint32_t hi = (uint32_t)(((uint64_t)n * m) >> 32);
#endif
        return (uint32_t)(((uint64_t)hi + n) >> s);
    }
};

// ------------------------------------------------------------ launch params
template <class R>
struct Consts {
    R tau0, smag2, sponge_tau, sigma;
    R sp_lo[3], sp_hi[3], u_inf[3], u_init[3], grav[3], center[3];
    R sp_lo_inv[3], sp_hi_inv[3];  // reciprocal sponge widths (0 where no sponge)
    // shifted equilibrium at rest density and u_inf: the absorbing target when
    // absorb_velocity (rest, then the even and odd parts of the 9 pairs)
    R ft_rest, ft_even[9], ft_odd[9];
};

struct LatParams {
    void *pop;                 // plane 0 of 19 planes, plane stride NP cells
    uint32_t *flags;           // N words: 0 fluid, 1 solid, 2/3 face, (rec+1)<<2 wall cell
    uint32_t *recs;            // nrec * RS words
    double *recd;              // FP64 engine: nrec * RD doubles (else null)
    const uint32_t *faces;     // face cells
    const uint32_t *face_info; // kind (0 velocity, 1 open, 2 free slip) | mirror axes << 2 | store mask << 8
    double *partials;          // per wall block: 8 doubles
    uint32_t *ticket;          // last-block counter of the force reduction
    double *hist;              // per step slot: 8 doubles (F, T)
    float4 *dump;              // macros() output
    uint32_t *err;             // error bits (ERR_*)
    uint64_t NP;               // plane stride (cells)
    uint32_t NX, NY, NZ, N;
    FastDiv div_nx, div_nxy;
    uint32_t nrec, nface;
    int per[3];
    int abs_u, total_p, wall_model, forcing, sponge_on, les_on, moving;
    uint32_t sp_w[6];          // sponge widths in cells, -x,+x,-y,+y,-z,+z
    const float *sp_tab;       // sponge ramp per x, then per y, then per z (NX + NY + NZ values)
    const double *sp_tabd;     // the same in FP64
    uint32_t xface_info[2];    // face info (kind | mirror << 2) of the -x and +x faces, for fused x faces
    // The face list is ordered planar cells of faces 0..5 (velocity or open
    // faces whose store mask is planar_mask(F), in-plane axes not periodic),
    // then the rest (edges, corners, free slip), then fused x-face cells.
    // fplan[F]: first list index of group F (F = 6: the rest); fblk[F]: the
    // face kernel's first block for group F.
    uint32_t fplan[7], fblk[7];
    // A planar group of a y or z face that lists its whole rectangle in cell
    // order (frect[F] = 1): cell k of the group is frect_b0 + u + v frect_sv
    // with k = v nu + u, nu = frect_nu.d, so the face kernel computes it and
    // the group's info (finfo[F]) instead of loading them.
    uint32_t frect[6], frect_b0[6], frect_sv[6], finfo[6];
    FastDiv frect_nu[6];
    int tma;                   // the staged bulk kernel applies (NX * element size % 16 == 0)
    // spinning part (Geometry::Spin, lattice.rs:87-92): every cell of the swept
    // box is a record, re-voxelized each step from the rotated surface
    const uint32_t *occ;       // body-frame occupancy bits on a fine grid
    float occ_lo[3];
    float occ_invh;
    int32_t occ_n[3];
    const float4 *tris;        // 3 per triangle: v0, e1, e2 (body frame)
    uint32_t ntri;
    int32_t box_lo[3];
    uint32_t box_n[3];
    uint32_t *qscr;            // 9 links x (nearest t, farthest t, hits) per box cell
    Consts<float> kf;
    Consts<double> kd;
};

struct StepParams {
    uint32_t seed;   // stochastic rounding seed of this step (lattice.rs:676)
    uint32_t seed_mix;  // seed * 0x85EBCA77 + 0x632BE5AB, the seed's term of sr_hash
    uint32_t next_seed_mix;  // the same for the next step
    uint32_t nface;          // face cells the face kernel handles this step
    uint32_t slot;   // history slot of this step
    float omega[3];  // angular velocity, rad per step
    double omega_d[3];
    float rot[9];    // body axes in lattice coordinates, row-major (columns = axes)
    float rot_prev[9];  // the same for the previous step
};

template <class R> __device__ __forceinline__ const Consts<R> &K(const LatParams &p);
template <> __device__ __forceinline__ const Consts<float> &K<float>(const LatParams &p) { return p.kf; }
template <> __device__ __forceinline__ const Consts<double> &K<double>(const LatParams &p) { return p.kd; }

// ------------------------------------------------------------ rounding
// Stochastic rounding (shader.rs:507-517): a value is rounded up with
// probability equal to its fractional part in units of the target format's
// last place, so slow changes below half an ulp still accumulate.  The
// reference adds uniform noise in [-1/2, 1/2) ulp from an integer hash of
// (cell * 19 + slot, step seed) and rounds to nearest.  Here the same
// distribution comes from the conversion instruction of sm_100a that rounds
// stochastically (cvt.rs): it adds random bits just below the destination's
// last place of the magnitude and truncates.  The random bits come from one
// hash per cell (the reference's mixer keyed by the cell and the step seed),
// spread over the cell's values by multiplication or by a 32-bit linear
// congruential sequence (Numerical Recipes constants).
__host__ __device__ __forceinline__ uint32_t sr_hash(uint32_t key, uint32_t seed) {
    uint32_t h = (key * 0x9E3779B1u) ^ (seed * 0x85EBCA77u + 0x632BE5ABu);
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    return h;
}
__device__ __forceinline__ uint32_t sr_hash_mix(uint32_t key, uint32_t mix) {
    uint32_t h = (key * 0x9E3779B1u) ^ mix;
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    return h;
}
struct Rng {
    uint32_t s;
    __device__ __forceinline__ uint32_t next() {
        s = s * 1664525u + 1013904223u;
        return s;
    }
    // a step whose two 16-bit halves are both usable as random fields (the
    // low bits of the sequence alone repeat with short periods)
    __device__ __forceinline__ uint32_t next2() {
        const uint32_t x = next();
        return x ^ (x >> 16);
    }
};

// {hi, lo} = two binary16 values rounded stochastically from a and b,
// saturating at the largest finite value.  The random field of a is
// rbits[28:16], that of b rbits[12:0]: with m the magnitude's bits below the
// binary16 last place (13 for a normal result, more for a subnormal one, kept
// to 13 places below it), the magnitude is rounded up when m + field carries
// into the last place.  Measured on B200 against this model, bit for bit, for
// normal, subnormal, overflowing and special inputs.
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float a, float b, uint32_t rbits) {
    uint32_t d;
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
    return d;
}
// the bfloat16 form: 16-bit fields, rbits[31:16] for a and rbits[15:0] for b
__device__ __forceinline__ uint32_t cvt_rs_bf16x2(float a, float b, uint32_t rbits) {
    uint32_t d;
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
    return d;
}
// Random bits for the pair K of a cell whose hash is h: the low and high
// words of the 64-bit product h * A_K (A_K odd, one per pair) exclusive-ored,
// so every field mixes the carries of the whole product and the pairs of a
// cell draw on different multipliers without a dependency chain.  (Either
// word alone is not enough: the low word's low bits depend only on the low
// bits of h, and the high word's are nearly the same function of h for every
// multiplier.)  Over 4e5 hashes the 19 fields of a cell correlate by at most
// 0.004 and the rounding variance of the cell's mass, momentum and stress
// equals that of independent fields.
template <int K>
__device__ __forceinline__ uint32_t pair_bits(uint32_t h) {
    constexpr uint32_t A[12] = {0x9E3779B1u, 0x85EBCA77u, 0xC2B2AE3Du, 0x27D4EB2Fu, 0x165667B1u, 0x7FEB352Du,
                                0x846CA68Bu, 0xCC9E2D51u, 0x1B873593u, 0xE6546B65u, 0x2C1B3C6Du, 0x297A2D39u};
    static_assert(K >= 0 && K < 12, "pair index");
    const uint64_t p = (uint64_t)h * A[K];
    return (uint32_t)p ^ (uint32_t)(p >> 32);
}

// FP16 stores (f - w) * 32768 (binary16's range holds the deviations with
// the scale; values beyond it saturate)
__device__ __forceinline__ __half sr_f16(float v, Rng &r) {
    return __ushort_as_half((unsigned short)(cvt_rs_f16x2(v * FP16_SCALE, 0.0f, r.next()) >> 16));
}
// BF16 stores (f - w) as is
__device__ __forceinline__ __nv_bfloat16 sr_bf16(float v, Rng &r) {
    return __ushort_as_bfloat16((unsigned short)(cvt_rs_bf16x2(v, 0.0f, r.next()) >> 16));
}

// ------------------------------------------------------------ storage
template <class S> struct Pop;
template <> struct Pop<float> {
    using real = float;
    static __device__ __forceinline__ float cvt(float v) { return v; }
    static __device__ __forceinline__ float ld(const float *p) { return *p; }
    static __device__ __forceinline__ float enc(float v, Rng &) { return v; }
};
template <> struct Pop<double> {
    using real = double;
    static __device__ __forceinline__ double cvt(double v) { return v; }
    static __device__ __forceinline__ double ld(const double *p) { return *p; }
    static __device__ __forceinline__ double enc(double v, Rng &) { return v; }
};
// 2-byte formats also round two values at once: rs2(a, b, bits) = {hi, lo}
// in storage units (values already scaled), bits(x) reinterprets 16 bits
template <> struct Pop<__half> {
    using real = float;
    static __device__ __forceinline__ float cvt(__half v) { return __half2float(v) * (1.0f / FP16_SCALE); }
    static __device__ __forceinline__ float ld(const __half *p) { return cvt(*p); }
    static __device__ __forceinline__ __half enc(float v, Rng &r) { return sr_f16(v, r); }
    static __device__ __forceinline__ uint32_t rs2(float a, float b, uint32_t bits) { return cvt_rs_f16x2(a, b, bits); }
    static __device__ __forceinline__ __half bits(uint32_t x) { return __ushort_as_half((unsigned short)x); }
};
template <> struct Pop<__nv_bfloat16> {
    using real = float;
    static __device__ __forceinline__ float cvt(__nv_bfloat16 v) { return __bfloat162float(v); }
    static __device__ __forceinline__ float ld(const __nv_bfloat16 *p) { return cvt(*p); }
    static __device__ __forceinline__ __nv_bfloat16 enc(float v, Rng &r) { return sr_bf16(v, r); }
    static __device__ __forceinline__ uint32_t rs2(float a, float b, uint32_t bits) { return cvt_rs_bf16x2(a, b, bits); }
    static __device__ __forceinline__ __nv_bfloat16 bits(uint32_t x) { return __ushort_as_bfloat16((unsigned short)x); }
};

// ------------------------------------------------------------ records
template <class R> struct Rec;
template <> struct Rec<float> {
    static __device__ __forceinline__ float fpost(const LatParams &p, uint32_t r, int i) { return __uint_as_float(p.recs[r * RS + R_FPOST + i - 1]); }
    static __device__ __forceinline__ void set_fpost(const LatParams &p, uint32_t r, int i, float v) { p.recs[r * RS + R_FPOST + i - 1] = __float_as_uint(v); }
    static __device__ __forceinline__ float macro(const LatParams &p, uint32_t r, int a) { return __uint_as_float(p.recs[r * RS + R_MACRO + a]); }
    static __device__ __forceinline__ void set_macro(const LatParams &p, uint32_t r, int a, float v) { p.recs[r * RS + R_MACRO + a] = __float_as_uint(v); }
    static __device__ __forceinline__ float ft(const LatParams &p, uint32_t r, int a) { return __uint_as_float(p.recs[r * RS + R_FT + a]); }
    static __device__ __forceinline__ void set_ft(const LatParams &p, uint32_t r, int a, float v) { p.recs[r * RS + R_FT + a] = __float_as_uint(v); }
};
template <> struct Rec<double> {
    static __device__ __forceinline__ double fpost(const LatParams &p, uint32_t r, int i) { return p.recd[r * RD + RD_FPOST + i - 1]; }
    static __device__ __forceinline__ void set_fpost(const LatParams &p, uint32_t r, int i, double v) {
        p.recd[r * RD + RD_FPOST + i - 1] = v;
        p.recs[r * RS + R_FPOST + i - 1] = __float_as_uint((float)v);
    }
    static __device__ __forceinline__ double macro(const LatParams &p, uint32_t r, int a) { return p.recd[r * RD + RD_MACRO + a]; }
    static __device__ __forceinline__ void set_macro(const LatParams &p, uint32_t r, int a, double v) {
        p.recd[r * RD + RD_MACRO + a] = v;
        p.recs[r * RS + R_MACRO + a] = __float_as_uint((float)v);
    }
    static __device__ __forceinline__ double ft(const LatParams &p, uint32_t r, int a) { return p.recd[r * RD + RD_FT + a]; }
    static __device__ __forceinline__ void set_ft(const LatParams &p, uint32_t r, int a, double v) {
        p.recd[r * RD + RD_FT + a] = v;
        p.recs[r * RS + R_FT + a] = __float_as_uint((float)v);
    }
};

// q of direction i (1..18) from the f16 pairs of a record
__device__ __forceinline__ float rec_q(const uint32_t *recs, uint32_t r, int i) {
    uint32_t w = recs[r * RS + R_Q + (i - 1) / 2];
    uint16_t h = ((i - 1) & 1) ? (uint16_t)(w >> 16) : (uint16_t)(w & 0xffffu);
    return __half2float(__ushort_as_half(h));
}

// ------------------------------------------------------------ neighbours
// Offsets of the six axis neighbours with periodic wrap (shader.rs:247-252).
struct Nb {
    int32_t xp, xm, yp, ym, zp, zm;
    __device__ __forceinline__ int32_t off(int dx, int dy, int dz) const {
        return (dx == 1 ? xp : (dx == -1 ? xm : 0)) + (dy == 1 ? yp : (dy == -1 ? ym : 0)) + (dz == 1 ? zp : (dz == -1 ? zm : 0));
    }
};
__device__ __forceinline__ Nb make_nb(const LatParams &p, uint32_t x, uint32_t y, uint32_t z) {
    Nb b;
    const int32_t nx = (int32_t)p.NX, nxy = (int32_t)(p.NX * p.NY);
    b.xp = x == p.NX - 1 ? -(nx - 1) : 1;
    b.xm = x == 0 ? (nx - 1) : -1;
    b.yp = y == p.NY - 1 ? -(int32_t)(p.NY - 1) * nx : nx;
    b.ym = y == 0 ? (int32_t)(p.NY - 1) * nx : -nx;
    b.zp = z == p.NZ - 1 ? -(int32_t)(p.NZ - 1) * nxy : nxy;
    b.zm = z == 0 ? (int32_t)(p.NZ - 1) * nxy : -nxy;
    return b;
}

__device__ __forceinline__ void coords(const LatParams &p, uint32_t n, uint32_t &x, uint32_t &y, uint32_t &z) {
    z = p.div_nxy.div(n);
    const uint32_t r = n - z * (p.NX * p.NY);
    y = p.div_nx.div(r);
    x = r - y * p.NX;
}

// ------------------------------------------------------------ AA access
// Input parity P (shader.rs:5-13): before a step of parity P the population
// arriving at cell n in direction i sits at P=0: (n, i), P=1: (n - c_i, opp i);
// the step writes its post-collision values to P=0: (n, opp i),
// P=1: (n + c_i, i).
template <class S, int P>
__device__ __forceinline__ void load_in(const LatParams &p, uint32_t n, const Nb &nb, typename Pop<S>::real *f) {
    const S *pop = (const S *)p.pop;
    const uint64_t NP = p.NP;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        if (P == 0 || i == 0) f[i] = Pop<S>::ld(pop + (uint64_t)i * NP + n);
        else f[i] = Pop<S>::ld(pop + (uint64_t)OPP(i) * NP + (uint32_t)((int32_t)n + nb.off(-CX(i), -CY(i), -CZ(i))));
    }
}

template <class S, int P>
__device__ __forceinline__ void store_out(const LatParams &p, uint32_t n, const Nb &nb, const typename Pop<S>::real *f, Rng &rng) {
    S *pop = (S *)p.pop;
    const uint64_t NP = p.NP;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        if (P == 0 || i == 0) pop[(uint64_t)OPP(i) * NP + n] = Pop<S>::enc(f[i], rng);
        else pop[(uint64_t)i * NP + (uint32_t)((int32_t)n + nb.off(CX(i), CY(i), CZ(i)))] = Pop<S>::enc(f[i], rng);
    }
}

// the post-collision populations a cell wrote in the previous step of
// parity Q (shader.rs:307-321)
template <class S, int Q>
__device__ __forceinline__ void load_prev_out(const LatParams &p, uint32_t n, const Nb &nb, typename Pop<S>::real *f) {
    const S *pop = (const S *)p.pop;
    const uint64_t NP = p.NP;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        if (Q == 0 || i == 0) f[i] = Pop<S>::ld(pop + (uint64_t)OPP(i) * NP + n);
        else f[i] = Pop<S>::ld(pop + (uint64_t)i * NP + (uint32_t)((int32_t)n + nb.off(CX(i), CY(i), CZ(i))));
    }
}

// writes a face cell's "previous" post-collision populations for parity Q
// (shader.rs:273-305).  Only the directions in `mask` are written: those
// that stream into a cell that collides.  The rest (leaving a non-periodic
// domain, or entering another face cell, which never collides) are read by
// no one.
template <class S, int Q>
__device__ __forceinline__ void store_prev_out(const LatParams &p, uint32_t n, const Nb &nb, uint32_t mask,
                                               const typename Pop<S>::real *f, Rng &rng) {
    S *pop = (S *)p.pop;
    const uint64_t NP = p.NP;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        if (!(mask & (1u << i))) continue;
        const auto v = Pop<S>::enc(f[i], rng);
        if (Q == 0 || i == 0) pop[(uint64_t)OPP(i) * NP + n] = v;
        else pop[(uint64_t)i * NP + (uint32_t)((int32_t)n + nb.off(CX(i), CY(i), CZ(i)))] = v;
    }
}

// ------------------------------------------------------------ projections
template <class R>
__device__ __forceinline__ R cdot(int i, R ux, R uy, R uz) {
    R t = 0;
    if (CX(i) == 1) t = t + ux; else if (CX(i) == -1) t = t - ux;
    if (CY(i) == 1) t = t + uy; else if (CY(i) == -1) t = t - uy;
    if (CZ(i) == 1) t = t + uz; else if (CZ(i) == -1) t = t - uz;
    return t;
}

// shifted equilibrium w (rho1 + rho (3cu + 4.5cu^2 - 1.5u^2)), shader.rs:367-377
template <class R>
__device__ __forceinline__ R feq_i(int i, R rho1, R rho, R ux, R uy, R uz, R usq) {
    R cu = cdot<R>(i, ux, uy, uz);
    return (R)WD(i) * (rho1 + rho * ((R)3 * cu + (R)4.5 * cu * cu - usq));
}

// 4.5 w (c c : Pi - tr Pi / 3), shader.rs:379-396; pi = xx yy zz xy xz yz
template <class R>
__device__ __forceinline__ R fneq_i(int i, const R *pi, R tr) {
    R t = -tr;
    if (CX(i) != 0) t = t + pi[0];
    if (CY(i) != 0) t = t + pi[1];
    if (CZ(i) != 0) t = t + pi[2];
    if (CX(i) * CY(i) != 0) t = t + (R)(2 * CX(i) * CY(i)) * pi[3];
    if (CX(i) * CZ(i) != 0) t = t + (R)(2 * CX(i) * CZ(i)) * pi[4];
    if (CY(i) * CZ(i) != 0) t = t + (R)(2 * CY(i) * CZ(i)) * pi[5];
    return (R)(4.5 * WD(i)) * t;
}

template <class R>
struct Moments {
    R rho1, jx, jy, jz, sxx, syy, szz, sxy, sxz, syz;
};

// shader.rs:341-365, from the sums s_k and differences d_k of the 9
// opposite pairs (2k+1, 2k+2)
template <class R>
__device__ __forceinline__ Moments<R> moments_sd(R f0, const R *s, const R *d) {
    Moments<R> m;
    m.rho1 = f0 + ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7])) + s[8];
    // odd members: 1 (1,0,0) 3 (0,1,0) 5 (0,0,1) 7 (1,1,0) 9 (1,0,1) 11 (0,1,1) 13 (1,-1,0) 15 (1,0,-1) 17 (0,1,-1)
    m.jx = (d[0] + d[3]) + (d[4] + d[6]) + d[7];
    m.jy = (d[1] + d[3]) + (d[5] - d[6]) + d[8];
    m.jz = (d[2] + d[4]) + (d[5] - d[7]) - d[8];
    m.sxx = (s[0] + s[3]) + (s[4] + s[6]) + s[7];
    m.syy = (s[1] + s[3]) + (s[5] + s[6]) + s[8];
    m.szz = (s[2] + s[4]) + (s[5] + s[7]) + s[8];
    m.sxy = s[3] - s[6];
    m.sxz = s[4] - s[7];
    m.syz = s[5] - s[8];
    return m;
}
template <class R>
__device__ __forceinline__ Moments<R> moments(const R *f) {
    R s[9], d[9];
#pragma unroll
    for (int k = 0; k < 9; k++) { s[k] = f[2 * k + 1] + f[2 * k + 2]; d[k] = f[2 * k + 1] - f[2 * k + 2]; }
    return moments_sd<R>(f[0], s, d);
}

// shader.rs:818-824: non-equilibrium stress from shifted moments
template <class R>
__device__ __forceinline__ void pi_neq(const Moments<R> &m, R rho, R ux, R uy, R uz, R *pi) {
    const R r3 = m.rho1 / (R)3;
    pi[0] = m.sxx - rho * ux * ux - r3;
    pi[1] = m.syy - rho * uy * uy - r3;
    pi[2] = m.szz - rho * uz * uz - r3;
    pi[3] = m.sxy - rho * ux * uy;
    pi[4] = m.sxz - rho * ux * uz;
    pi[5] = m.syz - rho * uy * uz;
}

// shader.rs:528-538: the sponge factor is the largest of six ramps, each
// depending on one coordinate, so it is the largest of three per-axis values
// tabulated at setup with the reference's arithmetic (1 - p / width)
template <class R> __device__ __forceinline__ const R *sp_table(const LatParams &p);
template <> __device__ __forceinline__ const float *sp_table<float>(const LatParams &p) { return p.sp_tab; }
template <> __device__ __forceinline__ const double *sp_table<double>(const LatParams &p) { return p.sp_tabd; }
template <class R>
__device__ __forceinline__ R sponge_at(const Consts<R> &, const LatParams &p, uint32_t x, uint32_t y, uint32_t z) {
    const R *t = sp_table<R>(p);
    return max(max(__ldg(t + x), __ldg(t + p.NX + y)), __ldg(t + p.NX + p.NY + z));
}

}  // namespace lbm
