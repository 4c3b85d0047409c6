// The static voxelizer on the GPU: voxelize_static / voxelize_static27
// (crates/cfd/src/voxel.rs:73-216 inside_grid, 218-296 bins, 298-326
// seg_tri, 361-490 voxelize_links), the same algorithm as the host
// restatement in voxel.cpp, with the same FP64 operations in the same order.
// The file is compiled without floating-point contraction (-fmad=false), so
// every product and sum rounds as on the host, and the solid cells and wall
// links are bit-identical to voxel.cpp's.
//
//  * inside_grid, per axis a (b = a+1, c = a+2 mod 3): one thread per
//    triangle finds the scan lines (j, k) its projection covers and the
//    crossing (t along a, orientation w), counted then written per line;
//    one thread per line sorts its crossings by t, picks the rule (winding
//    number for consistently oriented lines, parity for the others, no vote
//    for an odd count) and marks the line's points.  A point is inside when
//    most of its valid votes say so.
//  * bins: triangles listed per unit bin of their grown bounding box (count,
//    scan, fill; the order within a bin does not matter, as only the
//    nearest and farthest hit and the hit count are used).
//  * links: one thread per fluid cell of the part's region that has
//    triangles nearby or a solid neighbour: per direction the segment tests
//    against the bin's triangles, the cut link with q from the nearest hit
//    (0.5 without a hit), and a thin-sheet link (two hits, neighbour fluid)
//    whose reciprocal link the next pass gives the neighbour unless the
//    neighbour has that link already.
#include <cuda_runtime.h>
#include <thrust/copy.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/scan.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_wait.hpp"
#include "voxel.hpp"

namespace lbm {
namespace vg {

constexpr double EPS_B = 1.2345671e-5;  // voxel.rs:68-71, as voxel.cpp
constexpr double EPS_C = 2.7182818e-5;
constexpr int T = 256;

// std::min / std::max on doubles (the first argument when neither is smaller)
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

struct Region {
    int64_t slo[3];       // region point 0 in lattice cells (may be -1)
    uint32_t gd[3];       // region points per axis
    uint32_t dims[3];     // lattice
};

__device__ __forceinline__ uint64_t rid(const Region &r, uint64_t i, uint64_t j, uint64_t k) {
    return (k * r.gd[1] + j) * r.gd[0] + i;
}
__device__ __forceinline__ bool in_domain(const Region &r, int64_t i, int64_t j, int64_t k) {
    const int64_t p[3] = {i + r.slo[0], j + r.slo[1], k + r.slo[2]};
    for (int a = 0; a < 3; a++)
        if (p[a] < 0 || p[a] >= (int64_t)r.dims[a]) return false;
    return true;
}

// ------------------------------------------------------------ inside_grid
// crossings of the scan lines along axis a by triangle t (voxel.cpp
// parity_axis): FILL = false counts them per line, FILL = true writes them
template <bool FILL>
__global__ void __launch_bounds__(T) kv_crossings(const double *gv, const uint32_t *tris, uint32_t nt, int a, Region r, uint32_t *count,
                                                  const uint64_t *offs, double *ht, int8_t *hw) {
    const uint32_t t = blockIdx.x * T + threadIdx.x;
    if (t >= nt) return;
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    const uint32_t nb = r.gd[b], nc = r.gd[c];
    const uint32_t ids[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
    double p[3][3];
    for (int q = 0; q < 3; q++)
        for (int k = 0; k < 3; k++) p[q][k] = gv[3 * (uint64_t)ids[q] + k];
    double lo = INFINITY, hi = -INFINITY;
    for (int v = 0; v < 3; v++) { lo = dmin(lo, p[v][c]); hi = dmax(hi, p[v][c]); }
    const double k0f = dmax(ceil(lo - EPS_C), 0.0);
    const double k1f = floor(hi - EPS_C);
    if (k1f < 0.0 || nc == 0 || nb == 0) return;
    const uint64_t k0 = (uint64_t)k0f, k1 = min((uint64_t)k1f, (uint64_t)nc - 1);
    double blo = INFINITY, bhi = -INFINITY;
    for (int q = 0; q < 3; q++) { blo = dmin(blo, p[q][b]); bhi = dmax(bhi, p[q][b]); }
    const double j0f = dmax(ceil(blo - EPS_B), 0.0);
    const double j1f = floor(bhi - EPS_B);
    if (j1f < 0.0) return;
    const uint64_t j0 = (uint64_t)j0f, j1 = min((uint64_t)j1f, (uint64_t)nb - 1);
    for (uint64_t k = k0; k <= k1 && k < nc; k++) {
        const double pc = (double)k + EPS_C;
        for (uint64_t j = j0; j <= j1; j++) {
            const double pb = (double)j + EPS_B;
            // edge functions with the vertices in canonical (index) order, so a
            // line through a shared edge counts one crossing
            auto e = [&](int u, int v) -> double {
                const double *pu, *pv;
                double sg;
                if (ids[u] < ids[v]) { pu = p[u]; pv = p[v]; sg = 1.0; } else { pu = p[v]; pv = p[u]; sg = -1.0; }
                return sg * ((pv[b] - pu[b]) * (pc - pu[c]) - (pv[c] - pu[c]) * (pb - pu[b]));
            };
            const double e0 = e(1, 2), e1 = e(2, 0), e2 = e(0, 1);
            const bool inside = (e0 > 0.0 && e1 > 0.0 && e2 > 0.0) || (e0 < 0.0 && e1 < 0.0 && e2 < 0.0);
            if (!inside) continue;
            const uint64_t line = k * nb + j;
            const uint32_t slot = atomicAdd(&count[line], 1u);
            if (FILL) {
                const double sum = e0 + e1 + e2;
                ht[offs[line] + slot] = (e0 * p[0][a] + e1 * p[1][a] + e2 * p[2][a]) / sum;
                hw[offs[line] + slot] = sum > 0.0 ? 1 : -1;
            }
        }
    }
}

// one scan line (j, k) along axis a: its crossings sorted by t, the rule, and
// the votes of its points (voxel.cpp mark_line).  Bits: 1 << a inside,
// 1 << (3 + a) a valid vote.  Each launch handles one axis, whose lines do
// not share points, so the votes need no atomics.
__global__ void __launch_bounds__(T) kv_lines(int a, Region r, const uint32_t *count, const uint64_t *offs, double *ht, int8_t *hw,
                                              uint8_t *votes) {
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    const uint64_t nb = r.gd[b], nc = r.gd[c], na = r.gd[a];
    const uint64_t line = (uint64_t)blockIdx.x * T + threadIdx.x;
    if (line >= nb * nc) return;
    const uint64_t j = line % nb, k = line / nb;
    const uint32_t nl = count[line];
    double *t = ht + offs[line];
    int8_t *w = hw + offs[line];
    // insertion sort by t (the order among equal t does not change a vote)
    for (uint32_t q = 1; q < nl; q++) {
        const double tv = t[q];
        const int8_t wv = w[q];
        uint32_t s = q;
        while (s > 0 && tv < t[s - 1]) { t[s] = t[s - 1]; w[s] = w[s - 1]; s--; }
        t[s] = tv;
        w[s] = wv;
    }
    int wsum = 0;
    for (uint32_t q = 0; q < nl; q++) wsum += w[q];
    // no crossing: a valid outside vote; consistently oriented: winding rule;
    // otherwise parity when the count is even, no vote when it is odd
    const int mode = nl == 0 ? 1 : (wsum == 0 ? 1 : (nl % 2 == 0 ? 2 : 0));
    if (mode == 0) return;
    const uint8_t vbit = (uint8_t)(1u << (3 + a)), ibit = (uint8_t)(1u << a);
    uint32_t h = 0;
    int wind = 0;
    uint64_t pos[3];
    pos[b] = j;
    pos[c] = k;
    for (uint64_t i = 0; i < na; i++) {
        const double ta = (double)i;
        while (h < nl && t[h] < ta) { wind += w[h]; h++; }
        pos[a] = i;
        const bool ins = mode == 1 ? wind != 0 : (h % 2 == 1);
        votes[rid(r, pos[0], pos[1], pos[2])] |= (uint8_t)(vbit | (ins ? ibit : 0u));
    }
}

// inside = most valid votes say inside; also the region point's solid flag
__global__ void __launch_bounds__(T) kv_inside(uint64_t n, const uint8_t *votes, uint8_t *inside) {
    const uint64_t l = (uint64_t)blockIdx.x * T + threadIdx.x;
    if (l >= n) return;
    const uint32_t v = votes[l];
    const uint32_t valid = (v >> 3) & 7u, ins = v & 7u & valid;
    const int nv = __popc(valid), ni = __popc(ins);
    inside[l] = (nv > 0 && 2 * ni > nv) ? 1 : 0;
}

// ------------------------------------------------------------ bins
// voxel.cpp build_bins: the unit bins (origin lo, dims gd) a triangle's
// bounding box grown by `dilate` covers; false when it covers none
__device__ __forceinline__ bool bin_range(const double *verts, const uint32_t *tri, const double *lo, const uint32_t *gd, double dilate,
                                          uint64_t *r0, uint64_t *r1) {
    for (int k = 0; k < 3; k++) {
        double mn = INFINITY, mx = -INFINITY;
        for (int v = 0; v < 3; v++) { mn = dmin(mn, verts[3 * (uint64_t)tri[v] + k]); mx = dmax(mx, verts[3 * (uint64_t)tri[v] + k]); }
        mn = mn - dilate - lo[k];
        mx = mx + dilate - lo[k];
        if (mx < 0.0 || mn >= (double)gd[k]) return false;
        r0[k] = (uint64_t)dmax(floor(mn), 0.0);
        r1[k] = min((uint64_t)floor(mx), (uint64_t)gd[k] - 1);
    }
    return true;
}

struct BinSpec {
    double lo[3];
    uint32_t gd[3];
    double dilate;
};

template <bool FILL>
__global__ void __launch_bounds__(T) kv_bins(const double *verts, const uint32_t *tris, uint32_t nt, BinSpec s, uint32_t *count,
                                             const uint64_t *offs, uint32_t *list) {
    const uint32_t t = blockIdx.x * T + threadIdx.x;
    if (t >= nt) return;
    uint64_t r0[3], r1[3];
    if (!bin_range(verts, tris + 3 * (uint64_t)t, s.lo, s.gd, s.dilate, r0, r1)) return;
    for (uint64_t k = r0[2]; k <= r1[2]; k++)
        for (uint64_t j = r0[1]; j <= r1[1]; j++)
            for (uint64_t i = r0[0]; i <= r1[0]; i++) {
                const uint64_t bn = (k * s.gd[1] + j) * s.gd[0] + i;
                const uint32_t slot = atomicAdd(&count[bn], 1u);
                if (FILL) list[offs[bn] + slot] = t;
            }
}

// ------------------------------------------------------------ links
// voxel.cpp seg_tri (Moller-Trumbore on the segment o + s d, s in [0, 1])
__device__ __forceinline__ bool seg_tri(const double *o, const double *d, const double *t0, const double *t1, const double *t2, double *out) {
    double e1[3], e2[3], pv[3], tv[3], qv[3];
    for (int k = 0; k < 3; k++) { e1[k] = t1[k] - t0[k]; e2[k] = t2[k] - t0[k]; }
    pv[0] = d[1] * e2[2] - d[2] * e2[1]; pv[1] = d[2] * e2[0] - d[0] * e2[2]; pv[2] = d[0] * e2[1] - d[1] * e2[0];
    const double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
    if (fabs(det) < 1e-14) return false;
    const double inv = 1.0 / det;
    for (int k = 0; k < 3; k++) tv[k] = o[k] - t0[k];
    const double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv;
    if (!(u >= 0.0 && u <= 1.0)) return false;
    qv[0] = tv[1] * e1[2] - tv[2] * e1[1]; qv[1] = tv[2] * e1[0] - tv[0] * e1[2]; qv[2] = tv[0] * e1[1] - tv[1] * e1[0];
    const double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
    if (v < 0.0 || u + v > 1.0) return false;
    const double tt = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
    if (!(tt >= -1e-9 && tt <= 1.0)) return false;
    *out = dmax(tt, 0.0);
    return true;
}

struct Dirs {
    int8_t c[27][3];
    int8_t opp[27];
    int nd, rest;
};

// cells that can carry a link: fluid, in the lattice, with triangles in
// their bin or a solid neighbour (the others have no hit and no solid
// neighbour, so no link)
__global__ void __launch_bounds__(T) kv_active(Region r, Dirs D, const uint8_t *inside, const uint64_t *boffs, uint32_t *flag) {
    const uint64_t n = (uint64_t)r.gd[0] * r.gd[1] * r.gd[2];
    const uint64_t l = (uint64_t)blockIdx.x * T + threadIdx.x;
    if (l >= n) return;
    const int64_t i = (int64_t)(l % r.gd[0]), j = (int64_t)((l / r.gd[0]) % r.gd[1]), k = (int64_t)(l / ((uint64_t)r.gd[0] * r.gd[1]));
    bool act = false;
    if (!inside[l] && in_domain(r, i, j, k)) {
        act = boffs[l + 1] > boffs[l];
        for (int d = 0; d < D.nd && !act; d++) {
            const int64_t ni = i + D.c[d][0], nj = j + D.c[d][1], nk = k + D.c[d][2];
            if (ni >= 0 && nj >= 0 && nk >= 0 && ni < (int64_t)r.gd[0] && nj < (int64_t)r.gd[1] && nk < (int64_t)r.gd[2])
                act = inside[rid(r, ni, nj, nk)] != 0;
        }
    }
    flag[l] = act ? 1u : 0u;
}

// the links of active cell a (region point act[a]): mask, q per direction,
// and the q of each thin-sheet link's reciprocal (NaN: none) for the next pass
__global__ void __launch_bounds__(T) kv_links(Region r, Dirs D, const double *verts, const uint32_t *tris, const uint8_t *inside,
                                              const uint64_t *boffs, const uint32_t *blist, const uint32_t *act, uint32_t nact,
                                              uint32_t *mask1, float *q1, float *qthin) {
    const uint32_t a = blockIdx.x * T + threadIdx.x;
    if (a >= nact) return;
    const uint64_t l = act[a];
    const int64_t i = (int64_t)(l % r.gd[0]), j = (int64_t)((l / r.gd[0]) % r.gd[1]), k = (int64_t)(l / ((uint64_t)r.gd[0] * r.gd[1]));
    const double p[3] = {(double)(i + r.slo[0]), (double)(j + r.slo[1]), (double)(k + r.slo[2])};
    const uint32_t *cand = blist + boffs[l];
    const uint32_t ncand = (uint32_t)(boffs[l + 1] - boffs[l]);
    uint32_t mask = 0;
    for (int d = 0; d < D.nd; d++) {
        float qd = 1.0f, qt = __int_as_float(0x7fc00000);
        if (d != D.rest) {
            const int64_t ni = i + D.c[d][0], nj = j + D.c[d][1], nk = k + D.c[d][2];
            const double dv[3] = {(double)D.c[d][0], (double)D.c[d][1], (double)D.c[d][2]};
            double tmin = INFINITY, tmax = -INFINITY;
            int hits = 0;
            for (uint32_t q = 0; q < ncand; q++) {
                const uint32_t *tr = tris + 3 * (uint64_t)cand[q];
                double tt;
                if (seg_tri(p, dv, verts + 3 * (uint64_t)tr[0], verts + 3 * (uint64_t)tr[1], verts + 3 * (uint64_t)tr[2], &tt)) {
                    tmin = dmin(tmin, tt);
                    tmax = dmax(tmax, tt);
                    hits++;
                }
            }
            const bool in_region = ni >= 0 && nj >= 0 && nk >= 0 && ni < (int64_t)r.gd[0] && nj < (int64_t)r.gd[1] && nk < (int64_t)r.gd[2];
            const bool nsolid = in_region ? inside[rid(r, ni, nj, nk)] != 0 : (hits % 2 == 1);
            if (nsolid) {
                qd = hits > 0 ? (float)dmin(dmax(tmin, 1e-3), 1.0) : 0.5f;
                mask |= 1u << d;
            } else if (hits >= 2 && tmax - tmin > 1e-6) {
                qd = (float)dmin(dmax(tmin, 1e-3), 1.0);
                mask |= 1u << d;
                if (in_region) qt = (float)dmin(dmax(1.0 - tmax, 1e-3), 1.0);
            }
        }
        q1[(uint64_t)a * 27 + d] = qd;
        qthin[(uint64_t)a * 27 + d] = qt;
    }
    for (int d = D.nd; d < 27; d++) { q1[(uint64_t)a * 27 + d] = 1.0f; qthin[(uint64_t)a * 27 + d] = __int_as_float(0x7fc00000); }
    mask1[a] = mask;
}

// the reciprocal thin-sheet links: neighbour n = cell + c_d gets link opp d
// with q = 1 - tmax unless its own pass gave it that link; err counts
// neighbours that are not active cells (none can be: the sheet lies within
// one link of them, so their bin lists it)
__global__ void __launch_bounds__(T) kv_thin(Region r, Dirs D, const uint8_t *inside, const uint32_t *act, uint32_t nact, const uint32_t *aidx,
                                             const uint32_t *aflag, const uint32_t *mask1, const float *qthin, uint32_t *maskt, float *qt,
                                             uint32_t *err) {
    const uint32_t a = blockIdx.x * T + threadIdx.x;
    if (a >= nact) return;
    const uint64_t l = act[a];
    const int64_t i = (int64_t)(l % r.gd[0]), j = (int64_t)((l / r.gd[0]) % r.gd[1]), k = (int64_t)(l / ((uint64_t)r.gd[0] * r.gd[1]));
    for (int d = 0; d < D.nd; d++) {
        const float q = qthin[(uint64_t)a * 27 + d];
        if (q != q) continue;
        const int64_t ni = i + D.c[d][0], nj = j + D.c[d][1], nk = k + D.c[d][2];
        const uint64_t nl = rid(r, ni, nj, nk);
        if (inside[nl] || !in_domain(r, ni, nj, nk)) continue;
        if (!aflag[nl]) { atomicAdd(err, 1u); continue; }
        const uint32_t b = aidx[nl];
        const int o = D.opp[d];
        if (mask1[b] & (1u << o)) continue;
        atomicOr(&maskt[b], 1u << o);
        qt[(uint64_t)b * 27 + o] = q;  // one writer per (neighbour, direction)
    }
}

struct WallRec {  // WallCell's layout
    uint32_t cell, mask;
    float q[27];
};

// the walls in region order: cell index in the lattice, mask, q
__global__ void __launch_bounds__(T) kv_walls(Region r, const uint32_t *act, const uint32_t *sel, uint32_t nw, const uint32_t *mask1,
                                              const uint32_t *maskt, const float *q1, const float *qt, WallRec *out) {
    const uint32_t w = blockIdx.x * T + threadIdx.x;
    if (w >= nw) return;
    const uint32_t a = sel[w];
    const uint64_t l = act[a];
    const int64_t i = (int64_t)(l % r.gd[0]), j = (int64_t)((l / r.gd[0]) % r.gd[1]), k = (int64_t)(l / ((uint64_t)r.gd[0] * r.gd[1]));
    WallRec c;
    c.cell = (uint32_t)(((uint64_t)(k + r.slo[2]) * r.dims[1] + (uint64_t)(j + r.slo[1])) * r.dims[0] + (uint64_t)(i + r.slo[0]));
    c.mask = mask1[a] | maskt[a];
    for (int d = 0; d < 27; d++) c.q[d] = (mask1[a] >> d) & 1u ? q1[(uint64_t)a * 27 + d] : (((maskt[a] >> d) & 1u) ? qt[(uint64_t)a * 27 + d] : 1.0f);
    out[w] = c;
}

__global__ void __launch_bounds__(T) kv_solid(Region r, const uint8_t *inside, const uint32_t *sel, uint32_t ns, uint32_t *out) {
    const uint32_t s = blockIdx.x * T + threadIdx.x;
    if (s >= ns) return;
    const uint64_t l = sel[s];
    const int64_t i = (int64_t)(l % r.gd[0]), j = (int64_t)((l / r.gd[0]) % r.gd[1]), k = (int64_t)(l / ((uint64_t)r.gd[0] * r.gd[1]));
    out[s] = (uint32_t)(((uint64_t)(k + r.slo[2]) * r.dims[1] + (uint64_t)(j + r.slo[1])) * r.dims[0] + (uint64_t)(i + r.slo[0]));
}

__global__ void __launch_bounds__(T) kv_wall_flags(uint32_t nact, const uint32_t *mask1, const uint32_t *maskt, uint32_t *flag) {
    const uint32_t a = blockIdx.x * T + threadIdx.x;
    if (a < nact) flag[a] = (mask1[a] | maskt[a]) != 0u ? 1u : 0u;
}

__global__ void __launch_bounds__(T) kv_solid_flags(Region r, const uint8_t *inside, uint32_t *flag) {
    const uint64_t n = (uint64_t)r.gd[0] * r.gd[1] * r.gd[2];
    const uint64_t l = (uint64_t)blockIdx.x * T + threadIdx.x;
    if (l >= n) return;
    const int64_t i = (int64_t)(l % r.gd[0]), j = (int64_t)((l / r.gd[0]) % r.gd[1]), k = (int64_t)(l / ((uint64_t)r.gd[0] * r.gd[1]));
    flag[l] = (inside[l] && in_domain(r, i, j, k)) ? 1u : 0u;
}

__global__ void __launch_bounds__(T) kv_narrow(uint64_t n, const uint64_t *in, uint32_t *out) {
    const uint64_t l = (uint64_t)blockIdx.x * T + threadIdx.x;
    if (l < n) out[l] = (uint32_t)in[l];
}



}  // namespace vg

namespace {

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw VoxelError(e == cudaErrorMemoryAllocation ? 2 : 3, std::string(what) + ": " + cudaGetErrorString(e));
}

// device buffers of one call, freed when it ends
struct Pool {
    std::vector<void *> p;
    template <class X>
    X *get(uint64_t n) {
        void *q = nullptr;
        ck(cudaMalloc(&q, std::max<uint64_t>(n, 1) * sizeof(X)), "cudaMalloc");
        p.push_back(q);
        return (X *)q;
    }
    ~Pool() {
        for (void *q : p) cudaFree(q);
    }
};

constexpr double VOXEL_WAIT_S = 600.0;  // host-side limit on each wait for the voxelizer's kernels

unsigned blocks(uint64_t n) { return (unsigned)((n + vg::T - 1) / vg::T); }

// offs[0..n] = exclusive prefix sum of count[0..n-1] (count has n + 1
// entries, the last zero); returns the total
uint64_t scan(cudaStream_t st, const uint32_t *count, uint64_t *offs, uint64_t n) {
    thrust::exclusive_scan(thrust::cuda::par.on(st), count, count + n + 1, offs, (uint64_t)0);
    uint64_t tot = 0;
    ck(cudaMemcpyAsync(&tot, offs + n, 8, cudaMemcpyDeviceToHost, st), "scan total");
    ck(lbm::stream_wait(st, VOXEL_WAIT_S), "scan");
    return tot;
}

struct NonZero {
    __host__ __device__ bool operator()(uint32_t f) const { return f != 0u; }
};

// indices i < n with flag[i] != 0, in order
uint32_t select_idx(cudaStream_t st, const uint32_t *flag, uint64_t n, uint32_t *out) {
    auto end = thrust::copy_if(thrust::cuda::par.on(st), thrust::counting_iterator<uint32_t>(0), thrust::counting_iterator<uint32_t>((uint32_t)n), flag,
                               out, NonZero());
    ck(lbm::stream_wait(st, VOXEL_WAIT_S), "select");
    return (uint32_t)(end - out);
}

}  // namespace

StaticVoxels voxelize_static_gpu(const Surface &s, std::array<size_t, 3> dims, int lattice) {
    const auto &dirs = lattice == 27 ? dirs27() : dirs19();
    vg::Dirs D{};
    D.nd = (int)dirs.size();
    D.rest = lattice == 27 ? 13 : 0;
    for (int d = 0; d < D.nd; d++) {
        for (int k = 0; k < 3; k++) D.c[d][k] = (int8_t)dirs[d][k];
        D.opp[d] = (int8_t)(lattice == 27 ? 26 - d : (d == 0 ? 0 : (d % 2 == 1 ? d + 1 : d - 1)));
    }
    // the part's region: its bounding box grown by 2 cells, clipped to one
    // cell outside the lattice (voxel.cpp voxelize_links)
    double maxlen = 0.0;
    for (auto &d : dirs) maxlen = std::max(maxlen, std::sqrt((double)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])));
    std::array<double, 3> blo, bhi;
    for (int k = 0; k < 3; k++) { blo[k] = std::numeric_limits<double>::infinity(); bhi[k] = -blo[k]; }
    for (auto &p : s.verts)
        for (int k = 0; k < 3; k++) { blo[k] = std::min(blo[k], p[k]); bhi[k] = std::max(bhi[k], p[k]); }
    long long slo[3], shi[3];
    for (int k = 0; k < 3; k++) {
        slo[k] = std::max((long long)std::floor(blo[k] - 2.0), -1LL);
        shi[k] = std::min((long long)std::ceil(bhi[k] + 2.0), (long long)dims[k]);
    }
    StaticVoxels out;
    for (int k = 0; k < 3; k++) {
        out.lo[k] = (size_t)std::max(slo[k], 0LL);
        out.hi[k] = (size_t)std::max(std::min(shi[k], (long long)dims[k] - 1), 0LL);
    }
    if (s.tris.empty() || slo[0] > shi[0] || slo[1] > shi[1] || slo[2] > shi[2]) return out;
    vg::Region R{};
    for (int k = 0; k < 3; k++) {
        R.slo[k] = slo[k];
        R.gd[k] = (uint32_t)(shi[k] - slo[k] + 1);
        R.dims[k] = (uint32_t)dims[k];
    }
    const uint64_t glen = (uint64_t)R.gd[0] * R.gd[1] * R.gd[2];
    const uint32_t nt = (uint32_t)s.tris.size();
    cudaStream_t st = nullptr;
    ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            if (lbm::stream_wait(s, VOXEL_WAIT_S) != cudaErrorTimeout) cudaStreamDestroy(s);
        }
    } sg{st};
    Pool pool;
    // vertices (lattice units) and their region coordinates (the grid has
    // h = 1 and origin slo), triangles
    std::vector<double> hv(3 * s.verts.size()), hg(3 * s.verts.size());
    for (size_t i = 0; i < s.verts.size(); i++)
        for (int k = 0; k < 3; k++) {
            hv[3 * i + k] = s.verts[i][k];
            hg[3 * i + k] = (s.verts[i][k] - (double)slo[k]) / 1.0;
        }
    std::vector<uint32_t> ht(3 * (size_t)nt);
    for (size_t t = 0; t < nt; t++)
        for (int k = 0; k < 3; k++) ht[3 * t + k] = s.tris[t][k];
    double *verts = pool.get<double>(hv.size()), *gv = pool.get<double>(hg.size());
    uint32_t *tris = pool.get<uint32_t>(ht.size());
    ck(cudaMemcpyAsync(verts, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice, st), "upload vertices");
    ck(cudaMemcpyAsync(gv, hg.data(), hg.size() * 8, cudaMemcpyHostToDevice, st), "upload vertices");
    ck(cudaMemcpyAsync(tris, ht.data(), ht.size() * 4, cudaMemcpyHostToDevice, st), "upload triangles");

    // inside_grid: the votes of the three axes, then the majority
    uint8_t *votes = pool.get<uint8_t>(glen), *inside = pool.get<uint8_t>(glen);
    ck(cudaMemsetAsync(votes, 0, glen, st), "memset");
    for (int a = 0; a < 3; a++) {
        const uint64_t nlines = (uint64_t)R.gd[(a + 1) % 3] * R.gd[(a + 2) % 3];
        Pool ap;
        uint32_t *count = ap.get<uint32_t>(nlines + 1);
        uint64_t *offs = ap.get<uint64_t>(nlines + 1);
        ck(cudaMemsetAsync(count, 0, (nlines + 1) * 4, st), "memset");
        vg::kv_crossings<false><<<blocks(nt), vg::T, 0, st>>>(gv, tris, nt, a, R, count, nullptr, nullptr, nullptr);
        ck(cudaGetLastError(), "crossings");
        const uint64_t nh = scan(st, count, offs, nlines);
        double *hts = ap.get<double>(nh);
        int8_t *hws = ap.get<int8_t>(nh);
        ck(cudaMemsetAsync(count, 0, (nlines + 1) * 4, st), "memset");
        vg::kv_crossings<true><<<blocks(nt), vg::T, 0, st>>>(gv, tris, nt, a, R, count, offs, hts, hws);
        vg::kv_lines<<<blocks(nlines), vg::T, 0, st>>>(a, R, count, offs, hts, hws, votes);
        ck(cudaGetLastError(), "scan lines");
        ck(lbm::stream_wait(st, VOXEL_WAIT_S), "scan lines");
    }
    vg::kv_inside<<<blocks(glen), vg::T, 0, st>>>(glen, votes, inside);
    ck(cudaGetLastError(), "inside");

    // bins of the triangles near each region point
    vg::BinSpec B{};
    for (int k = 0; k < 3; k++) { B.lo[k] = (double)slo[k] - 0.5; B.gd[k] = R.gd[k]; }
    B.dilate = maxlen + 0.01;
    uint32_t *bcount = pool.get<uint32_t>(glen + 1);
    uint64_t *boffs = pool.get<uint64_t>(glen + 1);
    ck(cudaMemsetAsync(bcount, 0, (glen + 1) * 4, st), "memset");
    vg::kv_bins<false><<<blocks(nt), vg::T, 0, st>>>(verts, tris, nt, B, bcount, nullptr, nullptr);
    ck(cudaGetLastError(), "bins");
    const uint64_t nlist = scan(st, bcount, boffs, glen);
    uint32_t *blist = pool.get<uint32_t>(nlist);
    ck(cudaMemsetAsync(bcount, 0, (glen + 1) * 4, st), "memset");
    vg::kv_bins<true><<<blocks(nt), vg::T, 0, st>>>(verts, tris, nt, B, bcount, boffs, blist);
    ck(cudaGetLastError(), "bins");

    // the cells that can carry links, their links, the reciprocal thin links
    uint32_t *aflag = pool.get<uint32_t>(glen + 1);
    uint64_t *aoff = pool.get<uint64_t>(glen + 1);
    ck(cudaMemsetAsync(aflag, 0, (glen + 1) * 4, st), "memset");
    vg::kv_active<<<blocks(glen), vg::T, 0, st>>>(R, D, inside, boffs, aflag);
    ck(cudaGetLastError(), "active cells");
    uint32_t *act = pool.get<uint32_t>(glen);
    const uint32_t nact = select_idx(st, aflag, glen, act);
    (void)scan(st, aflag, aoff, glen);
    uint32_t *aidx = pool.get<uint32_t>(glen);
    // region point -> active index (32-bit), from the 64-bit prefix sum
    vg::kv_narrow<<<blocks(glen), vg::T, 0, st>>>(glen, aoff, aidx);
    uint32_t *mask1 = pool.get<uint32_t>(nact), *maskt = pool.get<uint32_t>(nact), *err = pool.get<uint32_t>(1);
    float *q1 = pool.get<float>((uint64_t)nact * 27), *qthin = pool.get<float>((uint64_t)nact * 27), *qt = pool.get<float>((uint64_t)nact * 27);
    ck(cudaMemsetAsync(maskt, 0, (uint64_t)std::max<uint32_t>(nact, 1) * 4, st), "memset");
    ck(cudaMemsetAsync(err, 0, 4, st), "memset");
    if (nact) vg::kv_links<<<blocks(nact), vg::T, 0, st>>>(R, D, verts, tris, inside, boffs, blist, act, nact, mask1, q1, qthin);
    ck(cudaGetLastError(), "links");
    if (nact) vg::kv_thin<<<blocks(nact), vg::T, 0, st>>>(R, D, inside, act, nact, aidx, aflag, mask1, qthin, maskt, qt, err);
    ck(cudaGetLastError(), "thin links");
    uint32_t herr = 0;
    ck(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st), "readback");
    ck(lbm::stream_wait(st, VOXEL_WAIT_S), "links");
    if (herr) throw VoxelError(1, "GPU voxelizer: a thin-sheet link reached a cell outside the candidate set");

    // walls and solid cells in region order, to the host
    uint32_t *wflag = pool.get<uint32_t>(nact), *wsel = pool.get<uint32_t>(nact);
    if (nact) vg::kv_wall_flags<<<blocks(nact), vg::T, 0, st>>>(nact, mask1, maskt, wflag);
    const uint32_t nw = select_idx(st, wflag, nact, wsel);
    vg::WallRec *wrec = pool.get<vg::WallRec>(nw);
    if (nw) vg::kv_walls<<<blocks(nw), vg::T, 0, st>>>(R, act, wsel, nw, mask1, maskt, q1, qt, wrec);
    ck(cudaGetLastError(), "walls");
    uint32_t *sflag = pool.get<uint32_t>(glen), *ssel = pool.get<uint32_t>(glen);
    vg::kv_solid_flags<<<blocks(glen), vg::T, 0, st>>>(R, inside, sflag);
    const uint32_t ns = select_idx(st, sflag, glen, ssel);
    uint32_t *solid = pool.get<uint32_t>(ns);
    if (ns) vg::kv_solid<<<blocks(ns), vg::T, 0, st>>>(R, inside, ssel, ns, solid);
    ck(cudaGetLastError(), "solid cells");
    out.solid.resize(ns);
    out.walls.resize(nw);
    static_assert(sizeof(vg::WallRec) == sizeof(WallCell), "wall record layout");
    if (ns) ck(cudaMemcpyAsync(out.solid.data(), solid, (size_t)ns * 4, cudaMemcpyDeviceToHost, st), "readback");
    if (nw) ck(cudaMemcpyAsync(out.walls.data(), wrec, (size_t)nw * sizeof(WallCell), cudaMemcpyDeviceToHost, st), "readback");
    ck(lbm::stream_wait(st, VOXEL_WAIT_S), "readback");
    return out;
}

}  // namespace lbm
