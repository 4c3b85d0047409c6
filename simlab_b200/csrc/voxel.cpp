// Triangle surface -> lattice geometry on the CPU (setup input of the time
// step).  Follows crates/cfd/src/voxel.rs:
//  * inside_grid (voxel.rs:73-216): ray parity along x, y and z through every
//    grid point with a majority vote; lines crossing an odd number of times do
//    not vote; consistently oriented lines use the non-zero winding rule;
//    canonical vertex order in the edge functions so a line through a shared
//    edge counts one crossing.
//  * Bins (voxel.rs:218-296): triangles listed per unit bin of their grown
//    bounding box.
//  * seg_tri (voxel.rs:298-326): Moller-Trumbore segment test.
//  * voxelize_links (voxel.rs:361-490): solid cells, wall links from fluid to
//    solid cells with q from the nearest hit (0.5 without a hit), reciprocal
//    thin-sheet links.
// Parallel over scan rows / cells with OpenMP; results are independent of the
// thread count (per-row work, sorted outputs).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "voxel.hpp"

namespace lbm {

namespace {
using P3 = std::array<double, 3>;

constexpr double EPS_B = 1.2345671e-5;  // voxel.rs:68-71
constexpr double EPS_C = 2.7182818e-5;

struct Hit { uint32_t j; double t; int w; };

void mark_line(const GridSpec &g, int a, int b, int c, size_t j, size_t k, const Hit *line, size_t nl, int mode,
               std::vector<std::atomic<uint32_t>> &votes) {
    size_t na = g.dims[a];
    uint32_t vbit = 1u << (3 + a), ibit = 1u << a;
    size_t h = 0;
    int wind = 0;
    for (size_t i = 0; i < na; i++) {
        double ta = (double)i;
        while (h < nl && line[h].t < ta) { wind += line[h].w; h++; }
        size_t pos[3];
        pos[a] = i; pos[b] = j; pos[c] = k;
        size_t id = (pos[2] * g.dims[1] + pos[1]) * g.dims[0] + pos[0];
        uint32_t bits = 0;
        if (mode != 0) {
            bits |= vbit;
            bool ins = mode == 1 ? wind != 0 : (h % 2 == 1);
            if (ins) bits |= ibit;
        }
        if (bits) votes[id].fetch_or(bits, std::memory_order_relaxed);
    }
}

void parity_axis(const Surface &s, const GridSpec &g, int a, std::vector<std::atomic<uint32_t>> &votes) {
    int b = (a + 1) % 3, c = (a + 2) % 3;
    size_t nb = g.dims[b], nc = g.dims[c];
    std::vector<P3> gv(s.verts.size());
    for (size_t i = 0; i < s.verts.size(); i++)
        for (int k = 0; k < 3; k++) gv[i][k] = (s.verts[i][k] - g.origin[k]) / g.h;
    std::vector<std::vector<uint32_t>> rows(nc);
    for (size_t t = 0; t < s.tris.size(); t++) {
        double lo = std::numeric_limits<double>::infinity(), hi = -lo;
        for (int v = 0; v < 3; v++) { lo = std::min(lo, gv[s.tris[t][v]][c]); hi = std::max(hi, gv[s.tris[t][v]][c]); }
        double k0f = std::max(std::ceil(lo - EPS_C), 0.0);
        double k1f = std::floor(hi - EPS_C);
        if (k1f < 0.0) continue;
        size_t k0 = (size_t)k0f;
        size_t k1 = std::min((size_t)k1f, nc ? nc - 1 : 0);
        for (size_t k = k0; k <= k1 && k < nc; k++) rows[k].push_back((uint32_t)t);
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long long kk = 0; kk < (long long)nc; kk++) {
        size_t k = (size_t)kk;
        double pc = (double)k + EPS_C;
        std::vector<Hit> hits;
        for (uint32_t t : rows[k]) {
            const uint32_t ids[3] = {s.tris[t][0], s.tris[t][1], s.tris[t][2]};
            const P3 p[3] = {gv[ids[0]], gv[ids[1]], gv[ids[2]]};
            double lo = std::numeric_limits<double>::infinity(), hi = -lo;
            for (int q = 0; q < 3; q++) { lo = std::min(lo, p[q][b]); hi = std::max(hi, p[q][b]); }
            double j0f = std::max(std::ceil(lo - EPS_B), 0.0);
            double j1f = std::floor(hi - EPS_B);
            if (j1f < 0.0) continue;
            size_t j0 = (size_t)j0f, j1 = std::min((size_t)j1f, nb ? nb - 1 : 0);
            for (size_t j = j0; j <= j1; j++) {
                double pb = (double)j + EPS_B;
                auto e = [&](int u, int v) -> double {
                    uint32_t iu = ids[u], iv = ids[v];
                    P3 pu, pv;
                    double sg;
                    if (iu < iv) { pu = p[u]; pv = p[v]; sg = 1.0; } else { pu = p[v]; pv = p[u]; sg = -1.0; }
                    return sg * ((pv[b] - pu[b]) * (pc - pu[c]) - (pv[c] - pu[c]) * (pb - pu[b]));
                };
                double e0 = e(1, 2), e1 = e(2, 0), e2 = e(0, 1);
                bool inside = (e0 > 0.0 && e1 > 0.0 && e2 > 0.0) || (e0 < 0.0 && e1 < 0.0 && e2 < 0.0);
                if (!inside) continue;
                double sum = e0 + e1 + e2;
                double ta = (e0 * p[0][a] + e1 * p[1][a] + e2 * p[2][a]) / sum;
                hits.push_back({(uint32_t)j, ta, sum > 0.0 ? 1 : -1});
            }
        }
        std::sort(hits.begin(), hits.end(), [](const Hit &x, const Hit &y) {
            if (x.j != y.j) return x.j < y.j;
            return x.t < y.t;  // total order on finite values
        });
        size_t i0 = 0;
        while (i0 < hits.size()) {
            uint32_t j = hits[i0].j;
            size_t i1 = i0;
            while (i1 < hits.size() && hits[i1].j == j) i1++;
            int wsum = 0;
            for (size_t q = i0; q < i1; q++) wsum += hits[q].w;
            int mode = wsum == 0 ? 1 : ((i1 - i0) % 2 == 0 ? 2 : 0);
            mark_line(g, a, b, c, j, k, hits.data() + i0, i1 - i0, mode, votes);
            i0 = i1;
        }
        std::vector<char> have(nb, 0);
        for (auto &h : hits) have[h.j] = 1;
        for (size_t j = 0; j < nb; j++)
            if (!have[j]) mark_line(g, a, b, c, j, k, nullptr, 0, 1, votes);
    }
}

struct Bins {
    P3 lo;
    std::array<size_t, 3> dims;
    std::vector<uint32_t> start, list;
    const uint32_t *get(const P3 &p, size_t &n) const {
        size_t ix[3];
        for (int k = 0; k < 3; k++) {
            double f = std::floor(p[k] - lo[k]);
            if (f < 0.0 || f >= (double)dims[k]) { n = 0; return nullptr; }
            ix[k] = (size_t)f;
        }
        size_t b = (ix[2] * dims[1] + ix[1]) * dims[0] + ix[0];
        n = start[b + 1] - start[b];
        return list.data() + start[b];
    }
};

Bins build_bins(const Surface &s, P3 lo, std::array<size_t, 3> dims, double dilate) {
    size_t nb = dims[0] * dims[1] * dims[2];
    auto range = [&](size_t t, size_t *r0, size_t *r1) -> bool {
        for (int k = 0; k < 3; k++) {
            double mn = std::numeric_limits<double>::infinity(), mx = -mn;
            for (int v = 0; v < 3; v++) { mn = std::min(mn, s.verts[s.tris[t][v]][k]); mx = std::max(mx, s.verts[s.tris[t][v]][k]); }
            mn = mn - dilate - lo[k];
            mx = mx + dilate - lo[k];
            if (mx < 0.0 || mn >= (double)dims[k]) return false;
            r0[k] = (size_t)std::max(std::floor(mn), 0.0);
            r1[k] = std::min((size_t)std::floor(mx), dims[k] - 1);
        }
        return true;
    };
    std::vector<uint32_t> counts(nb, 0);
    for (size_t t = 0; t < s.tris.size(); t++) {
        size_t r0[3], r1[3];
        if (!range(t, r0, r1)) continue;
        for (size_t k = r0[2]; k <= r1[2]; k++)
            for (size_t j = r0[1]; j <= r1[1]; j++)
                for (size_t i = r0[0]; i <= r1[0]; i++) counts[(k * dims[1] + j) * dims[0] + i]++;
    }
    Bins B;
    B.lo = lo; B.dims = dims;
    B.start.assign(nb + 1, 0);
    for (size_t i = 0; i < nb; i++) B.start[i + 1] = B.start[i] + counts[i];
    B.list.assign(B.start[nb], 0);
    std::vector<uint32_t> cur(B.start.begin(), B.start.end() - 1);
    for (size_t t = 0; t < s.tris.size(); t++) {  // ascending t: each bin sorted
        size_t r0[3], r1[3];
        if (!range(t, r0, r1)) continue;
        for (size_t k = r0[2]; k <= r1[2]; k++)
            for (size_t j = r0[1]; j <= r1[1]; j++)
                for (size_t i = r0[0]; i <= r1[0]; i++) B.list[cur[(k * dims[1] + j) * dims[0] + i]++] = (uint32_t)t;
    }
    return B;
}

}  // namespace

bool seg_tri(const double o[3], const double d[3], const double t0[3], const double t1[3], const double t2[3], double *out) {
    double e1[3], e2[3], pv[3], tv[3], qv[3];
    for (int k = 0; k < 3; k++) { e1[k] = t1[k] - t0[k]; e2[k] = t2[k] - t0[k]; }
    pv[0] = d[1] * e2[2] - d[2] * e2[1]; pv[1] = d[2] * e2[0] - d[0] * e2[2]; pv[2] = d[0] * e2[1] - d[1] * e2[0];
    double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
    if (std::fabs(det) < 1e-14) return false;
    double inv = 1.0 / det;
    for (int k = 0; k < 3; k++) tv[k] = o[k] - t0[k];
    double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv;
    if (!(u >= 0.0 && u <= 1.0)) return false;
    qv[0] = tv[1] * e1[2] - tv[2] * e1[1]; qv[1] = tv[2] * e1[0] - tv[0] * e1[2]; qv[2] = tv[0] * e1[1] - tv[1] * e1[0];
    double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
    if (v < 0.0 || u + v > 1.0) return false;
    double tt = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
    if (!(tt >= -1e-9 && tt <= 1.0)) return false;
    *out = std::max(tt, 0.0);
    return true;
}

std::vector<uint8_t> inside_grid(const Surface &s, const GridSpec &g) {
    size_t n = g.dims[0] * g.dims[1] * g.dims[2];
    std::vector<uint8_t> out(n, 0);
    if (n == 0 || s.tris.empty()) return out;
    std::vector<std::atomic<uint32_t>> votes(n);
    for (auto &v : votes) v.store(0, std::memory_order_relaxed);
    for (int a = 0; a < 3; a++) parity_axis(s, g, a, votes);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) {
        uint32_t v = votes[i].load(std::memory_order_relaxed);
        uint32_t valid = (v >> 3) & 7u, ins = v & 7u & valid;
        int nv = __builtin_popcount(valid), ni = __builtin_popcount(ins);
        out[i] = (nv > 0 && 2 * ni > nv) ? 1 : 0;
    }
    return out;
}

StaticVoxels voxelize_links(const Surface &s, std::array<size_t, 3> dims, const std::vector<std::array<int, 3>> &dirs,
                            const std::vector<int> &opp, int rest) {
    const size_t nd = dirs.size();
    double maxlen = 0.0;
    for (auto &d : dirs) maxlen = std::max(maxlen, std::sqrt((double)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])));
    P3 blo, bhi;
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
    GridSpec g;
    g.origin = {(double)slo[0], (double)slo[1], (double)slo[2]};
    g.h = 1.0;
    g.dims = {(size_t)(shi[0] - slo[0] + 1), (size_t)(shi[1] - slo[1] + 1), (size_t)(shi[2] - slo[2] + 1)};
    const auto &gd = g.dims;
    std::vector<uint8_t> inside = inside_grid(s, g);
    Bins bins = build_bins(s, {(double)slo[0] - 0.5, (double)slo[1] - 0.5, (double)slo[2] - 0.5}, gd, maxlen + 0.01);
    auto in_domain = [&](size_t i, size_t j, size_t k) {
        long long p[3] = {(long long)i + slo[0], (long long)j + slo[1], (long long)k + slo[2]};
        for (int a = 0; a < 3; a++) if (p[a] < 0 || p[a] >= (long long)dims[a]) return false;
        return true;
    };
    auto gidx = [&](size_t i, size_t j, size_t k) -> size_t {
        return ((size_t)((long long)k + slo[2]) * dims[1] + (size_t)((long long)j + slo[1])) * dims[0] + (size_t)((long long)i + slo[0]);
    };
    const size_t glen = gd[0] * gd[1] * gd[2];
    for (size_t l = 0; l < glen; l++) {
        if (!inside[l]) continue;
        size_t i = l % gd[0], j = (l / gd[0]) % gd[1], k = l / (gd[0] * gd[1]);
        if (in_domain(i, j, k)) out.solid.push_back((uint32_t)gidx(i, j, k));
    }
    auto is_solid = [&](long long i, long long j, long long k) {
        if (i < 0 || j < 0 || k < 0 || i >= (long long)gd[0] || j >= (long long)gd[1] || k >= (long long)gd[2]) return false;
        return inside[((size_t)k * gd[1] + (size_t)j) * gd[0] + (size_t)i] != 0;
    };
    struct Thin { size_t nl; int d; float q; };
    struct Cell { size_t l; uint32_t mask; std::array<float, 27> q; std::vector<Thin> thin; };
    std::vector<std::vector<Cell>> per_row(gd[2]);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long kk = 0; kk < (long long)gd[2]; kk++) {
        size_t k = (size_t)kk;
        for (size_t j = 0; j < gd[1]; j++)
            for (size_t i = 0; i < gd[0]; i++) {
                size_t l = (k * gd[1] + j) * gd[0] + i;
                if (inside[l] || !in_domain(i, j, k)) continue;
                double p[3] = {(double)((long long)i + slo[0]), (double)((long long)j + slo[1]), (double)((long long)k + slo[2])};
                size_t ncand;
                const uint32_t *cand = bins.get({p[0], p[1], p[2]}, ncand);
                Cell cell;
                cell.l = l; cell.mask = 0;
                cell.q.fill(1.0f);
                for (size_t d = 0; d < nd; d++) {
                    if ((int)d == rest) continue;
                    const auto &c = dirs[d];
                    long long ni = (long long)i + c[0], nj = (long long)j + c[1], nk = (long long)k + c[2];
                    double dv[3] = {(double)c[0], (double)c[1], (double)c[2]};
                    double tmin = std::numeric_limits<double>::infinity(), tmax = -tmin;
                    int hits = 0;
                    for (size_t q = 0; q < ncand; q++) {
                        const auto &tr = s.tris[cand[q]];
                        double tt;
                        if (seg_tri(p, dv, s.verts[tr[0]].data(), s.verts[tr[1]].data(), s.verts[tr[2]].data(), &tt)) {
                            tmin = std::min(tmin, tt);
                            tmax = std::max(tmax, tt);
                            hits++;
                        }
                    }
                    bool in_region = ni >= 0 && nj >= 0 && nk >= 0 && ni < (long long)gd[0] && nj < (long long)gd[1] && nk < (long long)gd[2];
                    bool nsolid = in_region ? is_solid(ni, nj, nk) : (hits % 2 == 1);
                    if (nsolid) {
                        cell.q[d] = hits > 0 ? (float)std::min(std::max(tmin, 1e-3), 1.0) : 0.5f;
                        cell.mask |= 1u << d;
                    } else if (hits >= 2 && tmax - tmin > 1e-6) {
                        cell.q[d] = (float)std::min(std::max(tmin, 1e-3), 1.0);
                        cell.mask |= 1u << d;
                        if (in_region)
                            cell.thin.push_back({((size_t)nk * gd[1] + (size_t)nj) * gd[0] + (size_t)ni, opp[d],
                                                 (float)std::min(std::max(1.0 - tmax, 1e-3), 1.0)});
                    }
                }
                if (cell.mask) per_row[k].push_back(std::move(cell));
            }
    }
    std::vector<Cell> cells;
    for (auto &r : per_row) for (auto &c : r) cells.push_back(std::move(c));
    std::unordered_map<size_t, size_t> at;
    for (size_t r = 0; r < cells.size(); r++) at[cells[r].l] = r;
    size_t nfirst = cells.size();
    for (size_t ci = 0; ci < nfirst; ci++) {
        std::vector<Thin> thin = cells[ci].thin;
        for (auto &t : thin) {
            size_t i = t.nl % gd[0], j = (t.nl / gd[0]) % gd[1], k = t.nl / (gd[0] * gd[1]);
            if (inside[t.nl] || !in_domain(i, j, k)) continue;
            auto it = at.find(t.nl);
            size_t r;
            if (it == at.end()) {
                Cell c;
                c.l = t.nl; c.mask = 0; c.q.fill(1.0f);
                cells.push_back(std::move(c));
                r = cells.size() - 1;
                at[t.nl] = r;
            } else {
                r = it->second;
            }
            if ((cells[r].mask & (1u << t.d)) == 0) {
                cells[r].mask |= 1u << t.d;
                cells[r].q[t.d] = t.q;
            }
        }
    }
    std::sort(cells.begin(), cells.end(), [](const Cell &a, const Cell &b) { return a.l < b.l; });
    out.walls.reserve(cells.size());
    for (auto &c : cells) {
        size_t i = c.l % gd[0], j = (c.l / gd[0]) % gd[1], k = c.l / (gd[0] * gd[1]);
        WallCell w;
        w.cell = (uint32_t)gidx(i, j, k);
        w.mask = c.mask;
        w.q = c.q;
        out.walls.push_back(w);
    }
    return out;
}

const std::vector<std::array<int, 3>> &dirs19() {
    static const std::vector<std::array<int, 3>> d = {
        {0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},   {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
        {1, 1, 0},  {-1, -1, 0}, {1, 0, 1},  {-1, 0, -1}, {0, 1, 1},  {0, -1, -1}, {1, -1, 0},
        {-1, 1, 0}, {1, 0, -1},  {-1, 0, 1}, {0, 1, -1},  {0, -1, 1}};
    return d;
}

const std::vector<std::array<int, 3>> &dirs27() {
    static std::vector<std::array<int, 3>> d = [] {
        std::vector<std::array<int, 3>> v(27);
        for (int i = 0; i < 27; i++) v[i] = {i % 3 - 1, (i / 3) % 3 - 1, i / 9 - 1};  // d3q27.rs:9-11
        return v;
    }();
    return d;
}

StaticVoxels voxelize_static(const Surface &s, std::array<size_t, 3> dims, int lattice) {
    if (lattice == 27) {
        std::vector<int> opp(27);
        for (int i = 0; i < 27; i++) opp[i] = 26 - i;
        return voxelize_links(s, dims, dirs27(), opp, 13);
    }
    std::vector<int> opp(19);
    for (int i = 0; i < 19; i++) opp[i] = i == 0 ? 0 : (i % 2 == 1 ? i + 1 : i - 1);
    return voxelize_links(s, dims, dirs19(), opp, 0);
}

}  // namespace lbm

namespace lbm {

// voxel.rs:562-584: splits triangles at their edge midpoints (1 into 4) until
// no edge is longer than max_edge
Surface subdivide(const Surface &s, double max_edge) {
    Surface o;
    o.verts = s.verts;
    std::vector<std::array<uint32_t, 3>> stack(s.tris.begin(), s.tris.end());
    auto len = [](const std::array<double, 3> &a, const std::array<double, 3> &b) {
        return std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
    };
    while (!stack.empty()) {
        const std::array<uint32_t, 3> t = stack.back();
        stack.pop_back();
        const auto a = o.verts[t[0]], b = o.verts[t[1]], c = o.verts[t[2]];
        if (std::max(std::max(len(a, b), len(b, c)), len(c, a)) <= max_edge || o.tris.size() > 50000000u) {
            o.tris.push_back(t);
            continue;
        }
        auto mid = [&](const std::array<double, 3> &p, const std::array<double, 3> &q) {
            o.verts.push_back({(p[0] + q[0]) / 2.0, (p[1] + q[1]) / 2.0, (p[2] + q[2]) / 2.0});
            return (uint32_t)(o.verts.size() - 1);
        };
        const uint32_t ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
        stack.push_back({t[0], ab, ca});
        stack.push_back({ab, t[1], bc});
        stack.push_back({ca, bc, t[2]});
        stack.push_back({ab, bc, ca});
    }
    return o;
}

// voxel.rs:507-560: occupancy on a grid of spacing h around the part (a margin
// of 2h), triangles as (v0, e1, e2) in f32, radius and axial extent
SpinVoxels voxelize_spin(const Surface &s, std::array<double, 3> axis, double h) {
    SpinVoxels v;
    if (s.verts.empty()) throw std::runtime_error("empty surface");
    std::array<double, 3> lo = s.verts[0], hi = s.verts[0];
    for (const auto &p : s.verts)
        for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    const double m = 2.0 * h;
    GridSpec g;
    for (int k = 0; k < 3; k++) {
        v.occ_lo[k] = lo[k] - m;
        v.occ_dims[k] = (size_t)std::ceil((hi[k] - lo[k] + 2.0 * m) / h) + 1;
    }
    g.origin = v.occ_lo;
    g.h = h;
    g.dims = v.occ_dims;
    v.occ_h = h;
    const std::vector<uint8_t> inside = inside_grid(s, g);
    v.occ_bits.assign((inside.size() + 31) / 32, 0u);
    for (size_t l = 0; l < inside.size(); l++)
        if (inside[l]) v.occ_bits[l >> 5] |= 1u << (l & 31);
    const Surface fine = subdivide(s, 1.5);
    v.tris.reserve(fine.tris.size());
    for (const auto &t : fine.tris) {
        const auto a = fine.verts[t[0]], b = fine.verts[t[1]], c = fine.verts[t[2]];
        v.tris.push_back({(float)a[0], (float)a[1], (float)a[2], 0.f, (float)(b[0] - a[0]), (float)(b[1] - a[1]), (float)(b[2] - a[2]), 0.f,
                          (float)(c[0] - a[0]), (float)(c[1] - a[1]), (float)(c[2] - a[2]), 0.f});
    }
    double amin = std::numeric_limits<double>::infinity(), amax = -amin;
    for (const auto &p : s.verts) {
        const double a = p[0] * axis[0] + p[1] * axis[1] + p[2] * axis[2];
        const double r2 = std::max(p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - a * a, 0.0);
        v.radius = std::max(v.radius, std::sqrt(r2));
        amin = std::min(amin, a);
        amax = std::max(amax, a);
    }
    v.axial[0] = amin;
    v.axial[1] = amax;
    return v;
}

}  // namespace lbm
