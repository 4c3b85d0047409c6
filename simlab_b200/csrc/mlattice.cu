// Host driver of the multi-level D3Q27 engine: the lbm_create_multi and
// lbm_multi_* functions of include/simlab_lbm.h.
//
// Mirrors `MultiLattice` of crates/cfd/src/mlattice.rs: setup validation
// (198-216), cell types and lists per level (404-478), records and flags of
// the finest level (178-192, 345-354, 430-446), initial moments (484-501),
// level constants (506-540), the initial state (664-686), the recursive
// sub-cycling schedule (786-842) and the readback (723-784, 883-905).
// Differences by design: one allocation per array (no buffer split), one CUDA
// stream per handle, device waits bounded by a host-side limit, forces summed
// in FP64.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/simlab_lbm.h"
#include "d3q27.h"
#include "host_wait.hpp"

namespace lbm_host {
void set_global_error(const std::string &msg);
}

namespace {

constexpr size_t HIST_CAP = 1024;  // finest steps per readback (mlattice.rs:283)

struct MErr : std::runtime_error {
    int code;
    MErr(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? LBM_ERR_NOMEM : LBM_ERR_CUDA;
        throw MErr(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

inline uint32_t fbits(float x) { uint32_t b; std::memcpy(&b, &x, 4); return b; }

// lattice.rs:172-189 / mlattice.rs:154-170: the host's f16 packing of q
uint16_t f16_bits(float x) {
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

size_t storage_bytes(int s) { return s == LBM_STORAGE_FP32 ? 4 : (s == LBM_STORAGE_FP64 ? 8 : 2); }

struct Level {
    lbm27::LevelParams p{};
    uint32_t src = 0, mslot = 1;
    uint64_t steps = 0;
};

}  // namespace

struct lbm_multi {
    lbm_multi_setup setup{};
    std::vector<lbm_level_box> boxes;
    std::vector<Level> lv;
    int storage = LBM_STORAGE_FP32;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    int device = 0;
    std::vector<void *> allocs;
    uint64_t memory_bytes = 0;
    uint32_t nrec = 0;
    uint32_t *recs = nullptr;
    double *recd = nullptr;
    void *wallf = nullptr;  // 27 reals per record, written by the wall kernel each finest step
    double *partials = nullptr;
    uint32_t *ticket = nullptr;
    double *hist = nullptr;       // HIST_CAP x 8 doubles
    double *hist_host = nullptr;  // pinned
    double *mass_d = nullptr;   // mass, non-finite count, then the grid sum's block partials and ticket
    float4 *dump = nullptr;
    // probes (mlattice.rs:243-305): surface vertices sampled on the finest
    // level, slice pixels each taken from the finest level that covers it
    uint32_t nvert = 0, npix = 0;
    float voff = 0.f;
    float *verts = nullptr;               // 8 floats per vertex (position, 0, normal, 0)
    double *vacc = nullptr;               // 2 doubles per vertex: sum of rho, count
    double *sacc = nullptr;               // 5 doubles per pixel: sums of rho, u, count
    std::vector<uint32_t *> pix;          // per level: (pixel, cell) pairs
    std::vector<uint32_t> npix_l;         // per level: number of pairs
    uint64_t fine_steps = 0;
    double timeout_s = 600.0;
    std::string err;

    void *dalloc(size_t bytes) {
        void *p = nullptr;
        ck(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc");
        allocs.push_back(p);
        memory_bytes += std::max<size_t>(bytes, 16);
        return p;
    }
    ~lbm_multi() {
        if (stream && lbm::stream_wait(stream, timeout_s) == cudaErrorTimeout) {
            lbm_host::set_global_error("multi-level lattice destroyed while its device work had not finished: buffers left allocated");
            return;
        }
        for (void *p : allocs) cudaFree(p);
        if (hist_host) cudaFreeHost(hist_host);
        if (ev) cudaEventDestroy(ev);
        if (stream) cudaStreamDestroy(stream);
    }
    void wait() {
        ck(cudaEventRecord(ev, stream), "cudaEventRecord");
        auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            cudaError_t q = cudaEventQuery(ev);
            if (q == cudaSuccess) return;
            if (q != cudaErrorNotReady) ck(q, "device wait");
            double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el > timeout_s) throw MErr(LBM_ERR_TIMEOUT, "device did not finish within " + std::to_string(timeout_s) + " s");
            if (el > 1e-3) std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    size_t sub_steps() const { return (size_t)1 << (lv.size() - 1); }
    uint32_t seed_of(uint32_t hslot, uint32_t src, uint32_t mw) const {  // mlattice.rs:692-703
        return ((uint32_t)fine_steps + hslot) * lbm::STEP_SEED_MUL + (src * lbm27::SEED_SRC_MUL + mw * lbm27::SEED_MW_MUL);
    }
    static uint32_t mix(uint32_t seed) { return seed * 0x85EBCA77u + 0x632BE5ABu; }

    // mlattice.rs:786-842: one step of level l and, nested in it, two steps
    // of each finer level with their ghost fills, then the restriction
    void schedule(size_t l, const lbm_step_in *fine, size_t &fine_i) {
        const size_t nl = lv.size(), finest = nl - 1;
        Level &L = lv[l];
        const uint32_t lsrc = L.src, lmw = 1u - L.mslot;
        const uint32_t hslot = (uint32_t)(fine_i % HIST_CAP);
        lbm27::StepArgs a{};
        a.src = lsrc;
        a.mw = lmw;
        a.seed_mix = mix(seed_of(hslot, lsrc, lmw));
        for (int k = 0; k < 9; k++) a.rot[k] = a.rot_prev[k] = (k % 4 == 0) ? 1.0f : 0.0f;
        if (l == finest && fine) {
            for (int k = 0; k < 3; k++) { a.omega[k] = (float)fine[fine_i].omega[k]; a.omega_d[k] = fine[fine_i].omega[k]; }
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    a.rot[3 * r + c] = (float)fine[fine_i].rot[r][c];
                    a.rot_prev[3 * r + c] = (float)fine[fine_i].rot_prev[r][c];
                }
        }
        if (l == 0) ck(lbm27::launch27_face(storage, L.p, a, stream), "face kernel");
        if (L.p.moving) ck(lbm27::launch27_revoxel(storage, L.p, a, stream), "re-voxelizer");
        ck(lbm27::launch27_step(storage, L.p, a, stream), "step kernel");
        L.src = 1u - lsrc;
        L.mslot = lmw;
        L.steps++;
        if (l == finest) {
            ck(lbm27::launch27_reduce(L.p, storage == LBM_STORAGE_FP64, partials, ticket, hist + (fine_i % HIST_CAP) * 8, stream), "reduce kernel");
            if (fine && fine[fine_i].sample) {
                // mlattice.rs:812-824: vertices with this step's rotation on the
                // finest level's new state, then the slices of every level
                lbm27::StepArgs after = a;
                after.src = L.src;
                ck(lbm27::launch27_sample_verts(storage, L.p, after, verts, nvert, voff, vacc, stream), "vertex probes");
                for (size_t q = 0; q < nl; q++)
                    ck(lbm27::launch27_sample_slices(storage, lv[q].p, lv[q].src, pix[q], npix_l[q], sacc, stream), "slice probes");
            }
            fine_i++;
        }
        if (l + 1 < nl) {
            const uint32_t mold = 1u - lmw;
            for (int sub = 0; sub < 2; sub++) {
                Level &C = lv[l + 1];
                lbm27::StepArgs g{};
                g.src = C.src;
                g.mold = mold;
                g.mnew = lmw;
                g.blend = 0.5f * (float)sub;
                g.seed_mix = mix(seed_of(0, g.src, 0));
                ck(lbm27::launch27_ghost(storage, C.p, g, stream), "ghost kernel");
                schedule(l + 1, fine, fine_i);
            }
            lbm27::StepArgs r{};
            r.src = L.src;
            r.seed_mix = mix(seed_of(0, r.src, 0));
            ck(lbm27::launch27_restrict(storage, L.p, r, stream), "restrict kernel");
        }
    }

    // mlattice.rs:723-784
    void run(const lbm_step_in *fine, uint64_t n, double *forces) {
        const size_t ss = sub_steps();
        if (n % ss != 0) throw MErr(LBM_ERR_INVALID, "step count must be a multiple of " + std::to_string(ss));
        const size_t max_coarse = std::max<size_t>(HIST_CAP / ss, 1);
        uint64_t done = 0;
        while (done < n) {
            const size_t nc = std::min<uint64_t>((n - done) / ss, max_coarse);
            size_t fine_i = 0;
            for (size_t k = 0; k < nc; k++) schedule(0, fine ? fine + done : nullptr, fine_i);
            const size_t nf = nc * ss;
            if (forces) {
                ck(cudaMemcpyAsync(hist_host, hist, nf * 8 * sizeof(double), cudaMemcpyDeviceToHost, stream), "history readback");
                wait();
                for (size_t k = 0; k < nf; k++) std::memcpy(forces + 6 * (done + k), hist_host + 8 * k, 6 * sizeof(double));
            }
            fine_steps += nf;
            done += nf;
        }
    }
};

namespace {

int mfail(lbm_multi *h, const MErr &e) {
    if (h) h->err = e.what(); else lbm_host::set_global_error(e.what());
    return e.code;
}

template <class F>
int mguard(lbm_multi *h, F &&fn) {
    try {
        fn();
        return LBM_OK;
    } catch (const MErr &e) {
        return mfail(h, e);
    } catch (const std::exception &e) {
        return mfail(h, MErr(LBM_ERR_INVALID, e.what()));
    }
}

template <class R>
void fill27(lbm27::Consts27<R> &k, const lbm_multi_setup &s, size_t l, size_t finest, const std::vector<std::array<double, 3>> &org) {
    const double tau_l = 0.5 + 3.0 * s.nu0 * (double)(1ull << l);  // mlattice.rs:486
    k.tau0 = (R)tau_l;
    k.smag2 = (R)(s.smagorinsky * s.smagorinsky);
    k.sponge_tau = (R)(l == 0 ? s.sponge_tau : 0.0);
    k.sigma = (R)(l == 0 ? s.sponge_sigma : 0.0);
    const double sc_l = (double)(1ull << (finest - l));
    for (int a = 0; a < 3; a++) {
        k.sp_lo[a] = (R)(l == 0 ? (double)s.sponge[2 * a] : 0.0);
        k.sp_hi[a] = (R)(l == 0 ? (double)s.sponge[2 * a + 1] : 0.0);
        k.u_inf[a] = (R)s.u_inf[a];
        k.u_init[a] = (R)s.u_init[a];
        k.grav[a] = (R)(s.body_force0[a] / (double)(1ull << l));  // mlattice.rs:531
        k.center[a] = (R)(l == finest ? s.center[a] : (s.center[a] - org[l][a]) / sc_l);
    }
}

template <class R>
void init_moments(lbm_multi *h, void *dst, uint64_t nodes, const lbm_multi_setup &s, double tau_l) {
    if (!nodes) return;
    std::vector<R> v(nodes * lbm27::MW, (R)0);
    for (uint64_t k = 0; k < nodes; k++) {
        R *c = &v[k * lbm27::MW];
        c[0] = (R)1;
        c[1] = (R)s.u_init[0];
        c[2] = (R)s.u_init[1];
        c[3] = (R)s.u_init[2];
        c[10] = (R)tau_l;
    }
    ck(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(R), cudaMemcpyHostToDevice, h->stream), "moment init");
    ck(lbm::stream_wait(h->stream, h->timeout_s), "moment init");
}

void create_multi(const lbm_multi_setup *setup, const lbm_geometry *geom, const lbm_probes *probes, lbm_multi *h) {
    if (!setup) throw MErr(LBM_ERR_INVALID, "setup is null");
    const lbm_multi_setup &s = *setup;
    if (s.nboxes && !s.boxes) throw MErr(LBM_ERR_INVALID, "boxes is null");
    if (s.nboxes > 8) throw MErr(LBM_ERR_INVALID, "at most 8 refinement boxes");
    if (s.storage < LBM_STORAGE_FP32 || s.storage > LBM_STORAGE_FP64) throw MErr(LBM_ERR_INVALID, "unknown storage");
    if (!(s.nu0 > 0.0) || !std::isfinite(s.nu0)) throw MErr(LBM_ERR_INVALID, "viscosity must be positive");
    for (int f = 0; f < 6; f++) {
        if (s.faces[f] < LBM_FACE_VELOCITY || s.faces[f] > LBM_FACE_FREE_SLIP) throw MErr(LBM_ERR_INVALID, "unknown face type");
        if (s.faces[f] == LBM_FACE_FREE_SLIP) throw MErr(LBM_ERR_UNSUPPORTED, "free-slip faces are not available on the D3Q27 lattice");
    }
    bool per0[3];
    for (int a = 0; a < 3; a++) {
        const bool p0 = s.faces[2 * a] == LBM_FACE_PERIODIC, p1 = s.faces[2 * a + 1] == LBM_FACE_PERIODIC;
        if (p0 != p1) throw MErr(LBM_ERR_INVALID, "periodic faces must come in pairs");
        per0[a] = p0;
    }
    if (geom && (geom->kind < 0 || geom->kind > 2)) throw MErr(LBM_ERR_INVALID, "unknown geometry kind");
    if (s.dims0[0] < 3 || s.dims0[1] < 3 || s.dims0[2] < 3) throw MErr(LBM_ERR_INVALID, "grid must be at least 3 cells in every direction");
    h->setup = s;
    h->boxes.assign(s.boxes, s.boxes + s.nboxes);
    h->setup.boxes = h->boxes.data();
    h->storage = s.storage;
    const size_t nl = (size_t)s.nboxes + 1, finest = nl - 1;
    // mlattice.rs:198-216
    if (nl > 1 && (per0[0] || per0[1] || per0[2])) throw MErr(LBM_ERR_INVALID, "periodic faces only work without refinement");
    auto dims = [&](size_t l) -> std::array<uint32_t, 3> {
        if (l == 0) return {s.dims0[0], s.dims0[1], s.dims0[2]};
        const lbm_level_box &b = h->boxes[l - 1];
        return {2 * (b.n[0] - 1) + 1, 2 * (b.n[1] - 1) + 1, 2 * (b.n[2] - 1) + 1};
    };
    for (size_t l = 1; l < nl; l++) {
        const lbm_level_box &b = h->boxes[l - 1];
        const auto pd = dims(l - 1);
        for (int k = 0; k < 3; k++) {
            const int64_t hi = (int64_t)b.lo[k] + (int64_t)b.n[k] - 1;
            const int margin = l == 1 ? 2 : 3;
            if (b.lo[k] < margin || hi > (int64_t)pd[k] - 1 - margin || b.n[k] < 8)
                throw MErr(LBM_ERR_INVALID, "refinement box " + std::to_string(l) + " does not fit inside its parent");
        }
    }
    std::vector<std::array<double, 3>> org(nl, {0, 0, 0});
    std::vector<double> scale(nl, 1.0);
    scale[0] = (double)(1ull << finest);
    for (size_t l = 1; l < nl; l++) {
        scale[l] = scale[l - 1] / 2.0;
        for (int k = 0; k < 3; k++) org[l][k] = org[l - 1][k] + h->boxes[l - 1].lo[k] * scale[l - 1];
    }
    // probes (mlattice.rs:243-305): each slice pixel (finest-level
    // coordinates) goes to the finest level whose interior, without its ghost
    // layer, holds the nearest node
    std::vector<float> vbuf;
    std::vector<std::vector<uint32_t>> pix_lists(nl);
    if (probes) {
        if (probes->nvert && !probes->verts) throw MErr(LBM_ERR_INVALID, "probe vertices are null");
        if (probes->nslices && !probes->slices) throw MErr(LBM_ERR_INVALID, "probe slices are null");
        if (probes->nvert >= 0xffffffffull) throw MErr(LBM_ERR_INVALID, "too many probe vertices");
        h->nvert = (uint32_t)probes->nvert;
        h->voff = (float)probes->vertex_offset;
        for (uint64_t v = 0; v < probes->nvert; v++) {
            const double *q = probes->verts + 6 * v;
            const float e[8] = {(float)q[0], (float)q[1], (float)q[2], 0.f, (float)q[3], (float)q[4], (float)q[5], 0.f};
            vbuf.insert(vbuf.end(), e, e + 8);
        }
        uint64_t base = 0;
        for (uint64_t sl = 0; sl < probes->nslices; sl++) {
            const lbm_slice_def &d = probes->slices[sl];
            for (uint32_t iv = 0; iv < d.nv; iv++)
                for (uint32_t iu = 0; iu < d.nu; iu++) {
                    const double pt[3] = {(double)(d.origin[0] + (int64_t)iu * d.u[0] + (int64_t)iv * d.v[0]),
                                          (double)(d.origin[1] + (int64_t)iu * d.u[1] + (int64_t)iv * d.v[1]),
                                          (double)(d.origin[2] + (int64_t)iu * d.u[2] + (int64_t)iv * d.v[2])};
                    for (size_t l = nl; l-- > 0;) {
                        const auto dl = dims(l);
                        const double lo = l == 0 ? 1.0 : 2.0;
                        bool ok = true;
                        uint32_t cell[3];
                        for (int k = 0; k < 3 && ok; k++) {
                            const double x = std::round((pt[k] - org[l][k]) / scale[l]);
                            if (x < lo || x > (double)dl[k] - 1.0 - lo) ok = false;
                            else cell[k] = (uint32_t)x;
                        }
                        if (ok) {
                            pix_lists[l].push_back((uint32_t)(base + (uint64_t)iv * d.nu + iu));
                            pix_lists[l].push_back((cell[2] * dl[1] + cell[1]) * dl[0] + cell[0]);
                            break;
                        }
                    }
                }
            base += (uint64_t)d.nu * d.nv;
            if (base >= 0xffffffffull) throw MErr(LBM_ERR_INVALID, "too many slice pixels");
        }
        h->npix = (uint32_t)base;
    }
    const auto fd = dims(finest);
    const uint64_t NF = (uint64_t)fd[0] * fd[1] * fd[2];

    // A spinning part on the finest level (no counterpart: the reference
    // spins parts on D3Q19 only): every swept-box cell is a record without
    // links, re-voxelized each finest step.
    const lbm_geometry *spin = (geom && geom->kind == 2) ? geom : nullptr;
    std::vector<lbm_wall_cell> boxwalls;
    lbm_geometry boxgeom{};
    if (spin) {
        for (int k = 0; k < 3; k++)
            if (spin->box_lo[k] < 1 || (int64_t)spin->box_lo[k] + (int64_t)spin->box_n[k] > (int64_t)fd[k] - 1 || spin->box_n[k] == 0)
                throw MErr(LBM_ERR_INVALID, "the spinning part's swept box leaves the finest level");
        if (!spin->occ_bits || (spin->ntri && !spin->tris) || !(spin->occ_h > 0.0))
            throw MErr(LBM_ERR_INVALID, "spinning part without occupancy grid or triangles");
        const uint64_t nb = (uint64_t)spin->box_n[0] * spin->box_n[1] * spin->box_n[2];
        if (nb >= 0x1fffffffull || spin->ntri >= 0x7fffffffull) throw MErr(LBM_ERR_INVALID, "swept box too large");
        boxwalls.resize(nb);
        uint64_t k = 0;
        for (uint32_t z = 0; z < spin->box_n[2]; z++)
            for (uint32_t y = 0; y < spin->box_n[1]; y++)
                for (uint32_t x = 0; x < spin->box_n[0]; x++, k++) {
                    boxwalls[k].cell = (uint32_t)((((uint64_t)z + spin->box_lo[2]) * fd[1] + (uint64_t)y + spin->box_lo[1]) * fd[0] + (uint64_t)x + spin->box_lo[0]);
                    boxwalls[k].mask = 0;
                    for (int i = 0; i < 27; i++) boxwalls[k].q[i] = 1.0f;
                }
        boxgeom.kind = 1;
        boxgeom.walls = boxwalls.data();
        boxgeom.nwalls = nb;
        geom = &boxgeom;
    }

    // records (mlattice.rs:178-192, 345-354): words in the reference layout
    const bool stat = geom && geom->kind == 1;
    const uint64_t nrec = stat ? geom->nwalls : 0;
    if (nrec >= 0x1fffffffull) throw MErr(LBM_ERR_INVALID, "too many wall records");
    h->nrec = (uint32_t)nrec;
    std::vector<uint32_t> words(nrec * lbm27::RS, 0u);
    std::vector<std::pair<uint32_t, uint32_t>> rec_of;
    for (uint64_t r = 0; r < nrec; r++) {
        const lbm_wall_cell &w = geom->walls[r];
        if (w.cell >= NF) throw MErr(LBM_ERR_INVALID, "wall cell index outside the finest level");
        uint32_t *o = words.data() + r * lbm27::RS;
        o[lbm27::R_MASK] = w.mask & 0x7ffdfffu;  // 27 directions, rest excluded
        o[lbm27::R_CELL] = w.cell;
        float qs[26];
        for (int k = 0; k < 26; k++) qs[k] = 1.0f;
        for (int i = 0; i < 27; i++)
            if (i != 13) qs[i < 13 ? i : i - 1] = w.q[i];
        for (int k = 0; k < 13; k++) o[lbm27::R_Q + k] = (uint32_t)f16_bits(qs[2 * k]) | ((uint32_t)f16_bits(qs[2 * k + 1]) << 16);
        rec_of.push_back({w.cell, (uint32_t)r + 1});
    }
    std::sort(rec_of.begin(), rec_of.end());
    std::vector<uint32_t> solid;
    if (stat) {
        solid.assign(geom->solid, geom->solid + geom->nsolid);
        for (uint32_t c : solid)
            if (c >= NF) throw MErr(LBM_ERR_INVALID, "solid cell index outside the finest level");
    }
    std::sort(solid.begin(), solid.end());

    ck(cudaGetDevice(&h->device), "cudaGetDevice");
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&h->ev, cudaEventDisableTiming), "cudaEventCreate");
    const size_t esz = storage_bytes(s.storage);
    const size_t rsz = s.storage == LBM_STORAGE_FP64 ? 8 : 4;  // moment buffers in the arithmetic type

    h->lv.assign(nl, Level());
    uint64_t max_n = 0;
    for (size_t l = 0; l < nl; l++) {
        Level &L = h->lv[l];
        lbm27::LevelParams &p = L.p;
        const auto d = dims(l);
        const uint64_t N = (uint64_t)d[0] * d[1] * d[2];
        if (N >= 0xffffffffull) throw MErr(LBM_ERR_INVALID, "level " + std::to_string(l) + " has too many cells");
        max_n = std::max(max_n, N);
        p.NX = d[0]; p.NY = d[1]; p.NZ = d[2]; p.N = (uint32_t)N;
        p.div_nx.init(d[0]);
        p.div_nxy.init(d[0] * d[1]);
        for (int a = 0; a < 3; a++) p.per[a] = l == 0 ? per0[a] : 0;
        p.n_sponge = 0;
        if (l == 0)
            for (int f = 0; f < 6; f++) p.n_sponge |= s.sponge[f] > 0;
        p.forcing = s.body_force0[0] != 0.0 || s.body_force0[1] != 0.0 || s.body_force0[2] != 0.0;
        p.abs_u = s.absorb_velocity != 0;
        p.total_p = s.total_pressure_inlet != 0;
        p.has_child = l + 1 < nl;
        p.has_parent = l > 0;
        if (p.has_child) {
            for (int k = 0; k < 3; k++) { p.ch_lo[k] = h->boxes[l].lo[k]; p.ch_n[k] = h->boxes[l].n[k]; }
            p.ch_nodes = p.ch_n[0] * p.ch_n[1] * p.ch_n[2];
        } else {
            for (int k = 0; k < 3; k++) { p.ch_lo[k] = 0; p.ch_n[k] = 1; }
            p.ch_nodes = 1;
        }
        for (int k = 0; k < 3; k++) p.pn[k] = (d[k] - 1) / 2 + 1;
        fill27<float>(p.kf, s, l, finest, org);
        fill27<double>(p.kd, s, l, finest, org);
        // cell types and lists (mlattice.rs:404-478)
        const uint32_t nx = d[0], ny = d[1], nz = d[2];
        std::vector<uint32_t> flags(N, 0u), faces, ghosts, restricted;
        size_t si = 0, fi = 0;
        for (uint64_t cc = 0; cc < N; cc++) {
            const uint32_t x = (uint32_t)(cc % nx), y = (uint32_t)((cc / nx) % ny), z = (uint32_t)(cc / ((uint64_t)nx * ny));
            int ty = 0;
            if (l == 0) {
                const bool on[6] = {x == 0, x == nx - 1, y == 0, y == ny - 1, z == 0, z == nz - 1};
                for (int f = 0; f < 6; f++)
                    if (on[f] && s.faces[f] != LBM_FACE_PERIODIC) ty = ty == 1 ? 1 : (s.faces[f] == LBM_FACE_VELOCITY ? 1 : 2);
            }
            const bool ghost = l > 0 && (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1);
            bool restr = p.has_child;
            if (restr) {
                const int q[3] = {(int)x, (int)y, (int)z};
                for (int k = 0; k < 3; k++) restr = restr && q[k] >= p.ch_lo[k] + 2 && q[k] <= p.ch_lo[k] + (int)p.ch_n[k] - 3;
            }
            uint32_t v = 0;
            if (ty) { v = lbm27::T_FACE | ((uint32_t)ty << 3); faces.push_back((uint32_t)cc); }
            else if (ghost) { v = lbm27::T_GHOST; ghosts.push_back((uint32_t)cc); }
            else if (restr) { v = lbm27::T_RESTRICT; restricted.push_back((uint32_t)cc); }
            if (l == finest) {
                while (si < solid.size() && solid[si] < cc) si++;
                while (si < solid.size() && solid[si] == cc) { if (v == 0) v = lbm27::T_SOLID; si++; }
                while (fi < rec_of.size() && rec_of[fi].first < cc) fi++;
                while (fi < rec_of.size() && rec_of[fi].first == cc) {
                    if ((v & 7u) == 0 || (v & 7u) == lbm27::T_SOLID) v = (v & 7u) | (rec_of[fi].second << 3);
                    fi++;
                }
            }
            flags[cc] = v;
        }
        p.nface = (uint32_t)faces.size();
        p.nghost = (uint32_t)ghosts.size();
        p.nrestrict = (uint32_t)restricted.size();
        // device arrays
        p.NP = (N + 255) / 256 * 256;
        p.pop = h->dalloc(2 * 27 * p.NP * esz);
        p.flags = (uint32_t *)h->dalloc(N * 4);
        ck(cudaMemcpyAsync(p.flags, flags.data(), N * 4, cudaMemcpyHostToDevice, h->stream), "flags upload");
        auto upload_list = [&](const std::vector<uint32_t> &v) -> const uint32_t * {
            if (v.empty()) return nullptr;
            uint32_t *d_ = (uint32_t *)h->dalloc(v.size() * 4);
            ck(cudaMemcpyAsync(d_, v.data(), v.size() * 4, cudaMemcpyHostToDevice, h->stream), "list upload");
            return d_;
        };
        p.faces = upload_list(faces);
        p.ghosts = upload_list(ghosts);
        p.restricted = upload_list(restricted);
        ck(lbm::stream_wait(h->stream, h->timeout_s), "upload");
        const double tau_l = 0.5 + 3.0 * s.nu0 * (double)(1ull << l);
        if (p.has_child) {
            p.mom_child = h->dalloc(2ull * p.ch_nodes * lbm27::MW * rsz);
            if (rsz == 8) init_moments<double>(h, p.mom_child, 2ull * p.ch_nodes, s, tau_l);
            else init_moments<float>(h, p.mom_child, 2ull * p.ch_nodes, s, tau_l);
        }
        if (p.has_parent) {
            const uint64_t pn = (uint64_t)p.pn[0] * p.pn[1] * p.pn[2];
            p.mom_up = h->dalloc(pn * lbm27::MW * rsz);
            if (rsz == 8) init_moments<double>(h, p.mom_up, pn, s, tau_l);
            else init_moments<float>(h, p.mom_up, pn, s, tau_l);
        }
    }
    for (size_t l = 0; l < nl; l++) {
        if (l > 0) h->lv[l].p.mom_parent = h->lv[l - 1].p.mom_child;
        if (l + 1 < nl) h->lv[l].p.mom_child_up = h->lv[l + 1].p.mom_up;
    }
    // shared (finest-level) buffers
    h->recs = (uint32_t *)h->dalloc(std::max<uint64_t>(nrec, 1) * lbm27::RS * 4);
    if (nrec) ck(cudaMemcpyAsync(h->recs, words.data(), words.size() * 4, cudaMemcpyHostToDevice, h->stream), "records upload");
    if (s.storage == LBM_STORAGE_FP64) {
        h->recd = (double *)h->dalloc(std::max<uint64_t>(nrec, 1) * 6 * 8);
        ck(cudaMemsetAsync(h->recd, 0, std::max<uint64_t>(nrec, 1) * 6 * 8, h->stream), "records init");
    }
    h->wallf = h->dalloc(std::max<uint64_t>(nrec, 1) * 27 * rsz);
    h->partials = (double *)h->dalloc((size_t)std::max<uint32_t>(lbm27::reduce27_blocks(h->nrec), 1) * 8 * 8);
    h->ticket = (uint32_t *)h->dalloc(16);
    ck(cudaMemsetAsync(h->ticket, 0, 16, h->stream), "ticket init");
    h->hist = (double *)h->dalloc(HIST_CAP * 8 * 8);
    ck(cudaMemsetAsync(h->hist, 0, HIST_CAP * 8 * 8, h->stream), "history init");
    h->verts = (float *)h->dalloc(std::max<size_t>(vbuf.size(), 8) * 4);
    if (!vbuf.empty()) ck(cudaMemcpyAsync(h->verts, vbuf.data(), vbuf.size() * 4, cudaMemcpyHostToDevice, h->stream), "upload vertices");
    h->vacc = (double *)h->dalloc(std::max<uint64_t>(h->nvert, 1) * 2 * sizeof(double));
    h->sacc = (double *)h->dalloc(std::max<uint64_t>(h->npix, 1) * 5 * sizeof(double));
    ck(cudaMemsetAsync(h->vacc, 0, std::max<uint64_t>(h->nvert, 1) * 2 * sizeof(double), h->stream), "memset");
    ck(cudaMemsetAsync(h->sacc, 0, std::max<uint64_t>(h->npix, 1) * 5 * sizeof(double), h->stream), "memset");
    for (size_t l = 0; l < nl; l++) {
        h->npix_l.push_back((uint32_t)(pix_lists[l].size() / 2));
        h->pix.push_back((uint32_t *)h->dalloc(std::max<size_t>(pix_lists[l].size(), 2) * 4));
        if (!pix_lists[l].empty())
            ck(cudaMemcpyAsync(h->pix[l], pix_lists[l].data(), pix_lists[l].size() * 4, cudaMemcpyHostToDevice, h->stream), "upload pixels");
    }
    ck(lbm::stream_wait(h->stream, h->timeout_s), "probe upload");  // host vectors go out of scope
    ck(cudaMallocHost(&h->hist_host, HIST_CAP * 8 * 8), "cudaMallocHost");
    h->mass_d = (double *)h->dalloc((2 + 2 * (size_t)lbm27::mass27_blocks()) * sizeof(double) + 16);
    ck(cudaMemset(h->mass_d, 0, (2 + 2 * (size_t)lbm27::mass27_blocks()) * sizeof(double) + 16), "memset");
    if (s.debug_dump) h->dump = (float4 *)h->dalloc(max_n * sizeof(float4));
    if (spin) {
        lbm27::LevelParams &p = h->lv[finest].p;
        p.moving = 1;
        const uint64_t nocc = (uint64_t)spin->occ_dims[0] * spin->occ_dims[1] * spin->occ_dims[2];
        const uint64_t wocc = (nocc + 31) / 32;
        p.occ = (const uint32_t *)h->dalloc(wocc * 4);
        ck(cudaMemcpy((void *)p.occ, spin->occ_bits, wocc * 4, cudaMemcpyHostToDevice), "upload occupancy");
        for (int k = 0; k < 3; k++) {
            p.occ_lo[k] = (float)spin->occ_lo[k];
            p.occ_n[k] = (int32_t)spin->occ_dims[k];
            p.box_lo[k] = spin->box_lo[k];
            p.box_n[k] = spin->box_n[k];
        }
        p.occ_invh = (float)(1.0 / spin->occ_h);
        p.ntri = (uint32_t)spin->ntri;
        p.tris = (const float4 *)h->dalloc(std::max<uint64_t>(spin->ntri, 1) * 48);
        if (spin->ntri) ck(cudaMemcpy((void *)p.tris, spin->tris, spin->ntri * 48, cudaMemcpyHostToDevice), "upload triangles");
        std::vector<uint32_t> q0((size_t)h->nrec * 39, 0u);
        for (size_t k = 0; k < q0.size(); k += 3) q0[k] = 0x7f7fffffu;  // nearest hit: FLT_MAX
        p.qscr = (uint32_t *)h->dalloc(q0.size() * 4);
        ck(cudaMemcpy(p.qscr, q0.data(), q0.size() * 4, cudaMemcpyHostToDevice), "upload link scratch");
    }
    for (size_t l = 0; l < nl; l++) {
        lbm27::LevelParams &p = h->lv[l].p;
        p.dump = h->dump;
        if (l == finest) { p.recs = h->recs; p.recd = h->recd; p.wallf = h->wallf; p.nrec = h->nrec; }
        else { p.recs = nullptr; p.recd = nullptr; p.wallf = nullptr; p.nrec = 0; }
        ck(lbm27::launch27_init(s.storage, p, h->stream), "init kernel");
    }
    h->wait();
}

}  // namespace

extern "C" {

int lbm_create_multi(const lbm_multi_setup *setup, const lbm_geometry *geom, const lbm_probes *probes, lbm_multi **out) {
    if (!out) { lbm_host::set_global_error("out is null"); return LBM_ERR_INVALID; }
    *out = nullptr;
    lbm_multi *h = new lbm_multi();
    int rc = mguard(nullptr, [&] { create_multi(setup, geom, probes, h); });
    if (rc != LBM_OK) { delete h; return rc; }
    *out = h;
    return LBM_OK;
}

void lbm_multi_destroy(lbm_multi *h) { delete h; }

int lbm_multi_last_error(const lbm_multi *h, char *buf, uint64_t len) {
    if (!h) return LBM_ERR_INVALID;
    if (buf && len) std::snprintf(buf, (size_t)len, "%s", h->err.c_str());
    return LBM_OK;
}

int lbm_multi_levels(const lbm_multi *h, uint32_t *levels) {
    if (!h || !levels) return LBM_ERR_INVALID;
    *levels = (uint32_t)h->lv.size();
    return LBM_OK;
}

int lbm_multi_sub_steps(const lbm_multi *h, uint32_t *sub_steps) {
    if (!h || !sub_steps) return LBM_ERR_INVALID;
    *sub_steps = (uint32_t)h->sub_steps();
    return LBM_OK;
}

int lbm_multi_level_dims(const lbm_multi *h, uint32_t *dims) {
    if (!h || !dims) return LBM_ERR_INVALID;
    for (size_t l = 0; l < h->lv.size(); l++) { dims[3 * l] = h->lv[l].p.NX; dims[3 * l + 1] = h->lv[l].p.NY; dims[3 * l + 2] = h->lv[l].p.NZ; }
    return LBM_OK;
}

int lbm_multi_level_cells(const lbm_multi *h, uint64_t *cells) {
    if (!h || !cells) return LBM_ERR_INVALID;
    for (size_t l = 0; l < h->lv.size(); l++) cells[l] = h->lv[l].p.N;
    return LBM_OK;
}

int lbm_multi_run(lbm_multi *h, const lbm_step_in *steps, uint64_t n, double *forces_out) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        if (n && !steps) throw MErr(LBM_ERR_INVALID, "steps is null");
        h->run(steps, n, forces_out);
    });
}

int lbm_multi_advance(lbm_multi *h, uint64_t n) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] { h->run(nullptr, n, nullptr); });
}

int lbm_multi_stream(lbm_multi *h, void **stream) {
    if (!h || !stream) return LBM_ERR_INVALID;
    *stream = (void *)h->stream;
    return LBM_OK;
}

int lbm_multi_synchronize(lbm_multi *h) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] { h->wait(); });
}

int lbm_multi_set_timeout(lbm_multi *h, double seconds) {
    if (!h || !(seconds > 0)) return LBM_ERR_INVALID;
    h->timeout_s = seconds;
    return LBM_OK;
}

int lbm_multi_macros(lbm_multi *h, uint32_t level, float *out) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        if (!out) throw MErr(LBM_ERR_INVALID, "out is null");
        if (level >= h->lv.size()) throw MErr(LBM_ERR_INVALID, "no such level");
        if (!h->dump) throw MErr(LBM_ERR_STATE, "macros() needs debug_dump");
        const Level &L = h->lv[level];
        ck(lbm27::launch27_dump(h->storage, L.p, L.src, h->stream), "dump kernel");
        ck(cudaMemcpyAsync(out, h->dump, (size_t)L.p.N * sizeof(float4), cudaMemcpyDeviceToHost, h->stream), "macros readback");
        h->wait();
    });
}

int lbm_multi_records(lbm_multi *h, uint32_t *out, uint64_t cap_words) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        const uint64_t words = (uint64_t)h->nrec * lbm27::RS;
        if (!out || cap_words < words) throw MErr(LBM_ERR_INVALID, "output too small for the records");
        if (words) ck(cudaMemcpyAsync(out, h->recs, words * 4, cudaMemcpyDeviceToHost, h->stream), "records readback");
        h->wait();
    });
}

int lbm_multi_reset_samples(lbm_multi *h) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        ck(cudaMemsetAsync(h->vacc, 0, std::max<uint64_t>(h->nvert, 1) * 2 * sizeof(double), h->stream), "memset");
        ck(cudaMemsetAsync(h->sacc, 0, std::max<uint64_t>(h->npix, 1) * 5 * sizeof(double), h->stream), "memset");
        h->wait();
    });
}

int lbm_multi_vertex_means(lbm_multi *h, float *out) {
    if (!h || (!out && h->nvert)) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        if (!h->nvert) return;
        std::vector<double> v(2 * (size_t)h->nvert);
        ck(cudaMemcpyAsync(v.data(), h->vacc, v.size() * 8, cudaMemcpyDeviceToHost, h->stream), "vertex readback");
        h->wait();
        for (uint32_t i = 0; i < h->nvert; i++) out[i] = v[2 * i + 1] > 0 ? (float)(v[2 * i] / v[2 * i + 1]) : NAN;
    });
}

int lbm_multi_slice_means(lbm_multi *h, float *out) {
    if (!h || (!out && h->npix)) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        if (!h->npix) return;
        std::vector<double> v(5 * (size_t)h->npix);
        ck(cudaMemcpyAsync(v.data(), h->sacc, v.size() * 8, cudaMemcpyDeviceToHost, h->stream), "slice readback");
        h->wait();
        for (uint32_t i = 0; i < h->npix; i++) {
            const double c = v[5 * i + 4];
            for (int a = 0; a < 4; a++) out[4 * i + a] = c > 0 ? (float)(v[5 * i + a] / c) : NAN;
        }
    });
}

int lbm_multi_get_info(const lbm_multi *h, lbm_info *out) {
    if (!h || !out) return LBM_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    out->steps_done = h->fine_steps;
    out->nrec = h->nrec;
    out->nface = h->lv.empty() ? 0 : h->lv[0].p.nface;
    out->nvert = h->nvert;
    out->npix = h->npix;
    out->memory_bytes = h->memory_bytes;
    for (const Level &L : h->lv) out->cells += L.p.N;
    out->storage = h->storage;
    out->collision = -1;
    return LBM_OK;
}

int lbm_multi_mass(lbm_multi *h, uint32_t level, double *mass, uint64_t *nonfinite) {
    if (!h) return LBM_ERR_INVALID;
    return mguard(h, [&] {
        if (!mass || !nonfinite) throw MErr(LBM_ERR_INVALID, "null output");
        if (level >= h->lv.size()) throw MErr(LBM_ERR_INVALID, "no such level");
        const Level &L = h->lv[level];
        ck(lbm27::launch27_mass(h->storage, L.p, L.src, h->mass_d + 2, h->mass_d, h->stream), "mass kernel");
        double hv[2];
        ck(cudaMemcpyAsync(hv, h->mass_d, 16, cudaMemcpyDeviceToHost, h->stream), "mass readback");
        h->wait();
        *mass = hv[0];
        *nonfinite = (uint64_t)hv[1];
    });
}

}  // extern "C"
