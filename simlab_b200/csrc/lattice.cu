// Host driver of the D3Q19 engine and the C ABI of include/simlab_lbm.h.
//
// Mirrors `Lattice` of crates/cfd/src/lattice.rs: setup validation (233-271),
// face list (283-324), wall records (454-482, record_words 202-218), flags
// (489-526), initial state (661-671), the per-step dispatch (701-753), field
// and record readback (785-841).  Differences by design: one allocation per
// buffer in HBM (no 4 GiB split), one CUDA stream per handle, device waits
// bounded by a host-side limit, forces summed in FP64.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/simlab_lbm.h"
#include "host_wait.hpp"
#include "lbm_kernels.h"
#include "voxel.hpp"

#ifndef LBM_SIDE_PRIORITY
#define LBM_SIDE_PRIORITY 1  // wall-cell stream at the device's greatest priority
#endif

namespace {

thread_local std::string g_error;

constexpr uint32_t KMAX = 512;  // steps per readback chunk (lattice.rs:134)

struct LbmError : std::runtime_error {
    int code;
    LbmError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? LBM_ERR_NOMEM : LBM_ERR_CUDA;
        throw LbmError(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

inline uint32_t fbits(float x) { uint32_t b; std::memcpy(&b, &x, 4); return b; }

// lattice.rs:172-189
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

inline double weight19(int i) { return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }

size_t storage_bytes(int s) { return s == LBM_STORAGE_FP32 ? 4 : (s == LBM_STORAGE_FP64 ? 8 : 2); }

}  // namespace

// creation errors of the other handle types land in the same message
namespace lbm_host {
void set_global_error(const std::string &msg) { g_error = msg; }
}  // namespace lbm_host

struct lbm_lattice {
    lbm_setup setup{};
    lbm::LatParams lp{};
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // wall-cell kernel, when it cannot touch the faces' slots
    cudaEvent_t fork = nullptr, join = nullptr;
    int device = 0;
    std::vector<void *> allocs;
    uint64_t steps_done = 0;
    uint64_t memory_bytes = 0;
    uint32_t nrec = 0, nface = 0, npix = 0, nvert = 0;
    double timeout_s = 600.0;
    std::string err;
    // sampling
    double *vacc = nullptr;     // 2 doubles per vertex (sum, count)
    double *sacc = nullptr;     // 5 doubles per pixel
    float *verts = nullptr;     // 8 floats per vertex
    int32_t *slicedef = nullptr;
    uint32_t nslices = 0;
    float voff = 0.f;
    double *hist_host = nullptr;  // pinned
    cudaEvent_t ev = nullptr;
    // kernel profiling: 4 events per profiled step (mode 1), or only the two
    // around the bulk kernel (mode 2)
    bool prof = false;
    int prof_mode = 0;
    std::vector<cudaEvent_t> prof_ev;
    uint64_t prof_steps = 0;
    uint64_t prof_launches = 0;  // kernels launched by the profiled steps
    uint64_t pop_bytes = 0;
    uint32_t nface_rest = 0;   // face cells the face kernel handles once x faces are fused
    bool xfuse = false;        // planar x faces are written by the staged kernel
    bool fused_valid = false;  // the last step wrote the fused x faces for the next one
    uint32_t *err_host = nullptr;  // pinned

    void *dalloc(size_t bytes) {
        void *p = nullptr;
        ck(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc");
        allocs.push_back(p);
        memory_bytes += std::max<size_t>(bytes, 16);
        return p;
    }
    ~lbm_lattice() {
        // bounded waits: if the device never finishes, the buffers it may
        // still use are left allocated rather than freed under it
        if ((stream && lbm::stream_wait(stream, timeout_s) == cudaErrorTimeout) ||
            (side && lbm::stream_wait(side, timeout_s) == cudaErrorTimeout)) {
            lbm_host::set_global_error("lattice destroyed while its device work had not finished: buffers left allocated");
            return;
        }
        for (void *p : allocs) cudaFree(p);
        if (hist_host) cudaFreeHost(hist_host);
        if (err_host) cudaFreeHost(err_host);
        if (ev) cudaEventDestroy(ev);
        for (cudaEvent_t e : prof_ev) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
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
            if (el > timeout_s) throw LbmError(LBM_ERR_TIMEOUT, "device did not finish within " + std::to_string(timeout_s) + " s");
            if (el > 1e-3) std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    int parity() const { return (int)(steps_done % 2); }
    void check_device_errors() {
        if (err_host && *err_host) {
            const uint32_t e = *err_host;
            *err_host = 0;
            cudaMemsetAsync(lp.err, 0, 4, stream);
            if (e & lbm::ERR_COPY_WAIT) throw LbmError(LBM_ERR_TIMEOUT, "a bulk-copy wait in the step kernel passed its iteration limit");
            throw LbmError(LBM_ERR_CUDA, "device error bits " + std::to_string(e));
        }
    }
};

namespace {

int fail(lbm_lattice *h, const LbmError &e) {
    if (h) h->err = e.what(); else g_error = e.what();
    return e.code;
}

template <class F>
int guard(lbm_lattice *h, F &&fn) {
    try {
        fn();
        return LBM_OK;
    } catch (const LbmError &e) {
        return fail(h, e);
    } catch (const std::exception &e) {
        return fail(h, LbmError(LBM_ERR_INVALID, e.what()));
    }
}

template <class R>
void fill_consts(lbm::Consts<R> &k, const lbm_setup &st) {
    k.tau0 = (R)(0.5 + 3.0 * st.nu);
    k.smag2 = (R)(st.smagorinsky * st.smagorinsky);
    k.sponge_tau = (R)st.sponge_tau;
    k.sigma = (R)st.sponge_sigma;
    for (int a = 0; a < 3; a++) {
        k.sp_lo[a] = (R)st.sponge[2 * a];
        k.sp_hi[a] = (R)st.sponge[2 * a + 1];
        k.u_inf[a] = (R)st.u_inf[a];
        k.u_init[a] = (R)st.u_init[a];
        k.grav[a] = (R)st.body_force[a];
        k.center[a] = (R)st.center[a];
        k.sp_lo_inv[a] = st.sponge[2 * a] ? (R)(1.0 / st.sponge[2 * a]) : (R)0;
        k.sp_hi_inv[a] = st.sponge[2 * a + 1] ? (R)(1.0 / st.sponge[2 * a + 1]) : (R)0;
    }
    const double usq = 1.5 * (st.u_inf[0] * st.u_inf[0] + st.u_inf[1] * st.u_inf[1] + st.u_inf[2] * st.u_inf[2]);
    k.ft_rest = (R)(-(1.0 / 3.0) * usq);
    for (int kk = 0; kk < 9; kk++) {
        const int i = 2 * kk + 1;
        const double w = kk < 3 ? 1.0 / 18.0 : 1.0 / 36.0;
        const double cu = lbm::CX(i) * st.u_inf[0] + lbm::CY(i) * st.u_inf[1] + lbm::CZ(i) * st.u_inf[2];
        k.ft_even[kk] = (R)(w * (4.5 * cu * cu - usq));
        k.ft_odd[kk] = (R)(w * 3.0 * cu);
    }
}

lbm::StepParams step_params(const lbm_lattice *h, const lbm_step_in &s, uint32_t slot, uint64_t step_index) {
    lbm::StepParams sp{};
    sp.seed = (uint32_t)step_index * lbm::STEP_SEED_MUL;  // lattice.rs:676
    sp.seed_mix = sp.seed * 0x85EBCA77u + 0x632BE5ABu;
    sp.next_seed_mix = ((uint32_t)(step_index + 1) * lbm::STEP_SEED_MUL) * 0x85EBCA77u + 0x632BE5ABu;
    sp.nface = h->fused_valid ? h->nface_rest : h->nface;
    sp.slot = slot;
    for (int a = 0; a < 3; a++) {
        sp.omega[a] = (float)s.omega[a];
        sp.omega_d[a] = s.omega[a];
    }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            sp.rot[r * 3 + c] = (float)s.rot[r][c];
            sp.rot_prev[r * 3 + c] = (float)s.rot_prev[r][c];
        }
    (void)h;
    return sp;
}

void create_impl(const lbm_setup *setup, const lbm_geometry *geom, const lbm_probes *probes, lbm_lattice *h) {
    if (!setup) throw LbmError(LBM_ERR_INVALID, "setup is null");
    const lbm_setup &st = *setup;
    const uint64_t NX = st.dims[0], NY = st.dims[1], NZ = st.dims[2];
    const uint64_t N = NX * NY * NZ;
    // lattice.rs:233-244
    if (N == 0 || N >= 0xffffffffull) throw LbmError(LBM_ERR_INVALID, "grid of " + std::to_string(N) + " cells is out of range");
    if (NX < 3 || NY < 3 || NZ < 3) throw LbmError(LBM_ERR_INVALID, "grid must be at least 3 cells in every direction");
    int per[3];
    for (int a = 0; a < 3; a++) {
        bool p0 = st.faces[2 * a] == LBM_FACE_PERIODIC, p1 = st.faces[2 * a + 1] == LBM_FACE_PERIODIC;
        if (p0 != p1) throw LbmError(LBM_ERR_INVALID, "periodic faces must come in pairs");
        per[a] = p0;
    }
    for (int f = 0; f < 6; f++)
        if (st.faces[f] < LBM_FACE_VELOCITY || st.faces[f] > LBM_FACE_FREE_SLIP) throw LbmError(LBM_ERR_INVALID, "unknown face type");
    if (st.storage < LBM_STORAGE_FP32 || st.storage > LBM_STORAGE_FP64) throw LbmError(LBM_ERR_INVALID, "unknown storage");
    if (st.collision != LBM_COLLISION_REGULARIZED && st.collision != LBM_COLLISION_BGK) throw LbmError(LBM_ERR_INVALID, "unknown collision");
    if (!(st.nu > 0.0) || !std::isfinite(st.nu)) throw LbmError(LBM_ERR_INVALID, "viscosity must be positive");
    if (geom && (geom->kind < 0 || geom->kind > 2)) throw LbmError(LBM_ERR_INVALID, "unknown geometry kind");
    h->setup = st;

    // face cells (lattice.rs:283-324) plus free slip: velocity sticks,
    // otherwise the later face in -x,+x,-y,+y,-z,+z order wins; free-slip
    // faces collect their mirror axes.
    std::vector<uint32_t> faces;
    std::vector<uint32_t> finfo;
    auto face_type = [&](uint64_t x, uint64_t y, uint64_t z, uint32_t &info) -> bool {
        bool on[6] = {x == 0, x == NX - 1, y == 0, y == NY - 1, z == 0, z == NZ - 1};
        int ty = -1;
        uint32_t mir = 0;
        for (int f = 0; f < 6; f++) {
            if (on[f] && st.faces[f] != LBM_FACE_PERIODIC) {
                int t = st.faces[f] == LBM_FACE_VELOCITY ? 0 : (st.faces[f] == LBM_FACE_OPEN ? 1 : 2);
                if (st.faces[f] == LBM_FACE_FREE_SLIP) mir |= 1u << (f / 2);
                ty = (ty == 0) ? 0 : t;
            }
        }
        if (ty < 0) return false;
        info = (uint32_t)ty | (ty == 2 ? (mir << 2) : 0u);
        return true;
    };
    // a face cell's populations matter only where they stream into a cell
    // that collides: bit i of the store mask is set when x + c_i is inside
    // the domain (periodic axes wrap) and not itself a face cell
    const uint64_t dimv[3] = {NX, NY, NZ};
    auto on_face = [&](const int64_t c[3]) {
        for (int a = 0; a < 3; a++)
            if (!per[a] && (c[a] == 0 || c[a] == (int64_t)dimv[a] - 1)) return true;
        return false;
    };
    auto store_mask = [&](uint64_t x, uint64_t y, uint64_t z) {
        uint32_t mask = 0;
        for (int i = 0; i < 19; i++) {
            int64_t c[3] = {(int64_t)x + lbm::CX(i), (int64_t)y + lbm::CY(i), (int64_t)z + lbm::CZ(i)};
            bool ok = true;
            for (int a = 0; a < 3; a++) {
                if (c[a] < 0 || c[a] >= (int64_t)dimv[a]) {
                    if (!per[a]) ok = false;
                    else c[a] = (c[a] + (int64_t)dimv[a]) % (int64_t)dimv[a];
                }
            }
            if (ok && !on_face(c)) mask |= 1u << i;
        }
        return mask;
    };
    for (uint64_t z = 0; z < NZ; z++)
        for (uint64_t y = 0; y < NY; y++) {
            bool edge = y == 0 || y == NY - 1 || z == 0 || z == NZ - 1;
            auto visit = [&](uint64_t x) {
                uint32_t info;
                if (face_type(x, y, z, info)) {
                    faces.push_back((uint32_t)((z * NY + y) * NX + x));
                    finfo.push_back(info | (store_mask(x, y, z) << 8));
                }
            };
            if (edge) { for (uint64_t x = 0; x < NX; x++) visit(x); }
            else { visit(0); visit(NX - 1); }
        }
    h->nface = (uint32_t)faces.size();

    // A spinning part (lattice.rs:260-271, 465-480): every cell of the swept
    // box is a record with no cut link and the initial state; the GPU
    // re-voxelizer rewrites its flag, links and q every step.
    const lbm_geometry *spin = (geom && geom->kind == 2) ? geom : nullptr;
    std::vector<lbm_wall_cell> boxwalls;
    lbm_geometry boxgeom{};
    if (spin) {
        for (int k = 0; k < 3; k++)
            if (spin->box_lo[k] < 1 || (int64_t)spin->box_lo[k] + (int64_t)spin->box_n[k] > (int64_t)st.dims[k] - 1 || spin->box_n[k] == 0)
                throw LbmError(LBM_ERR_INVALID, "the spinning part's swept box leaves the domain");
        if (!spin->occ_bits || (spin->ntri && !spin->tris) || !(spin->occ_h > 0.0))
            throw LbmError(LBM_ERR_INVALID, "spinning part without occupancy grid or triangles");
        if (spin->ntri >= 0x7fffffffull) throw LbmError(LBM_ERR_INVALID, "too many triangles");
        const uint64_t nb = (uint64_t)spin->box_n[0] * spin->box_n[1] * spin->box_n[2];
        if (nb >= 0x3fffffffull) throw LbmError(LBM_ERR_INVALID, "swept box too large");
        boxwalls.resize(nb);
        uint64_t k = 0;
        for (uint32_t z = 0; z < spin->box_n[2]; z++)
            for (uint32_t y = 0; y < spin->box_n[1]; y++)
                for (uint32_t x = 0; x < spin->box_n[0]; x++, k++) {
                    lbm_wall_cell &w = boxwalls[k];
                    w.cell = (uint32_t)((((uint64_t)z + spin->box_lo[2]) * NY + (uint64_t)y + spin->box_lo[1]) * NX + (uint64_t)x + spin->box_lo[0]);
                    w.mask = 0;
                    for (int i = 0; i < 27; i++) w.q[i] = 1.0f;
                }
        boxgeom.kind = 1;
        boxgeom.walls = boxwalls.data();
        boxgeom.nwalls = nb;
        geom = &boxgeom;
    }

    // wall records (lattice.rs:454-482; record_words 202-218)
    const bool stat = geom && geom->kind == 1;
    const uint64_t nrec = stat ? geom->nwalls : 0;
    if (nrec > lbm::MAX_RECORDS) throw LbmError(LBM_ERR_INVALID, "too many wall records");
    h->nrec = (uint32_t)nrec;
    std::vector<uint32_t> words(nrec * lbm::RS, 0);
    std::vector<double> wordsd;
    if (st.storage == LBM_STORAGE_FP64) wordsd.assign(nrec * lbm::RD, 0.0);
    {
        float fe[19];
        double fed[19];
        double usq = 1.5 * (st.u_init[0] * st.u_init[0] + st.u_init[1] * st.u_init[1] + st.u_init[2] * st.u_init[2]);
        for (int i = 0; i < 19; i++) {
            double cu = lbm::CX(i) * st.u_init[0] + lbm::CY(i) * st.u_init[1] + lbm::CZ(i) * st.u_init[2];
            fed[i] = weight19(i) * (3.0 * cu + 4.5 * cu * cu - usq);
            fe[i] = (float)fed[i];
        }
        for (uint64_t r = 0; r < nrec; r++) {
            const lbm_wall_cell &w = geom->walls[r];
            if (w.cell >= N) throw LbmError(LBM_ERR_INVALID, "wall cell index outside the grid");
            uint32_t *o = words.data() + r * lbm::RS;
            o[lbm::R_MASK] = w.mask & 0x7fffeu;  // directions 1..18
            o[lbm::R_CELL] = w.cell;
            for (int k = 0; k < 9; k++) o[lbm::R_Q + k] = (uint32_t)f16_bits(w.q[2 * k + 1]) | ((uint32_t)f16_bits(w.q[2 * k + 2]) << 16);
            for (int i = 1; i < 19; i++) o[lbm::R_FPOST + i - 1] = fbits(fe[i]);
            o[lbm::R_MACRO] = fbits(1.0f);
            for (int a = 0; a < 3; a++) o[lbm::R_MACRO + 1 + a] = fbits((float)st.u_init[a]);
            if (!wordsd.empty()) {
                double *d = wordsd.data() + r * lbm::RD;
                for (int i = 1; i < 19; i++) d[lbm::RD_FPOST + i - 1] = fed[i];
                d[lbm::RD_MACRO] = 1.0;
                for (int a = 0; a < 3; a++) d[lbm::RD_MACRO + 1 + a] = st.u_init[a];
            }
        }
    }
    // flags (lattice.rs:489-526)
    std::vector<uint32_t> flags(N, 0);
    for (size_t k = 0; k < faces.size(); k++) flags[faces[k]] = (finfo[k] & 3u) == 0 ? 2u : 3u;
    if (stat) {
        for (uint64_t s = 0; s < geom->nsolid; s++) {
            uint32_t c = geom->solid[s];
            if (c >= N) throw LbmError(LBM_ERR_INVALID, "solid cell index outside the grid");
            if (flags[c] == 0) flags[c] = 1;
        }
        for (uint64_t r = 0; r < nrec; r++) {
            uint32_t c = geom->walls[r].cell;
            if ((flags[c] & 3u) == 0) flags[c] = (uint32_t)(r + 1) << 2;  // a later record of the same cell wins
        }
    }

    // Planar x-face cells (x = 0 or NX - 1, y and z inside) whose inner
    // neighbour m = b +- 1 is a plain fluid cell are written by the staged
    // kernel while it collides m (flag bit FLAG_XFACE on m), one step ahead;
    // only the first step after setup or a state load needs the face kernel
    // for them.  They go to the end of the face list.
    const bool tma_ok = (NX * storage_bytes(st.storage)) % 16 == 0 && !per[0] && !per[1];
    std::vector<char> fused(faces.size(), 0);
    uint32_t xinfo[2] = {0, 0};
    // (not with a spinning part, whose re-voxelizer rewrites the box flags)
    if (tma_ok && !spin && !(std::getenv("SIMLAB_LBM_NO_TMA") && std::getenv("SIMLAB_LBM_NO_TMA")[0] == '1')) {
        for (size_t k = 0; k < faces.size(); k++) {
            const uint64_t c = faces[k], x = c % NX, y = (c / NX) % NY, z = c / (NX * NY);
            if (x != 0 && x != NX - 1) continue;
            // rows away from the y and z boundaries (periodic or not), so the
            // slots written stay inside the tile's linear slot range
            if (y == 0 || y == NY - 1 || z == 0 || z == NZ - 1) continue;
            const uint64_t m = x == 0 ? c + 1 : c - 1;
            if (flags[m] != 0) continue;
            fused[k] = 1;
            flags[m] |= lbm::FLAG_XFACE;
            xinfo[x == 0 ? 0 : 1] = finfo[k] & 0xffu;
        }
    }
    uint32_t fplan[7] = {0, 0, 0, 0, 0, 0, 0}, fblk[7] = {0, 0, 0, 0, 0, 0, 0};
    uint32_t rect[6] = {0, 0, 0, 0, 0, 0}, rect_b0[6] = {0, 0, 0, 0, 0, 0}, rect_sv[6] = {0, 0, 0, 0, 0, 0},
             rect_nu[6] = {1, 1, 1, 1, 1, 1}, rect_info[6] = {0, 0, 0, 0, 0, 0};
    {
        // face cells are independent; grouping them by kind and store mask
        // keeps each warp on one code path.  Planar cells of a velocity or
        // open face whose in-plane axes are not periodic come first, one
        // group per face: the face kernel handles them with compile-time
        // directions and plain strides.
        auto group = [&](size_t k) -> int {
            const uint32_t info = finfo[k];
            if (fused[k] || (info & 3u) == 2u) return 6;
            for (int f = 0; f < 6; f++) {
                const int a = f >> 1;
                if ((info >> 8) == lbm::planar_mask(f) && !per[a == 0 ? 1 : 0] && !per[a == 2 ? 1 : 2]) return f;
            }
            return 6;
        };
        std::vector<int> grp(faces.size());
        for (size_t k = 0; k < faces.size(); k++) grp[k] = group(k);
        std::vector<size_t> ord(faces.size());
        for (size_t k = 0; k < ord.size(); k++) ord[k] = k;
        std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
            if (fused[a] != fused[b]) return fused[a] < fused[b];
            if (grp[a] != grp[b]) return grp[a] < grp[b];
            return finfo[a] < finfo[b];
        });
        uint32_t cnt[7] = {0, 0, 0, 0, 0, 0, 0};
        for (size_t k = 0; k < faces.size(); k++) cnt[grp[k]]++;
        for (int f = 1; f < 7; f++) {
            fplan[f] = fplan[f - 1] + cnt[f - 1];
            fblk[f] = fblk[f - 1] + (cnt[f - 1] + (uint32_t)lbm::BLOCK - 1) / (uint32_t)lbm::BLOCK;
        }
        // a y or z face's planar group is the rectangle x in [2, NX-3] by the
        // other in-plane axis in [2, N-3] (interior points of non-periodic
        // axes), listed in cell order; checked cell by cell before the face
        // kernel relies on it
        for (int f = 2; f < 6; f++) {
            const int a = f >> 1, o = a == 1 ? 2 : 1;
            const uint64_t nu = NX >= 5 ? NX - 4 : 0, nv = dimv[o] >= 5 ? dimv[o] - 4 : 0;
            const uint64_t fixed = (f & 1) ? dimv[a] - 1 : 0;
            const uint64_t so = o == 1 ? NX : NX * NY, sa = a == 1 ? NX : NX * NY;
            const uint64_t b0 = 2 + 2 * so + fixed * sa;
            bool ok = cnt[f] > 0 && (uint64_t)cnt[f] == nu * nv;
            for (uint64_t k = 0; ok && k < cnt[f]; k++) ok = faces[ord[fplan[f] + k]] == b0 + k % nu + (k / nu) * so;
            rect[f] = ok ? 1u : 0u;
            if (ok) {
                rect_b0[f] = (uint32_t)b0;
                rect_sv[f] = (uint32_t)so;
                rect_nu[f] = (uint32_t)nu;
                rect_info[f] = finfo[ord[fplan[f]]];
            }
        }
        std::vector<uint32_t> f2(faces.size()), i2(faces.size());
        uint32_t rest = 0;
        for (size_t k = 0; k < ord.size(); k++) {
            f2[k] = faces[ord[k]];
            i2[k] = finfo[ord[k]];
            rest += fused[ord[k]] ? 0u : 1u;
        }
        faces.swap(f2);
        finfo.swap(i2);
        h->nface_rest = rest;
        h->xfuse = rest < faces.size();
    }

    // probes
    std::vector<float> vbuf;
    std::vector<int32_t> sd(4, 0);
    if (probes) {
        h->nvert = (uint32_t)probes->nvert;
        for (uint64_t v = 0; v < probes->nvert; v++) {
            const double *q = probes->verts + 6 * v;
            float e[8] = {(float)q[0], (float)q[1], (float)q[2], 0.f, (float)q[3], (float)q[4], (float)q[5], 0.f};
            vbuf.insert(vbuf.end(), e, e + 8);
        }
        h->nslices = (uint32_t)probes->nslices;
        sd[0] = (int32_t)probes->nslices;
        uint64_t npix = 0;
        for (uint64_t s = 0; s < probes->nslices; s++) {
            const lbm_slice_def &d = probes->slices[s];
            int32_t e[12] = {d.origin[0], d.origin[1], d.origin[2], (int32_t)d.nu, d.u[0], d.u[1], d.u[2], (int32_t)d.nv, d.v[0], d.v[1], d.v[2], 0};
            sd.insert(sd.end(), e, e + 12);
            npix += (uint64_t)d.nu * d.nv;
        }
        if (npix >= 0xffffffffull) throw LbmError(LBM_ERR_INVALID, "too many slice pixels");
        h->npix = (uint32_t)npix;
        h->voff = (float)probes->vertex_offset;
    }

    // device buffers
    ck(cudaGetDevice(&h->device), "cudaGetDevice");
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&h->ev, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaMallocHost((void **)&h->hist_host, KMAX * 8 * sizeof(double)), "cudaMallocHost");
    ck(cudaMallocHost((void **)&h->err_host, 16), "cudaMallocHost");
    lbm::LatParams &p = h->lp;
    const size_t sb = storage_bytes(st.storage);
    // planes padded to 256 cells; a guard after the last plane covers the
    // shifted tile ranges the staged kernel fetches (largest offset NX*NY+NX+1)
    const uint64_t NP = (N + lbm::PLANE_ALIGN - 1) / lbm::PLANE_ALIGN * lbm::PLANE_ALIGN;
    const uint64_t guard = (lbm::TILE_MAX + NX * NY + NX + 64 + lbm::PLANE_ALIGN - 1) / lbm::PLANE_ALIGN * lbm::PLANE_ALIGN;
    h->pop_bytes = (19 * NP + guard) * sb;
    p.pop = h->dalloc(h->pop_bytes);
    p.NP = NP;
    const uint64_t NFL = (N + lbm::TILE_MAX - 1) / lbm::TILE_MAX * lbm::TILE_MAX + lbm::TILE_MAX;  // flags padded past the last tile
    p.flags = (uint32_t *)h->dalloc(NFL * 4);
    p.err = (uint32_t *)h->dalloc(16);
    p.recs = (uint32_t *)h->dalloc(nrec * lbm::RS * 4);
    p.recd = st.storage == LBM_STORAGE_FP64 ? (double *)h->dalloc(nrec * lbm::RD * 8) : nullptr;
    p.faces = (uint32_t *)h->dalloc(faces.size() * 4);
    p.face_info = (uint32_t *)h->dalloc(finfo.size() * 4);
    const uint64_t nwb = (nrec + lbm::WBLOCK - 1) / lbm::WBLOCK;  // blocks of the wall-cell kernel
    p.partials = (double *)h->dalloc(std::max<uint64_t>(nwb, 1) * 8 * sizeof(double));
    p.ticket = (uint32_t *)h->dalloc(16);
    p.hist = (double *)h->dalloc(KMAX * 8 * sizeof(double));
    p.dump = st.debug_dump ? (float4 *)h->dalloc(N * 16) : nullptr;
    h->vacc = (double *)h->dalloc(std::max<uint64_t>(h->nvert, 1) * 2 * sizeof(double));
    h->sacc = (double *)h->dalloc(std::max<uint64_t>(h->npix, 1) * 5 * sizeof(double));
    h->verts = (float *)h->dalloc(std::max<size_t>(vbuf.size(), 8) * 4);
    h->slicedef = (int32_t *)h->dalloc(sd.size() * 4);
    p.NX = (uint32_t)NX; p.NY = (uint32_t)NY; p.NZ = (uint32_t)NZ; p.N = (uint32_t)N;
    p.div_nx.init((uint32_t)NX);
    p.div_nxy.init((uint32_t)(NX * NY));
    // the staged bulk kernel needs x-rows that keep 16-byte alignment and
    // non-periodic x and y (its in-place tiles own their slots only then)
    const char *no_tma = std::getenv("SIMLAB_LBM_NO_TMA");
    p.tma = (NX * sb) % 16 == 0 && !per[0] && !per[1] && !(no_tma && no_tma[0] == '1');
    p.nrec = (uint32_t)nrec; p.nface = (uint32_t)faces.size();
    for (int a = 0; a < 3; a++) p.per[a] = per[a];
    p.abs_u = st.absorb_velocity != 0;
    p.total_p = st.total_pressure_inlet != 0;
    p.wall_model = st.wall_model != 0;
    p.forcing = st.body_force[0] != 0.0 || st.body_force[1] != 0.0 || st.body_force[2] != 0.0;
    p.sponge_on = 0;
    for (int f = 0; f < 6; f++) {
        p.sponge_on |= st.sponge[f] > 0;
        p.sp_w[f] = st.sponge[f];
    }
    p.les_on = st.smagorinsky != 0.0;
    p.moving = 0;
    if (spin) {
        p.moving = 1;
        const uint64_t nocc = (uint64_t)spin->occ_dims[0] * spin->occ_dims[1] * spin->occ_dims[2];
        const uint64_t words_occ = (nocc + 31) / 32;
        p.occ = (const uint32_t *)h->dalloc(words_occ * 4);
        ck(cudaMemcpy((void *)p.occ, spin->occ_bits, words_occ * 4, cudaMemcpyHostToDevice), "upload occupancy");
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
        std::vector<uint32_t> q0((size_t)nrec * 27, 0u);
        for (size_t k = 0; k < q0.size(); k += 3) q0[k] = 0x7f7fffffu;  // nearest hit: FLT_MAX
        p.qscr = (uint32_t *)h->dalloc(q0.size() * 4);
        ck(cudaMemcpy(p.qscr, q0.data(), q0.size() * 4, cudaMemcpyHostToDevice), "upload link scratch");
    }
    fill_consts<float>(p.kf, st);
    fill_consts<double>(p.kd, st);
    p.xface_info[0] = xinfo[0];
    p.xface_info[1] = xinfo[1];
    for (int f = 0; f < 7; f++) { p.fplan[f] = fplan[f]; p.fblk[f] = fblk[f]; }
    for (int f = 0; f < 6; f++) {
        p.frect[f] = rect[f];
        p.frect_b0[f] = rect_b0[f];
        p.frect_sv[f] = rect_sv[f];
        p.finfo[f] = rect_info[f];
        p.frect_nu[f].init(rect_nu[f]);
    }
    // sponge ramps per axis (shader.rs:528-538): 1 - p / width inside a layer
    std::vector<float> tabf;
    std::vector<double> tabd;
    for (int a = 0; a < 3; a++) {
        const uint64_t na = st.dims[a];
        for (uint64_t q = 0; q < na; q++) {
            float sf = 0.f;
            double sd = 0.0;
            const float pf = (float)q, hf = (float)(na - 1) - pf;
            if (st.sponge[2 * a] > 0) { sf = std::max(sf, 1.0f - pf / (float)st.sponge[2 * a]); sd = std::max(sd, 1.0 - (double)q / st.sponge[2 * a]); }
            if (st.sponge[2 * a + 1] > 0) {
                sf = std::max(sf, 1.0f - hf / (float)st.sponge[2 * a + 1]);
                sd = std::max(sd, 1.0 - (double)(na - 1 - q) / st.sponge[2 * a + 1]);
            }
            tabf.push_back(std::min(sf, 1.0f));
            tabd.push_back(std::min(sd, 1.0));
        }
    }
    p.sp_tab = (const float *)h->dalloc(tabf.size() * 4);
    p.sp_tabd = (const double *)h->dalloc(tabd.size() * 8);
    // the wall kernel may overlap the face kernel when no wall cell is within
    // three cells of a non-periodic boundary (its slots then never meet the
    // faces' slots or the inner cells the faces read)
    bool walls_far = nrec > 0 && !faces.empty() && !spin;
    for (uint64_t r = 0; walls_far && r < nrec; r++) {
        const uint64_t c = geom->walls[r].cell;
        const uint64_t q[3] = {c % NX, (c / NX) % NY, c / (NX * NY)};
        for (int a = 0; a < 3; a++)
            if (!per[a] && (q[a] < 3 || q[a] + 4 > st.dims[a])) walls_far = false;
    }

    cudaStream_t s = h->stream;
    ck(cudaMemsetAsync(p.pop, 0, h->pop_bytes, s), "memset");
    ck(cudaMemsetAsync(p.flags, 0, NFL * 4, s), "memset");
    ck(cudaMemsetAsync(p.err, 0, 16, s), "memset");
    ck(cudaMemcpyAsync(p.flags, flags.data(), N * 4, cudaMemcpyHostToDevice, s), "upload flags");
    if (nrec) ck(cudaMemcpyAsync(p.recs, words.data(), words.size() * 4, cudaMemcpyHostToDevice, s), "upload records");
    if (!wordsd.empty()) ck(cudaMemcpyAsync(p.recd, wordsd.data(), wordsd.size() * 8, cudaMemcpyHostToDevice, s), "upload records");
    if (!faces.empty()) {
        ck(cudaMemcpyAsync((void *)p.faces, faces.data(), faces.size() * 4, cudaMemcpyHostToDevice, s), "upload faces");
        ck(cudaMemcpyAsync((void *)p.face_info, finfo.data(), finfo.size() * 4, cudaMemcpyHostToDevice, s), "upload faces");
    }
    if (!vbuf.empty()) ck(cudaMemcpyAsync(h->verts, vbuf.data(), vbuf.size() * 4, cudaMemcpyHostToDevice, s), "upload vertices");
    ck(cudaMemcpyAsync(h->slicedef, sd.data(), sd.size() * 4, cudaMemcpyHostToDevice, s), "upload slices");
    ck(cudaMemcpyAsync((void *)p.sp_tab, tabf.data(), tabf.size() * 4, cudaMemcpyHostToDevice, s), "upload sponge");
    ck(cudaMemcpyAsync((void *)p.sp_tabd, tabd.data(), tabd.size() * 8, cudaMemcpyHostToDevice, s), "upload sponge");
    if (walls_far) {
        // the wall-cell kernel is the longer of the two that run before the
        // bulk: its blocks go first on the SMs
        int prio_lo = 0, prio_hi = 0;
        ck(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "cudaDeviceGetStreamPriorityRange");
        ck(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, LBM_SIDE_PRIORITY ? prio_hi : prio_lo), "cudaStreamCreate");
        ck(cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming), "cudaEventCreate");
        ck(cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming), "cudaEventCreate");
    }
    ck(cudaMemsetAsync(p.ticket, 0, 16, s), "memset");
    ck(cudaMemsetAsync(p.hist, 0, KMAX * 8 * sizeof(double), s), "memset");
    ck(cudaMemsetAsync(h->vacc, 0, std::max<uint64_t>(h->nvert, 1) * 2 * sizeof(double), s), "memset");
    ck(cudaMemsetAsync(h->sacc, 0, std::max<uint64_t>(h->npix, 1) * 5 * sizeof(double), s), "memset");
    ck(lbm::launch_init(st.storage, p, s), "init kernel");
    h->wait();  // host vectors go out of scope after this
}

// steps == nullptr: n still steps (StepIn::still(false))
void run_impl(lbm_lattice *h, const lbm_step_in *steps, uint64_t n, double *forces_out, bool readback) {
    lbm::LatParams &p = h->lp;
    lbm_step_in still{};
    for (int a = 0; a < 3; a++) { still.rot[a][a] = 1.0; still.rot_prev[a][a] = 1.0; }
    for (uint64_t c0 = 0; c0 < n; c0 += KMAX) {
        const uint32_t len = (uint32_t)std::min<uint64_t>(KMAX, n - c0);
        if (p.nrec == 0) ck(cudaMemsetAsync(p.hist, 0, len * 8 * sizeof(double), h->stream), "memset");
        for (uint32_t k = 0; k < len; k++) {
            const lbm_step_in &si = steps ? steps[c0 + k] : still;
            const uint64_t idx = h->steps_done;
            lbm::StepParams sp = step_params(h, si, k, idx);
            cudaEvent_t *evs = nullptr;
            cudaEvent_t ev4[4];
            if (h->prof) {
                const size_t need = 4 * (h->prof_steps + 1);
                while (h->prof_ev.size() < need) {
                    cudaEvent_t e;
                    ck(cudaEventCreate(&e), "cudaEventCreate");
                    h->prof_ev.push_back(e);
                }
                evs = h->prof_ev.data() + 4 * h->prof_steps;
                if (h->prof_mode == 2) {
                    // bulk kernel only: the face and wall events are not recorded
                    ev4[0] = nullptr; ev4[1] = nullptr; ev4[2] = evs[2]; ev4[3] = evs[3];
                    evs = ev4;
                }
                h->prof_steps++;
                // the kernels launch_step enqueues for this step
                h->prof_launches += (sp.nface ? 1u : 0u) + (p.nrec ? 1u : 0u) + 1u + (p.moving ? 2u + (p.ntri ? 1u : 0u) : 0u);
                if (si.sample) h->prof_launches += (h->nvert ? 1u : 0u) + (h->npix ? 1u : 0u);
            }
            ck(lbm::launch_step(h->setup.storage, p, sp, (int)(idx % 2), h->setup.collision, h->stream, h->side, h->fork, h->join, evs),
               "step kernels");
            if (si.sample && (h->nvert || h->npix))
                ck(lbm::launch_sample(h->setup.storage, p, sp, (int)(idx % 2), h->verts, h->nvert, h->voff, h->vacc, h->slicedef,
                                      h->nslices, h->npix, h->sacc, h->stream),
                   "sample kernels");
            h->steps_done++;
            h->fused_valid = h->xfuse;
        }
        if (readback) {
            ck(cudaMemcpyAsync(h->hist_host, p.hist, len * 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "history readback");
            ck(cudaMemcpyAsync(h->err_host, p.err, 4, cudaMemcpyDeviceToHost, h->stream), "error readback");
            h->wait();
            h->check_device_errors();
            if (forces_out)
                for (uint32_t k = 0; k < len; k++)
                    for (int j = 0; j < 6; j++) forces_out[(c0 + k) * 6 + j] = h->hist_host[k * 8 + j];
        }
    }
}

}  // namespace

// ============================================================== C ABI
extern "C" {

const char *lbm_version(void) { return "simlab-lbm-b200 0.1 (sm_100a)"; }

int lbm_global_error(char *buf, uint64_t len) {
    if (buf && len) std::snprintf(buf, (size_t)len, "%s", g_error.c_str());
    return LBM_OK;
}

int lbm_last_error(const lbm_lattice *h, char *buf, uint64_t len) {
    if (!h) return lbm_global_error(buf, len);
    if (buf && len) std::snprintf(buf, (size_t)len, "%s", h->err.c_str());
    return LBM_OK;
}

uint64_t lbm_max_cells(int32_t storage) {
    (void)storage;
    return 0xfffffffeull;  // cell indices are 32-bit, as in the reference
}

int lbm_create(const lbm_setup *setup, const lbm_geometry *geom, const lbm_probes *probes, lbm_lattice **out) {
    if (!out) { g_error = "out is null"; return LBM_ERR_INVALID; }
    *out = nullptr;
    lbm_lattice *h = new lbm_lattice();
    try {
        create_impl(setup, geom, probes, h);
    } catch (const LbmError &e) {
        g_error = e.what();
        delete h;
        return e.code;
    } catch (const std::exception &e) {
        g_error = e.what();
        delete h;
        return LBM_ERR_INVALID;
    }
    *out = h;
    return LBM_OK;
}

void lbm_destroy(lbm_lattice *h) { delete h; }

int lbm_run(lbm_lattice *h, const lbm_step_in *steps, uint64_t n, double *forces_out) {
    if (!h) return LBM_ERR_INVALID;
    if (n && !steps) return fail(h, LbmError(LBM_ERR_INVALID, "steps is null"));
    return guard(h, [&] { run_impl(h, steps, n, forces_out, true); });
}

int lbm_advance(lbm_lattice *h, uint64_t n) {
    if (!h) return LBM_ERR_INVALID;
    return guard(h, [&] { run_impl(h, nullptr, n, nullptr, false); });
}

int lbm_stream(lbm_lattice *h, void **stream) {
    if (!h || !stream) return LBM_ERR_INVALID;
    *stream = (void *)h->stream;
    return LBM_OK;
}

int lbm_synchronize(lbm_lattice *h) {
    if (!h) return LBM_ERR_INVALID;
    return guard(h, [&] { h->wait(); });
}

int lbm_profile(lbm_lattice *h, int32_t enable) {
    if (!h) return LBM_ERR_INVALID;
    return guard(h, [&] {
        h->wait();
        if (enable < 0 || enable > 2) throw LbmError(LBM_ERR_INVALID, "profile mode must be 0, 1 or 2");
        h->prof = enable != 0;
        h->prof_mode = enable;
        h->prof_steps = 0;
        h->prof_launches = 0;
    });
}

int lbm_get_kernel_times(lbm_lattice *h, lbm_kernel_times *out) {
    if (!h || !out) return LBM_ERR_INVALID;
    return guard(h, [&] {
        h->wait();
        out->steps = h->prof_steps;
        out->launches = h->prof_launches;
        out->faces_ms = out->walls_ms = out->bulk_ms = 0.0;
        for (uint64_t k = 0; k < h->prof_steps; k++) {
            cudaEvent_t *e = h->prof_ev.data() + 4 * k;
            float a = 0, b = 0, c;
            if (h->prof_mode != 2) {
                ck(cudaEventElapsedTime(&a, e[0], e[1]), "cudaEventElapsedTime");
                ck(cudaEventElapsedTime(&b, e[1], e[2]), "cudaEventElapsedTime");
            }
            ck(cudaEventElapsedTime(&c, e[2], e[3]), "cudaEventElapsedTime");
            out->faces_ms += a;
            out->walls_ms += b;
            out->bulk_ms += c;
        }
    });
}

int lbm_selftest_copy_wait(uint64_t limit_ns, uint32_t *gave_up, uint64_t *waited_us) {
    if (!gave_up || !waited_us || limit_ns == 0 || limit_ns > 10000000000ull) {
        g_error = "lbm_selftest_copy_wait: null output or limit outside (0, 10 s]";
        return LBM_ERR_INVALID;
    }
    uint32_t *d = nullptr;
    uint32_t hst[2] = {0, 0};
    cudaError_t e = cudaMalloc((void **)&d, sizeof(hst));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(hst));
    if (e == cudaSuccess) e = lbm::launch_wait_selftest(d, limit_ns, 0);
    if (e == cudaSuccess) e = cudaMemcpy(hst, d, sizeof(hst), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        g_error = std::string("lbm_selftest_copy_wait: ") + cudaGetErrorString(e);
        return LBM_ERR_CUDA;
    }
    *gave_up = hst[0];
    *waited_us = hst[1];
    return LBM_OK;
}

int lbm_set_timeout(lbm_lattice *h, double seconds) {
    if (!h || !(seconds > 0)) return LBM_ERR_INVALID;
    h->timeout_s = seconds;
    return LBM_OK;
}

int lbm_macros(lbm_lattice *h, float *out) {
    if (!h || !out) return LBM_ERR_INVALID;
    return guard(h, [&] {
        if (!h->setup.debug_dump) throw LbmError(LBM_ERR_STATE, "macros() needs debug_dump");
        const int q = 1 - h->parity();
        ck(lbm::launch_dump(h->setup.storage, h->lp, q, h->stream), "dump kernel");
        ck(cudaMemcpyAsync(out, h->lp.dump, (size_t)h->lp.N * 16, cudaMemcpyDeviceToHost, h->stream), "dump readback");
        h->wait();
    });
}

int lbm_records(lbm_lattice *h, uint32_t *out, uint64_t cap_words) {
    if (!h || (!out && cap_words)) return LBM_ERR_INVALID;
    return guard(h, [&] {
        uint64_t words = (uint64_t)h->nrec * lbm::RS;
        if (cap_words < words) throw LbmError(LBM_ERR_INVALID, "record buffer too small");
        if (words) ck(cudaMemcpyAsync(out, h->lp.recs, words * 4, cudaMemcpyDeviceToHost, h->stream), "record readback");
        h->wait();
    });
}

int lbm_reset_samples(lbm_lattice *h) {
    if (!h) return LBM_ERR_INVALID;
    return guard(h, [&] {
        ck(cudaMemsetAsync(h->vacc, 0, std::max<uint64_t>(h->nvert, 1) * 2 * sizeof(double), h->stream), "memset");
        ck(cudaMemsetAsync(h->sacc, 0, std::max<uint64_t>(h->npix, 1) * 5 * sizeof(double), h->stream), "memset");
        h->wait();
    });
}

int lbm_vertex_means(lbm_lattice *h, float *out) {
    if (!h || (!out && h->nvert)) return LBM_ERR_INVALID;
    return guard(h, [&] {
        if (!h->nvert) return;
        std::vector<double> v(2 * (size_t)h->nvert);
        ck(cudaMemcpyAsync(v.data(), h->vacc, v.size() * 8, cudaMemcpyDeviceToHost, h->stream), "vertex readback");
        h->wait();
        for (uint32_t i = 0; i < h->nvert; i++) out[i] = v[2 * i + 1] > 0 ? (float)(v[2 * i] / v[2 * i + 1]) : NAN;
    });
}

int lbm_slice_means(lbm_lattice *h, float *out) {
    if (!h || (!out && h->npix)) return LBM_ERR_INVALID;
    return guard(h, [&] {
        if (!h->npix) return;
        std::vector<double> v(5 * (size_t)h->npix);
        ck(cudaMemcpyAsync(v.data(), h->sacc, v.size() * 8, cudaMemcpyDeviceToHost, h->stream), "slice readback");
        h->wait();
        for (uint32_t i = 0; i < h->npix; i++) {
            double c = v[5 * i + 4];
            for (int a = 0; a < 4; a++) out[4 * i + a] = c > 0 ? (float)(v[5 * i + a] / c) : NAN;
        }
    });
}

int lbm_get_info(const lbm_lattice *h, lbm_info *out) {
    if (!h || !out) return LBM_ERR_INVALID;
    out->steps_done = h->steps_done;
    out->nrec = h->nrec;
    out->nface = h->nface;
    out->npix = h->npix;
    out->nvert = h->nvert;
    out->memory_bytes = h->memory_bytes;
    out->cells = h->lp.N;
    out->storage = h->setup.storage;
    out->collision = h->setup.collision;
    return LBM_OK;
}

int lbm_mass(lbm_lattice *h, double *mass, uint64_t *nonfinite) {
    if (!h) return LBM_ERR_INVALID;
    return guard(h, [&] {
        // out[2], then the block partials and the ticket of the grid sum
        const size_t nb = lbm::mass_blocks();
        double *dm = nullptr;
        ck(cudaMallocAsync((void **)&dm, (2 + 2 * nb) * sizeof(double) + 16, h->stream), "cudaMallocAsync");
        ck(cudaMemsetAsync(dm, 0, (2 + 2 * nb) * sizeof(double) + 16, h->stream), "memset");
        ck(lbm::launch_mass(h->setup.storage, h->lp, 1 - h->parity(), dm + 2, dm, h->stream), "mass kernel");
        double hv[2];
        ck(cudaMemcpyAsync(hv, dm, 16, cudaMemcpyDeviceToHost, h->stream), "mass readback");
        ck(cudaFreeAsync(dm, h->stream), "cudaFreeAsync");
        h->wait();
        if (mass) *mass = hv[0];
        if (nonfinite) *nonfinite = (uint64_t)hv[1];
    });
}

// checkpoint blob: header, populations, records (u32), records (f64, FP64 only)
struct StateHeader { uint64_t magic, cells, steps_done, nrec; int32_t storage, collision, fused_valid, _pad; };
static const uint64_t STATE_MAGIC = 0x4c424d5354415431ull;

int lbm_state_size(const lbm_lattice *h, uint64_t *bytes) {
    if (!h || !bytes) return LBM_ERR_INVALID;
    *bytes = sizeof(StateHeader) + 19 * h->lp.NP * storage_bytes(h->setup.storage) + (uint64_t)h->nrec * lbm::RS * 4 +
             (h->lp.recd ? (uint64_t)h->nrec * lbm::RD * 8 : 0) + (h->lp.moving ? (uint64_t)h->lp.N * 4 : 0);  // a spinning part's flags change
    return LBM_OK;
}

int lbm_save_state(lbm_lattice *h, void *buf, uint64_t bytes) {
    if (!h || !buf) return LBM_ERR_INVALID;
    return guard(h, [&] {
        uint64_t need;
        lbm_state_size(h, &need);
        if (bytes < need) throw LbmError(LBM_ERR_INVALID, "state buffer too small");
        StateHeader hd{STATE_MAGIC, h->lp.N, h->steps_done, h->nrec, h->setup.storage, h->setup.collision, h->fused_valid ? 1 : 0, 0};
        char *o = (char *)buf;
        std::memcpy(o, &hd, sizeof hd);
        o += sizeof hd;
        const uint64_t pb = 19ull * h->lp.NP * storage_bytes(h->setup.storage);
        ck(cudaMemcpyAsync(o, h->lp.pop, pb, cudaMemcpyDeviceToHost, h->stream), "state readback");
        o += pb;
        if (h->nrec) ck(cudaMemcpyAsync(o, h->lp.recs, (size_t)h->nrec * lbm::RS * 4, cudaMemcpyDeviceToHost, h->stream), "state readback");
        o += (size_t)h->nrec * lbm::RS * 4;
        if (h->lp.recd && h->nrec) ck(cudaMemcpyAsync(o, h->lp.recd, (size_t)h->nrec * lbm::RD * 8, cudaMemcpyDeviceToHost, h->stream), "state readback");
        o += h->lp.recd ? (size_t)h->nrec * lbm::RD * 8 : 0;
        if (h->lp.moving) ck(cudaMemcpyAsync(o, h->lp.flags, (size_t)h->lp.N * 4, cudaMemcpyDeviceToHost, h->stream), "state readback");
        h->wait();
    });
}

int lbm_load_state(lbm_lattice *h, const void *buf, uint64_t bytes) {
    if (!h || !buf) return LBM_ERR_INVALID;
    return guard(h, [&] {
        uint64_t need;
        lbm_state_size(h, &need);
        if (bytes < need) throw LbmError(LBM_ERR_INVALID, "state buffer too small");
        StateHeader hd;
        std::memcpy(&hd, buf, sizeof hd);
        if (hd.magic != STATE_MAGIC || hd.cells != h->lp.N || hd.nrec != h->nrec || hd.storage != h->setup.storage)
            throw LbmError(LBM_ERR_INVALID, "state does not belong to this lattice");
        const char *o = (const char *)buf + sizeof hd;
        const uint64_t pb = 19ull * h->lp.NP * storage_bytes(h->setup.storage);
        ck(cudaMemcpyAsync(h->lp.pop, o, pb, cudaMemcpyHostToDevice, h->stream), "state upload");
        o += pb;
        if (h->nrec) ck(cudaMemcpyAsync(h->lp.recs, o, (size_t)h->nrec * lbm::RS * 4, cudaMemcpyHostToDevice, h->stream), "state upload");
        o += (size_t)h->nrec * lbm::RS * 4;
        if (h->lp.recd && h->nrec) ck(cudaMemcpyAsync(h->lp.recd, o, (size_t)h->nrec * lbm::RD * 8, cudaMemcpyHostToDevice, h->stream), "state upload");
        o += h->lp.recd ? (size_t)h->nrec * lbm::RD * 8 : 0;
        if (h->lp.moving) ck(cudaMemcpyAsync(h->lp.flags, o, (size_t)h->lp.N * 4, cudaMemcpyHostToDevice, h->stream), "state upload");
        h->wait();
        h->steps_done = hd.steps_done;
        // the blob holds the fused x faces' slots when its step wrote them
        h->fused_valid = h->xfuse && hd.fused_valid != 0;
    });
}

// ------------------------------------------------------------ voxelizer
struct lbm_voxels {
    lbm::StaticVoxels v;
};

static lbm::Surface make_surface(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris) {
    lbm::Surface s;
    s.verts.resize(nverts);
    for (uint64_t i = 0; i < nverts; i++) s.verts[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
    s.tris.resize(ntris);
    for (uint64_t t = 0; t < ntris; t++) {
        for (int k = 0; k < 3; k++)
            if (tris[3 * t + k] >= nverts) throw LbmError(LBM_ERR_INVALID, "triangle vertex index out of range");
        s.tris[t] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
    }
    return s;
}

int lbm_voxelize_static(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris, const uint32_t dims[3],
                        int32_t lattice, lbm_voxels **out) {
    if (!out || !dims || (nverts && !verts) || (ntris && !tris)) { g_error = "null argument"; return LBM_ERR_INVALID; }
    *out = nullptr;
    return guard(nullptr, [&] {
        if (lattice != 19 && lattice != 27) throw LbmError(LBM_ERR_INVALID, "lattice must be 19 or 27");
        lbm::Surface s = make_surface(verts, nverts, tris, ntris);
        lbm_voxels *v = new lbm_voxels();
        v->v = lbm::voxelize_static(s, {dims[0], dims[1], dims[2]}, lattice);
        *out = v;
    });
}

int lbm_voxelize_static_gpu(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris, const uint32_t dims[3],
                            int32_t lattice, lbm_voxels **out) {
    if (!out || !dims || (nverts && !verts) || (ntris && !tris)) { g_error = "null argument"; return LBM_ERR_INVALID; }
    *out = nullptr;
    return guard(nullptr, [&] {
        if (lattice != 19 && lattice != 27) throw LbmError(LBM_ERR_INVALID, "lattice must be 19 or 27");
        if (nverts >= 0xffffffffull || ntris >= 0xffffffffull) throw LbmError(LBM_ERR_INVALID, "surface too large");
        lbm::Surface s = make_surface(verts, nverts, tris, ntris);
        lbm_voxels *v = new lbm_voxels();
        try {
            v->v = lbm::voxelize_static_gpu(s, {dims[0], dims[1], dims[2]}, lattice);
        } catch (const lbm::VoxelError &e) {
            delete v;
            throw LbmError(e.code == 2 ? LBM_ERR_NOMEM : (e.code == 3 ? LBM_ERR_CUDA : LBM_ERR_INVALID), e.what());
        } catch (...) {
            delete v;
            throw;
        }
        *out = v;
    });
}

int lbm_voxels_counts(const lbm_voxels *v, uint64_t *nsolid, uint64_t *nwalls) {
    if (!v) return LBM_ERR_INVALID;
    if (nsolid) *nsolid = v->v.solid.size();
    if (nwalls) *nwalls = v->v.walls.size();
    return LBM_OK;
}

int lbm_voxels_copy(const lbm_voxels *v, uint32_t *solid, lbm_wall_cell *walls) {
    if (!v) return LBM_ERR_INVALID;
    if (solid && !v->v.solid.empty()) std::memcpy(solid, v->v.solid.data(), v->v.solid.size() * 4);
    if (walls)
        for (size_t r = 0; r < v->v.walls.size(); r++) {
            walls[r].cell = v->v.walls[r].cell;
            walls[r].mask = v->v.walls[r].mask;
            for (int k = 0; k < 27; k++) walls[r].q[k] = v->v.walls[r].q[k];
        }
    return LBM_OK;
}

void lbm_voxels_free(lbm_voxels *v) { delete v; }

struct lbm_spin_voxels {
    lbm::SpinVoxels v;
};

int lbm_voxelize_spin(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris, const double axis[3], double h,
                      lbm_spin_voxels **out) {
    if (!out || !axis || (nverts && !verts) || (ntris && !tris)) { g_error = "null argument"; return LBM_ERR_INVALID; }
    if (!(h > 0.0)) { g_error = "grid spacing must be positive"; return LBM_ERR_INVALID; }
    return guard(nullptr, [&] {
        lbm::Surface s;
        s.verts.resize(nverts);
        for (uint64_t k = 0; k < nverts; k++) s.verts[k] = {verts[3 * k], verts[3 * k + 1], verts[3 * k + 2]};
        s.tris.resize(ntris);
        for (uint64_t k = 0; k < ntris; k++) {
            for (int j = 0; j < 3; j++)
                if (tris[3 * k + j] >= nverts) throw LbmError(LBM_ERR_INVALID, "triangle index out of range");
            s.tris[k] = {tris[3 * k], tris[3 * k + 1], tris[3 * k + 2]};
        }
        lbm_spin_voxels *v = new lbm_spin_voxels();
        v->v = lbm::voxelize_spin(s, {axis[0], axis[1], axis[2]}, h);
        *out = v;
    });
}

int lbm_spin_voxels_info(const lbm_spin_voxels *v, lbm_spin_info *out) {
    if (!v || !out) return LBM_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < 3; k++) { out->occ_lo[k] = v->v.occ_lo[k]; out->occ_dims[k] = (uint32_t)v->v.occ_dims[k]; }
    out->occ_h = v->v.occ_h;
    out->occ_words = v->v.occ_bits.size();
    out->ntri = v->v.tris.size();
    out->radius = v->v.radius;
    out->axial[0] = v->v.axial[0];
    out->axial[1] = v->v.axial[1];
    return LBM_OK;
}

int lbm_spin_voxels_copy(const lbm_spin_voxels *v, uint32_t *occ_bits, float *tris) {
    if (!v || !occ_bits || (!tris && !v->v.tris.empty())) return LBM_ERR_INVALID;
    std::memcpy(occ_bits, v->v.occ_bits.data(), v->v.occ_bits.size() * 4);
    for (size_t k = 0; k < v->v.tris.size(); k++) std::memcpy(tris + 12 * k, v->v.tris[k].data(), 48);
    return LBM_OK;
}

void lbm_spin_voxels_free(lbm_spin_voxels *v) { delete v; }

int lbm_inside_grid(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris, const double origin[3], double h,
                    const uint32_t dims[3], uint8_t *out) {
    if (!origin || !dims || !out || (nverts && !verts) || (ntris && !tris)) { g_error = "null argument"; return LBM_ERR_INVALID; }
    return guard(nullptr, [&] {
        lbm::Surface s = make_surface(verts, nverts, tris, ntris);
        lbm::GridSpec g;
        g.origin = {origin[0], origin[1], origin[2]};
        g.h = h;
        g.dims = {dims[0], dims[1], dims[2]};
        std::vector<uint8_t> in = lbm::inside_grid(s, g);
        std::memcpy(out, in.data(), in.size());
    });
}

}  // extern "C"
