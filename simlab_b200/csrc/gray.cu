// Gray-level D3Q19 lattice and its discrete adjoint (lbm_gray_* and
// lbm_backward of include/simlab_lbm.h).  No counterpart in the reference.
//
// Forward step (state P = post-collision populations, shifted by the weights,
// two sets A/B, direction i of cell n at i * NP + n):
//   faces   x = 0 cells hold feq(1, u_in); x = NX-1 cells copy the cell at x-1
//   stream  g_i(n) = P_i(n - c_i), periodic in y and z
//   collide BGK plus the Brinkman drag of the exact-difference method
//           (Kupershtokh 2004): P_i = (1 - w) g_i + w_i [w rho1 + 3 (w - a) c_i.j
//           + B Q_i / rho], Q_i = 4.5 (c_i.j)^2 - 1.5 j.j, B = w - 1 + (1 - a)^2,
//           a = alpha * gamma (w the BGK rate): momentum j becomes (1 - a) j
//   force   F = sum of a j over cells (what the gray body takes from the fluid)
//
// Adjoint.  The collision's Jacobian depends on the pre-collision state only
// through rho and j, so the reverse sweep needs 4 numbers per cell and step,
// not 19: with mu the adjoint of a cell's post-collision populations,
//   L0 = sum mu_i w_i, L1 = sum mu_i w_i c_i, M = sum mu_i w_i c_i c_i^T,
//   Qm = 4.5 j.M.j - 1.5 (j.j) L0,
//   lambda_k = (1 - w) mu_k + w L0 - B Qm / rho^2
//              + c_k . [3 (w - a) L1 + B (9 M j - 3 L0 j) / rho] + s_t a e.c_k
//   dJ/da   += -3 L1.j - 2 (1 - a) Qm / rho + s_t e.j
// (e the objective's weight vector of the cell, s_t the window weight of
// step t).  mu of a cell is pulled from the neighbours' lambda of the next step
// (the adjoint of the pull), plus the outlet copy's share at x = NX-2.
//
// Checkpoints: the full state every K steps; a reverse segment recomputes its
// K forward steps from its checkpoint, storing only (rho - 1, j) per cell and
// step, then runs the adjoint over them.  When the moments of every step fit
// in HBM and the caller allows it, the first forward pass keeps them and no
// segment is recomputed.
//
// Traffic per cell update (FP32): forward 152 B (19 loads + 19 stores) + 4 B
// of a; moments 16 B more when kept; adjoint 152 B + 16 B of moments + 4 B.
// FP16 storage halves the forward's population traffic and the checkpoints;
// the moments, the adjoint and the arithmetic stay FP32 (the rounding is not
// differentiated: the gradient is the adjoint of the FP32 update along the
// stored trajectory).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/simlab_lbm.h"
#include "lbm_device.cuh"
#include "host_wait.hpp"

namespace lbm_host {
void set_global_error(const std::string &msg);
}

namespace gray {

using lbm::CX;
using lbm::CY;
using lbm::CZ;
using lbm::FastDiv;
using lbm::WD;

constexpr int BLK = 256;

// feq_in: the inlet equilibrium (shifted by the weights); feq_q: the same
// as the storage holds it (rounded to nearest in FP16 storage), which the
// x = 1 cells pull from the inlet column
template <class R>
struct GConsts {
    R omega, feq_in[19], feq_q[19], center[3], dir[3];
};

struct GParams {
    uint32_t NX, NY, NZ, N;
    uint64_t NP;
    FastDiv div_nx, div_nxy;
    uint32_t box_lo[3], box_n[3];
    const void *a;       // R per cell: alpha * gamma (0 outside the design box)
    // step-kernel blocks holding design-box cells: block b's slot among them
    // (-1: none), so the force sum reads one partial per such block
    const int32_t *box_slot;
    uint32_t nbox_blocks;
    GConsts<float> kf;
    GConsts<double> kd;
};

template <class R> __device__ __forceinline__ const GConsts<R> &KG(const GParams &p);
template <> __device__ __forceinline__ const GConsts<float> &KG<float>(const GParams &p) { return p.kf; }
template <> __device__ __forceinline__ const GConsts<double> &KG<double>(const GParams &p) { return p.kd; }

__device__ __forceinline__ void coords(const GParams &p, uint32_t n, uint32_t &x, uint32_t &y, uint32_t &z) {
    z = p.div_nxy.div(n);
    const uint32_t r = n - z * (p.NX * p.NY);
    y = p.div_nx.div(r);
    x = r - y * p.NX;
}

// offset of the neighbour n + (dx, dy, dz), periodic in y and z (x never wraps)
struct Off {
    int32_t yp, ym, zp, zm;
    __device__ __forceinline__ int32_t at(int dx, int dy, int dz) const {
        return dx + (dy == 1 ? yp : (dy == -1 ? ym : 0)) + (dz == 1 ? zp : (dz == -1 ? zm : 0));
    }
};
__device__ __forceinline__ Off make_off(const GParams &p, uint32_t y, uint32_t z) {
    Off o;
    const int32_t nx = (int32_t)p.NX, nxy = (int32_t)(p.NX * p.NY);
    o.yp = y == p.NY - 1 ? -(int32_t)(p.NY - 1) * nx : nx;
    o.ym = y == 0 ? (int32_t)(p.NY - 1) * nx : -nx;
    o.zp = z == p.NZ - 1 ? -(int32_t)(p.NZ - 1) * nxy : nxy;
    o.zm = z == 0 ? (int32_t)(p.NZ - 1) * nxy : -nxy;
    return o;
}

// objective weight vector: force along dir, or moment about center along dir
template <class R>
__device__ __forceinline__ void weight_vec(const GConsts<R> &k, int objective, uint32_t x, uint32_t y, uint32_t z, R *e) {
    if (objective == 0) { e[0] = k.dir[0]; e[1] = k.dir[1]; e[2] = k.dir[2]; return; }
    const R r[3] = {(R)x - k.center[0], (R)y - k.center[1], (R)z - k.center[2]};
    e[0] = k.dir[1] * r[2] - k.dir[2] * r[1];
    e[1] = k.dir[2] * r[0] - k.dir[0] * r[2];
    e[2] = k.dir[0] * r[1] - k.dir[1] * r[0];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-block FP64 sums of 6 values from the blocks that hold a slot (0 ..
// count-1); the last of them to finish adds the partials in slot order and
// writes out[0..5] (the order, so the sum, does not depend on scheduling)
__device__ __forceinline__ void block_reduce6_at(double *v, uint32_t slot, uint32_t count, double *partials, uint32_t *ticket, double *out) {
    __shared__ double sh[BLK / 32][6];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 6; j++) v[j] = warp_sum(v[j]);
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = v[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < BLK / 32; w++) t += sh[w][threadIdx.x];
        partials[slot * 8 + threadIdx.x] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == count - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < count; b += BLK)
        for (int j = 0; j < 6; j++) acc[j] += __ldcg(&partials[b * 8 + j]);
    for (int j = 0; j < 6; j++) acc[j] = warp_sum(acc[j]);
    __syncthreads();
    if (lane == 0)
        for (int j = 0; j < 6; j++) sh[warp][j] = acc[j];
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0;
        for (int w = 0; w < BLK / 32; w++) t += sh[w][threadIdx.x];
        out[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// Storage S of the populations: float, double, or __half (FP32 arithmetic,
// f - w scaled by 32768 and rounded stochastically, as the engine stores
// FP16); rn() rounds a constant to nearest (inlet and initial values).
template <class S> struct GS {
    using R = typename lbm::Pop<S>::real;
    static __device__ __forceinline__ S rn(R v) { return (S)v; }
};
template <> struct GS<__half> {
    using R = float;
    static __device__ __forceinline__ __half rn(float v) { return __float2half_rn(v * 32768.0f); }
};

template <class S>
__global__ void __launch_bounds__(BLK) kg_init(const __grid_constant__ GParams p, S *P) {
    using R = typename GS<S>::R;
    const uint32_t n = blockIdx.x * BLK + threadIdx.x;
    if (n >= p.N) return;
    const GConsts<R> &k = KG<R>(p);
#pragma unroll
    for (int i = 0; i < 19; i++) P[(uint64_t)i * p.NP + n] = GS<S>::rn(k.feq_in[i]);
}

// one step of the bulk (1 <= x <= NX-2).  The x faces are read in place of
// being written: the inlet column x = 0 holds the inlet equilibrium, so the
// x = 1 cells pull feq_q for the directions coming from it; the outlet
// column x = NX-1 is a copy of x = NX-2, so the x = NX-2 cells pull those
// directions from their own column.  The face columns in memory are never
// read.  MOM: (rho - 1, j) of every cell's
// pre-collision state into 4 planes of NP; FORCE: the force a * j and its
// moment about the centre of every design-box cell into fm, summed in FP64
// over the grid (fixed order: block partials, then the last block).  FP16
// storage rounds stochastically from a hash of the cell and the step
// (seed_mix), so a segment recomputed from its checkpoint repeats the first
// pass bit for bit.
template <class S, bool MOM, bool FORCE>
__device__ __forceinline__ void step_cell(const GParams &p, const S *__restrict__ src, S *__restrict__ dst, typename GS<S>::R *__restrict__ mom,
                                          uint32_t seed_mix, uint32_t n, double *fm) {
    using R = typename GS<S>::R;
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    if (x < 1 || x + 1 >= p.NX) return;
    const GConsts<R> &k = KG<R>(p);
    const Off o = make_off(p, y, z);
    R g[19];
    const bool outlet = x + 2 == p.NX;
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const int32_t dx = CX(i) == -1 ? (outlet ? 0 : 1) : -CX(i);
        const R v = lbm::Pop<S>::cvt(src[(uint64_t)i * p.NP + (uint32_t)((int32_t)n + dx + o.at(0, -CY(i), -CZ(i)))]);
        g[i] = (CX(i) == 1 && x == 1) ? k.feq_q[i] : v;
    }
    R rho1 = 0, j[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 19; i++) {
        rho1 += g[i];
        if (CX(i)) j[0] += CX(i) * g[i];
        if (CY(i)) j[1] += CY(i) * g[i];
        if (CZ(i)) j[2] += CZ(i) * g[i];
    }
    const R an = ((const R *)p.a)[n];
    const R w = k.omega, rho = (R)1 + rho1, irho = (R)1 / rho;
    const R jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
    const R B = w - (R)1 + ((R)1 - an) * ((R)1 - an);
    const R c1 = (R)3 * (w - an), bq = B * irho;
    lbm::Rng rng{lbm::sr_hash_mix(n, seed_mix)};
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const R cj = (R)CX(i) * j[0] + (R)CY(i) * j[1] + (R)CZ(i) * j[2];
        const R Q = (R)4.5 * cj * cj - (R)1.5 * jj;
        dst[(uint64_t)i * p.NP + n] = lbm::Pop<S>::enc(((R)1 - w) * g[i] + (R)WD(i) * (w * rho1 + c1 * cj + bq * Q), rng);
    }
    if (MOM) {
        mom[n] = rho1;
        mom[p.NP + n] = j[0];
        mom[2 * p.NP + n] = j[1];
        mom[3 * p.NP + n] = j[2];
    }
    if (FORCE) {
        const uint32_t bx = x - p.box_lo[0], by = y - p.box_lo[1], bz = z - p.box_lo[2];
        if (bx < p.box_n[0] && by < p.box_n[1] && bz < p.box_n[2]) {
            const double F[3] = {(double)(an * j[0]), (double)(an * j[1]), (double)(an * j[2])};
            const double r[3] = {(double)x - (double)k.center[0], (double)y - (double)k.center[1], (double)z - (double)k.center[2]};
            fm[0] = F[0]; fm[1] = F[1]; fm[2] = F[2];
            fm[3] = r[1] * F[2] - r[2] * F[1];
            fm[4] = r[2] * F[0] - r[0] * F[2];
            fm[5] = r[0] * F[1] - r[1] * F[0];
        }
    }
}

// Forward steps are launched with programmatic stream serialization: every
// block lets the next step's grid launch as soon as it starts, and waits for
// the previous step's grid to complete (memory included) before it touches
// global memory, so the next grid's blocks fill the SMs this grid's last wave
// leaves free instead of starting after a launch gap.  Without the launch
// attribute both instructions do nothing.
template <class S, bool MOM, bool FORCE>
__global__ void __launch_bounds__(BLK, 4) kg_step(const __grid_constant__ GParams p, const S *__restrict__ src, S *__restrict__ dst,
                                               typename GS<S>::R *__restrict__ mom, double *partials, uint32_t *ticket, double *out,
                                               uint32_t seed_mix) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const uint32_t n = blockIdx.x * BLK + threadIdx.x;
    double fm[6] = {0, 0, 0, 0, 0, 0};
    if (n < p.N) step_cell<S, MOM, FORCE>(p, src, dst, mom, seed_mix, n, fm);
    if (FORCE) {
        const int32_t slot = p.box_slot[blockIdx.x];  // the same for the whole block
        if (slot >= 0) block_reduce6_at(fm, (uint32_t)slot, p.nbox_blocks, partials, ticket, out);
    }
}

// one reverse step t: lin = lambda of step t+1 (pre-collision adjoint),
// lout = lambda of step t, mom = (rho - 1, j) of step t
template <class R>
__global__ void __launch_bounds__(BLK) kg_adjoint(const __grid_constant__ GParams p, const R *__restrict__ lin, R *__restrict__ lout,
                                                  const R *__restrict__ mom, double *__restrict__ grad, int objective, R swin) {
    // launched like the forward steps (programmatic stream serialization)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const uint32_t n = blockIdx.x * BLK + threadIdx.x;
    if (n >= p.N) return;
    uint32_t x, y, z;
    coords(p, n, x, y, z);
    if (x < 1 || x + 1 >= p.NX) return;
    const GConsts<R> &k = KG<R>(p);
    const Off o = make_off(p, y, z);
    // mu_i: the pull of step t+1 read P_i(n) at n + c_i; the outlet copy read
    // P_i(n) at x = NX-1 for the cells n + x + c_i with c_ix = -1
    R mu[19];
#pragma unroll
    for (int i = 0; i < 19; i++) {
        R v = 0;
        const uint32_t xn = x + CX(i);
        if (xn >= 1 && xn + 1 < p.NX) v = lin[(uint64_t)i * p.NP + (uint32_t)((int32_t)n + o.at(CX(i), CY(i), CZ(i)))];
        if (CX(i) == -1 && x + 2 == p.NX) v += lin[(uint64_t)i * p.NP + (uint32_t)((int32_t)n + o.at(0, CY(i), CZ(i)))];
        mu[i] = v;
    }
    const R rho1 = mom[n], j[3] = {mom[p.NP + n], mom[2 * p.NP + n], mom[3 * p.NP + n]};
    const R an = ((const R *)p.a)[n];
    const R w = k.omega, rho = (R)1 + rho1, irho = (R)1 / rho;
    const R jj = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
    const R B = w - (R)1 + ((R)1 - an) * ((R)1 - an);
    R L0 = 0, L1[3] = {0, 0, 0}, M[6] = {0, 0, 0, 0, 0, 0};  // xx yy zz xy xz yz
#pragma unroll
    for (int i = 0; i < 19; i++) {
        const R m = (R)WD(i) * mu[i];
        L0 += m;
        if (CX(i)) { L1[0] += CX(i) * m; M[0] += m; }
        if (CY(i)) { L1[1] += CY(i) * m; M[1] += m; }
        if (CZ(i)) { L1[2] += CZ(i) * m; M[2] += m; }
        if (CX(i) * CY(i)) M[3] += (R)(CX(i) * CY(i)) * m;
        if (CX(i) * CZ(i)) M[4] += (R)(CX(i) * CZ(i)) * m;
        if (CY(i) * CZ(i)) M[5] += (R)(CY(i) * CZ(i)) * m;
    }
    const R Mj[3] = {M[0] * j[0] + M[3] * j[1] + M[4] * j[2], M[3] * j[0] + M[1] * j[1] + M[5] * j[2],
                     M[4] * j[0] + M[5] * j[1] + M[2] * j[2]};
    const R Qm = (R)4.5 * (j[0] * Mj[0] + j[1] * Mj[1] + j[2] * Mj[2]) - (R)1.5 * jj * L0;
    R e[3];
    weight_vec<R>(k, objective, x, y, z, e);
    const R s0 = w * L0 - B * Qm * irho * irho;
    R V[3];
#pragma unroll
    for (int c = 0; c < 3; c++) V[c] = (R)3 * (w - an) * L1[c] + B * ((R)9 * Mj[c] - (R)3 * L0 * j[c]) * irho + swin * an * e[c];
#pragma unroll
    for (int kk = 0; kk < 19; kk++)
        lout[(uint64_t)kk * p.NP + n] = ((R)1 - w) * mu[kk] + s0 + (R)CX(kk) * V[0] + (R)CY(kk) * V[1] + (R)CZ(kk) * V[2];
    const uint32_t bx = x - p.box_lo[0], by = y - p.box_lo[1], bz = z - p.box_lo[2];
    if (bx < p.box_n[0] && by < p.box_n[1] && bz < p.box_n[2]) {
        const R ga = -(R)3 * (L1[0] * j[0] + L1[1] * j[1] + L1[2] * j[2]) - (R)2 * ((R)1 - an) * Qm * irho +
                     swin * (e[0] * j[0] + e[1] * j[1] + e[2] * j[2]);
        grad[((uint64_t)bz * p.box_n[1] + by) * p.box_n[0] + bx] += (double)ga;
    }
}

}  // namespace gray

namespace {

struct GErr : std::runtime_error {
    int code;
    GErr(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
inline void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw GErr(e == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr size_t HCHUNK = 1024;  // steps per force readback

}  // namespace

struct lbm_gray {
    lbm_gray_setup setup{};
    gray::GParams p{};
    int storage = LBM_STORAGE_FP32;
    size_t ssz = 4;  // bytes per stored population
    size_t rsz = 4;  // bytes per real (arithmetic, moments, adjoint)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<void *> allocs;
    void *P[2] = {nullptr, nullptr};
    void *a = nullptr;
    double *partials = nullptr;
    uint32_t *ticket = nullptr;
    double *hist = nullptr, *hist_host = nullptr;
    uint32_t cur = 0;
    uint64_t steps_done = 0;
    double timeout_s = 600.0;
    double t_fwd = 0, t_rec = 0, t_rev = 0;
    std::string err;
    // adjoint work space, kept between calls
    void *L[2] = {nullptr, nullptr};
    void *mom = nullptr;
    size_t mom_slots = 0;
    void *ckpt = nullptr;
    size_t ckpt_slots = 0;
    double *grad = nullptr;

    uint32_t nblk() const { return (p.N + gray::BLK - 1) / gray::BLK; }
    uint64_t nbox() const { return (uint64_t)p.box_n[0] * p.box_n[1] * p.box_n[2]; }
    size_t set_bytes() const { return (size_t)19 * p.NP * ssz; }   // a population set (or checkpoint)
    size_t lset_bytes() const { return (size_t)19 * p.NP * rsz; }  // an adjoint set
    void *dalloc(size_t bytes) {
        void *q = nullptr;
        ck(cudaMalloc(&q, std::max<size_t>(bytes, 16)), "cudaMalloc");
        allocs.push_back(q);
        return q;
    }
    void dfree(void *&q) {
        if (!q) return;
        auto it = std::find(allocs.begin(), allocs.end(), q);
        if (it != allocs.end()) allocs.erase(it);
        cudaFree(q);
        q = nullptr;
    }
    ~lbm_gray() {
        if (stream && lbm::stream_wait(stream, timeout_s) == cudaErrorTimeout) {
            lbm_host::set_global_error("gray lattice destroyed while its device work had not finished: buffers left allocated");
            return;
        }
        for (void *q : allocs) cudaFree(q);
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
            if (el > timeout_s) throw GErr(LBM_ERR_TIMEOUT, "device did not finish within " + std::to_string(timeout_s) + " s");
            if (el > 1e-3) std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    // fn((S *)nullptr) with S the population storage type
    template <class F>
    void typed(F &&fn) {
        if (storage == LBM_STORAGE_FP64) fn((double *)nullptr);
        else if (storage == LBM_STORAGE_FP16) fn((__half *)nullptr);
        else fn((float *)nullptr);
    }
    void reset() {
        typed([&](auto *t) {
            using S = std::remove_pointer_t<decltype(t)>;
            gray::kg_init<S><<<nblk(), gray::BLK, 0, stream>>>(p, (S *)P[0]);
            gray::kg_init<S><<<nblk(), gray::BLK, 0, stream>>>(p, (S *)P[1]);
        });
        ck(cudaGetLastError(), "init kernel");
        cur = 0;
        steps_done = 0;
    }
    // one forward step, the current set into the other (faces read in place); out:
    // null (no forces) or 8 doubles for the force and moment of the step
    // stochastic-rounding seed of step steps_done + 1 (the engine's rule)
    uint32_t seed_mix() const {
        const uint32_t seed = (uint32_t)((steps_done + 1) * 2654435761ull);
        return seed * 0x85EBCA77u + 0x632BE5ABu;
    }
    void step(void *mom_slot, double *out) {
        typed([&](auto *t) {
            using S = std::remove_pointer_t<decltype(t)>;
            using R = typename gray::GS<S>::R;
            const uint32_t mix = seed_mix();
            const S *src = (const S *)P[cur];
            S *dst = (S *)P[1 - cur];
            // programmatic stream serialization (the kernel's first lines say how it is used)
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(nblk());
            cfg.blockDim = dim3(gray::BLK);
            cfg.dynamicSmemBytes = 0;
            cfg.stream = stream;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            R *ms = (R *)mom_slot;
            double *pt = out ? partials : nullptr;
            uint32_t *tk = out ? ticket : nullptr;
            if (mom_slot && out) ck(cudaLaunchKernelEx(&cfg, gray::kg_step<S, true, true>, p, src, dst, ms, pt, tk, out, mix), "step kernel");
            else if (mom_slot) ck(cudaLaunchKernelEx(&cfg, gray::kg_step<S, true, false>, p, src, dst, ms, pt, tk, out, mix), "step kernel");
            else if (out) ck(cudaLaunchKernelEx(&cfg, gray::kg_step<S, false, true>, p, src, dst, ms, pt, tk, out, mix), "step kernel");
            else ck(cudaLaunchKernelEx(&cfg, gray::kg_step<S, false, false>, p, src, dst, ms, pt, tk, out, mix), "step kernel");
        });
        ck(cudaGetLastError(), "step kernel");
        cur = 1 - cur;
        steps_done++;
    }
    void run(uint64_t n, double *forces) {
        uint64_t done = 0;
        while (done < n) {
            const uint64_t m = std::min<uint64_t>(HCHUNK, n - done);
            for (uint64_t k = 0; k < m; k++) step(nullptr, forces ? hist + 8 * k : nullptr);
            if (forces) {
                ck(cudaMemcpyAsync(hist_host, hist, m * 8 * sizeof(double), cudaMemcpyDeviceToHost, stream), "force readback");
                wait();
                for (uint64_t k = 0; k < m; k++) std::memcpy(forces + 6 * (done + k), hist_host + 8 * k, 6 * sizeof(double));
            }
            done += m;
        }
    }
    double backward(const lbm_adjoint_spec &sp, double *grad_out);
};

double lbm_gray::backward(const lbm_adjoint_spec &sp, double *grad_out) {
    const uint64_t T = sp.steps;
    if (T == 0 || sp.t0 < 1 || sp.t1 < sp.t0 || sp.t1 > T) throw GErr(LBM_ERR_INVALID, "objective window must satisfy 1 <= t0 <= t1 <= steps");
    if (sp.checkpoint_every == 0) throw GErr(LBM_ERR_INVALID, "checkpoint_every must be positive");
    if (sp.objective != 0 && sp.objective != 1) throw GErr(LBM_ERR_INVALID, "objective must be 0 (force) or 1 (moment)");
    const uint64_t K = std::min<uint64_t>(sp.checkpoint_every, T);
    const uint64_t nseg = (T + K - 1) / K;
    const size_t mom_bytes = (size_t)4 * p.NP * rsz;
    // Moments of the trailing segments are kept from the first pass when the
    // caller allows it, as many as fit in 80 % of the free device memory
    // beside K slots for recomputing the others; those others restart from
    // their checkpoints.
    size_t free_b = 0, total_b = 0;
    ck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const double avail = 0.8 * (double)(free_b + (mom ? mom_slots * mom_bytes : 0) + (ckpt ? ckpt_slots * set_bytes() : 0));
    uint64_t keep_seg = 0;  // trailing segments whose moments the first pass keeps
    if (!sp.recompute) {
        if ((double)T * mom_bytes < avail) keep_seg = nseg;
        else {
            const double per_seg = (double)K * mom_bytes, fixed = (double)K * mom_bytes + (double)nseg * set_bytes();
            keep_seg = avail > fixed ? std::min<uint64_t>(nseg - 1, (uint64_t)((avail - fixed) / per_seg)) : 0;
        }
    }
    const uint64_t keep_from = (nseg - keep_seg) * K;  // steps keep_from+1 .. T are kept
    const bool all_kept = keep_seg == nseg;
    const uint64_t kept_steps = T - std::min<uint64_t>(keep_from, T);
    const size_t need_mom = (all_kept ? 0 : K) + kept_steps, need_ck = all_kept ? 0 : nseg - keep_seg;
    if (mom_slots < need_mom || ckpt_slots < need_ck) {
        dfree(mom);
        dfree(ckpt);
        mom_slots = ckpt_slots = 0;
        mom = dalloc(need_mom * mom_bytes);
        mom_slots = need_mom;
        if (need_ck) {
            ckpt = dalloc(need_ck * set_bytes());
            ckpt_slots = need_ck;
        }
    }
    const uint64_t kbase = all_kept ? 0 : K;  // first moment slot of the kept steps
    auto kept_slot = [&](uint64_t step1) { return (char *)mom + (kbase + (step1 - keep_from - 1)) * mom_bytes; };
    if (!L[0]) { L[0] = dalloc(lset_bytes()); L[1] = dalloc(lset_bytes()); }
    const uint64_t nb = nbox();
    if (!grad) grad = (double *)dalloc(std::max<uint64_t>(nb, 1) * 8);
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    auto elapsed = [&]() {
        ck(cudaEventRecord(e1, stream), "cudaEventRecord");
        wait();
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        return (double)ms;
    };
    t_fwd = t_rec = t_rev = 0;
    // first forward pass: the objective, checkpoints, kept moments
    reset();
    std::vector<double> dsum(T + 1, 0.0);
    ck(cudaEventRecord(e0, stream), "cudaEventRecord");
    uint64_t t = 0;
    while (t < T) {
        const uint64_t m = std::min<uint64_t>(HCHUNK, T - t);
        for (uint64_t k = 0; k < m; k++) {
            if (t < keep_from && t % K == 0)
                ck(cudaMemcpyAsync((char *)ckpt + (t / K) * set_bytes(), P[cur], set_bytes(), cudaMemcpyDeviceToDevice, stream), "checkpoint");
            step(t >= keep_from ? kept_slot(t + 1) : nullptr, hist + 8 * k);
            t++;
        }
        ck(cudaMemcpyAsync(hist_host, hist, m * 8 * sizeof(double), cudaMemcpyDeviceToHost, stream), "force readback");
        wait();
        for (uint64_t k = 0; k < m; k++) {
            const double *f = hist_host + 8 * k + (sp.objective == 1 ? 3 : 0);
            dsum[t - m + k + 1] = sp.dir[0] * f[0] + sp.dir[1] * f[1] + sp.dir[2] * f[2];
        }
    }
    t_fwd = elapsed();
    double J = 0;
    for (uint64_t s2 = sp.t0; s2 <= sp.t1; s2++) J += dsum[s2];
    J /= (double)(sp.t1 - sp.t0 + 1);
    // reverse sweep
    ck(cudaMemsetAsync(L[0], 0, lset_bytes(), stream), "adjoint init");
    ck(cudaMemsetAsync(L[1], 0, lset_bytes(), stream), "adjoint init");
    ck(cudaMemsetAsync(grad, 0, std::max<uint64_t>(nb, 1) * 8, stream), "gradient init");
    const double swin = 1.0 / (double)(sp.t1 - sp.t0 + 1);
    uint32_t lc = 0;  // L[lc] = lambda of step s+1
    for (uint64_t seg = nseg; seg-- > 0;) {
        const uint64_t c = seg * K, cend = std::min<uint64_t>(c + K, T);
        const bool kept = c >= keep_from;
        if (!kept) {
            ck(cudaEventRecord(e0, stream), "cudaEventRecord");
            ck(cudaMemcpyAsync(P[cur], (char *)ckpt + seg * set_bytes(), set_bytes(), cudaMemcpyDeviceToDevice, stream), "restore");
            steps_done = c;  // the recomputed steps round with the first pass's seeds
            for (uint64_t s2 = c; s2 < cend; s2++) step((char *)mom + (s2 - c) * mom_bytes, nullptr);
            t_rec += elapsed();
        }
        ck(cudaEventRecord(e0, stream), "cudaEventRecord");
        for (uint64_t s2 = cend; s2 > c; s2--) {
            const void *mslot = kept ? (const void *)kept_slot(s2) : (const void *)((char *)mom + (s2 - 1 - c) * mom_bytes);
            const double sw = (s2 >= sp.t0 && s2 <= sp.t1) ? swin : 0.0;
            typed([&](auto *tp) {
                using R = typename gray::GS<std::remove_pointer_t<decltype(tp)>>::R;
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3(nblk());
                cfg.blockDim = dim3(gray::BLK);
                cfg.dynamicSmemBytes = 0;
                cfg.stream = stream;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                ck(cudaLaunchKernelEx(&cfg, gray::kg_adjoint<R>, p, (const R *)L[lc], (R *)L[1 - lc], (const R *)mslot, grad, sp.objective, (R)sw),
                   "adjoint kernel");
            });
            lc = 1 - lc;
        }
        t_rev += elapsed();
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<double> g(std::max<uint64_t>(nb, 1));
    ck(cudaMemcpyAsync(g.data(), grad, nb * 8, cudaMemcpyDeviceToHost, stream), "gradient readback");
    wait();
    for (uint64_t b2 = 0; b2 < nb; b2++) grad_out[b2] = setup.alpha * g[b2];
    reset();
    return J;
}

namespace {

int gfail(lbm_gray *h, const GErr &e) {
    if (h) h->err = e.what(); else lbm_host::set_global_error(e.what());
    return e.code;
}
template <class F>
int gguard(lbm_gray *h, F &&fn) {
    try {
        fn();
        return LBM_OK;
    } catch (const GErr &e) {
        return gfail(h, e);
    } catch (const std::exception &e) {
        return gfail(h, GErr(LBM_ERR_INVALID, e.what()));
    }
}

template <class R>
void fill(gray::GConsts<R> &k, const lbm_gray_setup &s) {
    k.omega = (R)(1.0 / (0.5 + 3.0 * s.nu));
    const double usq = 1.5 * (s.u_in[0] * s.u_in[0] + s.u_in[1] * s.u_in[1] + s.u_in[2] * s.u_in[2]);
    for (int i = 0; i < 19; i++) {
        const double cu = lbm::CX(i) * s.u_in[0] + lbm::CY(i) * s.u_in[1] + lbm::CZ(i) * s.u_in[2];
        k.feq_in[i] = (R)(lbm::WD(i) * (3.0 * cu + 4.5 * cu * cu - usq));
        k.feq_q[i] = k.feq_in[i];
        if (s.storage == LBM_STORAGE_FP16)
            k.feq_q[i] = (R)(__half2float(__float2half_rn((float)k.feq_in[i] * 32768.0f)) * (1.0f / 32768.0f));
    }
    for (int c = 0; c < 3; c++) { k.center[c] = (R)s.center[c]; k.dir[c] = (R)0; }
}

void create_gray(const lbm_gray_setup *s, lbm_gray *h) {
    if (!s) throw GErr(LBM_ERR_INVALID, "setup is null");
    const uint64_t N = (uint64_t)s->dims[0] * s->dims[1] * s->dims[2];
    if (s->dims[0] < 4 || s->dims[1] < 1 || s->dims[2] < 1) throw GErr(LBM_ERR_INVALID, "grid must be at least 4 cells along x");
    if (N >= 0x7fffffffull) throw GErr(LBM_ERR_INVALID, "grid of " + std::to_string(N) + " cells is out of range");
    if (s->storage != LBM_STORAGE_FP32 && s->storage != LBM_STORAGE_FP64 && s->storage != LBM_STORAGE_FP16)
        throw GErr(LBM_ERR_UNSUPPORTED, "the gray lattice stores FP32, FP64 or FP16");
    if (!(s->nu > 0.0)) throw GErr(LBM_ERR_INVALID, "viscosity must be positive");
    if (!(s->alpha > 0.0 && s->alpha <= 1.0)) throw GErr(LBM_ERR_INVALID, "alpha must be in (0, 1]");
    for (int k = 0; k < 3; k++)
        if (s->box_n[k] == 0 || (uint64_t)s->box_lo[k] + s->box_n[k] > s->dims[k]) throw GErr(LBM_ERR_INVALID, "design box outside the grid");
    if (s->box_lo[0] < 1 || s->box_lo[0] + s->box_n[0] > s->dims[0] - 1) throw GErr(LBM_ERR_INVALID, "design box must leave the x faces out");
    h->setup = *s;
    h->storage = s->storage;
    h->rsz = s->storage == LBM_STORAGE_FP64 ? 8 : 4;
    h->ssz = s->storage == LBM_STORAGE_FP64 ? 8 : (s->storage == LBM_STORAGE_FP16 ? 2 : 4);
    gray::GParams &p = h->p;
    p.NX = s->dims[0]; p.NY = s->dims[1]; p.NZ = s->dims[2]; p.N = (uint32_t)N;
    p.NP = (N + 255) / 256 * 256;
    p.div_nx.init(p.NX);
    p.div_nxy.init(p.NX * p.NY);
    for (int k = 0; k < 3; k++) { p.box_lo[k] = s->box_lo[k]; p.box_n[k] = s->box_n[k]; }
    fill<float>(p.kf, *s);
    fill<double>(p.kd, *s);
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&h->ev, cudaEventDisableTiming), "cudaEventCreate");
    h->P[0] = h->dalloc(h->set_bytes());
    h->P[1] = h->dalloc(h->set_bytes());
    h->a = h->dalloc(N * h->rsz);
    ck(cudaMemsetAsync(h->a, 0, N * h->rsz, h->stream), "field init");
    p.a = h->a;
    {
        // the step kernel's blocks that hold design-box cells, numbered in block order
        std::vector<int32_t> slot(h->nblk(), -1);
        for (uint32_t z = s->box_lo[2]; z < s->box_lo[2] + s->box_n[2]; z++)
            for (uint32_t y = s->box_lo[1]; y < s->box_lo[1] + s->box_n[1]; y++)
                for (uint32_t x = s->box_lo[0]; x < s->box_lo[0] + s->box_n[0]; x++)
                    slot[(((uint64_t)z * s->dims[1] + y) * s->dims[0] + x) / gray::BLK] = 0;
        uint32_t nb = 0;
        for (auto &v : slot)
            if (v == 0) v = (int32_t)nb++;
        h->p.nbox_blocks = nb;
        int32_t *d = (int32_t *)h->dalloc(slot.size() * 4);
        ck(cudaMemcpy(d, slot.data(), slot.size() * 4, cudaMemcpyHostToDevice), "upload box blocks");
        h->p.box_slot = d;
        h->partials = (double *)h->dalloc((size_t)std::max<uint32_t>(nb, 1) * 8 * 8);
    }
    h->ticket = (uint32_t *)h->dalloc(16);
    ck(cudaMemsetAsync(h->ticket, 0, 16, h->stream), "ticket init");
    h->hist = (double *)h->dalloc(HCHUNK * 8 * 8);
    ck(cudaMallocHost(&h->hist_host, HCHUNK * 8 * 8), "cudaMallocHost");
    h->reset();
    h->wait();
}

}  // namespace

extern "C" {

int lbm_gray_create(const lbm_gray_setup *setup, lbm_gray **out) {
    if (!out) { lbm_host::set_global_error("out is null"); return LBM_ERR_INVALID; }
    *out = nullptr;
    lbm_gray *h = new lbm_gray();
    int rc = gguard(nullptr, [&] { create_gray(setup, h); });
    if (rc != LBM_OK) { delete h; return rc; }
    *out = h;
    return LBM_OK;
}

void lbm_gray_destroy(lbm_gray *h) { delete h; }

int lbm_gray_last_error(const lbm_gray *h, char *buf, uint64_t len) {
    if (!h) return LBM_ERR_INVALID;
    if (buf && len) std::snprintf(buf, (size_t)len, "%s", h->err.c_str());
    return LBM_OK;
}

int lbm_gray_set_field(lbm_gray *h, const double *gamma) {
    if (!h) return LBM_ERR_INVALID;
    return gguard(h, [&] {
        if (!gamma) throw GErr(LBM_ERR_INVALID, "gamma is null");
        const gray::GParams &p = h->p;
        std::vector<double> a((size_t)p.N, 0.0);
        const uint64_t nb = (uint64_t)p.box_n[0] * p.box_n[1] * p.box_n[2];
        for (uint64_t b = 0; b < nb; b++) {
            const double g = gamma[b];
            if (!(g >= 0.0 && g <= 1.0)) throw GErr(LBM_ERR_INVALID, "gamma must lie in [0, 1]");
            const uint32_t x = (uint32_t)(b % p.box_n[0]), y = (uint32_t)((b / p.box_n[0]) % p.box_n[1]), z = (uint32_t)(b / ((uint64_t)p.box_n[0] * p.box_n[1]));
            a[((uint64_t)(p.box_lo[2] + z) * p.NY + p.box_lo[1] + y) * p.NX + p.box_lo[0] + x] = h->setup.alpha * g;
        }
        if (h->rsz == 8) {
            ck(cudaMemcpyAsync(h->a, a.data(), a.size() * 8, cudaMemcpyHostToDevice, h->stream), "field upload");
            h->wait();
        } else {
            std::vector<float> af(a.begin(), a.end());
            ck(cudaMemcpyAsync(h->a, af.data(), af.size() * 4, cudaMemcpyHostToDevice, h->stream), "field upload");
            h->wait();
        }
    });
}

int lbm_gray_reset(lbm_gray *h) {
    if (!h) return LBM_ERR_INVALID;
    return gguard(h, [&] { h->reset(); h->wait(); });
}

int lbm_gray_run(lbm_gray *h, uint64_t n, double *forces_out) {
    if (!h) return LBM_ERR_INVALID;
    return gguard(h, [&] { h->run(n, forces_out); if (!forces_out) h->wait(); });
}

int lbm_backward(lbm_gray *h, const lbm_adjoint_spec *spec, double *objective, double *dJ_dgamma) {
    if (!h) return LBM_ERR_INVALID;
    return gguard(h, [&] {
        if (!spec || !objective || !dJ_dgamma) throw GErr(LBM_ERR_INVALID, "null argument");
        lbm_adjoint_spec sp = *spec;
        for (int c = 0; c < 3; c++) { h->p.kf.dir[c] = (float)sp.dir[c]; h->p.kd.dir[c] = sp.dir[c]; }
        *objective = h->backward(sp, dJ_dgamma);
    });
}

int lbm_gray_backward_times(const lbm_gray *h, double *forward_ms, double *recompute_ms, double *reverse_ms) {
    if (!h || !forward_ms || !recompute_ms || !reverse_ms) return LBM_ERR_INVALID;
    *forward_ms = h->t_fwd;
    *recompute_ms = h->t_rec;
    *reverse_ms = h->t_rev;
    return LBM_OK;
}

int lbm_gray_stream(lbm_gray *h, void **stream) {
    if (!h || !stream) return LBM_ERR_INVALID;
    *stream = (void *)h->stream;
    return LBM_OK;
}

}  // extern "C"
