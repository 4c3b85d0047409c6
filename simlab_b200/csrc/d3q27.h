// Launch parameters and launchers of the multi-level D3Q27 time step
// (d3q27_kernels.cu), shared with the host driver (mlattice.cu).
//
// Reference semantics: crates/cfd/src/mshader.rs (velocity set and record
// layout 30-48, access 199-228, collision 612-699, level kernels 702-793) and
// crates/cfd/src/d3q27.rs.
//
// HBM layout of a level: two population sets (A/B) of 27 planes each, set s
// direction i of cell n at (s * 27 + i) * NP + n, the plane stride NP being
// the cell count rounded up to 256 (every plane 512-byte aligned at 2-byte
// storage).  One u32 flag per cell: type in the low 3 bits (0 fluid, 1 solid,
// 2 face, 3 ghost, 4 restricted), wall record + 1 (or the face kind) above.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lbm_device.cuh"

namespace lbm27 {

// velocity set (d3q27.rs:1-29): direction i has velocity (i%3-1, (i/3)%3-1,
// i/9-1), the rest population is 13, the opposite of i is 26-i, and SLOT
// numbers the moving directions 0..25 in per-link arrays
__host__ __device__ __forceinline__ constexpr int CX(int i) { return i % 3 - 1; }
__host__ __device__ __forceinline__ constexpr int CY(int i) { return (i / 3) % 3 - 1; }
__host__ __device__ __forceinline__ constexpr int CZ(int i) { return i / 9 - 1; }
__host__ __device__ __forceinline__ constexpr int OPP27(int i) { return 26 - i; }
__host__ __device__ __forceinline__ constexpr int SLOT(int i) { return i < 13 ? i : i - 1; }
__host__ __device__ __forceinline__ constexpr double WD(int i) {
    return (CX(i) * CX(i) + CY(i) * CY(i) + CZ(i) * CZ(i)) == 0 ? 8.0 / 27.0
         : (CX(i) * CX(i) + CY(i) * CY(i) + CZ(i) * CZ(i)) == 1 ? 2.0 / 27.0
         : (CX(i) * CX(i) + CY(i) * CY(i) + CZ(i) * CZ(i)) == 2 ? 1.0 / 54.0
                                                                 : 1.0 / 216.0;
}

constexpr uint32_t RS = 24, R_MASK = 0, R_CELL = 1, R_Q = 2, R_FT = 15;  // record words (mshader.rs:32-36)
constexpr uint32_t MW = 12;                                               // words per exported moment node
// terms of a level step's rounding seed (mlattice.rs:704): (finest step + slot)
// * 2654435761 + source set * 7919 + moment slot * 104729
constexpr uint32_t SEED_SRC_MUL = 7919u, SEED_MW_MUL = 104729u;
constexpr uint32_t T_FLUID = 0, T_SOLID = 1, T_FACE = 2, T_GHOST = 3, T_RESTRICT = 4;

template <class R>
struct Consts27 {
    R tau0, smag2, sponge_tau, sigma;
    R sp_lo[3], sp_hi[3], u_inf[3], u_init[3], grav[3], center[3];
};

struct LevelParams {
    void *pop;                  // 2 sets x 27 planes of NP cells
    uint64_t NP;
    uint32_t *flags;
    const uint32_t *faces, *ghosts, *restricted;
    uint32_t nface, nghost, nrestrict;
    uint32_t NX, NY, NZ, N;
    lbm::FastDiv div_nx, div_nxy;
    int per[3];
    int n_sponge, forcing, abs_u, total_p;
    // refinement: this level's exports and the neighbouring levels' buffers
    int has_child, has_parent;
    int ch_lo[3];
    uint32_t ch_n[3];           // the child box in this level's nodes
    uint32_t ch_nodes;
    uint32_t pn[3];             // this level's nodes seen from its parent ((d - 1) / 2 + 1)
    void *mom_child;            // R, 2 slots x ch_nodes x MW: surface moments for the child's ghosts
    void *mom_up;               // R, pn nodes x MW: even-node moments for the parent's restriction
    const void *mom_parent;     // the parent's mom_child (ghost fill)
    const void *mom_child_up;   // the child's mom_up (restriction)
    // wall records (finest level only; nrec = 0 elsewhere)
    uint32_t *recs;
    double *recd;               // FP64 engine: 6 doubles (F, T) per record
    void *wallf;                // R, 27 per record: the wall populations the step substitutes
    uint32_t nrec;
    float4 *dump;
    // a spinning part on this (finest) level: every swept-box cell is a
    // record, re-voxelized each finest step from the step's rotation
    int moving;
    const uint32_t *occ;        // body-frame occupancy bits
    float occ_lo[3];
    float occ_invh;
    int32_t occ_n[3];
    const float4 *tris;         // 3 per triangle: v0, e1, e2 (body frame)
    uint32_t ntri;
    int32_t box_lo[3];
    uint32_t box_n[3];
    uint32_t *qscr;             // 13 positive links x (nearest t, farthest t, hits) per box cell
    Consts27<float> kf;
    Consts27<double> kd;
};

struct StepArgs {
    uint32_t src;       // source population set
    uint32_t mw;        // moment slot this step writes (mom_child)
    uint32_t mold, mnew;  // ghost fill: the parent's moment slots at the start and end of its step
    uint32_t seed_mix;  // stochastic rounding: the step seed's term of the hash
    float blend;        // ghost fill: time fraction between mold and mnew
    float omega[3];     // wall angular velocity, rad per finest step
    double omega_d[3];
    float rot[9];       // body axes in lattice coordinates (row-major, columns = axes)
    float rot_prev[9];  // the same one finest step earlier
};

// storage: lbm_storage (0 FP32, 1 FP16, 2 BF16, 3 FP64)
cudaError_t launch27_init(int storage, const LevelParams &p, cudaStream_t st);
cudaError_t launch27_face(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st);
cudaError_t launch27_step(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st);
cudaError_t launch27_ghost(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st);
cudaError_t launch27_restrict(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st);
cudaError_t launch27_dump(int storage, const LevelParams &p, uint32_t src, cudaStream_t st);
// probes (mshader.rs:563-602): surface vertices on the finest level with the
// step's rotation, and the (pixel, cell) pairs of the slice pixels a level
// owns; FP64 running sums in vacc (2 per vertex) and sacc (5 per pixel)
cudaError_t launch27_sample_verts(int storage, const LevelParams &p, const StepArgs &a, const float *verts, uint32_t nvert, float voff,
                                  double *vacc, cudaStream_t st);
cudaError_t launch27_sample_slices(int storage, const LevelParams &p, uint32_t src, const uint32_t *pix, uint32_t npix, double *sacc,
                                   cudaStream_t st);
// FP64 mass and non-finite count into out[0], out[1]; scratch: 2 doubles per
// block of mass27_blocks() blocks, then a u32 ticket that starts at zero
uint32_t mass27_blocks();
cudaError_t launch27_mass(int storage, const LevelParams &p, uint32_t src, double *scratch, double *out, cudaStream_t st);
// FP64 sum of the records' force and moment into out[0..5] (deterministic
// order: per-block partials, the last block sums them)
cudaError_t launch27_reduce(const LevelParams &p, int fp64, double *partials, uint32_t *ticket, double *out, cudaStream_t st);
uint32_t reduce27_blocks(uint32_t nrec);
// re-voxelize the spinning part's swept box for the rotation in `a` (finest level)
cudaError_t launch27_revoxel(int storage, const LevelParams &p, const StepArgs &a, cudaStream_t st);

}  // namespace lbm27
