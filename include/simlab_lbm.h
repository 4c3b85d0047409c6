/*
 * simlab_lbm.h -- C ABI of the B200 lattice-Boltzmann engine.
 *
 * This is the boundary that replaces the lattice layer of SimLab's
 * `crates/cfd` (the Rust `Lattice` type in crates/cfd/src/lattice.rs and the
 * voxelizer entry points in crates/cfd/src/voxel.rs).  Each declaration names
 * the reference item it stands in for.  Everything is in lattice units (cell
 * size 1, time step 1, reference density 1), as in the reference.
 *
 * Conventions
 *  - Every function returns an int status: 0 (LBM_OK) or a negative
 *    lbm_status code.  The message of the last failure is available from
 *    lbm_last_error() (per handle) or lbm_global_error() (creation errors).
 *  - No exception or C++ type crosses the boundary; all arrays are plain host
 *    memory owned by the caller, sizes are element counts.
 *  - A handle is driven by one thread at a time (the reference drives a
 *    `Lattice` from one job thread); it owns one CUDA stream.
 *  - Cell index everywhere is (z * NY + y) * NX + x.
 */
#ifndef SIMLAB_LBM_H
#define SIMLAB_LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* Status codes.  The reference returns anyhow::Result with bail! messages
 * (e.g. lattice.rs:233-244, 414-419); the message text is kept in the handle. */
typedef enum {
    LBM_OK = 0,
    LBM_ERR_INVALID = -1,     /* bad argument or setup (reference: bail!) */
    LBM_ERR_NOMEM = -2,       /* device allocation failed (lattice.rs:417-419) */
    LBM_ERR_CUDA = -3,        /* a CUDA call failed */
    LBM_ERR_TIMEOUT = -4,     /* a device wait passed its host-side limit */
    LBM_ERR_UNSUPPORTED = -5, /* feature not available for this configuration */
    LBM_ERR_STATE = -6        /* call not valid in the handle's state (e.g. macros without debug_dump) */
} lbm_status;

/* Face boundary conditions, faces ordered -x, +x, -y, +y, -z, +z.
 * VELOCITY/OPEN/PERIODIC mirror `FaceBc` (lattice.rs:35-43).  FREE_SLIP has
 * no counterpart in the reference: the face cell holds the mirror image of
 * its inner neighbour's post-collision populations (specular reflection). */
typedef enum {
    LBM_FACE_VELOCITY = 0,
    LBM_FACE_OPEN = 1,
    LBM_FACE_PERIODIC = 2,
    LBM_FACE_FREE_SLIP = 3
} lbm_face_bc;

/* Population storage, `Storage` (lattice.rs:11-32) plus BF16 and FP64.
 * All storage keeps f_i - w_i; FP16 scales it by 32768 with stochastic
 * rounding (shader.rs:73, 507-517).  Arithmetic is FP32 except FP64. */
typedef enum {
    LBM_STORAGE_FP32 = 0,
    LBM_STORAGE_FP16 = 1,
    LBM_STORAGE_BF16 = 2,
    LBM_STORAGE_FP64 = 3
} lbm_storage;

/* Collision operator.  REGULARIZED is the reference's (shader.rs:15-17,
 * 835-837); BGK is plain single-relaxation BGK (no counterpart). */
typedef enum {
    LBM_COLLISION_REGULARIZED = 0,
    LBM_COLLISION_BGK = 1
} lbm_collision;

/* `LatticeSetup` (lattice.rs:45-76), field for field, plus `collision`. */
typedef struct {
    uint32_t dims[3];
    int32_t faces[6];          /* lbm_face_bc, -x,+x,-y,+y,-z,+z */
    double nu;                 /* lattice kinematic viscosity; tau0 = 0.5 + 3 nu */
    double smagorinsky;        /* C_s (0 = no turbulence model) */
    double u_inf[3];
    double u_init[3];
    double body_force[3];      /* uniform acceleration (Guo forcing) */
    uint32_t sponge[6];        /* viscosity sponge width per face, cells */
    double sponge_tau;
    double sponge_sigma;
    int32_t absorb_velocity;
    int32_t total_pressure_inlet;
    int32_t storage;           /* lbm_storage */
    int32_t collision;         /* lbm_collision */
    double center[3];          /* moment reference point and spin centre */
    int32_t debug_dump;        /* keep a buffer for lbm_macros() */
    int32_t wall_model;        /* Spalding wall model in wall cells */
} lbm_setup;

/* `WallCell` (voxel.rs:328-335): a wall-adjacent fluid cell, its cut-link
 * mask (bit i = direction i) and q per direction (1.0 where no wall). */
typedef struct {
    uint32_t cell;
    uint32_t mask;
    float q[27];
} lbm_wall_cell;

/* `Geometry` (lattice.rs:87-92).  kind 0 = None, 1 = Static, 2 = Spin.
 * Spin: the part's `SpinVoxels` (voxel.rs:492-505, from lbm_voxelize_spin)
 * and the swept box of lattice cells that holds every cell it can reach;
 * every box cell becomes a record the GPU re-voxelizes each step from the
 * step's rotation (StepIn::rot, rot_prev). */
typedef struct {
    int32_t kind;
    int32_t _pad;
    const uint32_t *solid;     /* solid cell indices (StaticVoxels::solid) */
    uint64_t nsolid;
    const lbm_wall_cell *walls;/* StaticVoxels::walls */
    uint64_t nwalls;
    /* kind 2 */
    const uint32_t *occ_bits;  /* body-frame occupancy, one bit per point of occ_lo + occ_h (i, j, k), x fastest */
    double occ_lo[3];
    double occ_h;
    uint32_t occ_dims[3];
    uint32_t _pad2;
    const float *tris;         /* 12 floats per triangle: v0, e1, e2, each padded to 4 (body coordinates) */
    uint64_t ntri;
    int32_t box_lo[3];
    uint32_t box_n[3];
} lbm_geometry;

/* `SliceDef` (shader.rs:77-84). */
typedef struct {
    int32_t origin[3];
    int32_t u[3];
    int32_t v[3];
    uint32_t nu;
    uint32_t nv;
} lbm_slice_def;

/* `Probes` (lattice.rs:94-102).  verts: 6 doubles per vertex (position
 * relative to the centre in body coordinates, then the unit normal). */
typedef struct {
    const double *verts;
    uint64_t nvert;
    const lbm_slice_def *slices;
    uint64_t nslices;
    double vertex_offset;
} lbm_probes;

/* `StepIn` (lattice.rs:104-113).  rot[r][c]: row-major 3x3, columns are the
 * body axes in lattice coordinates; omega in rad per step. */
typedef struct {
    double rot[3][3];
    double rot_prev[3][3];
    double omega[3];
    int32_t sample;
    int32_t _pad;
} lbm_step_in;

/* Public fields of `Lattice` (lattice.rs:148-170). */
typedef struct {
    uint64_t steps_done;
    uint32_t nrec;
    uint32_t nface;
    uint32_t npix;
    uint32_t nvert;
    uint64_t memory_bytes;
    uint64_t cells;
    int32_t storage;           /* storage actually used */
    int32_t collision;
} lbm_info;

typedef struct lbm_lattice lbm_lattice;
typedef struct lbm_voxels lbm_voxels;

/* Library version string. */
const char *lbm_version(void);

/* Message of the last failure of a call that had no handle (creation,
 * voxelizer).  Copies at most len-1 bytes and a terminating zero. */
int lbm_global_error(char *buf, uint64_t len);

/* Message of the last failure on this handle. */
int lbm_last_error(const lbm_lattice *h, char *buf, uint64_t len);

/* Lattice::max_cells (lattice.rs:221-227): largest grid this storage can
 * hold by the layout alone (device memory budgets are the caller's). */
uint64_t lbm_max_cells(int32_t storage);

/* Lattice::new (lattice.rs:229-673): validates the setup, builds face list,
 * records and flags, allocates device memory and writes the initial state
 * (equilibrium at u_init).  `probes` may be NULL. */
int lbm_create(const lbm_setup *setup, const lbm_geometry *geom, const lbm_probes *probes, lbm_lattice **out);

/* Drop (frees every device buffer of the handle). */
void lbm_destroy(lbm_lattice *h);

/* Lattice::run (lattice.rs:699-753): advances n steps; forces_out receives
 * 6 doubles per step, the force and the moment about `center` on the
 * geometry after each step (lattice units).  Blocks until the forces are on
 * the host; returns LBM_ERR_TIMEOUT if the device does not finish within the
 * handle's wait limit (lbm_set_timeout). */
int lbm_run(lbm_lattice *h, const lbm_step_in *steps, uint64_t n, double *forces_out);

/* Enqueues n still steps (StepIn::still(false)) on the handle's stream and
 * returns without waiting; the forces stay in device memory.  For timing the
 * resident time step (no reference counterpart). */
int lbm_advance(lbm_lattice *h, uint64_t n);

/* The handle's CUDA stream (cudaStream_t), for event timing. */
int lbm_stream(lbm_lattice *h, void **stream);

/* Waits for the handle's stream with the wait limit. */
int lbm_synchronize(lbm_lattice *h);

/* Per-kernel device time of the steps enqueued while profiling is on,
 * from CUDA events recorded around each kernel on the handle's stream (no
 * reference counterpart; for the roofline figures), and the number of
 * kernels those steps launched.  Enabling clears the totals;
 * lbm_kernel_times waits for the stream and returns them. */
typedef struct {
    uint64_t steps;
    double faces_ms;
    double walls_ms;
    double bulk_ms;
    uint64_t launches;
} lbm_kernel_times;
/* Per-kernel device timing of the following steps with CUDA events on the
 * lattice's streams: enable 1 times the face, wall and bulk kernels (four
 * events per step), 2 only the bulk kernel (two events per step, so the
 * timed steps carry fewer stream operations; faces_ms and walls_ms stay 0),
 * 0 stops.  Starting clears the totals. */
int lbm_profile(lbm_lattice *h, int32_t enable);
int lbm_get_kernel_times(lbm_lattice *h, lbm_kernel_times *out);

/* Host-side limit on device waits, seconds (default 600). */
int lbm_set_timeout(lbm_lattice *h, double seconds);

/* Self-test of the step kernel's bounded waits (no reference counterpart):
 * one device thread waits on a bulk-copy barrier phase that nothing completes,
 * with the kernels' own wait routine and a limit of limit_ns (0 < limit_ns <=
 * 10 s).  *gave_up = 1 when the wait ended at its limit, as the step kernel's
 * waits end with LBM_ERR_TIMEOUT instead of hanging; *waited_us = the time it
 * waited.  No fault and no hang: the device stays usable. */
int lbm_selftest_copy_wait(uint64_t limit_ns, uint32_t *gave_up, uint64_t *waited_us);

/* Lattice::macros (lattice.rs:818-835): (rho, ux, uy, uz) of every cell,
 * NaN for solid and face cells; needs debug_dump.  out: 4 * cells floats. */
int lbm_macros(lbm_lattice *h, float *out);

/* Lattice::records (lattice.rs:837-841): the wall records, 40 u32 words per
 * record in the reference's layout (shader.rs:62-69).  out: cap_words u32. */
int lbm_records(lbm_lattice *h, uint32_t *out, uint64_t cap_words);

/* Lattice::reset_samples / vertex_means / slice_means (lattice.rs:785-816).
 * vertex_means: nvert floats; slice_means: 4 floats per pixel. */
int lbm_reset_samples(lbm_lattice *h);
int lbm_vertex_means(lbm_lattice *h, float *out);
int lbm_slice_means(lbm_lattice *h, float *out);

/* Public fields of Lattice (lattice.rs:148-170). */
int lbm_get_info(const lbm_lattice *h, lbm_info *out);

/* Global mass and the non-finite count over all fluid cells, summed in
 * FP64 on the device (no reference counterpart; the reference checks forces
 * for NaN in tunnel.rs:1142-1144). */
int lbm_mass(lbm_lattice *h, double *mass, uint64_t *nonfinite);

/* Checkpoint: size in bytes of the state blob, then save/load it (all
 * populations, records and the step counter).  No reference counterpart. */
int lbm_state_size(const lbm_lattice *h, uint64_t *bytes);
int lbm_save_state(lbm_lattice *h, void *buf, uint64_t bytes);
int lbm_load_state(lbm_lattice *h, const void *buf, uint64_t bytes);

/* voxelize_static / voxelize_static27 (voxel.rs:346-359, 361-490): solid
 * cells and wall links of a closed triangle surface given in lattice
 * coordinates.  lattice: 19 or 27.  The result is read with
 * lbm_voxels_counts / lbm_voxels_copy and freed with lbm_voxels_free. */
int lbm_voxelize_static(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris,
                        const uint32_t dims[3], int32_t lattice, lbm_voxels **out);
/* lbm_voxelize_static on the current CUDA device (no counterpart in the
 * reference, which voxelizes on the CPU): the same solid cells and wall links,
 * bit for bit (FP64 throughout, every product and sum rounded separately),
 * returned in the same host handle.  Runs on a stream of its own and returns
 * when the result is on the host; device scratch is allocated and freed
 * within the call. */
int lbm_voxelize_static_gpu(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris,
                            const uint32_t dims[3], int32_t lattice, lbm_voxels **out);
int lbm_voxels_counts(const lbm_voxels *v, uint64_t *nsolid, uint64_t *nwalls);
int lbm_voxels_copy(const lbm_voxels *v, uint32_t *solid, lbm_wall_cell *walls);
void lbm_voxels_free(lbm_voxels *v);

/* voxelize_spin (voxel.rs:507-560): body-frame geometry of a spinning part
 * given in body coordinates (lattice units, origin at the spin centre):
 * occupancy bits on a grid of spacing h (the reference uses 0.125) and the
 * surface split into triangles of at most 1.5 cells per edge. */
typedef struct lbm_spin_voxels lbm_spin_voxels;
typedef struct {
    double occ_lo[3];
    double occ_h;
    uint32_t occ_dims[3];
    uint32_t _pad;
    uint64_t occ_words;        /* u32 words of occupancy bits */
    uint64_t ntri;
    double radius;             /* largest distance of the surface from the axis */
    double axial[2];           /* extent along the axis */
} lbm_spin_info;
int lbm_voxelize_spin(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris, const double axis[3], double h,
                      lbm_spin_voxels **out);
int lbm_spin_voxels_info(const lbm_spin_voxels *v, lbm_spin_info *out);
int lbm_spin_voxels_copy(const lbm_spin_voxels *v, uint32_t *occ_bits, float *tris);
void lbm_spin_voxels_free(lbm_spin_voxels *v);

/* inside_grid (voxel.rs:73-95): inside test for every point of the grid
 * origin + h * (i, j, k); out: dims[0]*dims[1]*dims[2] bytes (0/1). */
int lbm_inside_grid(const double *verts, uint64_t nverts, const uint32_t *tris, uint64_t ntris,
                    const double origin[3], double h, const uint32_t dims[3], uint8_t *out);

/* ------------------------------------------------------------------------
 * Multi-level D3Q27 lattice: `MultiLattice` of crates/cfd/src/mlattice.rs
 * with the collision of crates/cfd/src/mshader.rs.  Pull streaming over two
 * population sets per level, the cumulant-type collision (deviatoric second
 * moments relaxed with the viscous rate, every higher cumulant to
 * equilibrium), Bouzidi walls with momentum exchange on the finest level,
 * nested node-aligned boxes of half the cell size stepped twice per parent
 * step.  Faces of type FREE_SLIP are not available here (LBM_ERR_UNSUPPORTED).
 * ------------------------------------------------------------------------ */

/* `LevelBox` (mlattice.rs:15-21): lo is the parent node of the level's node
 * 0, n the number of parent nodes it spans per axis (dims = 2 (n - 1) + 1). */
typedef struct {
    int32_t lo[3];
    uint32_t n[3];
} lbm_level_box;

/* `MultiSetup` (mlattice.rs:23-47), field for field. */
typedef struct {
    uint32_t dims0[3];          /* coarsest level size, cells */
    uint32_t nboxes;            /* number of refinement boxes (levels - 1) */
    const lbm_level_box *boxes; /* boxes of levels 1.., each in its parent's node coordinates */
    int32_t faces[6];           /* lbm_face_bc: VELOCITY, OPEN or PERIODIC (periodic only without boxes) */
    double nu0;                 /* lattice viscosity on the coarsest level (doubles per finer level) */
    double smagorinsky;
    double u_inf[3];
    double u_init[3];
    double body_force0[3];      /* acceleration on the coarsest level (halves per finer level) */
    uint32_t sponge[6];         /* sponge widths on the coarsest level, cells */
    double sponge_tau;
    double sponge_sigma;
    int32_t absorb_velocity;
    int32_t total_pressure_inlet;
    int32_t storage;            /* lbm_storage */
    int32_t debug_dump;
    double center[3];           /* moment reference, finest-level coordinates */
} lbm_multi_setup;

typedef struct lbm_multi lbm_multi;

/* MultiLattice::new (mlattice.rs:195-688).  Geometry (kind 0 or 1) is in the
 * finest level's cell indices; wall records use D3Q27 directions
 * (i = (cx+1) + 3 (cy+1) + 9 (cz+1)).  Same validation messages as the
 * reference ("refinement box 1 does not fit inside its parent", "periodic
 * faces only work without refinement", ...).  probes (`MProbes`,
 * mlattice.rs:79-84) may be NULL: vertices relative to `center` in body
 * coordinates, slices in finest-level cells. */
int lbm_create_multi(const lbm_multi_setup *setup, const lbm_geometry *geom, const lbm_probes *probes, lbm_multi **out);
void lbm_multi_destroy(lbm_multi *h);
int lbm_multi_last_error(const lbm_multi *h, char *buf, uint64_t len);

/* sub_steps / level_dims / level_cells (mlattice.rs:705-721).  levels: the
 * number of levels; dims: 3 per level; cells: 1 per level. */
int lbm_multi_levels(const lbm_multi *h, uint32_t *levels);
int lbm_multi_sub_steps(const lbm_multi *h, uint32_t *sub_steps);
int lbm_multi_level_dims(const lbm_multi *h, uint32_t *dims);
int lbm_multi_level_cells(const lbm_multi *h, uint64_t *cells);

/* MultiLattice::run (mlattice.rs:723-784): n finest steps, a multiple of
 * sub_steps; forces_out: 6 doubles per finest step (force and moment about
 * center on the geometry, finest lattice units). */
int lbm_multi_run(lbm_multi *h, const lbm_step_in *steps, uint64_t n, double *forces_out);

/* n finest still steps (a multiple of sub_steps) enqueued without waiting
 * (for timing; no reference counterpart). */
int lbm_multi_advance(lbm_multi *h, uint64_t n);
int lbm_multi_stream(lbm_multi *h, void **stream);
int lbm_multi_synchronize(lbm_multi *h);
int lbm_multi_set_timeout(lbm_multi *h, double seconds);

/* MultiLattice::macros (mlattice.rs:883-901): (rho, ux, uy, uz) per cell of
 * one level, NaN except plain fluid cells; needs debug_dump. */
int lbm_multi_macros(lbm_multi *h, uint32_t level, float *out);

/* MultiLattice::records (mlattice.rs:903-905): 24 u32 words per record
 * (mask, cell, q as 13 f16 pairs in slot order, force, moment, 3 zero). */
int lbm_multi_records(lbm_multi *h, uint32_t *out, uint64_t cap_words);

/* MultiLattice::reset_samples / vertex_means / slice_means
 * (mlattice.rs:844-881).  Surface vertices are sampled on the finest level
 * (trilinear density around each vertex, rotated by the step's StepIn::rot),
 * each slice pixel (slice coordinates in finest-level cells) on the finest
 * level whose interior, without its ghost layer, holds it
 * (mlattice.rs:266-305); both after every finest step whose StepIn::sample is
 * set.  vertex_means: nvert floats (NaN where nothing was sampled);
 * slice_means: 4 floats (rho, ux, uy, uz) per pixel. */
int lbm_multi_reset_samples(lbm_multi *h);
int lbm_multi_vertex_means(lbm_multi *h, float *out);
int lbm_multi_slice_means(lbm_multi *h, float *out);

/* steps_done counts finest steps; nrec, memory_bytes, storage, nvert, npix
 * as lbm_info; cells = the sum of the levels' cells. */
int lbm_multi_get_info(const lbm_multi *h, lbm_info *out);

/* FP64 mass and non-finite count over the plain fluid cells of one level
 * (no reference counterpart). */
int lbm_multi_mass(lbm_multi *h, uint32_t level, double *mass, uint64_t *nonfinite);

/* ------------------------------------------------------------------------
 * Gray-level lattice and its discrete adjoint (no counterpart in the
 * reference, which has no adjoint and no gray level).  A D3Q19 BGK lattice
 * whose cells carry a solid fraction gamma in [0, 1]; a cell removes the
 * fraction a = alpha * gamma of its momentum each step (Brinkman drag, added
 * to BGK with the exact-difference method: the post-collision state gains
 * feq(rho, (1 - a) u) - feq(rho, u)).  Faces: equilibrium velocity inlet at
 * -x, zero-gradient outlet at +x (the outlet cell copies its inner
 * neighbour), periodic in y and z.  The force on the gray body is the
 * momentum it removes, sum over cells of a * j; its moment is taken about
 * `center`.
 *
 * lbm_backward gives d(objective)/d(gamma) for every design-box cell by a
 * hand-written discrete adjoint of the whole step (faces, pull streaming,
 * collision, objective), with checkpoints of the full state every
 * checkpoint_every steps and the forward recomputed segment by segment.
 * ------------------------------------------------------------------------ */
typedef struct {
    uint32_t dims[3];
    uint32_t box_lo[3];         /* design box: first cell and size per axis */
    uint32_t box_n[3];
    int32_t storage;            /* LBM_STORAGE_FP32, _FP64, or _FP16 (populations stored as FP16, arithmetic,
                                   moments and adjoint FP32) */
    double nu;                  /* lattice viscosity, tau = 0.5 + 3 nu */
    double u_in[3];             /* inlet velocity (and initial state) */
    double alpha;               /* momentum fraction removed per step at gamma = 1 (0 < alpha <= 1) */
    double center[3];           /* moment reference */
} lbm_gray_setup;

/* The objective: J = mean over steps t0..t1 (1-based, inclusive) of
 * dir . F_t (objective 0) or dir . M_t (objective 1), F_t and M_t the force
 * and moment on the gray body after step t. */
typedef struct {
    uint64_t steps;             /* forward steps from the initial state */
    uint64_t t0, t1;
    uint32_t checkpoint_every;  /* full-state checkpoint interval */
    int32_t objective;          /* 0 force, 1 moment */
    double dir[3];
    int32_t recompute;          /* 1: recompute every segment from its checkpoint; 0: keep the
                                   per-step moments of the first pass when they fit in HBM */
    int32_t _pad;
} lbm_adjoint_spec;

typedef struct lbm_gray lbm_gray;

int lbm_gray_create(const lbm_gray_setup *setup, lbm_gray **out);
void lbm_gray_destroy(lbm_gray *h);
int lbm_gray_last_error(const lbm_gray *h, char *buf, uint64_t len);
/* gamma: box_n[0] * box_n[1] * box_n[2] values, x fastest, each in [0, 1] */
int lbm_gray_set_field(lbm_gray *h, const double *gamma);
/* back to the initial state (equilibrium at u_in), step counter 0 */
int lbm_gray_reset(lbm_gray *h);
/* n steps; forces_out: 6 doubles per step (force, then moment about center) */
int lbm_gray_run(lbm_gray *h, uint64_t n, double *forces_out);
/* From the initial state: the objective and its gradient with respect to
 * every design-box cell's gamma (box order, x fastest).  Leaves the lattice
 * in the state after spec->steps steps. */
int lbm_backward(lbm_gray *h, const lbm_adjoint_spec *spec, double *objective, double *dJ_dgamma);
/* Device time of the last lbm_backward, milliseconds: first forward pass,
 * recomputed forward segments, reverse sweep. */
int lbm_gray_backward_times(const lbm_gray *h, double *forward_ms, double *recompute_ms, double *reverse_ms);
int lbm_gray_stream(lbm_gray *h, void **stream);

/* Allocation-free force and moment sum over wall records (no counterpart in
 * the reference).  For callers that cannot allocate device memory where they
 * need the sum: hosts whose device memory is all handed out by their own pool
 * allocator, embedded callers with a fixed device footprint, latency-critical
 * loops that cannot afford cudaMalloc/cudaFree (which may synchronise the
 * device).  records_dev: nrec D3Q19 records of 40 u32 words in device memory
 * (the layout of lbm_records; the 24-word records of lbm_multi_records are
 * not accepted); forces_dev: 6 doubles in device memory (force, then moment);
 * stream: a cudaStream_t (NULL for the default stream).  The sum is over the
 * records' float force words in FP64, also for FP64-storage lattices (whose
 * lbm_run forces sum the double copies, so the two differ at float rounding).
 * The call enqueues the work and returns; it allocates and frees nothing.
 * Scratch: a fixed array inside this library, 256 KiB on every device that
 * loads it, kept until the process exits and shared by all calls on that
 * device: calls whose work overlaps on the GPU race and must be ordered by
 * the caller.  At most lbm_record_forces_noalloc_max() records (1,048,576);
 * more is rejected with LBM_ERR_INVALID.  The first call on a device looks up
 * the scratch's device address (kept for the life of the process, so the
 * device's context must not be reset in between); make that first call
 * before any stream capture.  Errors: message from lbm_noalloc_error. */
int lbm_record_forces_noalloc(const uint32_t *records_dev, uint64_t nrec, double *forces_dev, void *stream);
uint64_t lbm_record_forces_noalloc_max(void);
int lbm_noalloc_error(char *buf, uint64_t len);

#ifdef __cplusplus
}
#endif

#endif /* SIMLAB_LBM_H */
