/*
 * pgmpm.h -- C-ABI of the B200-native MLS-MPM step (libpgmpm.so).
 *
 * Plain C: pointers, sizes and an int status.  No torch or C++ types cross
 * this boundary.  Every entry point returns PGMPM_OK (0) or a negative
 * PGMPM_ERR_* code; pgmpm_last_error() gives the message of the last failure
 * on the calling thread.  A solver handle is not thread-safe: use one handle
 * per host thread.  Streams are explicit (cudaStream_t passed as void*; NULL
 * is the legacy default stream).
 *
 * What each entry point replaces in pedroscortes/physgrad (file:line):
 *   pgmpm_create / pgmpm_destroy
 *       physgrad::mpm::MPMSolver<T>(MPMSolverConfig) + initialize() +
 *       ~MPMSolver()/cleanup()            src/mpm_solver.h:156-187, 506-532
 *       MPMSolver<T,64>(int3, cell, origin, SimulationParams)
 *                                         src/material_point_method.h:450-453
 *       DifferentiableMPMSystem::initializeSystem
 *                                         src/differentiable_mpm.h:711-728
 *   pgmpm_upload
 *       MPMSolver<T>::addParticles        src/mpm_solver.h:190-226
 *       MPMSolver<T,64>::addParticles     src/material_point_method.h:455-477
 *   pgmpm_step
 *       MPMSolver<T>::step / run          src/mpm_solver.h:229-329
 *       MPMSolver<T,64>::step             src/material_point_method.h:479-500
 *       G2P2GKernelLauncher::launchG2P2G  src/mpm_g2p2g_kernels.h:494-515
 *   pgmpm_download / pgmpm_download_grid
 *       getParticles() / getGrid()        src/mpm_solver.h:322-324,
 *                                         src/material_point_method.h:503-504
 *   pgmpm_set_scene_params
 *       the per-call dt and gravity of
 *       DifferentiableMPMSystem::simulationStep(dt, gravity)
 *                                         src/differentiable_mpm.h:748
 *       and of launch_mpm_timestep_forward src/pytorch_autograd.cu:371-382
 *   pgmpm_get_metrics
 *       MPMSolver<T>::getMetrics          src/mpm_solver.h:324 (struct :72-101)
 *   pgmpm_forward_checkpointed / pgmpm_backward
 *       DifferentiableMPMSystem::simulationStep / computeGradients /
 *       getParticleGradients              src/differentiable_mpm.h:748-797
 *       (CheckpointStrategy::UNIFORM      src/differentiable_mpm.h:66)
 *   pgmpm_set_tuning / pgmpm_autotune
 *       MPMSolverConfig::cuda_block_size  src/mpm_solver.h:51 and
 *       kernels::KernelConfig             src/mpm_g2p2g_kernels.h:68-75
 *   launch_mpm_timestep_forward / launch_mpm_timestep_backward
 *       same names and arguments as       src/pytorch_autograd.cu:371-402
 *   pgmpm_radix_sort_pairs
 *       no reference counterpart (the reference does not sort); exported so
 *       the integer sort can be checked bit for bit on its own.
 */
#ifndef PGMPM_H
#define PGMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGMPM_ABI_VERSION 5

#if defined(__GNUC__)
#define PGMPM_API __attribute__((visibility("default")))
#else
#define PGMPM_API
#endif

/* ---- status codes ---------------------------------------------------- */
#define PGMPM_OK 0
#define PGMPM_ERR_ARG -1         /* invalid argument */
#define PGMPM_ERR_CUDA -2        /* CUDA runtime error (message in last_error) */
#define PGMPM_ERR_STATE -3       /* call not valid in the solver's state */
#define PGMPM_ERR_UNSUPPORTED -4 /* material / physics combination not built */
#define PGMPM_ERR_OOM -5         /* device allocation failed */
#define PGMPM_ERR_SIMULATION -6  /* device flagged escape / non-finite state */

/* ---- device status flags (pgmpm_check_status) ------------------------- */
#define PGMPM_FLAG_ESCAPE 1u      /* a particle left [0.5dx, (n-2.5)dx) (MLS) */
#define PGMPM_FLAG_NONFINITE 2u   /* non-finite position seen */
#define PGMPM_FLAG_TILE_RANGE 4u  /* stencil fell outside its tile (internal) */
#define PGMPM_FLAG_BAD_MATERIAL 8u /* material id outside [0, n_materials): used 0 */
#define PGMPM_FLAG_TILE_POOL 16u   /* sparse grid: the tile pool was full (results invalid) */

/* ---- enums ------------------------------------------------------------ */
#define PGMPM_PHYSICS_MLS 0        /* MLS-MPM + APIC + stress + walls */
#define PGMPM_PHYSICS_REF_COMPAT 1 /* reference CPU path: PIC, floor stencil, gravity */

#define PGMPM_BC_NONE 0
#define PGMPM_BC_STICKY 1   /* v = 0 on wall nodes */
#define PGMPM_BC_SLIP 2     /* normal component = 0 on wall nodes */
#define PGMPM_BC_SEPARATE 3 /* normal component clamped to leave the wall */

/* MaterialType values of src/mpm_data_structures.h:54-61 */
#define PGMPM_MAT_ELASTIC 0
#define PGMPM_MAT_ELASTOPLASTIC 1
#define PGMPM_MAT_FLUID 2
#define PGMPM_MAT_SAND 3
#define PGMPM_MAT_SNOW 4
#define PGMPM_MAT_JELLY 5

#define PGMPM_MODEL_FIXED_COROTATED 0
#define PGMPM_MODEL_NEO_HOOKEAN 1
#define PGMPM_MODEL_EOS_FLUID 2

/* pointer location flags for upload / download / backward */
#define PGMPM_PTR_HOST 0
#define PGMPM_PTR_DEVICE 1

typedef struct pgmpm_solver_s* pgmpm_solver;

/* One scene: a dense background grid of n[0] x n[1] x n[2] nodes with
 * spacing dx starting at origin (node (i,j,k) at origin + (i,j,k) dx). */
typedef struct {
    int32_t n[3];
    int32_t physics;            /* PGMPM_PHYSICS_* */
    int32_t boundary;           /* PGMPM_BC_* (MLS only; REF_COMPAT has none) */
    int32_t boundary_thickness; /* wall thickness in nodes */
    float dx;
    float origin[3];
    float dt;
    float gravity[3];
} pgmpm_scene_desc;

/* Material (src/mpm_data_structures.h:63-75 MaterialParameters subset).
 * ELASTIC / JELLY: model FIXED_COROTATED or NEO_HOOKEAN.
 * ELASTOPLASTIC: the neo-Hookean predictor with the von Mises return mapping
 *   of src/material_point_method.h:375-402 (the deviatoric Cauchy stress is
 *   scaled down to yield_stress; stateless, as there); model is ignored.
 * FLUID: model EOS_FLUID, p = -K (J - 1), plus the Newtonian viscous stress
 *   2 viscosity sym(grad v) of src/mpm_kernels.cu:131-149 (grad v = APIC C).
 * SAND and SNOW have no implementation in the reference and return
 * PGMPM_ERR_UNSUPPORTED.  Differentiation (pgmpm_forward_checkpointed,
 * pgmpm_backward) covers every supported material, the von Mises cap and the
 * fluid viscosity included (dL/dE: Young's modulus or bulk modulus). */
typedef struct {
    int32_t type;          /* PGMPM_MAT_* */
    int32_t model;         /* PGMPM_MODEL_*; FLUID requires EOS_FLUID */
    float youngs_modulus;  /* E; the bulk modulus K for FLUID (reference convention) */
    float poisson_ratio;
    float density;
    float yield_stress;    /* ELASTOPLASTIC: von Mises yield stress (Pa), > 0 */
    float viscosity;       /* FLUID: dynamic viscosity (Pa s), >= 0 (0: inviscid) */
} pgmpm_material;

typedef struct {
    int64_t total_steps;
    int64_t num_particles;
    int64_t active_nodes;      /* grid nodes with mass > 0 in the last step */
    double last_step_ms;       /* device time of the last timed step (events) */
    double average_step_ms;
    double particle_steps_per_s;
    double sort_ms, p2g_ms, grid_ms, g2p_ms; /* per-kernel device ms, last profiled step */
    int32_t p2g_block, p2g_ppt, g2p_block, graph_enabled;
    int32_t p2g_variant, g2p_variant, p2g_tiles_per_sm, g2p_tiles_per_sm;
} pgmpm_metrics;

/* Options of pgmpm_create_ex (zero-initialise; unset fields keep defaults). */
typedef struct {
    /* 1: a sparse grid.  Only the 4^3 node tiles that particles reach are
     * stored, in a pool of slots found through a hash of the tile's
     * coordinates, so memory follows the occupied region, not the domain:
     * a 2048^3 domain holds what its particles touch.  One MLS scene, at
     * most 4091 nodes per axis; the default kernels (P2G variant 4, G2P
     * variant 2, bin sort); no differentiation.  A step that finds the
     * pool full sets PGMPM_FLAG_TILE_POOL (create again with more tiles). */
    int32_t sparse_grid;
    int32_t reserved;
    /* sparse: tiles the pool must hold (0: max(4096, particles / 128)); the
     * pool is the next power of two of twice that, about 5.5 KB per slot. */
    int64_t max_tiles;
} pgmpm_create_options;

/* ---- lifecycle ---------------------------------------------------------- */
PGMPM_API const char* pgmpm_last_error(void);
/* Empties the calling thread's last error message, so that a caller of the
 * void launch_* entry points can tell whether one of them failed. */
PGMPM_API void pgmpm_clear_error(void);
PGMPM_API int pgmpm_abi_version(void);

/* Create a solver over n_scenes scenes (n_scenes = 1 for a plain solver).
 * particle_counts[s]: particles of scene s.  materials: table indexed by the
 * per-particle material id.  device: CUDA ordinal. */
PGMPM_API int pgmpm_create(const pgmpm_scene_desc* scenes, int32_t n_scenes, const int64_t* particle_counts,
                 const pgmpm_material* materials, int32_t n_materials, int32_t device, pgmpm_solver* out);
/* pgmpm_create with options (NULL: as pgmpm_create).  The reference's
 * sparse structures (src/sparse_data_structures.h) are separate from its
 * MPM grid; this makes the MPM grid itself sparse. */
PGMPM_API int pgmpm_create_ex(const pgmpm_scene_desc* scenes, int32_t n_scenes, const int64_t* particle_counts,
                              const pgmpm_material* materials, int32_t n_materials, int32_t device,
                              const pgmpm_create_options* options, pgmpm_solver* out);
PGMPM_API int pgmpm_destroy(pgmpm_solver s);

/* Replace the material table (same count), e.g. a new Young's modulus
 * between optimisation iterations.  Host pointer. */
PGMPM_API int pgmpm_set_materials(pgmpm_solver s, const pgmpm_material* materials, int32_t n_materials);

/* Change the time step and gravity of one scene between steps (gravity NULL
 * keeps it).  The next step's P2G payload is recomputed with the new dt.  A
 * recording of pgmpm_forward_checkpointed made before a change can no longer
 * be differentiated (pgmpm_backward then fails with PGMPM_ERR_STATE); so
 * does one made before pgmpm_set_materials.  Ordered after prior work on the
 * legacy default stream; returns when the change is in place. */
PGMPM_API int pgmpm_set_scene_params(pgmpm_solver s, int32_t scene, float dt, const float* gravity);

/* Upload particle state, scenes back to back in scene order.
 * x,v [N][3]; C,F [N][9] row-major (NULL C = 0, NULL F = I); m,V0 [N];
 * mat [N] (NULL = material 0).  ptr_kind: PGMPM_PTR_HOST / _DEVICE. */
PGMPM_API int pgmpm_upload(pgmpm_solver s, const float* x, const float* v, const float* C, const float* F,
                 const float* m, const float* V0, const int32_t* mat, int32_t ptr_kind, void* stream);

/* Download the state in upload order.  Any output pointer may be NULL. */
PGMPM_API int pgmpm_download(pgmpm_solver s, float* x, float* v, float* C, float* F, int32_t ptr_kind, void* stream);

/* Grid of one scene in the reference layout (index k*nx*ny + j*nx + i):
 * mass [nodes], velocity [nodes][3] after the last step's grid update. */
PGMPM_API int pgmpm_download_grid(pgmpm_solver s, int32_t scene, float* mass, float* velocity, int32_t ptr_kind,
                        void* stream);

/* ---- simulation ------------------------------------------------------------ */
PGMPM_API int pgmpm_step(pgmpm_solver s, int32_t n_steps, void* stream);

/* One host-buffer call: upload state, advance n_steps, download state.
 * Pointers are host memory (pinned for full PCIe speed). */
PGMPM_API int pgmpm_advance_host(pgmpm_solver s, const float* x_in, const float* v_in, const float* C_in,
                       const float* F_in, const float* m, const float* V0, const int32_t* mat,
                       int32_t n_steps, float* x_out, float* v_out, float* C_out, float* F_out, void* stream);

/* Device error flags accumulated since the last call (PGMPM_FLAG_*);
 * synchronises the stream and clears them. */
PGMPM_API int pgmpm_check_status(pgmpm_solver s, uint32_t* flags, void* stream);

/* ---- tuning ---------------------------------------------------------------- */
/* p2g_block, g2p_block: threads per block; ppt: particles per P2G chunk.
 * 0 keeps the current value.  use_graph: capture each step as a CUDA graph. */
PGMPM_API int pgmpm_set_tuning(pgmpm_solver s, int32_t p2g_block, int32_t ppt, int32_t g2p_block, int32_t use_graph);
/* Kernel variants.  p2g_variant 0: (cell, z-slice) register accumulation
 * over occupied 4^3 cell tiles (persistent, p2g_tiles_per_sm blocks per SM);
 * 1: per-particle shared-memory atomics over chunks of ppt particles;
 * 2: one thread per cell with 108 register accumulators;
 * 3: variant 2 with each cell's accumulators split over two lanes (MLS
 * forward; p2g_tiles_per_sm capped at 5);
 * 4: variant 3's lane pairs walking equal runs of each tile's sorted
 * particles instead of one cell each, cells shared by runs merged in shared
 * memory (MLS forward with the bin sort; with the radix step sort it runs
 * variant 3);
 * 5: variant 4, fused with G2P: from the second step of a chain, each
 * step's G2P kernel also does the next step's P2G (one lane per run of a
 * tile's sorted particles, the tile's node velocities staged in shared
 * memory, the payload never written to memory), so a step is the sort, the
 * grid update and that one kernel.  The pending P2G carries over to the
 * next pgmpm_step call; uploads, material or scene changes and
 * differentiation recompute it.  MLS with the bin sort (else variant 4's
 * rules apply); p2g_tiles_per_sm 4 or 6 (its register budget).
 * pgmpm_create picks 4 for MLS solvers that use the bin sort, else 3 from
 * 2^20 particles and 2 below; REF_COMPAT runs variant 2 for 2-5.
 * g2p_variant 0: tile-staged gather (g2p_tiles_per_sm blocks per SM);
 * 1: direct gather in sorted order; 2: direct gather in physical order.
 * Negative keeps a value. */
PGMPM_API int pgmpm_set_kernel_variants(pgmpm_solver s, int32_t p2g_variant, int32_t g2p_variant,
                                        int32_t p2g_tiles_per_sm, int32_t g2p_tiles_per_sm);
/* Per-step grouping of particles by cell.  PGMPM_SORT_BINS: a counting sort
 * over the cells, O(N + occupied cells + tiles) per step with 8 bytes of
 * scratch per cell; the keys come out sorted, particles that share a cell in
 * atomic-arrival order.  PGMPM_SORT_RADIX: the stable LSD radix sort, O(N)
 * per pass (the order of a stable CPU sort of the keys).  pgmpm_create picks
 * BINS when the grids hold at most about 8 cells per particle, else RADIX. */
#define PGMPM_SORT_BINS 0
#define PGMPM_SORT_RADIX 1
PGMPM_API int pgmpm_set_step_sort(pgmpm_solver s, int32_t kind);
/* Time candidate (block, ppt) settings on the solver's own state (restored
 * afterwards) and keep the fastest. */
PGMPM_API int pgmpm_autotune(pgmpm_solver s, int32_t reps, void* stream);
/* profile != 0: time each kernel group with events on the next steps
 * (graphs disabled while profiling). */
PGMPM_API int pgmpm_set_profiling(pgmpm_solver s, int32_t profile);
PGMPM_API int pgmpm_get_metrics(pgmpm_solver s, pgmpm_metrics* out);

/* ---- differentiation (MLS physics) ------------------------------------------ */
/* Run n_steps from the current state, storing the state every
 * checkpoint_every steps, so that pgmpm_backward can differentiate them. */
PGMPM_API int pgmpm_forward_checkpointed(pgmpm_solver s, int32_t n_steps, int32_t checkpoint_every, void* stream);
/* on != 0 (the default): a pgmpm_forward_checkpointed with the bin sort and
 * split steps records every step's sort (order, tile lists and cell ranges)
 * and keys, about 12 bytes per particle + 530 bytes per cell tile per step,
 * when the tape and the record take at most 1/16 of the device memory and
 * leave a quarter of it free.  pgmpm_backward's replays
 * then keep the recorded sorts instead of sorting again; a replayed step
 * sorts again only when the previous step's G2P, rounding differently from
 * the forward, put a particle in another cell.  Takes effect at the next
 * pgmpm_forward_checkpointed.  on = 2 records too, but every replayed step
 * after a segment's first sorts again (a check of that path: the gradients
 * are those of on = 0).  No reference counterpart (the reference keeps no
 * sort). */
PGMPM_API int pgmpm_set_sort_record(pgmpm_solver s, int32_t on);
/* Replayed steps that sorted again (see pgmpm_set_sort_record) over the
 * solver's life; waits for the device.  No reference counterpart. */
PGMPM_API int pgmpm_get_replay_resorts(pgmpm_solver s, int64_t* steps);
/* Reverse pass over the last pgmpm_forward_checkpointed call.  g*_out: dL/d
 * of the final state (upload order, any may be NULL = 0).  g*_in: receives
 * dL/d of the initial state (any may be NULL).  gE [n_materials]: dL/dE per
 * material (dL/dK for FLUID); may be NULL. */
PGMPM_API int pgmpm_backward(pgmpm_solver s, const float* gx_out, const float* gv_out, const float* gC_out,
                   const float* gF_out, float* gx_in, float* gv_in, float* gC_in, float* gF_in, float* gE,
                   int32_t ptr_kind, void* stream);

/* ---- output ---------------------------------------------------------------------- */
/* Particle output in the legacy VTK format (binary, POLYDATA): points x, one
 * vertex per particle, and point data "velocity" (v), "J" (det F) and
 * "material" (id), each written when its array is given.  Host arrays in
 * upload order; x: [n][3], v: [n][3], F: [n][9] row-major, mat: [n].  Needs
 * no GPU.  This is the data output that MPMSolver::outputData()
 * (src/mpm_solver.h:501-504) leaves as a stub. */
PGMPM_API int pgmpm_vtk_write_particles(const char* path, int64_t n, const float* x, const float* v, const float* F,
                                        const int32_t* mat, double time);
/* The solver's particles (downloaded, upload order) to `path` as above, with
 * material ids when the solver has more than one material. */
PGMPM_API int pgmpm_write_vtk(pgmpm_solver s, const char* path, double time, void* stream);

/* ---- spatial hash grid (particle neighbourhoods) ------------------------------ */
/* physgrad::sparse::SpatialHashGrid<float, uint32_t> (src/sparse_data_structures.h:44-296,
 * used by src/fsi_coupling.h:72) on the GPU.  Cells of size cell_size tile
 * [domain_min, domain_max); a point's cell id is morton(cell) % total_cells
 * with the cell clamped to the resolution, as getCellID (:143-151).  The
 * table (per-cell counts and starts, particle indices sorted by cell, stable
 * within a cell, and the cell id of each particle) equals buildHashTable's
 * (:155-190) bit for bit. */
typedef struct pgmpm_hashgrid_s* pgmpm_hashgrid;
typedef struct {
    float average_particles_per_cell; /* over occupied cells (HashTableStats, :243-272) */
    float load_factor;                /* occupied / total cells */
    uint32_t max_particles_per_cell;
    uint32_t occupied_cells;
    float memory_usage_mb;            /* the host class's accounting */
    uint32_t total_cells;
    uint32_t resolution[3];
} pgmpm_hashgrid_info;
/* SpatialHashGrid(cell_size, domain_min, domain_max, max_particles) (:76-97). */
PGMPM_API int pgmpm_hashgrid_create(float cell_size, const float* domain_min, const float* domain_max,
                                    int64_t max_particles, int32_t device, pgmpm_hashgrid* out);
PGMPM_API int pgmpm_hashgrid_destroy(pgmpm_hashgrid g);
/* buildHashTable(positions [n][3], n) (:155-190). */
PGMPM_API int pgmpm_hashgrid_build(pgmpm_hashgrid g, const float* positions, int64_t n, int32_t ptr_kind,
                                   void* stream);
/* getNeighbors(x, y, z, radius) (:206-240) for nq query points [nq][3]:
 * query i's list is indices[offsets[i] .. offsets[i+1]), offsets has nq + 1
 * entries and *total = offsets[nq].  As the host class, a list holds every
 * particle of the (2 ceil(radius / cell_size) + 1)^3 cells around the query's
 * cell in that method's order, without a distance test.  indices are
 * written only when capacity >= *total (else call again with room for it). */
PGMPM_API int pgmpm_hashgrid_neighbors(pgmpm_hashgrid g, const float* queries, int64_t nq, float radius,
                                       int64_t* offsets, uint32_t* indices, int64_t capacity, int64_t* total,
                                       int32_t ptr_kind, void* stream);
/* getCellParticleCounts / getCellStartIndices (total_cells entries),
 * getParticleIndices and the cell ids (n entries) of the last build; NULL
 * skips an array. */
PGMPM_API int pgmpm_hashgrid_get_table(pgmpm_hashgrid g, uint32_t* counts, uint32_t* starts,
                                       uint32_t* particle_indices, uint32_t* cell_ids, int32_t ptr_kind,
                                       void* stream);
/* getStats() (:243-272); before a build the particle fields are zero. */
PGMPM_API int pgmpm_hashgrid_stats(pgmpm_hashgrid g, pgmpm_hashgrid_info* out);

/* ---- consumers of the particles ------------------------------------------------ */
/* CouplingConfig of src/sph_mpm_coupling.h:391-407 (the fields its forces use). */
typedef struct {
    float coupling_stiffness;        /* k, normal spring (default there 1e5) */
    float coupling_damping;          /* c, normal damping (1e3) */
    float friction_coefficient;      /* mu (0.3) */
    float coupling_radius;           /* pairs closer than this (0.15) */
    int32_t enable_two_way_coupling; /* 1: add the fluid forces to sph_force */
    int32_t reserved;
} pgmpm_sph_coupling_config;
/* SPHMPMCouplingSystem::findCouplingPairs + computeCouplingForces +
 * getNumCouplingPairs + getTotalCouplingEnergy (src/sph_mpm_coupling.h:
 * 453-575) with the solver's particles (one scene, their current x and v)
 * as the MPM side: every (SPH, MPM) pair closer than the radius, normal
 * force k (r - d) + c (dv . n) along n = (x_mpm - x_sph) / d, friction
 * -mu k (r - d) along the tangential relative velocity, nothing when
 * d < 1e-6.  sph_x, sph_v [n_sph][3]; sph_force [n_sph][3]: the fluid forces
 * are ADDED (as the reference adds them to SPHParticle::force), two-way only;
 * mpm_force [N][3] (may be NULL): overwritten with each particle's summed
 * solid force, upload order.  n_pairs, energy (sum of k (r - d)^2 / 2) may be
 * NULL.  Pairs are found through the spatial hash grid of this library over
 * the scene's grid domain, with cells of half a radius (one radius when that
 * would make more than max(4 N, 2^20) cells).  Synchronises stream. */
PGMPM_API int pgmpm_sph_coupling(pgmpm_solver s, const pgmpm_sph_coupling_config* cfg, const float* sph_x,
                                 const float* sph_v, int64_t n_sph, float* sph_force, float* mpm_force,
                                 int64_t* n_pairs, double* energy, int32_t ptr_kind, void* stream);
/* The energy monitor of FSISimulationManager (computeTotalEnergy,
 * src/fsi_coupling.h:837-858): sum of m |v|^2 / 2 over the particles,
 * per material id (per_material [n_materials], may be NULL) and in total
 * (may be NULL); with a fluid and a solid material, the two sets that
 * monitor sums.  FP64 sums.  Synchronises stream. */
PGMPM_API int pgmpm_kinetic_energy(pgmpm_solver s, double* per_material, double* total, void* stream);

/* ---- inspection ------------------------------------------------------------------ */
#define PGMPM_ARRAY_USER_INDEX 0   /* physical slot -> upload index */
#define PGMPM_ARRAY_KEYS 1         /* cell key per physical slot (input of the next sort) */
#define PGMPM_ARRAY_SORTED_KEYS 2  /* sorted keys of the last step */
#define PGMPM_ARRAY_SORTED_ORDER 3 /* sorted position -> physical slot, last step */
/* Copy one u32 array of N entries (see PGMPM_ARRAY_*) for inspection; no
 * reference counterpart (exposes the integer sort for bit-exact checks). */
PGMPM_API int pgmpm_get_array(pgmpm_solver s, int32_t which, uint32_t* out, int32_t ptr_kind, void* stream);

/* ---- building blocks ---------------------------------------------------------- */
/* Stable LSD radix sort of (key, value) pairs by the low key_bits bits of the
 * key (device pointers; vals_in NULL = 0..n-1).  Bit-identical to a stable
 * CPU sort. */
PGMPM_API int pgmpm_radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                           uint32_t* vals_out, int64_t n, int32_t key_bits, void* stream);

/* Same stable sort, for callers that may not allocate device memory (a host
 * framework that owns the GPU memory budget, or a loop that cannot afford
 * cudaMalloc's device-wide synchronisation).  No reference counterpart: the
 * reference has no sort.  It calls no allocator.  Its scratch is a fixed
 * array in the library's device image (about 8.9 MB per GPU that loads the
 * library, held until exit), so n is limited to PGMPM_NOALLOC_MAX_PAIRS
 * (larger n returns PGMPM_ERR_ARG).  keys_out and vals_out must not overlap
 * the inputs or each other (PGMPM_ERR_ARG).  The first call on a device
 * looks up the array's address and may load the module: make it before any
 * stream capture.  The address is kept for the process's life, so a
 * cudaDeviceReset of a device after this entry point has been called on it
 * is not supported.  Calls share the array, so calls that overlap on the GPU
 * race; the caller orders them.  Asynchronous on `stream`. */
#define PGMPM_NOALLOC_MAX_PAIRS (1 << 20)
PGMPM_API int pgmpm_radix_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                             uint32_t* vals_out, int64_t n, int32_t key_bits, void* stream);

/* Reference-shaped launcher (src/pytorch_autograd.cu:371-382): one
 * REF_COMPAT MPM step of num_particles particles on the unit cube with a
 * grid_resolution^3 grid (dx = 1/grid_resolution).  positions, velocities
 * [n][3], masses [n], gravity [3] are device pointers; stream is a
 * cudaStream_t.  Errors are reported through pgmpm_last_error(). */
PGMPM_API void launch_mpm_timestep_forward(float* positions, float* velocities, const float* masses, int num_particles,
                                 int grid_resolution, float dt, const float* gravity, void* stream);

/* Reference-shaped launcher (src/pytorch_autograd.cu:384-402): the reverse of
 * the step launch_mpm_timestep_forward ran from saved_positions,
 * saved_velocities (that step's inputs).  grad_positions, grad_velocities:
 * dL/d of the step's outputs; writes dL/d of its inputs to
 * grad_input_positions, grad_input_velocities [n][3] and grad_masses [n]
 * (may be NULL), and adds dL/dgravity to grad_gravity [3] (may be NULL), as
 * the reference's kernel does.  Masses and gravity are those of the last
 * forward call with the same device, particle count and resolution (an
 * error if there was none).  Device pointers; asynchronous on stream. */
PGMPM_API void launch_mpm_timestep_backward(const float* grad_positions, const float* grad_velocities,
                                  float* grad_input_positions, float* grad_input_velocities, float* grad_masses,
                                  float* grad_gravity, const float* saved_positions, const float* saved_velocities,
                                  int num_particles, int grid_resolution, float dt, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PGMPM_H */
