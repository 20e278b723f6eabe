/*
 * banana_b200 -- C ABI of the B200-native FLIP / APIC / AFLIP fluid step, pressure PCG,
 * uniform-grid cell sort and neighbour search.
 *
 * This is the drop-in boundary.  The reference (ttnghia/Banana) drives the hot path
 * through its solver plugin API:
 *   ParticleSolver<N,Real>              Simulation/ParticleSolvers/ParticleSolver.h:39-105
 *   ParticleSolverFactory / Registered   Simulation/ParticleSolvers/ParticleSolverFactory.h:32-60
 *   PIC_Solver::advanceFrame             Simulation/ParticleSolvers/PICFluid/PIC_Solver.cpp:267-311
 *   FLIP_Solver::advanceVelocity         Simulation/ParticleSolvers/PICFluid/FLIP_Solver.cpp:42-53
 * A host C++ class registered in that factory (banana_b200/host/FLIP_GPU_Solver.h) owns one
 * bnn_flip handle and forwards advanceFrame / particle I/O to the functions below.
 *
 * Conventions: every function returns an int status (BNN_OK = 0).  Arrays are HOST
 * pointers unless the parameter name ends in _dev.  Particle arrays are AoS float3
 * (x,y,z per particle), the layout of glm::vec3 in ParticleSimulationData::positions
 * (ParticleSolverData.h:197).  Grid arrays use the reference Array<3,T> layout
 * (k*Sy + j)*Sx + i (BananaCore/Banana/Array/Array.h:276).  A handle is driven by one
 * host thread at a time; distinct handles may be used from distinct threads.
 * No function calls exit(): failures that the reference turns into exit(EXIT_FAILURE)
 * (__BNN_REQUIRE, Macros.h:225-233, and ExitIfPressureProjectionFailed,
 * PIC_Solver.cpp:901-906) come back as status codes.
 */
#ifndef BANANA_B200_H
#define BANANA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define BNN_OK                    0
#define BNN_ERR_INVALID_ARGUMENT  1  /* __BNN_REQUIRE failures in the reference */
#define BNN_ERR_OUT_OF_MEMORY     2
#define BNN_ERR_PCG_NOT_CONVERGED 3  /* PCGSolver::solve_precond returned false */
#define BNN_ERR_DEVICE_CHECK      4  /* a kernel's own range / state check failed */
#define BNN_ERR_TIMEOUT           5  /* a bounded device-side wait gave up */
#define BNN_ERR_CUDA              6
#define BNN_ERR_NOT_SUPPORTED     7
#define BNN_ERR_CAPACITY          8  /* output buffer too small (neighbour lists) */

/* ---- enums ----------------------------------------------------------------------- */
#define BNN_SOLVER_FLIP   0  /* FLIP_3DSolver  (FLIP_Solver.cpp)  */
#define BNN_SOLVER_APIC   1  /* APIC_3DSolver  (APIC_Solver.cpp)  */
#define BNN_SOLVER_AFLIP  2  /* AFLIP_3DSolver (AFLIP_Solver.cpp) */
#define BNN_SOLVER_PIC    3  /* PIC_3DSolver (PIC_Solver.cpp): semi-Lagrangian grid advection,
                                particles only mark the fluid */

#define BNN_PCG_FP32      0  /* FP32 vectors, FP64 dot/norm reductions */
#define BNN_PCG_FP64      1  /* FP64 vectors and reductions */
#define BNN_PCG_REFINED   2  /* FP32 inner PCG + FP64 outer residual (iterative refinement) */
#define BNN_PCG_MODE_MASK 0x0f
/* OR-ed into a BNN_PCG_* mode: the single-reduction form of the same iteration (Chronopoulos
 * & Gear: both inner products of an iteration in one grid-wide reduction, the same iterates
 * up to rounding).  Without it the solve takes PCGSolver::solve_precond's own step order
 * (PCGSolver.cpp:143-199: the two inner products one after the other, two reductions per
 * iteration). */
#define BNN_PCG_SINGLE_REDUCTION 0x10

#define BNN_PRECOND_JACOBI 0 /* PCGSolver::JACOBI (PCGSolver.cpp:232-237,273-284) */

#define BNN_FIELD_U        0 /* face velocities, sizes (G+1)GG, G(G+1)G, GG(G+1) */
#define BNN_FIELD_V        1
#define BNN_FIELD_W        2
#define BNN_FIELD_PHI      3 /* fluid SDF on cells (PIC_Data.h fluidSDF) */
#define BNN_FIELD_PRESSURE 4 /* pressure scattered onto cells, 0 where not fluid */
#define BNN_FIELD_OLD_U    5 /* FLIP backup velocities (FLIP_Data.h oldVels) */
#define BNN_FIELD_OLD_V    6
#define BNN_FIELD_OLD_W    7
#define BNN_FIELD_ACTIVE   8 /* active cell index + 1 on cells, 0 = not fluid */
#define BNN_FIELD_WEIGHT_U 9 /* face weights (PIC_Data.h weights); 1 without dynamic boundaries */
#define BNN_FIELD_WEIGHT_V 10
#define BNN_FIELD_WEIGHT_W 11
#define BNN_FIELD_BOUNDARY_SDF 12 /* boundary SDF on the (G+1)^3 nodes (PIC_Data.h boundarySDF) */

/* Values of SimulationParameters / PIC_Parameters / GlobalParameters the step reads
 * (ParticleSolverData.h:87-175, PIC_Data.h:31-40, ParticleSolverData.h:37-75). */
typedef struct bnn_params {
    float    box_min[3];             /* SimulationDomainBox BoxMin (before NExpandCells padding) */
    float    box_max[3];             /* SimulationDomainBox BoxMax */
    float    cell_size;              /* CellSize */
    uint32_t n_expand_cells;         /* NExpandCells (default 2) */
    float    cfl_factor;             /* CFLFactor (default 1) */
    float    min_timestep;           /* MinTimestep (default 1e-6) */
    float    max_timestep;           /* MaxTimestep (default 1/30) */
    float    frame_duration;         /* FrameDuration (default 1/30) */
    float    pic_flip_ratio;         /* PIC_FLIP_ratio (default 0.97) */
    float    cg_relative_tolerance;  /* CGRelativeTolerance */
    uint32_t max_cg_iteration;       /* MaxCGIteration */
    uint32_t advection_steps;        /* AdvectionSteps (default 1) */
    int32_t  solver_kind;            /* BNN_SOLVER_* */
    int32_t  pcg_mode;               /* BNN_PCG_*, optionally | BNN_PCG_SINGLE_REDUCTION */
    int32_t  preconditioner;         /* BNN_PRECOND_* */
    float    refine_tolerance;       /* BNN_PCG_REFINED: outer max-norm relative tolerance */
    float    refine_inner_tolerance; /* BNN_PCG_REFINED: inner FP32 relative tolerance (1e-2 is
                                        fastest on the 256^3 dam break to an outer 1e-8) */
    int32_t  apply_gravity;          /* GlobalParameters ApplyGravity (default 1) */
    uint32_t max_particles;          /* particle capacity; 0 = size to the first set_particles */
    int32_t  correct_position;       /* CorrectPosition (default 0): neighbour-spring pass after
                                        moveParticles, PIC_Solver::correctParticlePositions */
    float    repulsive_force_stiffness; /* RepulsiveForceStiffness (default 50) */
    float    ratio_cell_size_p_radius;  /* RatioCellSizePRadius (default 2): particle radius =
                                           cell_size / ratio */
} bnn_params;

/* What one call of bnn_flip_step did.  stage_ms are CUDA-event times of the stages:
 * 0 move, 1 sort, 2 p2g, 3 extrapolate+backup+gravity, 4 fluid sdf, 5 system, 6 pcg,
 * 7 update+extrapolate, 8 g2p, 9 whole step. */
typedef struct bnn_step_stats {
    double   dt;               /* sub-step size used (PIC_Solver.cpp:284-290) */
    double   frame_time;       /* frameLocalTime after the sub-step */
    uint32_t frame_finished;   /* 1 when frame_time reached FrameDuration */
    uint32_t pcg_iterations;   /* PCGSolver::iterations() (inner total for refinement) */
    double   pcg_residual;     /* PCGSolver::residual(): max|r| of the last iterate */
    uint32_t pcg_success;
    uint32_t n_active;         /* rows of the pressure system */
    uint32_t outer_iterations; /* refinement sweeps (BNN_PCG_REFINED) */
    uint32_t zero_phi_cells;   /* interior cells with fluid SDF exactly 0 (left out) */
    float    stage_ms[10];
    uint32_t device_flags;     /* bit 0: particle outside the grid, bit 1: fluid in the
                                  outer cell ring, bit 2: PCG hit MaxCGIteration */
    float    pcg_kernel_ms;    /* device time of the persistent PCG launch(es) alone */
} bnn_step_stats;

typedef struct bnn_flip bnn_flip;

/* Create a solver: grid setup as SimulationParameters::makeReady + PIC_Data::makeReady
 * (ParticleSolverData.cpp:229-272, PIC_Data.cpp:128-144). */
int bnn_flip_create(const bnn_params* params, bnn_flip** out);
int bnn_flip_destroy(bnn_flip* h);
/* Grid cell counts G (after padding) */
int bnn_flip_grid_dims(bnn_flip* h, int32_t g[3]);
/* Replace all particles (PIC_ParticleData::addParticles, PIC_Data.cpp:73-82, into an
 * empty solver); grid velocities are reset to 0 as after makeReady. */
int bnn_flip_set_particles(bnn_flip* h, const float* pos, const float* vel, uint32_t n);
/* Particles in the order they were given (ParticleSolverInterface.h:128-149 reads
 * positions / velocities as raw host arrays between frames). */
int bnn_flip_get_particles(bnn_flip* h, float* pos, float* vel);
int bnn_flip_num_particles(bnn_flip* h, uint32_t* n);
/* Replace the face velocities of one component (BNN_FIELD_U/V/W; count = its face count),
 * e.g. from a saved memory state (PIC_Solver::loadMemoryState, PIC_Solver.cpp:158-206);
 * the next sub-step's CFL uses the new field. */
int bnn_flip_set_grid(bnn_flip* h, int32_t field, const float* in, size_t count);
/* Copy one grid field (BNN_FIELD_*) of `count` floats to host. */
int bnn_flip_get_grid(bnn_flip* h, int32_t field, float* out, size_t count);
/* One iteration of PIC_Solver::advanceFrame's sub-step loop (CFL, moveParticles,
 * advanceVelocity; PIC_Solver.cpp:277-305).  A new frame starts when the previous one
 * finished. */
int bnn_flip_step(bnn_flip* h, bnn_step_stats* stats);
/* PIC_Solver::advanceFrame: sub-steps until FrameDuration is reached. */
int bnn_flip_advance_frame(bnn_flip* h, uint32_t* substeps);
/* Device pointers of the particle arrays (SoA x,y,z,vx,vy,vz, current sorted order),
 * valid until the next step; lets a caller keep data on the device (and change it: the
 * next step then moves the particles from what the arrays hold). */
int bnn_flip_device_particles(bnn_flip* h, float** xyz_vxyz_dev, uint32_t** ids_dev);
/* The cudaStream_t every kernel of this handle is launched on (for events / ordering). */
int bnn_flip_stream(bnn_flip* h, void** stream);
/* Same sub-step as bnn_flip_step, but the particles come from pinned host AoS arrays and
 * are written back to them: upload, step, download in one stream (end-to-end timing). */
int bnn_flip_step_host(bnn_flip* h, float* pos, float* vel, bnn_step_stats* stats);

/* Device bytes the handle holds now (grids, particle, row and PCG arrays). */
int bnn_flip_device_bytes(bnn_flip* h, uint64_t* bytes);
/* Device bytes a scene with these parameters and n particles is expected to hold (the
 * admission test of scene batches). */
int bnn_scene_bytes_estimate(const bnn_params* params, uint32_t n, uint64_t* bytes);

/* ---- scene batches -----------------------------------------------------------------
 * Many independent scenes on one GPU (serving).  Each scene is a full solver (same
 * results as a lone handle); bnn_batch_step advances every scene by one sub-step,
 * stepping scenes concurrently from worker threads on their own streams.  A batch is
 * driven by one host thread.  No counterpart in the reference, which runs one scene per
 * ParticleSolver object (ParticleSolver.h:39-105). */
typedef struct bnn_batch bnn_batch;
/* How bnn_batch_step advances the scenes.  STAGED (the default): the scenes the staged
 * step takes (FLIP, BNN_PCG_REFINED in its default step order, the domain box as the only
 * boundary, no position correction, particles present) advance together, one kernel launch
 * per stage of the sub-step over all of them; the others as in PER_SCENE.  PER_SCENE: every
 * scene runs bnn_flip_step on its own stream, from a pool of host threads.  Both compute
 * for every scene exactly what bnn_flip_step computes for it alone. */
#define BNN_BATCH_STAGED    0
#define BNN_BATCH_PER_SCENE 1
/* OR-ed into BNN_BATCH_STAGED: launch the staged step's kernels one by one instead of
 * replaying the CUDA graphs captured from them (same kernels, same results) */
#define BNN_BATCH_NO_GRAPHS 0x100
typedef struct bnn_batch_params {
    uint64_t hbm_budget_bytes; /* admission budget over bnn_scene_bytes_estimate; 0 = none */
    uint32_t worker_threads;   /* host threads stepping scenes; 0 = min(16, cores) */
    uint32_t step_mode;        /* BNN_BATCH_STAGED (optionally | BNN_BATCH_NO_GRAPHS) or BNN_BATCH_PER_SCENE */
} bnn_batch_params;
typedef struct bnn_batch_stats {
    uint32_t scenes;           /* scenes stepped */
    uint32_t failed;           /* scenes whose step returned an error */
    uint64_t particle_steps;   /* particles advanced by one sub-step, summed over scenes */
    uint64_t pcg_iterations;   /* summed over scenes */
    double   wall_ms;          /* host wall time of the batch step */
    double   max_scene_ms;     /* slowest scene's step */
    uint32_t staged_scenes;    /* scenes advanced by the staged (one launch per stage) step */
    uint16_t graph_instantiations; /* segments of the staged step captured and built into a new
                                      CUDA graph in this step (0-2) */
    uint16_t graph_updates;    /* segments captured again and written into the existing graph
                                  (same launches, other shapes; 0-2) */
} bnn_batch_stats;
int bnn_batch_create(const bnn_batch_params* params, bnn_batch** out);
int bnn_batch_destroy(bnn_batch* b);
/* BNN_ERR_CAPACITY when the scene's estimate does not fit the remaining budget. */
int bnn_batch_add_scene(bnn_batch* b, const bnn_params* params, const float* pos, const float* vel, uint32_t n,
                        uint32_t* scene_id);
int bnn_batch_remove_scene(bnn_batch* b, uint32_t scene_id);
/* One sub-step of every scene; returns the first failing scene's status (all scenes are
 * stepped regardless). */
int bnn_batch_step(bnn_batch* b, bnn_batch_stats* stats);
/* Particle count, sub-steps done and the stats of its last sub-step; returns the status
 * of that sub-step. */
int bnn_batch_scene_info(bnn_batch* b, uint32_t scene_id, uint32_t* n, uint64_t* steps, bnn_step_stats* last);
int bnn_batch_get_scene(bnn_batch* b, uint32_t scene_id, float* pos, float* vel);
/* Sum of the admitted scenes' estimates and of the bytes they hold now. */
int bnn_batch_memory(bnn_batch* b, uint64_t* admitted, uint64_t* held);

/* ---- tile shapes of the P2G + fluid SDF pass -------------------------------------
 * The FLIP pass (P2G of the three face components with the fluid SDF) runs in tiles of
 * 30 x tz face columns walking yc face layers along y; every shape computes the same bits
 * (fixed per-cell and per-face summation orders).  By default a tuner times every shape the
 * first time it meets a kind of launch (a lone scene's resolution bucket, ceil((G + 1) / 32)
 * cells per axis; a batch's scene count and total cells, in powers of two) and keeps the
 * fastest (the default shape 0 unless another is 3% faster).  No counterpart in the reference (its P2G is a serial loop, FLIP_Solver.cpp:57-95). */
/* Number of shapes; tz[i], yc[i] of each (arrays of at least `cap` entries, may be NULL). */
int bnn_tile_shapes(int32_t* tz, int32_t* yc, int32_t cap);
/* Use shape `shape` (0 .. bnn_tile_shapes() - 1) for every launch of the process, or -1 to
 * tune (the default).  BNN_ERR_INVALID_ARGUMENT outside that range. */
int bnn_set_tile_shape(int32_t shape);
/* The tuner's choices as JSON lines, NUL-terminated, into buf (cap bytes); *needed = bytes
 * the whole text takes with its NUL.  BNN_ERR_CAPACITY when cap is smaller. */
int bnn_tile_tuning(char* buf, size_t cap, size_t* needed);

/* ---- standalone kernels (device pointers, stream = cudaStream_t or NULL) ---------- */

/* Grid::getCellIdx + getCellLinearizedIndex (Grid.h:108-111,156-162) for every point and
 * the canonical sorted index (stable: by linear cell id, ties in input order), i.e.
 * Grid::getParticleIdxSortedByCell (Grid.cpp:299-309) of a one-thread collectIndexToCells.
 * cell_start_dev (optional) receives the C+1 bucket offsets.  Points outside the grid
 * are clamped onto its border and counted in *out_of_range. */
int bnn_cell_sort(const float* pos_dev, uint32_t n, const float bmin[3], float cell_size, const int32_t ncells[3],
                  uint32_t* cell_id_dev, uint32_t* sorted_idx_dev, uint32_t* cell_start_dev, uint32_t* out_of_range,
                  void* stream);

/* The same cell sort (same outputs, bit for bit) without allocating any device memory.
 * No counterpart in the reference (its Grid sort is host code).  It is for callers that
 * cannot call cudaMalloc when they need a sort: an application whose own pool allocator
 * has already reserved all device memory (a further cudaMalloc would fail or steal from
 * the pool), or a loop on a latency budget where cudaMalloc / cudaFree would synchronise
 * the device and stall work queued on other streams.  The caller still passes the inputs
 * and outputs; the sort's scratch lives in a fixed array compiled into the library
 * (about 21 MiB, held on every GPU that loads the library until the process exits).
 * Limits: n <= 1,048,576 points and <= 2,097,152 cells; larger sizes return
 * BNN_ERR_CAPACITY.  The first call on a device (and the first after that device's
 * context was reset) looks up the array's device address, so make that first call before
 * any stream capture.  Every call uses the one array, which keeps the previous call's
 * contents: calls that overlap on the GPU (several streams or host threads at once) race
 * and must be serialised by the caller.  Synchronises `stream` before returning. */
int bnn_cell_sort_noalloc(const float* pos_dev, uint32_t n, const float bmin[3], float cell_size,
                          const int32_t ncells[3], uint32_t* cell_id_dev, uint32_t* sorted_idx_dev,
                          uint32_t* cell_start_dev, uint32_t* out_of_range, void* stream);

/* NeighborSearch::z_sort (NeighborSearch.cpp:57-86): Morton code of each point's hash key
 * and the permutation sorting by it (ties in input order). */
int bnn_z_sort(const float* pos_dev, uint32_t n, float radius, uint64_t* zvalue_dev, uint32_t* perm_dev, void* stream);

/* NeighborSearch::find_neighbors for one self-searching point set (NeighborSearch.cpp:
 * 219-226, query3D :530-692): neighbours of each point are all other points with
 * |x-y|^2 < r^2.  Output CSR: offsets_dev (n+1), idx_dev (capacity entries).  A list holds
 * its points in the order the 27 cells around the point are visited (z, y, x major; a
 * cell's points in sorted-index order), deterministic but not ascending -- the
 * reference's own order depends on its thread schedule, so lists compare as sets.
 * *total receives the entry count; BNN_ERR_CAPACITY when it exceeds capacity (offsets are
 * still written). */
int bnn_neighbors(const float* pos_dev, uint32_t n, float radius, uint64_t* offsets_dev, uint32_t* idx_dev,
                  uint64_t capacity, uint64_t* total, void* stream);

/* Standalone Jacobi PCG (PCGSolver::solve_precond, PCGSolver.cpp:143-199) on a 7-point
 * system given in host memory: diag[n], nbr[6n] neighbour rows in column order
 * (-z,-y,-x,+x,+y,+z; -1 = none), one off-diagonal value for every neighbour, rhs[n].
 * mode BNN_PCG_*.  x_out receives the solution in FP64. */
typedef struct bnn_pcg_stats {
    uint32_t iterations;
    uint32_t outer_iterations;
    double   residual;
    uint32_t success;
    float    ms;
} bnn_pcg_stats;
int bnn_pcg_solve_7pt(uint32_t n, const float* diag, const int32_t* nbr, float offdiag, const float* rhs, float tol,
                      uint32_t max_iter, int32_t mode, float inner_tol, double* x_out, bnn_pcg_stats* stats);

/* Self-test of the bounded wait of the PCG grid barrier (no counterpart in the reference,
 * whose solver has no device-side waits).  One block waits at a barrier sized for two
 * blocks, so the wait can only end by giving up: after 4096 polls and limit_seconds
 * (0 < limit_seconds <= 10) of wall time, the limit a solve uses being 1 s.
 * *barrier_status receives BNN_ERR_TIMEOUT when the wait gave up as designed, *elapsed_ms
 * how long the block polled.  The device stays usable afterwards.  The probe runs on the
 * default stream and synchronizes the device, so it is not for use while solves run. */
int bnn_pcg_barrier_probe(float limit_seconds, int32_t* barrier_status, float* elapsed_ms);

/* Library version / last CUDA error text / number of kernels this library has launched
 * in this process (diagnostics; no counterpart in the reference). */
/* ---- boundary objects ------------------------------------------------------------- */

#define BNN_GEOMETRY_BOX     0  /* GeometryObjects::BoxObject (GeometryObjects.cpp:246-268) */
#define BNN_GEOMETRY_SPHERE  1  /* GeometryObjects::SphereObject, unit sphere in object space */

/* One boundary object of "AdditionalBoundaryObjects" (ParticleSolver::generateBoundaries,
 * ParticleSolver.cpp:242-295; BoundaryObject.h:41-60): the fluid stays inside it (its
 * signed distance is taken with bNegativeInside = false).  Its current transformation is
 * given as the world-to-object map (GeometryObject::invTransform, the inverse of
 * translate * rotate * scale of the current animation frame) and the uniform scale. */
typedef struct bnn_boundary_object {
    int32_t geometry;          /* BNN_GEOMETRY_* */
    int32_t dynamic;           /* 1: animated ("Animation" present, SimulationObject.cpp:80-82) */
    float   box_min[3];        /* box corners in object space */
    float   box_max[3];
    float   inv_transform[12]; /* rows of the 3x4 world-to-object affine map */
    float   uniform_scale;
    int32_t transformed;       /* 0: the map is the identity and is not applied */
} bnn_boundary_object;

/* Sets the boundary objects besides the domain box (at most 15).  As in the reference,
 * the static ones are united with the domain box into one CSG object and the dynamic
 * ones stay separate; particles are projected back inside every one after each
 * advection.  update_grid != 0 with at least one dynamic object recomputes the grid's
 * boundary SDF from the objects as given (PIC_Solver::advanceScene + computeBoundarySDF,
 * PIC_Solver.cpp:70-118,1157-1168); from then on the solve uses the face weights, the
 * solid part of the fluid SDF and constrainGridVelocity.  The reference moves dynamic
 * objects before every sub-step after the first frame: call this then with their new
 * transformations and update_grid = 1.  Until a first update the boundary SDF is 0
 * everywhere (weights 1), as in the reference.  n = 0 restores the plain domain box. */
int bnn_flip_set_boundaries(bnn_flip* h, const bnn_boundary_object* objs, uint32_t n, int32_t update_grid);

/* ---- anisotropic kernels (surface reconstruction output) -------------------------- */

/* AnisotropicKernelGenerator<3, float> (Simulation/SurfaceReconstruction/
 * AniKernelGenerator.h:35-45,51; computeAniKernels AniKernelGenerator.cpp:53-101), as
 * PIC_Solver::saveFrameData runs it for "AniKernel" output (PIC_Solver.cpp:248-252):
 * per particle a smoothed centre and a 3x3 kernel matrix (column-major, glm::mat3 memory
 * order).  Neighbours are the other particles within kernel_ratio x particle_radius;
 * particles with fewer than neighbor_threshold of them get default_spray_size x identity. */
typedef struct bnn_aniso_params {
    float    particle_radius;     /* kernel radius = kernel_ratio x particle_radius */
    float    kernel_ratio;        /* 8 */
    float    default_spray_size;  /* 0.75 */
    float    position_blending;   /* 0.5 */
    float    axis_ratio;          /* 8 */
    uint32_t neighbor_threshold;  /* 25 */
} bnn_aniso_params;

typedef struct bnn_aniso_stats {
    float    grid_bmin[3];        /* the cell grid the particles were sorted on */
    float    grid_cell_size;
    int32_t  grid_dims[3];
    uint32_t sprays;              /* particles below the neighbour threshold */
    float    ms;                  /* device time of the kernel pass */
} bnn_aniso_stats;

/* The reference defaults for one particle radius */
int bnn_aniso_default_params(float particle_radius, bnn_aniso_params* out);
/* Over a device array of n points (AoS x,y,z); outputs are device arrays in input order:
 * centers n x 3, matrices n x 9.  The points are sorted on a cell grid of a quarter
 * kernel radius spanning their bounding box (reported in stats). */
int bnn_anisotropic_kernels(const float* pos_dev, uint32_t n, const bnn_aniso_params* params, float* centers_dev,
                            float* matrices_dev, bnn_aniso_stats* stats, void* stream);
/* Over the solver's current particles on its own grid; params NULL (or particle_radius
 * <= 0) takes the solver's particle radius (CellSize / RatioCellSizePRadius).  Outputs are
 * host arrays in the order the particles were given (as bnn_flip_get_particles). */
int bnn_flip_anisotropic_kernels(bnn_flip* h, const bnn_aniso_params* params, float* centers, float* matrices,
                                 bnn_aniso_stats* stats);

const char* bnn_version(void);
const char* bnn_last_error(void);
uint64_t bnn_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* BANANA_B200_H */
