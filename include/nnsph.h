/*
 * nnsph.h — C ABI of the B200 SPH step (libnnsph.so).
 *
 * The reference (chunleili/nonNewton) has no FFI: its step is driven through the
 * Python object API on the global `meta` (SPH/main.py:19-23) — `meta.pd` fields
 * (SPH/main.py:697-723), `meta.ns` (SPH/main.py:764-853) and the solver returned by
 * `build_solver()` (SPH/main.py:196-203). The Python package `nonnewton_b200`
 * keeps that object API and binds the entry points below with ctypes; each entry
 * point names the reference method it replaces.
 *
 * Conventions
 *  - Every function returns an int status: NN_OK (0) or a negative NN_ERR_*.
 *    No C++ exception crosses this boundary. nn_last_error() gives a message.
 *  - Pointers in nn_state are DEVICE pointers owned by the caller (torch tensors),
 *    laid out in particle-id order exactly like the reference's Taichi fields.
 *    Several scenes may be packed one after another (segmented arrays); scene s
 *    owns ids [start, start + n).
 *  - The context owns every scratch buffer (sorted working set, cell table,
 *    neighbour lists, solver vectors). They are allocated by nn_ctx_create /
 *    nn_set_scenes only; stepping allocates nothing.
 *  - All work is enqueued on the context's stream (nn_ctx_set_stream); calls on
 *    one context are not thread-safe, calls on distinct contexts are.
 */
#ifndef NNSPH_H
#define NNSPH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NNSPH_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define NN_OK                     0
#define NN_ERR_INVALID_ARG       -1
#define NN_ERR_CUDA              -2
#define NN_ERR_OOM               -3
#define NN_ERR_NEIGHBOR_OVERFLOW -4  /* a particle had more neighbours than max_neighbors */
#define NN_ERR_NOT_CONVERGED     -5  /* reported through nn_stats, not returned by nn_step */
#define NN_ERR_NAN               -6  /* non-finite value found in the state */
#define NN_ERR_STATE             -7  /* call out of order (e.g. no state bound) */
#define NN_ERR_CAPACITY          -8  /* more particles / scenes / cells than the context holds */

/* ---- materials, phases (SPH/main.py:26-39, 676) -------------------------- */
#define NN_FLUID 0
#define NN_SOLID 1
/* phase_id ranges used by the reference loader (SPH/main.py:633-661):
   fluid 0.., static 1000.., rigid 2000.., elastic 3000.. */
#define NN_PHASE_STATIC_BASE  1000
#define NN_PHASE_RIGID_BASE   2000
#define NN_PHASE_ELASTIC_BASE 3000

/* ---- feature flags of a scene ------------------------------------------ */
#define NN_F_SURFACE_TENSION   (1u << 0) /* SurfaceTension, SPH/main.py:1378-1414 */
#define NN_F_VISCOSITY         (1u << 1) /* explicit ViscosityModel, SPH/main.py:1417-1468 */
#define NN_F_NONNEWTON         (1u << 2) /* NonNewton strain rate + law, SPH/main.py:332-492 */
#define NN_F_IMPLICIT_VISCOSITY (1u << 3) /* Weiler 2018 CG (stub at SPH/main.py:1477-1513) */
#define NN_F_ELASTICITY        (1u << 4) /* Becker 2009, SPH/main.py:1182-1375 */
#define NN_F_DIVERGENCE        (1u << 5) /* divergence solve, SPH/main.py:1550 */
#define NN_F_CFL               (1u << 6) /* CFL time step (extension: the reference has none) */
#define NN_F_QUIRKS            (1u << 7) /* reproduce the reference's documented quirks */
#define NN_F_CARREAU_TEXTBOOK  (1u << 8) /* (1+(K g)^2)^((n-1)/2) instead of SPH/main.py:431-437 */
#define NN_F_RIGID             (1u << 9) /* RigidBodySolver shape matching, SPH/main.py:1099-1158 */

/* non-Newtonian laws, SPH/main.py:347-355 */
#define NN_NEWTONIAN        0
#define NN_POWER_LAW        1
#define NN_CROSS            2
#define NN_CASSON           3
#define NN_CARREAU          4
#define NN_BINGHAM          5
#define NN_HERSCHEL_BULKLEY 6

/* Parameters of one scene. Mirrors `Parameter` (SPH/main.py:594-621), the DFSPH
   settings (SPH/main.py:1523-1535), NonNewton.initParameters (SPH/main.py:357-368),
   Viscosity_Weiler2018 (SPH/main.py:1479-1485) and Elasticity (SPH/main.py:1188-1189).
   Set `size` to sizeof(nn_scene_params). */
typedef struct nn_scene_params {
  uint32_t size;
  uint32_t flags;                 /* NN_F_* */
  double domain_start[3];         /* domainStart */
  double domain_end[3];           /* domainEnd */
  double particle_radius;         /* particleRadius; h = 4 r (SPH/main.py:606) */
  double support_radius;          /* h */
  double volume0;                 /* 0.8 (2r)^3 (SPH/main.py:607) */
  double density0;                /* rho0 */
  double gravity[3];              /* gravitation */
  double dt;                      /* timeStepSize (initial step when NN_F_CFL) */
  double sticky_coeff;            /* 0.999 */
  double collision_coeff;         /* 0.5 */
  double padding;                 /* = h (SPH/main.py:615) */
  double viscosity;               /* explicit model coefficient (SPH/main.py:620-621) */
  double boundary_viscosity;      /* boundaryViscosity */
  double surface_tension;         /* 0.01 (SPH/main.py:1382) */
  double eps;                     /* m_eps 1e-5 (SPH/main.py:1526) */
  int32_t max_iterations_v;       /* maxIterationsV */
  int32_t max_iterations;         /* maxIterations */
  double max_error_v;             /* maxErrorV, percent */
  double max_error;               /* maxError, percent */
  /* non-Newtonian law */
  int32_t nonnewton_method;       /* NN_NEWTONIAN.. */
  int32_t pad0;
  double power_index, consistency_index, viscosity0, viscosity_inf;
  double critical_strain_rate, mu_c, yield_stress;
  /* implicit viscosity (Weiler 2018) */
  int32_t visco_max_iter;
  int32_t pad1;
  double visco_max_error;         /* relative residual of the CG */
  double visco_boundary;          /* viscosityBoundary (kinematic, times rho0) */
  /* elasticity */
  double youngs_modulus, poisson_ratio;
  /* CFL (extension) */
  double cfl_factor, cfl_min_dt, cfl_max_dt;
  /* rigid bodies: RigidBodySolver.substep runs coupling_interval times per step */
  int32_t coupling_interval;      /* couplingInterval (SPH/main.py:616, 930) */
  int32_t pad2;
} nn_scene_params;

/* One scene of a segmented particle array. */
typedef struct nn_scene_desc {
  uint32_t size;                  /* sizeof(nn_scene_desc) */
  int32_t start;                  /* first particle id of the scene */
  int32_t n;                      /* particles of the scene */
  int32_t n_fluid;                /* fluid particles (ids start .. start+n_fluid-1) */
  nn_scene_params params;
} nn_scene_desc;

/* Caller-owned device state, particle-id order (ParticleData, SPH/main.py:707-723).
   vec3 fields are [n][3] float32, scalars [n]. Optional fields may be NULL. */
typedef struct nn_state {
  uint32_t size;                  /* sizeof(nn_state) */
  int32_t n;
  float* x;                       /* [n,3] */
  float* x_0;                     /* [n,3] rest positions (elasticity) */
  float* v;                       /* [n,3] */
  float* acceleration;            /* [n,3] */
  float* volume;                  /* [n] */
  float* m;                       /* [n] */
  float* density;                 /* [n] */
  float* pressure;                /* [n] (unused by DFSPH, kept for the API) */
  float* dfsph_factor;            /* [n] */
  float* density_adv;             /* [n] */
  int32_t* material;              /* [n] NN_FLUID / NN_SOLID */
  int32_t* is_dynamic;            /* [n] */
  int32_t* phase_id;              /* [n] */
  /* optional outputs */
  float* strain_rate_norm;        /* [n] NonNewton.strainRateNorm */
  float* nonnewton_viscosity;     /* [n] NonNewton.nonNewtonViscosity */
  float* stress;                  /* [n,6] Elasticity.m_stress (Voigt 00,11,22,01,02,12) */
  float* rotations;               /* [n,9] Elasticity.m_rotations (row-major) */
} nn_state;

/* Per-scene statistics of the last step (SPH/main.py:1704, 1785 print these). */
typedef struct nn_stats {
  uint32_t size;
  int32_t status;                 /* NN_OK or NN_ERR_* seen by the device */
  int32_t iterations_v;           /* divergence solve: counter as printed at 1704 */
  int32_t iterations;             /* pressure solve: counter as printed at 1785 */
  int32_t cg_iterations;          /* implicit viscosity CG iterations */
  int32_t max_neighbors_seen;
  double avg_density_err_v;       /* last divergence error (FP64 reduction) */
  double avg_density_err;         /* last pressure error (FP64 reduction) */
  double cg_residual;             /* final relative CG residual */
  double dt;                      /* time step used by the last step */
  double max_density;             /* printed at SPH/main.py:1548 */
  int64_t steps;                  /* steps taken since nn_initialize */
  double max_avg_density_err;     /* largest avg_density_err at the end of any step since
                                     nn_set_scenes: the DFSPH error of every step, not only
                                     the last */
  int32_t nonpressure_folded;     /* 1 when the last nn_step took the fluid's non-pressure
                                     terms (compute_non_pressure_forces, 1557-1567) from the
                                     divergence loop's last density change instead of the
                                     force pass: every scene with fluid runs the divergence
                                     solve, none needs the explicit viscosity or quirk mode,
                                     and the loop ran as many bodies as in the step before */
} nn_stats;

typedef struct nn_ctx nn_ctx;

/* Passes of one step, each the sm_100a replacement of a reference method. */
enum nn_pass {
  NN_PASS_SEARCH = 0,                 /* NeighborhoodSearchSparse.run_search, 822-829 */
  NN_PASS_STATIC_BOUNDARY_VOLUME,     /* SPHBase.compute_static_boundary_volume, 1010-1019 */
  NN_PASS_MOVING_BOUNDARY_VOLUME,     /* SPHBase.compute_moving_boundary_volume, 1026-1035 */
  NN_PASS_CLEAR_ACCELERATIONS,        /* SPHBase.clear_accelerations, 942-951 */
  NN_PASS_DENSITIES,                  /* SPHBase.compute_densities, 975-984 */
  NN_PASS_DFSPH_FACTOR,               /* DFSPHSolver.compute_DFSPH_factor, 1569-1593 */
  NN_PASS_DIVERGENCE_SOLVE,           /* DFSPHSolver.divergence_solve, 1683-1713 */
  NN_PASS_NON_PRESSURE_FORCES,        /* DFSPHSolver.compute_non_pressure_forces, 1557-1567 */
  NN_PASS_NON_PRESSURE_ADVECT,        /* DFSPHSolver.non_pressure_advect, 1843-1848 */
  NN_PASS_PRESSURE_SOLVE,             /* DFSPHSolver.pressure_solve, 1762-1791 */
  NN_PASS_ELASTICITY,                 /* Elasticity.substep, 1241-1244 */
  NN_PASS_ADVECT,                     /* SPHBase.advect, 1086-1093 */
  NN_PASS_ENFORCE_BOUNDARY,           /* SPHBase.enforce_boundary_3D (FLUID then SOLID), 936-937 */
  NN_PASS_SUBSTEP,                    /* DFSPHSolver.substep, 1546-1555 */
  NN_PASS_RIGID,                      /* RigidBodySolver.substep (all bodies), 1108-1111 */
  NN_PASS_COUNT
};

/* step flags */
#define NN_STEP_SYNC_STATE  (1u << 0)  /* write the state back to nn_state after the last step */
#define NN_STEP_HOST_LOOP   (1u << 1)  /* drive solver loops from the host (no CUDA graph) */
#define NN_STEP_RESUME      (1u << 2)  /* continue from the state the last nn_step left resident on
                                          the device instead of reading nn_state again (for one launch
                                          per step without a write-back in between); NN_ERR_STATE if
                                          anything since that step changed the context or its state */

/* ---- context ------------------------------------------------------------
   Replaces: initialize() allocations (SPH/main.py:1870-1895) — ParticleData sizes,
   NeighborhoodSearchSparse.__init__ (SPH/main.py:766-791). */
int nn_ctx_create(int32_t max_particles, int32_t max_scenes, int32_t max_neighbors,
                  int64_t max_cells, nn_ctx** out);
int nn_ctx_destroy(nn_ctx* ctx);
int nn_ctx_set_stream(nn_ctx* ctx, void* cuda_stream);
const char* nn_last_error(const nn_ctx* ctx);
int nn_abi_version(void);
/* Bytes of the arithmetic type of this build: 4 for libnnsph.so (float, the product),
   8 for libnnsph64.so (the same kernels in double, the FP64 reference run). */
int nn_real_bytes(void);

/* Bind caller-owned state (meta.pd). */
int nn_bind_state(nn_ctx* ctx, const nn_state* state);
/* Describe the scenes packed in the bound state (segmented arrays). */
int nn_set_scenes(nn_ctx* ctx, int32_t nscenes, const nn_scene_desc* scenes);

/* solver.initialize() (SPH/main.py:957-960) and, for elastic phases, the
   Elasticity constructor (SPH/main.py:1186-1239): rest neighbourhoods and volumes. */
int nn_initialize(nn_ctx* ctx);

/* solver.step() (SPH/main.py:915-940), nsteps times. The state is read from
   nn_state at the start; with NN_STEP_SYNC_STATE it is written back at the end. */
int nn_step(nn_ctx* ctx, int32_t nsteps, uint32_t flags);

/* One sub-step method on the bound state (reads and writes nn_state). */
int nn_run_pass(nn_ctx* ctx, int32_t pass);

/* animate_particles (SPH/main.py:283-309), which SPHBase.step calls after advect: the
   next nn_step moves every particle of `scene`, static ones included, by
   displacement[3] (the sum of the scene's animeFile rows for the current frame),
   between advection and the boundary clamp; the step then clears it. Enqueued on the
   context's stream. */
int nn_set_animation(nn_ctx* ctx, int32_t scene, const float* displacement);

/* meta.ns.num_neighbors / meta.ns.neighbors (SPH/main.py:780-781) materialised in
   particle-id space, each row sorted by id and padded with -1. Device outputs:
   num_neighbors [n] int32, neighbors [n, width] int32. */
int nn_get_neighbors(nn_ctx* ctx, int32_t* num_neighbors, int32_t* neighbors, int32_t width);

/* Neighbour-list capacity per particle (the reference's fixed 60-wide list,
   SPH/main.py:777-781, which it overruns silently). Re-allocates the lists for
   `max_neighbors` entries (1..1024), clears NN_ERR_NEIGHBOR_OVERFLOW from every
   scene's status word and drops the captured step graphs; the next nn_step or
   nn_run_pass(NN_PASS_SEARCH) searches again. The caller re-runs the overflowed
   step from its own copy of the state before it (x and v are the only state a step
   carries over; the rest is recomputed or lives in the context). With elastic
   particles the rest lists are re-sized too and rebuilt by the next nn_initialize
   (from the rest positions x_0, so the rest state is the same); nn_step and
   nn_run_pass return NN_ERR_STATE until then. Synchronises the device. */
int nn_set_neighbor_cap(nn_ctx* ctx, int32_t max_neighbors);

/* The status word and the largest neighbour count of the last search of `scene`
   (nn_stats.status and .max_neighbors_seen), copied into host_out[0..1] in stream
   order without waiting: host_out should be pinned host memory. nn_status_wait
   blocks until the latest such copy has landed. Lets a caller check a step for
   overflow when it next needs to, not right after enqueueing it. */
int nn_status_async(nn_ctx* ctx, int32_t scene, int32_t* host_out);
int nn_status_wait(nn_ctx* ctx);

/* Statistics of scene `scene` (copies from the device; synchronises the stream). */
int nn_get_stats(nn_ctx* ctx, int32_t scene, nn_stats* out);

/* Statistics of scenes [first, first + count) in one device-to-host copy. */
int nn_get_stats_range(nn_ctx* ctx, int32_t first, int32_t count, nn_stats* out);

/* Kernel launches enqueued by this context since creation (for launch accounting). */
int64_t nn_launch_count(const nn_ctx* ctx);

/* Kernels of the step that nn_time_kernel can time on their own. */
enum nn_kernel_id {
  NN_K_PRESSURE_UPDATE = 0,   /* pressure_solve_iteration_kernel */
  NN_K_DENSITY_ADV,           /* compute_density_adv + FP64 error reduction */
  NN_K_DIVERGENCE_UPDATE,     /* divergence_solver_iteration_kernel */
  NN_K_DENSITY_CHANGE,        /* compute_density_change + FP64 error reduction */
  NN_K_DENSITY_FACTOR,        /* compute_densities + compute_DFSPH_factor (with the divergence
                                 solve's first density change when a scene runs it, as in the step) */
  NN_K_BUILD_LISTS,           /* store_neighbors */
  NN_K_CG_MATVEC,             /* implicit viscosity matrix-vector product */
  NN_K_NONPRESSURE,           /* surface tension + explicit viscosity */
  NN_K_DENSITY_CHANGE_NP,     /* compute_density_change with the non-pressure terms */
  NN_K_CG_SETUP,              /* implicit viscosity setup: A v, diagonal blocks, first residual */
  NN_K_COUNT
};
/* Average duration in ms of `reps` launches of one kernel on the current slots,
   timed with CUDA events on the context stream (measurement hook, no reference
   counterpart). Solver masks are set to "iterating" first, so the kernel does its
   full work; it mutates solver scratch and, for the update kernels, velocities.
   NN_K_BUILD_LISTS first re-sorts the slots by their current positions (one search),
   as a step's build sees them, and times the list build alone. */
int nn_time_kernel(nn_ctx* ctx, int32_t kernel, int32_t reps, float* ms_out);

/* Neighbour search that allocates no device memory. No counterpart in the
   reference: it exists for callers that cannot call cudaMalloc themselves or through
   this library (code that runs where allocation is forbidden or would deadlock, such
   as inside a host callback, or a host framework that owns every device allocation).
   Its scratch is a file-scope device array of NN_NOALLOC_SCRATCH_BYTES that every GPU
   loading the library holds until the process exits. Inputs and outputs are device
   buffers of the caller: x [n,3] float32; num_neighbors [n] and neighbors [n,width]
   int32. num_neighbors[i] is particle i's full neighbour count. Row i holds, sorted
   by id and padded with -1, the smallest ids among the neighbours the search stored,
   at most `width` of them: the same rows as nn_get_neighbors of a context whose
   neighbour cap is NN_NOALLOC_MAX_NEIGHBORS. The search stores every neighbour
   unless the count exceeds NN_NOALLOC_MAX_NEIGHBORS; such a count is this call's
   overflow signal, which the caller reads from num_neighbors without a host
   synchronisation: that row is incomplete (it is drawn from the first
   NN_NOALLOC_MAX_NEIGHBORS neighbours found, in cell order).
   The grid covers the domain of the scene (positions outside it are clamped into the
   border cells). Returns NN_ERR_CAPACITY beyond NN_NOALLOC_MAX_PARTICLES particles or
   when the domain needs more than NN_NOALLOC_MAX_CELLS cells of edge support_radius,
   and NN_ERR_CUDA, launching nothing, when a CUDA error from earlier work is pending.
   The first call in each CUDA context looks up the array's address in that context;
   make it before any stream capture. All calls share the array: calls that overlap on
   the GPU race. Work is enqueued on `cuda_stream` (NULL = legacy default stream). */
#define NN_NOALLOC_MAX_PARTICLES 16384
#define NN_NOALLOC_MAX_NEIGHBORS 64
#define NN_NOALLOC_MAX_CELLS     (1 << 18)
#define NN_NOALLOC_SCRATCH_BYTES (8u << 20)
int nn_neighbors_noalloc(const float* x, int32_t n, const double* domain_start, const double* domain_end,
                         double support_radius, int32_t width, int32_t* num_neighbors, int32_t* neighbors,
                         void* cuda_stream);

/* Autotuned launch shape: threads per block for the neighbour passes. 0 = default. */
int nn_set_block_size(nn_ctx* ctx, int32_t threads);

/* All tuning knobs at once (0 = default): threads per block of the neighbour passes
   (32..1024), neighbour chains each thread keeps in flight (1, 2 or 4 for every pass;
   0 = each pass its own measured depth, the default), and the cell
   factor f (cells of edge h / f searched with a (2f+1)-cell stencil; 1 or 2). A new
   cell factor takes effect at the next nn_set_scenes, which must follow. */
int nn_set_tuning(nn_ctx* ctx, int32_t block, int32_t unroll, int32_t cell_factor);

/* Tuning knob of the cell layout (0 = default, 1..4): x cells per cell edge. Cells
   are h/x_split long in x and h / cell_factor in y and z; the list build then tests
   the x cells within h of each particle's cell, (2 x_split + 1) / x_split of h in x
   instead of 3 h, in the same 9 contiguous rows. The neighbour sets do not depend on
   it. Takes effect at the next nn_set_scenes, which must follow. */
int nn_set_x_split(nn_ctx* ctx, int32_t x_split);

/* ---- Surface reconstruction (SPH/surf_recon/srtool.py, SRTool) ------------------
   The particle-to-mesh step after the simulation: fluid field on a vertex grid (an
   isotropic poly6 splat and the anisotropic Yu-Turk splat), one value-weighted
   Gaussian smoothing pass, dual contouring (one vertex per crossing cube from a
   clamped QEF around the mass point, two triangles per crossing edge), optional
   per-vertex normals. Replaces SRTool.dual_contouring (srtool.py:1264-1304) and
   export_mesh's data (1802-1838); the Python mirror is nonnewton_b200/surface.py.

   Vertex (x, y, z) of the grid lies at origin + (x, y, z) * voxel_size; linear index
   x + dims[0] * (y + dims[1] * z). Taichi's sparse fields are emulated: a block of
   NN_SR_BLOCK^3 vertices is active once any of its vertices is written, and the
   smoothing and contouring passes visit every vertex of the active blocks (what a
   struct-for over the reference's pointer/dense hierarchy visits). */
#define NN_SR_BLOCK 32
typedef struct nn_sr_params {
  int32_t size;                 /* sizeof(nn_sr_params) */
  int32_t dims[3];              /* vertices per axis */
  double origin[3];             /* bounding_box_extent[0] */
  double voxel_size;            /* SRTool(voxel_size) */
  double particle_radius;       /* SRTool(particle_radius): splat volume 4/3 pi r^3 */
  double smooth_radius;         /* dual_contouring(smooth_radius) */
  double isolevel;              /* dual_contouring(isolevel) */
  int32_t use_smooth_field;     /* dual_contouring(use_smooth_fluid_field) */
  int32_t smooth_iterations;    /* smooth_sdf(iteration), 1 in the reference */
  int32_t smooth_cells;         /* smooth_sdf(radius), 1 in the reference */
  int32_t record_normals;       /* SRTool(record_normals) */
} nn_sr_params;

typedef struct nn_sr_ctx nn_sr_ctx;

/* Capacities: particles, vertex grid cells, mesh vertices and triangle indices
   (SRTool(max_num_particles, max_num_vertices, max_num_indices)); options
   NN_SR_VELOCITY (SRTool(record_velocity=True)) adds the vertex velocity field. */
#define NN_SR_VELOCITY 1
int nn_sr_create(int32_t max_particles, int64_t max_cells, int32_t max_vertices, int32_t max_indices,
                 int32_t options, nn_sr_ctx** out);
int nn_sr_destroy(nn_sr_ctx* ctx);
const char* nn_sr_last_error(const nn_sr_ctx* ctx);

/* SRTool.dual_contouring for `n` particles at device positions pos [n,3] f32 (and,
   with velocities vel [n,3] f32 on a context created with NN_SR_VELOCITY, the
   velocity splat of srtool.py:1159-1190 and the mesh velocities of
   process_velocity, 1351-1381; vel NULL records none), enqueued on `cuda_stream`;
   the mesh stays in the context. NN_ERR_CAPACITY when the grid,
   the mesh or a voxel's particle list (NN_SR_MAX_PER_VOXEL, the reference's 64) is
   too small; NN_ERR_INVALID_ARG for particles outside the grid. Synchronises the
   stream once (to read the mesh sizes). */
#define NN_SR_MAX_PER_VOXEL 64
int nn_sr_dual_contouring(nn_sr_ctx* ctx, const nn_sr_params* params, const float* pos, const float* vel,
                          int32_t n, void* cuda_stream);

/* The same pipeline with marching cubes in place of dual contouring
   (SRTool.marching_cube_impl, srtool.py:1765-1800, which has no caller in the
   reference: its public entry is dual_contouring alone). Each cube emits one vertex
   per crossing edge, in edge order, as the reference does (vertices are not shared
   between cubes). The triangles come from this library's own case table, derived
   from the corner states by a face walk (in-corners kept separate on ambiguous
   faces), not from the reference's 256-case table; the surface is closed. Same
   arguments, errors and synchronisation as nn_sr_dual_contouring. */
int nn_sr_marching_cubes(nn_sr_ctx* ctx, const nn_sr_params* params, const float* pos, const float* vel,
                         int32_t n, void* cuda_stream);

/* The mesh of the last call: counts, and copies into caller device buffers when
   non-NULL: vertices [num_vertices,3] f32, indices [num_indices] i32 (triangles),
   normals [num_vertices,3] f32 (when record_normals was set), velocities
   [num_vertices,3] f32 (when velocities were given). Vertices are numbered
   by the linear index of their cube (marching cubes: then by edge), triangles
   ordered by cube and then by edge (dual contouring: the x, y, z edges of the cube's
   first corner; marching cubes: the case table's order). */
int nn_sr_get_mesh(nn_sr_ctx* ctx, int32_t* num_vertices, int32_t* num_indices, float* vertices,
                   int32_t* indices, float* normals, float* velocities, void* cuda_stream);

/* Stage outputs for parity checks (device buffers, each optional): the field [cells]
   f32, the active-block flags [blocks] u8 (blocks of NN_SR_BLOCK^3 in x-fastest
   order), the anisotropic kernels G [n,9] and centres x_bar [n,3] f32, and the
   smoothing's standard deviation (host double). `stage` 0 = after the splats,
   1 = after smoothing (the field the contouring reads). */
int nn_sr_get_stage(nn_sr_ctx* ctx, int32_t stage, float* field, uint8_t* active_blocks, float* G, float* xbar,
                    double* sd, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* NNSPH_H */
