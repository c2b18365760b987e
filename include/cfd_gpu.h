/* cfd_gpu.h - C ABI of the B200 steady SIMPLE solver (laminar and k-omega SST)
 * on structured C-grids.
 *
 * This is the boundary a host program binds to. It replaces the internals of
 * the reference's C++ class cfd::solver::SimpleSolver and its TurbulenceModel
 * plug-in (include/cfd/solver/SimpleSolver.hpp:159-274,
 * include/cfd/solver/TurbulenceModel.hpp:155-206, include/cfd/solver/KOmegaSST.hpp:174-257).
 * Plain pointers and sizes only. Every array is FP64 and in the reference's
 * own ordering: cells c = j*cellsI + i (Mesh::cellIndex, Mesh.hpp:168), faces
 * j-faces first then i-faces (Mesh.cpp:138-156), Vec2 arrays as (x, y) pairs.
 *
 * Errors: every entry point returns a cfd_status. Non-zero codes map one to
 * one onto cfd::ErrorCode (include/cfd/core/Error.hpp:37-46) plus one; the
 * message of the last failure on the calling thread is cfd_last_error().
 * As in the reference, a diverging solve is not an error: it shows up as
 * non-finite residuals in the monitor (src/app/SolverWorker.cpp:169-181).
 *
 * Threading: a handle is single-owner, like SimpleSolver. Calls on one handle
 * come from one host thread at a time. A handle owns one CUDA stream.
 */
#ifndef CFD_GPU_H
#define CFD_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int cfd_status;
enum {
  CFD_OK = 0,
  CFD_INVALID_ARGUMENT = 1, /* ErrorCode::InvalidArgument */
  CFD_OUT_OF_RANGE = 2,
  CFD_NOT_FOUND = 3,
  CFD_IO_FAILURE = 4,
  CFD_NOT_IMPLEMENTED = 5,
  CFD_INITIALIZATION_FAILURE = 6, /* also: CUDA device or allocation failure */
  CFD_NUMERICAL_FAILURE = 7,
  CFD_INTERNAL = 8 /* also: a bounded wait between a solve's CTAs gave up
                     (cfd_last_error says which); that launch's results are
                     not valid, and the device stays usable */
};

typedef struct cfd_solver_t* cfd_handle;

/* flow::BoundaryKind (include/cfd/flow/BoundaryConditions.hpp:34-72). */
enum { CFD_BC_INTERNAL = 0, CFD_BC_INLET = 1, CFD_BC_OUTLET = 2, CFD_BC_FARFIELD = 3,
       CFD_BC_NOSLIP_WALL = 4 };
/* mesh::BoundaryType (include/cfd/mesh/Mesh.hpp:42-48). */
enum { CFD_FACE_INTERIOR = 0, CFD_FACE_WALL = 1, CFD_FACE_FARFIELD = 2, CFD_FACE_OUTLET = 3,
       CFD_FACE_WAKECUT = 4 };

/* A structured face-based mesh, as cfd::mesh::Mesh exposes it (Mesh.hpp:121-190).
 * The arrays are read during cfd_gpu_create only and may be freed after it. */
typedef struct cfd_mesh_desc {
  int nodes_i, nodes_j;          /* Mesh::nodesI/nodesJ; cells = (ni-1)*(nj-1) */
  int cell_count, face_count;
  const double* cell_centroids;  /* 2*cells */
  const double* cell_areas;      /* cells */
  const double* face_centres;    /* 2*faces */
  const double* face_normals;    /* 2*faces, unit, out of the owner */
  const double* face_areas;      /* faces */
  const int* face_owner;         /* faces */
  const int* face_neighbour;     /* faces, -1 on a boundary */
  const int* face_boundary;      /* faces, CFD_FACE_* */
  const int* face_partner;       /* faces, wake-cut partner face or -1 */
  const double* nodes;           /* 2 * nodes_i * nodes_j, row-major (j, i); may be NULL
                                    (then cfd_gpu_forces is unavailable) */
} cfd_mesh_desc;

/* flow::FaceCondition per face (BoundaryConditions.hpp:101-107). */
typedef struct cfd_face_bc {
  const int* kind;         /* faces, CFD_BC_* */
  const double* velocity;  /* 2*faces */
  const double* pressure;  /* faces */
} cfd_face_bc;

/* solver::SimpleSettings (SimpleSolver.hpp:86-132) plus the precision form. */
typedef struct cfd_settings {
  double velocity_relaxation;      /* 0.5 */
  double pressure_relaxation;      /* 0.2 */
  int momentum_sweeps;             /* 3 */
  int pressure_iterations;         /* 200 */
  double pressure_tolerance;       /* 0.01 */
  int scheme;                      /* 0 upwind, 1 second-order upwind */
  double turbulence_relaxation;    /* 0.5 */
  double inflow_intensity;         /* 0.001 (TurbulenceInflow) */
  double inflow_viscosity_ratio;   /* 1.0 */
  double inflow_length_scale;      /* 0.0 */
  int non_orthogonal_correctors;   /* 1 */
  double non_orthogonal_blend;     /* 1.0 */
  int precision;                   /* 0 plain FP64 (the drop-in), 1 mixed FP32/FP64 */
  int inner_iterations;            /* mixed form: cap on the multigrid-CG iterations of one
                                      pressure correction (0: pressure_iterations); 16 */
} cfd_settings;

/* solver::SolverMonitor (SimpleSolver.hpp:135-154), flattened; plus the
 * model's maxWallYPlus (TurbulenceModel.hpp:205). */
typedef struct cfd_monitor {
  double continuity, momentum_x, momentum_y;
  double mass_imbalance, max_divergence;
  int pressure_iterations;
  int pad_;
  double turbulence_first, turbulence_second;
  double min_energy, max_energy, min_dissipation, max_dissipation;
  double min_eddy_viscosity, max_eddy_viscosity;
  double max_eddy_viscosity_ratio;
  double max_wall_yplus;
} cfd_monitor;

/* Fields readable with cfd_gpu_read_field. (F) marks a per-face array in
 * reference face order; (2N) a Vec2 per cell; the rest are per cell. */
enum {
  CFD_FIELD_U = 0, CFD_FIELD_V, CFD_FIELD_P, CFD_FIELD_RHO, CFD_FIELD_MU_EFF,
  CFD_FIELD_MASS_FLUX /*F*/, CFD_FIELD_DIVERGENCE, CFD_FIELD_MU_MOLECULAR,
  CFD_FIELD_GRAD_U /*2N*/, CFD_FIELD_GRAD_V /*2N*/, CFD_FIELD_GRAD_P /*2N*/,
  CFD_FIELD_MOM_DIAG, CFD_FIELD_MOM_SOURCE_U, CFD_FIELD_MOM_SOURCE_V,
  CFD_FIELD_MOM_UPPER /*F*/, CFD_FIELD_MOM_LOWER /*F*/, CFD_FIELD_MOMENTUM_DIAGONAL,
  CFD_FIELD_P_DIAG, CFD_FIELD_P_SOURCE, CFD_FIELD_P_UPPER /*F*/, CFD_FIELD_NET_FLUX,
  CFD_FIELD_P_CORRECTION,
  CFD_FIELD_K, CFD_FIELD_OMEGA, CFD_FIELD_MUT, CFD_FIELD_WALL_DISTANCE, CFD_FIELD_STRAIN,
  CFD_FIELD_F1, CFD_FIELD_F2, CFD_FIELD_CROSS_DIFFUSION, CFD_FIELD_PRODUCTION,
  CFD_FIELD_GRAD_K /*2N*/, CFD_FIELD_GRAD_OMEGA /*2N*/,
  CFD_FIELD_T_DIAG_K, CFD_FIELD_T_SOURCE_K, CFD_FIELD_T_DIAG_W, CFD_FIELD_T_SOURCE_W,
  CFD_FIELD_COUNT
};

/* Stop points for cfd_gpu_iterate_partial: the iteration returns right after
 * the named stage. The stage list follows SimpleSolver::iterate()
 * (SimpleSolver.cpp:662-794) and KOmegaSST::update (KOmegaSST.cpp:531-548). */
enum {
  CFD_STAGE_GRADIENTS = 0,        /* interpolateFaceValues + computeGradients */
  CFD_STAGE_MOMENTUM_ASSEMBLY,    /* assembleMomentum + applyRelaxation, u and v */
  CFD_STAGE_MOMENTUM_SOLVE,       /* Gauss-Seidel sweeps */
  CFD_STAGE_RHIE_CHOW,            /* computeRhieChowFluxes */
  CFD_STAGE_PRESSURE_ASSEMBLY,    /* assemblePressureCorrection */
  CFD_STAGE_PRESSURE_SOLVE,       /* conjugateGradient */
  CFD_STAGE_CORRECT,              /* correct */
  CFD_STAGE_SST_BLENDING,         /* computeStrain + computeBlending + production */
  CFD_STAGE_SST_ASSEMBLY,         /* k and omega systems, relaxed */
  CFD_STAGE_SST_SOLVE,            /* Gauss-Seidel sweeps (floors not yet applied) */
  CFD_STAGE_END                   /* the whole iteration */
};

/* SimpleSolver::create (SimpleSolver.cpp:30-80): validates, copies the mesh
 * metrics and face conditions to the device, precomputes face geometry.
 * settings may be NULL for the reference defaults. */
cfd_status cfd_gpu_create(const cfd_mesh_desc* mesh, const cfd_face_bc* conditions,
                          const cfd_settings* settings, cfd_handle* out);

/* SimpleSolver::setTurbulenceModel (SimpleSolver.cpp:212-230).
 * model: 0 = none (nullptr), 1 = LaminarModel, 2 = KOmegaSST. */
cfd_status cfd_gpu_set_turbulence(cfd_handle h, int model);

/* SimpleSolver::initialise (SimpleSolver.cpp:133-210); arrays per cell. */
cfd_status cfd_gpu_initialise(cfd_handle h, const double* u, const double* v, const double* p,
                              const double* rho, const double* mu);

/* n x SimpleSolver::iterate() (SimpleSolver.cpp:662-794) in one device launch.
 * last (may be NULL) gets the final iteration's monitor, history (may be
 * NULL) n monitors. Returns after the device has finished. */
cfd_status cfd_gpu_iterate(cfd_handle h, int n, cfd_monitor* last, cfd_monitor* history);

/* Iterate until worst() of the residuals < tol (SolverWorker.cpp:182-185),
 * a non-finite residual, or cap iterations. Residuals are checked on the
 * device every iteration; *taken gets the iterations run. */
cfd_status cfd_gpu_converge(cfd_handle h, int cap, double tol, int* taken, cfd_monitor* last);

/* One iteration stopped right after `stage` (CFD_STAGE_*): for stage-by-stage
 * parity checks. The state afterwards is partial; re-load or re-initialise. */
cfd_status cfd_gpu_iterate_partial(cfd_handle h, int stage, cfd_monitor* last);

/* SimpleSolver::field()/massFlux()/divergence() and friends: copy one device
 * field to host memory in reference order (see CFD_FIELD_*). */
cfd_status cfd_gpu_read_field(cfd_handle h, int which, double* out);

/* Surface data and forces (post::extractSurface + post::integrateForces,
 * src/post/SurfaceData.cpp:101-348, src/post/Forces.cpp:23-130), computed on
 * the device in FP64 from the current field: wall Cp, the two-point wall
 * shear, and the force and quarter-chord moment coefficients in wind axes. */
typedef struct cfd_forces {
  double lift_coefficient, drag_coefficient, moment_coefficient;
  double pressure_drag_coefficient, friction_drag_coefficient;
  double lift, drag, pitching_moment;
  double stagnation_chord_fraction;
  int stations;     /* wall stations: upper (leading edge -> trailing edge) then lower */
  int leading_edge; /* number of lower-surface stations */
  /* findSeparation (SurfaceData.cpp:179-203): x/c where the wall shear first
   * turns negative walking away from the leading edge, or -1 */
  double separation_upper_chord_fraction, separation_lower_chord_fraction;
} cfd_forces;

/* speed, alpha_deg, density and reference_pressure describe the freestream
 * (FreestreamConditions); chord the section. cp and cf (may be NULL) receive
 * one value per station in the order of `stations`. Needs mesh nodes. */
cfd_status cfd_gpu_forces(cfd_handle h, double speed, double alpha_deg, double density,
                          double reference_pressure, double chord, cfd_forces* out, double* cp,
                          double* cf);

/* post::StreamlineOptions (include/cfd/post/Streamlines.hpp:16-33). */
typedef struct cfd_streamline_options {
  int max_steps;           /* RK4 steps in each direction, 4000 */
  double step_fraction;    /* step length / sqrt(cell area), 0.35 */
  double stall_fraction;   /* stop below this fraction of the reference speed, 1e-4 */
  double reference_speed;  /* 1.0 */
  int trace_backwards;     /* 1: trace upstream from each seed too */
} cfd_streamline_options;
void cfd_default_streamline_options(cfd_streamline_options* out);

/* post::traceStreamlines (src/post/Streamlines.cpp:80-197) through the
 * solver's current velocity field, on the device (one thread per seed and
 * direction; RK4 with the reference's cell location, across the wake cut).
 * seeds: host (x, y) pairs; options may be NULL for the defaults. lengths
 * (host, count ints) gets each seed's point count, 0 where the reference
 * drops the seed (outside the domain, or fewer than 4 points); points (host)
 * the curves one after another, upstream end first, (x, y) per point, when
 * `capacity` points fit (else CFD_OUT_OF_RANGE; points may be NULL to ask);
 * *total (may be NULL) the points needed. Needs mesh nodes. */
cfd_status cfd_gpu_streamlines(cfd_handle h, const double* seeds, int count,
                               const cfd_streamline_options* options, int* lengths, double* points,
                               long long capacity, long long* total);

/* Overwrite the solver state (a warm start, or a state to continue from):
 * u, v, p per cell; mass_flux per face (may be NULL to keep); k, omega, mut
 * per cell (NULL unless SST); mu_eff per cell (may be NULL). */
cfd_status cfd_gpu_load_state(cfd_handle h, const double* u, const double* v, const double* p,
                              const double* mass_flux, const double* k, const double* omega,
                              const double* mut, const double* mu_eff);

/* SimpleSolver::setSettings (SimpleSolver.hpp:194). */
cfd_status cfd_gpu_set_settings(cfd_handle h, const cfd_settings* settings);
/* The reference defaults of SimpleSettings. */
void cfd_default_settings(cfd_settings* out);

/* Sizes: {cellsI, cellsJ, cells, faces}. */
cfd_status cfd_gpu_dims(cfd_handle h, int* out4);
/* SST freestream values {kInflow, omegaInflow}; referenceMassFlow. */
cfd_status cfd_gpu_scalars(cfd_handle h, double* out3);

cfd_status cfd_gpu_destroy(cfd_handle h);

const char* cfd_last_error(void);

/* Make `device` the CUDA device this thread's later calls create solves on
 * (one process per GPU: each rank selects its own). No reference
 * counterpart: the reference has no device. */
cfd_status cfd_set_device(int device);

/* ---- the pressure-correction CG as a device primitive -----------------------
 * A symmetric five-point system on a structured block, in the layout of the
 * reference's LinearSystem (LinearSystem.hpp:29-71): diag and source per cell,
 * one off-diagonal per face in reference face order (upper; the solve uses it
 * for both rows, so lower must equal it). A j = 0 face of column i couples to
 * across_j0[i] when that is >= 0 (the wake cut; Mesh.cpp:78-87). Every
 * pointer is device memory. */
typedef struct cfd_cg_system {
  int cells_i, cells_j;
  const double* diag;     /* cells */
  const double* upper;    /* faces */
  const double* source;   /* cells */
  const int* across_j0;   /* cells_i entries, or NULL for none */
} cfd_cg_system;

/* conjugateGradient (LinearSystem.hpp:315-316, LinearSystem.cpp:118-210) on
 * the device: x (device, cells) is the starting guess in and the solution
 * out; report (host, 4 doubles, may be NULL) = {iterations, initial residual,
 * final residual, converged}; both residuals are L1 norms as in the
 * reference. Allocates its scratch (two coefficient arrays, seven vectors) for
 * the call. stream: a cudaStream_t, or NULL for the legacy default stream.
 * Returns after the solve has finished. A wake-map entry >= cells_i*cells_j
 * is refused with CFD_INVALID_ARGUMENT, and x is then left unchanged. */
cfd_status cfd_cg_solve(const cfd_cg_system* system, double* x, double tolerance,
                        int max_iterations, double* report, void* stream);

/* The same solve for callers that cannot allocate device memory: a host
 * application whose memory manager owns the whole device, or a loop that must
 * not block on cudaFree's device-wide synchronisation. No counterpart in the
 * reference. It calls no cudaMalloc, cudaFree or allocating library routine:
 * its scratch is a fixed device array inside this library (4.75 MiB per GPU
 * that loads it, kept until exit), so blocks are limited to
 * (cells_i+1)*(cells_j+1) <= 65536 nodes; larger ones return
 * CFD_OUT_OF_RANGE. All calls on a device share that array; calls that
 * overlap on the GPU race and must be serialised by the caller. The first call
 * on each device resolves the array's address (cudaGetSymbolAddress, with
 * that device current); make that first call before any stream capture
 * begins. Like cfd_cg_solve, every call returns after its solve has finished.
 * Results equal cfd_cg_solve's. */
cfd_status cfd_cg_solve_noalloc(const cfd_cg_system* system, double* x, double tolerance,
                                int max_iterations, double* report, void* stream);

/* ---- the solve engine: continuous batching of many solves ------------------
 * A request loop over one GPU (no counterpart in the reference, which runs one
 * solve per worker thread; its polar sweep runs points one after another,
 * src/post/Polar.cpp:86-124). Requests queue until their device memory fits
 * the budget; admitted solves stay resident, and every engine step advances
 * all of them together (one launch per cluster shape, one thread-block
 * cluster per solve, `chunk` iterations). A solve retires when its residuals
 * pass the tolerance (converged), go non-finite (diverged: restarted once
 * from the freestream, as the reference's RetryCold) or reach its iteration
 * cap; its forces are integrated on the device and its memory freed for the
 * queue. */
typedef struct cfd_engine_t* cfd_engine;

typedef struct cfd_request {
  char designation[8];           /* NACA four digits, e.g. "2412" */
  int grid_surface_points, grid_wake_points, grid_normal_points;
  double grid_first_layer_height;
  double grid_upstream_chords, grid_downstream_chords, grid_vertical_chords;
  double alpha_deg, reynolds, speed, density;
  int model;                     /* 0 laminar, 2 k-omega SST */
  double tolerance;              /* worst() of the residuals */
  int max_iterations;
  cfd_settings settings;
} cfd_request;

/* Outcomes (pointStatus, Polar.cpp:79-84), plus a request that never started
 * because its solver could not be built or initialised (cfd_result.error
 * then holds the library's status code). */
enum { CFD_SOLVE_CONVERGED = 0, CFD_SOLVE_ITERATION_LIMIT = 1, CFD_SOLVE_DIVERGED = 2,
       CFD_SOLVE_FAILED = 3 };

typedef struct cfd_result {
  int id;
  int status;                    /* CFD_SOLVE_* (pointStatus, Polar.cpp:79-84) */
  int iterations;
  int retried_cold;
  int cells;
  int cluster_size;              /* CTAs per solve the engine ran it with */
  double continuity, momentum_x, momentum_y;
  double lift_coefficient, drag_coefficient, moment_coefficient;
  double pressure_drag_coefficient, friction_drag_coefficient;
  double submitted_s, started_s, finished_s;  /* engine clock, seconds */
  double separation_upper_chord_fraction, separation_lower_chord_fraction;  /* or -1 */
  double alpha_deg;              /* the incidence solved (a sweep's points get theirs here) */
  int continued;                 /* 1: started from the previous sweep point's u and p */
  int error;                     /* CFD_SOLVE_FAILED: why the solve could not start */
  double mesh_s;                 /* seconds the request's C-grid took to generate (0: cached) */
} cfd_result;

/* memory_budget_bytes: device memory the resident solves may hold (0: 80 %
 * of the free memory). chunk: iterations per engine step. */
cfd_status cfd_engine_create(unsigned long long memory_budget_bytes, int chunk, cfd_engine* out);
/* Queue a request; *id identifies its result. Its C-grid is generated on the
 * engine's host worker threads (or taken from the engine's cache), and the
 * request is admitted once the grid is ready; a grid the generator refuses
 * makes the request fail (CFD_SOLVE_FAILED, error = the generator's code). */
cfd_status cfd_engine_submit(cfd_engine e, const cfd_request* request, int* id);
/* One step: wait for the chunk the previous step launched (setting up the
 * requests that can join meanwhile), retire finished solves, admit what fits
 * the memory freed, and launch the next `chunk` iterations of every resident
 * solve, returning while they run. active/queued (may be NULL) report the
 * resident solves (those running) and the queued requests afterwards; keep
 * stepping while either is non-zero. */
cfd_status cfd_engine_step(cfd_engine e, int* active, int* queued);
/* post::sweepAngles (src/post/Polar.cpp:36-77): the angles from start to end
 * (a descending sweep when end < start) in steps of |step|, the point count
 * rounded when the step divides the range, at most 400 points; the
 * reference's refusals (non-finite bounds, step <= 0, an empty or too long
 * sweep) return CFD_INVALID_ARGUMENT with its message. out may be NULL to
 * query *count. */
cfd_status cfd_sweep_angles(double start, double end, double step, double* out, int capacity,
                            int* count);
/* A polar sweep as the reference runs one (startPolarSweep / updatePolar,
 * src/app/Panels.cpp:1601-1797): one solve of `base` per angle of
 * cfd_sweep_angles(start, end, step), each started when the previous point
 * has retired. continued = 1 starts every point after the first from the
 * previous point's u and p (k and omega from their freestream and wall seeds,
 * as Panels.cpp:1145-1156 rebuilds the solver), except after a point that
 * diverged even on its cold retry. The points get the ids first_id ..
 * first_id + count - 1 in sweep order; many sweeps (and single requests)
 * share the GPU. */
cfd_status cfd_engine_submit_sweep(cfd_engine e, const cfd_request* base, double start, double end,
                                   double step, int continued, int* first_id, int* count);
/* Move up to `capacity` finished results into `out`; *count gets how many. */
cfd_status cfd_engine_results(cfd_engine e, cfd_result* out, int capacity, int* count);
/* Launch shapes of the solves the engine starts from now on: 0 (default) by
 * grid size, as a lone solve would run (the mixed form on clusters of at most
 * 8 CTAs), which suits a few dozen concurrent solves (a polar); 1 tuned per
 * grid for a saturated GPU (serving streams): the
 * cluster size with the most solve-iterations per second when as many solves
 * as fit run at once, measured once per grid and kept for the process. Either
 * way a grid always runs with the same shape, so results do not depend on
 * what else is in the engine. */
cfd_status cfd_engine_set_shape_policy(cfd_engine e, int policy);

/* Pressure coefficient at every wall station of a finished solve (upper
 * surface from the leading edge, then the lower), as cfd_gpu_forces returns
 * it (post::extractSurface, SurfaceData.cpp:101-348). cp = NULL only stores
 * the station count; otherwise capacity must hold it, and the data are
 * released after the copy. Diverged solves have none. */
cfd_status cfd_engine_surface(cfd_engine e, int id, double* cp, int capacity, int* stations);
/* Seconds on the engine clock (for submit-time bookkeeping by callers). */
double cfd_engine_clock(cfd_engine e);
cfd_status cfd_engine_destroy(cfd_engine e);

/* ---- batches: many solves in one launch ------------------------------------
 * A batch is a descriptor table over existing handles (each keeps its own
 * device state). One launch runs every solve of the table, one thread-block
 * cluster each, so uneven sizes, angles and sections share the GPU. Each
 * solve keeps its own cluster size (set at create or by CFD_CLUSTER_SIZE);
 * solves of different sizes run as one launch per size, side by side on
 * streams forked from and joined back to the caller's, so small clusters can
 * fill SMs that wide ones leave idle. The reference runs one solve per worker
 * thread (src/app/SolverWorker.cpp); this has no counterpart there. The
 * handles must outlive the batch and must not be iterated on their own while
 * a batch launch is in flight. */
typedef struct cfd_batch_t* cfd_batch;

cfd_status cfd_batch_create(const cfd_handle* solvers, int count, cfd_batch* out);
/* n iterations of every solve; tol >= 0 lets each solve stop on its own at
 * convergence or divergence. taken (may be NULL) gets count iteration counts,
 * last (may be NULL) count monitors. Synchronous. */
cfd_status cfd_batch_iterate(cfd_batch b, int n, double tol, int* taken, cfd_monitor* last);
/* Enqueue n iterations on `stream` (a cudaStream_t; NULL means the batch's
 * own stream, not the legacy default stream) and return without waiting;
 * for callers that time with events on their own stream. */
cfd_status cfd_batch_launch(cfd_batch b, int n, void* stream);
/* The same launch replayed from a CUDA graph: the n-iteration launch is
 * captured on the batch's stream the first time (and again when n changes)
 * and then launched as a graph on `stream` (NULL: the batch's stream). The
 * results are those of cfd_batch_launch. */
cfd_status cfd_batch_graph_launch(cfd_batch b, int n, void* stream);
/* Monitors of the last launch (count entries); synchronises first. */
cfd_status cfd_batch_monitors(cfd_batch b, int* taken, cfd_monitor* last);
/* Cluster size (CTAs per solve) and threads per CTA of the batch's largest
 * group of solves. */
cfd_status cfd_batch_shape(cfd_batch b, int* cluster_size, int* threads);
cfd_status cfd_batch_destroy(cfd_batch b);

#ifdef __cplusplus
}
#endif
#endif /* CFD_GPU_H */
