/*
 * diff_smoke.h -- C ABI of the B200 smoke solver (sm_100a).
 *
 * Two levels of entry points:
 *
 *   1. Operator level, one function per launcher of the reference's kernel
 *      ABI (solvers/smoke/operators.h:40-72).  Argument order and meaning
 *      follow the reference; views become plain pointer triples and
 *      std::uint32_t iteration counts become an XsPressureSolve block.
 *   2. Step level (xs_smoke_*), the composition of Model::forward_step,
 *      jvp_step and vjp_step (solvers/smoke/model.cpp:341-389) over a caller
 *      owned workspace, plus domain construction (model.cpp:32-183).
 *
 * Every function returns an XsStatus and, except xs_warm_start_create, never
 * allocates device memory: the caller owns every buffer, sized with the
 * *_workspace_bytes queries.  All
 * work is enqueued on the given stream; nothing synchronises unless stated.
 * Pointers to cell masks may be NULL, meaning "no colliders" (every cell is
 * fluid); kernels then take the mask-free path.
 *
 * Layout (solvers/smoke/operators.cu:36-47): cell (x,y,z) lives at
 * x + nx*(y + ny*z); face component a has extent +1 along axis a.  State and
 * tangent fields are FP32, adjoint fields FP64 (cuda_types.h:81-129).
 */
#ifndef DIFF_SMOKE_H
#define DIFF_SMOKE_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum XsStatus {
    XS_OK = 0,
    XS_CUDA_ERROR = 1,          /* a CUDA call failed; xs_last_cuda_error() holds its code */
    XS_NOT_CONVERGED = 2,       /* a pressure solve hit its iteration cap */
    XS_NUMERICAL_ERROR = 3,     /* NaN/Inf or breakdown inside a solve */
    XS_INVALID_ARGUMENT = 4,    /* sizes, pointers or modes rejected before launch */
    XS_TIMEOUT = 5,             /* a bounded device-side wait gave up */
    XS_CAPACITY_EXCEEDED = 6    /* the grid is larger than a fixed-size entry point admits */
} XsStatus;

/* cuda_types.h:13-19 */
typedef struct XsGrid {
    uint32_t nx, ny, nz;
    float cell_size;
    float time_step;
} XsGrid;

/* cuda_types.h:21-24; modes use ScalarBoundaryMode {fixed_value=0,
 * zero_gradient=1, periodic=2} (data.ixx:14-18), faces x-,x+,y-,y+,z-,z+ */
typedef struct XsScalarBoundary {
    uint32_t modes[6];
    float values[6];
} XsScalarBoundary;

/* cuda_types.h:26-29; modes use VelocityBoundaryMode {fixed_value=0,
 * zero_gradient=1, normal_fixed_tangent_zero_gradient=2, periodic=3}
 * (data.ixx:20-25); values[3*face + component] */
typedef struct XsVelocityBoundary {
    uint32_t modes[6];
    float values[18];
} XsVelocityBoundary;

/* CenteredVectorView / StaggeredVectorView (cuda_types.h:45-79) */
typedef struct XsVector { float* x; float* y; float* z; } XsVector;
typedef struct XsVec3 { float x, y, z; } XsVec3;
/* CenteredVectorAdjointView / StaggeredVectorAdjointView (:95-129) */
typedef struct XsAdjointVector { double* x; double* y; double* z; } XsAdjointVector;

/* Inflow sphere (no reference counterpart): cells whose centre lies inside
 * are set to (density, temperature) by the source operator.  Inflow arrays
 * are HOST arrays of at most XS_MAX_INFLOWS entries; they travel to the
 * device as kernel parameters. */
#define XS_MAX_INFLOWS 8
typedef struct XsInflow {
    float center[3];
    float radius;
    float density;
    float temperature;
} XsInflow;

/* Pressure solve settings; replaces the reference's `iterations` argument
 * of projection_forward/jvp/vjp (operators.h:69-71). */
typedef enum XsPressureSolverKind {
    XS_SOLVER_JACOBI_PCG = 0,            /* to a relative residual */
    XS_SOLVER_RED_BLACK_GAUSS_SEIDEL = 1 /* fixed sweep count, as operators.cu:1007-1010 */
} XsPressureSolverKind;

typedef struct XsPressureSolve {
    uint32_t kind;            /* XsPressureSolverKind */
    uint32_t max_iterations;  /* PCG cap, or the RBGS sweep count */
    double tolerance;         /* ||b - A p||_2 <= tolerance * ||b||_2, FP64 */
    const float* initial_guess; /* PCG warm start (device, N cells) or NULL */
    uint32_t scale_guess;     /* 1: start from alpha * guess with the energy-optimal
                                 alpha = (g.b) / (g.A g); 0: from the guess as given */
} XsPressureSolve;

/* Opaque handle of the learned warm-start network (no reference counterpart). */
typedef struct XsWarmStartNet XsWarmStartNet;

/* Written by a pressure solve into device memory (inside the workspace) and
 * read back with xs_read_solve_stats. */
typedef struct XsSolveStats {
    uint32_t iterations;          /* CG iterations over all refinement passes */
    uint32_t status;              /* XsStatus of the solve */
    uint32_t refinements;         /* FP64 true-residual passes taken */
    uint32_t warm_start_used;     /* 1 if the initial guess was kept */
    double rhs_norm;              /* ||b||_2 */
    double initial_residual;      /* ||b - A p0||_2 / ||b||_2 of the accepted start */
    double final_residual;        /* ||b - A p||_2 / ||b||_2, p in FP64 */
    double guess_scale;           /* alpha applied to the guess (1 if unscaled, 0 if none) */
    uint32_t coarse_iterations;   /* CG iterations of the coarse-grid correction of the start (0: none) */
    uint32_t smoothed_iterations; /* iterations that also updated the minimal-residual smoothed sequence */
} XsSolveStats;

/* ------------------------------------------------------------------------ */
/* operator level (operators.h:40-72)                                        */
/* ------------------------------------------------------------------------ */

/* operators.h:40 -- destination[i] += source[i] */
XsStatus xs_accumulate(cudaStream_t stream, const double* source, double* destination, uint64_t count);

/* operators.h:42-44; inflows may be NULL / 0.  `which` selects the inflow
 * value: 0 density, 1 temperature. */
XsStatus xs_source_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* state, const float* source,
                           const XsInflow* inflows, uint32_t inflow_count, uint32_t which, float* output);
XsStatus xs_source_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* state_tangent, const float* source_tangent,
                       const XsInflow* inflows, uint32_t inflow_count, float* output_tangent);
XsStatus xs_source_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const double* output_adjoint,
                       const XsInflow* inflows, uint32_t inflow_count, double* state_adjoint, double* source_adjoint);

/* operators.h:46-48; parameters are device scalars as in the reference */
XsStatus xs_buoyancy_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* density, const float* temperature,
                             XsVector external_acceleration, const float* ambient_temperature, const float* density_buoyancy,
                             const float* temperature_buoyancy, XsVector force);
XsStatus xs_buoyancy_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* density, const float* temperature,
                         const float* density_tangent, const float* temperature_tangent, XsVector external_acceleration_tangent,
                         const float* ambient_temperature, const float* density_buoyancy, const float* temperature_buoyancy,
                         const float* ambient_temperature_tangent, const float* density_buoyancy_tangent,
                         const float* temperature_buoyancy_tangent, XsVector force_tangent);
/* parameter adjoints are reduced per block, then added once per block (no
 * per-cell global atomics, unlike operators.cu:334-336) */
XsStatus xs_buoyancy_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* density, const float* temperature,
                         const float* ambient_temperature, const float* density_buoyancy, const float* temperature_buoyancy,
                         XsAdjointVector force_adjoint, double* density_adjoint, double* temperature_adjoint,
                         XsAdjointVector external_acceleration_adjoint, double* ambient_temperature_adjoint,
                         double* density_buoyancy_adjoint, double* temperature_buoyancy_adjoint);

/* operators.h:50-52 */
XsStatus xs_integrate_velocity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, XsVector force,
                                       XsVector output);
XsStatus xs_integrate_velocity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity_tangent,
                                   XsVector force_tangent, XsVector output_tangent);
XsStatus xs_integrate_velocity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsAdjointVector output_adjoint,
                                   XsAdjointVector velocity_adjoint, XsAdjointVector force_adjoint);

/* operators.h:54-56 */
XsStatus xs_advect_velocity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity,
                                    XsVelocityBoundary boundary, XsVector output);
XsStatus xs_advect_velocity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, XsVector velocity_tangent,
                                XsVelocityBoundary boundary, XsVector output_tangent);
XsStatus xs_advect_velocity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, XsVelocityBoundary boundary,
                                XsAdjointVector output_adjoint, XsAdjointVector velocity_adjoint);

/* operators.h:58-60; collider_velocity components may be NULL (zero) */
XsStatus xs_constrain_velocity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector collider_velocity,
                                       XsVector velocity, XsVelocityBoundary boundary, XsVector output);
XsStatus xs_constrain_velocity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity_tangent,
                                   XsVelocityBoundary boundary, XsVector output_tangent);
XsStatus xs_constrain_velocity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsAdjointVector output_adjoint,
                                   XsVelocityBoundary boundary, XsAdjointVector velocity_adjoint);

/* operators.h:62-64 */
XsStatus xs_advect_scalar_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* collider_value,
                                  const float* source, XsVector velocity, XsScalarBoundary scalar_boundary,
                                  XsVelocityBoundary velocity_boundary, float* output);
XsStatus xs_advect_scalar_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* source, const float* source_tangent,
                              XsVector velocity, XsVector velocity_tangent, XsScalarBoundary scalar_boundary,
                              XsVelocityBoundary velocity_boundary, float* output_tangent);
XsStatus xs_advect_scalar_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* source, XsVector velocity,
                              XsScalarBoundary scalar_boundary, XsVelocityBoundary velocity_boundary, const double* output_adjoint,
                              double* source_adjoint, XsAdjointVector velocity_adjoint);

/* operators.h:66-68 (VorticityView: operators.h:8-36).  cache holds, in
 * order, centered velocity (3N), vorticity (3N), magnitude (N), normal (3N),
 * normalizer (N) as 11 consecutive N-float arrays. */
XsStatus xs_vorticity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, const float* confinement,
                              float* cache, XsVector force);
/* scratch: 10 consecutive N-float arrays */
XsStatus xs_vorticity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity_tangent, const float* confinement,
                          const float* confinement_tangent, const float* cache, XsVector force_tangent, float* scratch);
/* scratch: 10 consecutive N-double arrays */
XsStatus xs_vorticity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* confinement, const float* cache,
                          XsAdjointVector force_adjoint, XsAdjointVector velocity_adjoint, double* confinement_adjoint, double* scratch);

/* Bytes of workspace a projection / pressure solve on this grid needs. */
size_t xs_projection_workspace_bytes(XsGrid grid);

/* operators.h:69-71 with the solver settings block.  `pressure` (N floats)
 * receives the solution, `rhs` (N floats) the right-hand side.  The solve
 * statistics land in the workspace (xs_read_solve_stats). */
XsStatus xs_projection_forward(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                               const uint32_t* cell_mask, XsVector velocity, XsVelocityBoundary velocity_boundary,
                               XsScalarBoundary pressure_boundary, float* pressure, float* rhs, XsVector output, void* workspace);
XsStatus xs_projection_jvp(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                           const uint32_t* cell_mask, XsVector velocity_tangent, XsVelocityBoundary velocity_boundary,
                           XsScalarBoundary pressure_boundary, float* pressure_tangent, float* rhs_tangent, XsVector output_tangent,
                           void* workspace);
/* PCG kind: adjoint solve A lambda = g with A symmetric; RBGS kind: the
 * reversed sweeps of operators.cu:1025-1028. */
XsStatus xs_projection_vjp(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                           const uint32_t* cell_mask, XsAdjointVector output_adjoint, XsVelocityBoundary velocity_boundary,
                           XsScalarBoundary pressure_boundary, double* pressure_adjoint, double* rhs_adjoint,
                           XsAdjointVector velocity_adjoint, void* workspace);

/* Stand-alone pressure solve on a right-hand side computed elsewhere: the
 * system red-black Gauss-Seidel converges to (operators.cu:885-902). */
XsStatus xs_pressure_solve(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                           const uint32_t* cell_mask, XsScalarBoundary pressure_boundary, const float* rhs, float* pressure,
                           void* workspace);

/* No counterpart in the reference.  The same pressure solve as
 * xs_pressure_solve for callers that cannot allocate device memory (hosts
 * that only hand over their input and output buffers, or that forbid
 * allocations outside their own pool): it takes no workspace and calls no
 * allocator; its scratch is one library-owned device array sized for at
 * most XS_STATIC_SOLVE_MAX_CELLS cells (about 9.1 MiB: seven FP32 vectors
 * plus the FP64 iterate at 64^3, held by each GPU the entry point runs on
 * until the process exits).  Larger grids return XS_CAPACITY_EXCEEDED
 * without launching.  All calls share that array: calls that overlap on the
 * GPU race, so order them on one stream.  The first call on a device
 * resolves the array's address (make it before any stream capture).
 * host_stats may be NULL; when given, the call synchronises the stream and
 * copies the solve statistics into it, and returns their status (a barrier
 * timeout, no convergence).  With NULL it does not synchronise, and a
 * failure inside the solve goes unreported: the status then covers only the
 * argument checks and the launches. */
#define XS_STATIC_SOLVE_MAX_CELLS (64u * 64u * 64u)
XsStatus xs_pressure_solve_static(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                                  const uint32_t* cell_mask, XsScalarBoundary pressure_boundary, const float* rhs, float* pressure,
                                  XsSolveStats* host_stats);

/* No counterpart in the reference.  The exact solve the warm start's
 * coarse-grid correction uses: A x = rhs (the pressure operator without
 * fixed values) on a grid without colliders or anchor cell and with at most
 * XS_SEPARABLE_SOLVE_MAX cells per axis, by the eigenbases of the three 1D
 * operators the operator separates into.  XS_INVALID_ARGUMENT for other
 * grids.  scratch: xs_separable_solve_scratch_bytes() bytes of device
 * memory. */
#define XS_SEPARABLE_SOLVE_MAX 256u
size_t xs_separable_solve_scratch_bytes(void);
XsStatus xs_separable_solve(cudaStream_t stream, XsGrid grid, XsScalarBoundary pressure_boundary, uint32_t pressure_anchor,
                            const double* rhs, float* x, void* scratch);

/* Byte offset of the XsSolveStats record inside a projection or step
 * workspace (device memory), for asynchronous copies that do not
 * synchronise. */
size_t xs_solve_stats_offset(void);

/* Synchronises the stream and copies the last solve's statistics. */
XsStatus xs_read_solve_stats(cudaStream_t stream, const void* workspace, XsSolveStats* host_stats);

/* ------------------------------------------------------------------------ */
/* domain (model.cpp:32-183)                                                 */
/* ------------------------------------------------------------------------ */

/* Collider (data.ixx:55-70): shape 0 = ellipsoid (size = radii), 1 = box
 * (size = half extents). */
typedef struct XsCollider {
    uint32_t shape;
    float center[3];
    float size[3];
    float velocity[3];
    float density;
    float temperature;
} XsCollider;

/* Rasterises colliders on the device (model.cpp:49-71, 79-155) into the
 * cell mask, collider face velocity, density and temperature, and returns
 * the pressure anchor (model.cpp:72-77) in *pressure_anchor (host).
 * colliders is a host array.  Synchronises the stream. */
XsStatus xs_smoke_build_domain(cudaStream_t stream, XsGrid grid, XsScalarBoundary pressure_boundary, const XsCollider* colliders,
                               uint32_t collider_count, uint32_t* cell_mask, XsVector collider_velocity, float* collider_density,
                               float* collider_temperature, uint32_t* pressure_anchor);

/* ------------------------------------------------------------------------ */
/* step level (model.cpp:341-389)                                            */
/* ------------------------------------------------------------------------ */

/* Configuration and device domain of a model (data.ixx:72-83, 198-204). */
typedef struct XsSmokeModel {
    XsGrid grid;
    XsVelocityBoundary velocity_boundary;
    XsScalarBoundary pressure_boundary;
    XsScalarBoundary density_boundary;
    XsScalarBoundary temperature_boundary;
    uint32_t vorticity_confinement_enabled;
    uint32_t pressure_anchor;
    XsPressureSolve pressure;
    const XsInflow* inflows;      /* host array, at most XS_MAX_INFLOWS */
    uint32_t inflow_count;
    const uint32_t* cell_mask;    /* NULL when there are no colliders */
    XsVector collider_velocity;   /* faces, may be NULL */
    const float* collider_density;
    const float* collider_temperature;
    /* optional timing events (created by the caller with timing enabled),
     * recorded on the step's stream around each pressure solve; NULL: none */
    cudaEvent_t solve_begin;
    cudaEvent_t solve_end;
    /* learned warm start of the forward pressure solve (NULL: zero guess).
     * The network's grid times its factor must equal `grid`; the guess is
     * energy-scaled and PCG falls back to zero when it does not help.  Not
     * used by the JVP and VJP solves. */
    XsWarmStartNet* warm_start;
    /* number of previous forward solutions kept in the workspace (0..5; 0:
     * off).  The forward PCG then starts from the A-norm-optimal (Galerkin)
     * combination of those solutions, followed by one energy-optimal step
     * along the learned correction of its residual, if any.  The ring
     * is part of the workspace (xs_smoke_workspace_bytes counts it) and is
     * emptied by xs_smoke_reset_warm_start, which must run once after the
     * workspace is allocated. */
    uint32_t warm_start_history;
    /* coarse-grid correction of the forward and adjoint starts (0: off;
     * otherwise the coarsening factor per axis, which must divide the grid;
     * needs warm_start_history > 0 and no colliders).  The ring's start takes
     * 6 damped Jacobi sweeps; their residual is restricted to the coarse
     * grid and solved there: exactly when its operator separates (no anchor
     * cell, at most XS_SEPARABLE_SOLVE_MAX cells per coarse axis), otherwise
     * by Jacobi-PCG to 1e-2 relative residual (from the same kind of start
     * one level further down, when the coarse grid divides again).  The
     * solution is interpolated back and the start takes one energy-optimal
     * step along it (before the learned correction's step), in rounds
     * (warm_start_rounds).  It removes the smooth error that fine-grid CG
     * reduces slowest. */
    uint32_t warm_start_coarsening;
    /* rounds of sweeps and coarse-grid correction before a forward solve
     * (0: the defaults, two without a learned warm start and one before its
     * step; at most 8).  Adjoint solves always take three. */
    uint32_t warm_start_rounds;
    /* optional per-stage timing of xs_smoke_forward_step (NULL: none): an
     * array of XS_STEP_STAGES + 1 events created by the caller with timing
     * enabled, recorded on the step's stream at the stage boundaries:
     * [0] start, [1] sources and forces done, [2] integration, [3] advection
     * and constraint, [4] pressure right-hand side, [5] warm start (the fine
     * PCG launch follows), [6] fine pressure solve, [7] ring update,
     * [8] projection, [9] scalar advection (end of the step). */
    cudaEvent_t* stage_events;
} XsSmokeModel;
#define XS_STEP_STAGES 9

/* State / Control / Parameters (data.ixx:117-134) */
typedef struct XsState { float* density; float* temperature; XsVector velocity; } XsState;
typedef struct XsControl { float* density_source; float* temperature_source; XsVector external_acceleration; } XsControl;
typedef struct XsParameters {
    float* ambient_temperature; float* density_buoyancy; float* temperature_buoyancy; float* vorticity_confinement;
} XsParameters;
/* StepCache (data.ixx:189-196); vorticity holds the 11 N-float arrays of
 * xs_vorticity_forward's cache */
typedef struct XsStepCache {
    float* sourced_density; float* sourced_temperature; XsVector force; float* vorticity;
    XsVector forced_velocity; XsVector advected_velocity;
} XsStepCache;
/* adjoint / tangent counterparts (data.ixx:136-172) */
typedef struct XsStateAdjoint { double* density; double* temperature; XsAdjointVector velocity; } XsStateAdjoint;
typedef struct XsControlAdjoint { double* density_source; double* temperature_source; XsAdjointVector external_acceleration; } XsControlAdjoint;
typedef struct XsParameterAdjoint {
    double* ambient_temperature; double* density_buoyancy; double* temperature_buoyancy; double* vorticity_confinement;
} XsParameterAdjoint;

typedef enum XsExecutionMode { XS_MODE_FORWARD = 0, XS_MODE_DIFFERENTIABLE = 1 } XsExecutionMode;

/* Bytes of ExecutionContext scratch (model.ixx:17-49) for a model. */
size_t xs_smoke_workspace_bytes(const XsSmokeModel* model, uint32_t mode);

/* Model::forward_step (model.cpp:341-349) */
XsStatus xs_smoke_forward_step(cudaStream_t stream, const XsSmokeModel* model, XsState state, XsControl control, XsParameters parameters,
                               XsState next_state, XsStepCache step_cache, void* workspace);
/* Model::jvp_step (model.cpp:351-359) */
XsStatus xs_smoke_jvp_step(cudaStream_t stream, const XsSmokeModel* model, XsState state, XsParameters parameters, XsState next_state,
                           XsStepCache step_cache, XsState state_tangent, XsControl control_tangent, XsParameters parameter_tangent,
                           XsState next_state_tangent, void* workspace);
/* Model::vjp_step (model.cpp:361-389); accumulates into previous_state_adjoint,
 * control_adjoint and parameter_adjoint */
XsStatus xs_smoke_vjp_step(cudaStream_t stream, const XsSmokeModel* model, XsState state, XsParameters parameters, XsState next_state,
                           XsStepCache step_cache, XsStateAdjoint next_state_adjoint, XsStateAdjoint previous_state_adjoint,
                           XsControlAdjoint control_adjoint, XsParameterAdjoint parameter_adjoint, void* workspace);

/* The example driver's per-step metrics (examples/smoke/forward/
 * simulation.cu:59-85) into metrics[6] (device): density sum, density max,
 * temperature max, max centred speed, sum of squared divergence before and
 * after projection, over fluid cells.  Overwrites metrics; the maxima start
 * at 0, as the example zeroes its metrics buffer before the reduction
 * (simulation.cpp:97-98). */
/* The example driver's controls (examples/smoke/forward/simulation.cu:35-57,
 * launch_write_control): at step `step` (time step * dt), two Gaussian jets
 * of the given radius whose amplitudes 0.75 + 0.25 sin(2 pi t / period)
 * pulse in antiphase; per cell, the density and temperature sources are the
 * rates times the summed jet weights and the external acceleration is the
 * weighted sum of the jets' accelerations.  Overwrites all five fields. */
XsStatus xs_smoke_write_control(cudaStream_t stream, XsGrid grid, uint64_t step, float pulse_period, XsVec3 left_center,
                                XsVec3 right_center, float source_radius, float density_source_rate, float temperature_source_rate,
                                XsVec3 left_acceleration, XsVec3 right_acceleration, float* density_source, float* temperature_source,
                                XsVector external_acceleration);

XsStatus xs_smoke_reduce_metrics(cudaStream_t stream, const XsSmokeModel* model, const float* density, const float* temperature,
                                 XsVector pre_projection_velocity, XsVector post_projection_velocity, double* metrics);

/* Statistics of the last forward pressure solve of a step (workspace). */
XsStatus xs_smoke_read_solve_stats(cudaStream_t stream, const XsSmokeModel* model, const void* workspace, uint32_t mode,
                                   XsSolveStats* forward_stats, XsSolveStats* adjoint_stats);

/* Device pointers, inside the workspace, of the pressure (FP32 copy of the
 * solution) and of the right-hand side of the last forward pressure solve:
 * the (divergence, pressure) pairs the warm-start network trains on. */
XsStatus xs_smoke_pressure_fields(const XsSmokeModel* model, void* workspace, float** pressure, float** rhs);

/* With a ring of previous solutions: device pointers, inside the workspace,
 * of the ring's Galerkin start x0 of the last forward solve and of its
 * residual b - A x0 (recomputed on the stream by this call): with the
 * solution, the (residual, correction) pairs the network learns when it
 * serves a model that keeps a ring. */
XsStatus xs_smoke_warm_start_fields(cudaStream_t stream, const XsSmokeModel* model, void* workspace, float** ring_start, float** residual);

/* Empties the rings of previous solutions (model->warm_start_history > 0):
 * after allocating the workspace and when a new trajectory starts.  A
 * differentiable workspace (mode) also keeps a ring of previous adjoint
 * pressure solutions, which starts the adjoint solves of a reverse pass the
 * same way; both are emptied. */
XsStatus xs_smoke_reset_warm_start(cudaStream_t stream, const XsSmokeModel* model, void* workspace, uint32_t mode);

/* ------------------------------------------------------------------------ */
/* learned pressure warm start (no reference counterpart)                    */
/* ------------------------------------------------------------------------ */

/* 3x3x3 convolution with zero padding on tcgen05 tensor cores: out = relu?(
 * conv(input, weights) + bias).  input [batch][nz][ny][nx][in_channels] and
 * output [..][out_channels] BF16 (NDHWC); weights [27][out][in] BF16 with tap
 * = (dz * 3 + dy) * 3 + dx; bias FP32 or NULL.  Channels 16, 32 or 64;
 * nx * ny >= 128 with min(nx, 128) dividing 128, nx and 128 / that dividing ny.
 * error_flag (device int, may be NULL) is set if a bounded wait expired. */
XsStatus xs_conv3d_bf16(cudaStream_t stream, uint32_t batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t in_channels,
                        uint32_t out_channels, const void* input, const void* weights, const float* bias, void* output, uint32_t relu,
                        int* error_flag);

/* Weight gradient of xs_conv3d_bf16 on tcgen05: weight_grad[27][out][in]
 * (FP32) = (accumulate ? weight_grad : 0) + sum over voxels of
 * input[v + tap][in] * output_grad[v][out] (output_grad is the gradient of
 * the pre-activation, BF16 NDHWC).  partial is FP32 scratch of
 * xs_conv3d_weight_grad_scratch_floats() elements; the per-CTA partial sums
 * are added in a fixed order, so the result is deterministic. */
XsStatus xs_conv3d_weight_grad_bf16(cudaStream_t stream, uint32_t batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t in_channels,
                                    uint32_t out_channels, const void* input, const void* output_grad, float* partial, float* weight_grad,
                                    uint32_t accumulate, int* error_flag);
size_t xs_conv3d_weight_grad_scratch_floats(uint32_t batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t in_channels,
                                            uint32_t out_channels);

/* The warm-start network: a 4-level U-Net (16/32/64/64 channels, 3x3x3
 * convolutions on tcgen05, BF16 activations, FP32 accumulation, FP32 master
 * weights and Adam state) mapping the right-hand side of the pressure system
 * on its grid (nx x ny x nz cells, each a multiple of 8, every level a valid
 * xs_conv3d_bf16 shape) to a pressure guess.  `factor` is the ratio of the
 * fluid grid to the network grid used by xs_warm_start_guess and by a model
 * that carries the network (1, 2, 3 or 4).  The handle owns its device
 * memory (one allocation at creation). */
XsStatus xs_warm_start_create(XsWarmStartNet** net, uint32_t max_batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t factor);
XsStatus xs_warm_start_destroy(XsWarmStartNet* net);
/* Number of FP32 parameters (layer by layer, each [27][out][in]). */
size_t xs_warm_start_parameter_count(void);
/* He-normal initialisation from a seed; resets the Adam state.  Synchronises. */
XsStatus xs_warm_start_initialize(XsWarmStartNet* net, cudaStream_t stream, uint64_t seed);
/* Host copies of the FP32 parameters.  set resets the Adam state.  Both synchronise. */
XsStatus xs_warm_start_set_parameters(XsWarmStartNet* net, cudaStream_t stream, const float* parameters);
XsStatus xs_warm_start_get_parameters(XsWarmStartNet* net, cudaStream_t stream, float* parameters);
/* guess[b] = network(rhs[b]) on the network grid, in units of the predicted
 * pressure's RMS; rhs and guess are [batch][cells] FP32 (device). */
XsStatus xs_warm_start_predict(XsWarmStartNet* net, cudaStream_t stream, uint32_t batch, const float* rhs, float* guess);
/* Loss mean_{b,v} (out_b - p_b / rms(p_b))^2 into *loss (device double, may
 * be NULL) and its gradient with respect to the parameters into gradient
 * (device, parameter_count floats, may be NULL; the network keeps its own copy). */
XsStatus xs_warm_start_gradient(XsWarmStartNet* net, cudaStream_t stream, uint32_t batch, const float* rhs, const float* pressure,
                                float* gradient, double* loss);
/* Training loss: kind 0 (default) the normalised L2 loss above; kind 1 the
 * energy loss mean_b 1 - (g.Ap)^2 / ((g.Ag)(p.Ap)) with g = output channel 0
 * and A the 7-point pressure operator of the network grid under
 * pressure_boundary (no solids): the squared relative A-norm error of the
 * energy-optimally scaled guess.  Takes effect at the next gradient. */
XsStatus xs_warm_start_set_loss(XsWarmStartNet* net, uint32_t kind, XsScalarBoundary pressure_boundary);
/* One Adam update from the last gradient. */
XsStatus xs_warm_start_adam_step(XsWarmStartNet* net, cudaStream_t stream, float learning_rate, float beta1, float beta2, float epsilon);
/* xs_warm_start_gradient followed by Adam (beta 0.9 / 0.999, epsilon 1e-8). */
XsStatus xs_warm_start_train_step(XsWarmStartNet* net, cudaStream_t stream, uint32_t batch, const float* rhs, const float* pressure,
                                  float learning_rate, double* loss);
/* Guess on a fluid grid of factor x the network grid: restriction (sum of
 * the factor^3 children), network, trilinear prolongation to the fine cell
 * centres.  guess: cells FP32 (device). */
XsStatus xs_warm_start_guess(XsWarmStartNet* net, cudaStream_t stream, XsGrid grid, const float* rhs, float* guess);
/* Synchronises; XS_TIMEOUT if a bounded wait inside a network kernel expired. */
XsStatus xs_warm_start_status(XsWarmStartNet* net, cudaStream_t stream);

/* Number of kernel launches the library has issued since load (for launch
 * accounting). */
uint64_t xs_launch_count(void);
/* cudaError_t of the last failed CUDA call on this thread (0 if none). */
int xs_last_cuda_error(void);
/* Human-readable text of an XsStatus. */
const char* xs_status_string(int status);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* DIFF_SMOKE_H */
