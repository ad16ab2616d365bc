// Pressure solver interface shared between translation units.
#pragma once

#include "common.cuh"

namespace xs {

constexpr int kPartialSlots = 4;
constexpr int kMaxPersistentBlocks = 4096;

// Device-side solver control block (first bytes of a pressure workspace).
struct SolverState {
    unsigned int count;   // grid-barrier arrivals
    unsigned int gen;     // grid-barrier generation
    unsigned int error;   // set when a bounded wait gave up
    unsigned int pad;
    double sum[kPartialSlots];  // totals of the last grid reduction
    XsSolveStats stats;
};

struct PressureWorkspace {
    SolverState* state;
    double* partials;
    double* x64;  // FP64 solution iterate (also the reverse-sweep hand-off)
    float* z;     // preconditioned residual r / diag
    float* p0;
    float* p1;
    float* q;
    float* e;     // FP32 correction of the current CG pass
    float* s;     // minimal-residual smoothed residual (warm starts)
    float* y;     // smoothed correction (warm starts)
    size_t bytes;
};

// Division by a runtime constant for numerators below 2^31:
// q = (n * m) >> shift with m = floor(2^shift / d) + 1, shift = 31 + ceil(log2 d).
struct FastDiv {
    uint64_t m;
    uint32_t shift;
};

// Geometry of the collider-free fast path of the pressure operator.  Face
// kinds: 0 Neumann (dropped), 1 fixed value (counts in the diagonal),
// 2 periodic (wraps).
struct FastGeom {
    uint32_t nx, ny, nz, n, groups;
    FastDiv dnx, dny;
    uint32_t anchor;  // n when there is none
    uint32_t kind[6];
};

PressureWorkspace carve_pressure_workspace(void* base, const Grid& g);
size_t pressure_workspace_bytes(const Grid& g);

// Solves the pressure system for rhs_f (forward, FP32, fixed boundary values
// enter b) or rhs_d (adjoint, FP64, no fixed values).  pressure_out receives
// an FP32 copy, solution_out an FP64 copy (either may be null); the FP64
// iterate stays in the workspace (carved->x64).
XsStatus solve_pressure(cudaStream_t stream, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                        const XsScalarBoundary& pb, const float* rhs_f, const double* rhs_d, float* pressure_out,
                        double* solution_out, void* workspace, PressureWorkspace* carved);

// The reference's reversed red-black sweeps (operators.cu:1025-1028).
XsStatus reverse_rbgs(cudaStream_t stream, const Grid& g, uint32_t sweeps, uint32_t anchor, const uint32_t* mask,
                      const XsScalarBoundary& pb, double* pressure_adjoint, double* rhs_adjoint, void* workspace);

XsStatus read_solve_stats(cudaStream_t stream, const void* workspace, const Grid& g, XsSolveStats* out);

// Warm-start subspace: a ring of the last `history` forward solutions plus
// at most one extra vector (kMaxBasis in all) spanning the Galerkin start.
constexpr int kMaxHistory = 5;
constexpr int kMaxBasis = kMaxHistory + 1;
struct WarmHistory {
    float* slots[kMaxBasis];
    float* products[kMaxBasis];  // A slot, computed when the slot is written
    uint32_t history;   // ring slots (0: off)
    uint32_t forward_rounds;  // start rounds before a forward solve (0: defaults)
    uint32_t* meta;     // device: [0] valid slots, [1] next slot
    float* start;       // the start vector of the last forward solve (N)
    float* ring_start;  // the Galerkin start from the ring alone (N)
    float* residual;    // b - A ring_start (N)
    float* extra_product;  // A of the extra vector of a combination or of a line step's direction (N)
    double* partials;
    double* coef;
    // coarse-grid correction of the start (coarsening > 0): the residual
    // restricted by `coarsening` per axis, solved on the coarse grid to
    // kCoarseTolerance by Jacobi-PCG, interpolated back (trilinear)
    uint32_t coarsening;
    Grid coarse;            // the coarse grid
    float* correction;      // the interpolated coarse solution (N)
    double* coarse_rhs;     // the restricted residual (coarse cells)
    float* coarse_solution; // (coarse cells)
    void* coarse_solver;    // pressure workspace of the coarse grid
    // the coarse solve's own start (coarsening2 > 0): pre-sweeps from zero,
    // the coarsest grid's solution for their residual, one line step
    uint32_t coarsening2;     // factor from the coarse grid to the coarsest
    Grid coarsest;
    float* coarse_start;      // (coarse cells)
    float* coarse_tmp;        // (coarse cells)
    float* coarse_residual;   // (coarse cells)
    float* coarse_product;    // A of a coarse line step's direction (coarse cells)
    float* coarse_correction; // the interpolated coarsest solution (coarse cells)
    double* coarsest_rhs;     // (coarsest cells)
    float* coarsest_solution; // (coarsest cells)
    void* coarsest_solver;    // pressure workspace of the coarsest grid
    // eigenbases of the coarse grid's axes (coarse grids within kSpectralMax)
    float* spectral_basis;    // 6 kSpectralMax^2 (each axis' basis and its transpose)
    float* spectral_eigen;    // 3 kSpectralMax
};
// Exact coarse solve for operators that separate by axis (spectral.cu):
// grids of at most kSpectralMax cells per axis, no anchor cell, no colliders.
constexpr int kSpectralMax = 256;
struct SpectralAxes {
    int n[3];
    int kind[3];  // per axis: zero-gradient / fixed-value ends, or periodic
};
// Whether the coarse operator of grid c (boundary modes of pb, anchor cell or
// none) separates; fills the axis description.
bool spectral_axes(const Grid& c, const XsScalarBoundary& pb, uint32_t anchor, SpectralAxes& out);
// x = A^-1 rhs on grid c by the axes' eigenbases (built into basis /
// eigen: 6 kSpectralMax^2 and 3 kSpectralMax floats).
XsStatus spectral_solve(cudaStream_t st, const Grid& c, const SpectralAxes& ax, float* basis, float* eigen, const double* rhs, float* x);
constexpr double kCoarseTolerance = 1e-2;
constexpr uint32_t kCoarseMaxIterations = 1000;
// Damped Jacobi sweeps (weight 2/3) on the start before its residual is
// restricted: they remove the high-frequency part of the error, which the
// coarse grid cannot represent and CG would otherwise meet first.  The
// adjoint starts take nine per round: their ring predicts far less, and at
// 256^3 nine sweeps in each of three rounds leave 3-5 adjoint iterations
// per solve instead of 5-16 (3.7 % less time per reverse step; the forward
// starts measured fastest with six).
constexpr int kCoarsePreSweeps = 6;
constexpr int kAdjointPreSweeps = 9;
// The coarse grid's own coarsening for the start of its solve: 4 when its
// extents allow (divisible, at least 8 cells after), else 2, else none.
uint32_t second_coarsening(const Grid& coarse);
// The coarse grid of g for a coarsening factor (false: none, or g not divisible).
bool coarse_grid(const Grid& g, uint32_t coarsening, Grid& coarse);
size_t warm_history_bytes(const Grid& g, uint32_t history, uint32_t coarsening = 0);
WarmHistory carve_warm_history(void* base, const Grid& g, uint32_t history, uint32_t coarsening = 0);
// out = the A-norm-optimal combination of the valid ring vectors (use_ring)
// and the n_extra vectors in `extra`, for the right-hand side rhs (+ fixed
// boundary values), or for the FP64 adjoint right-hand side rhs_d (no fixed
// values) when given.  out must not be one of the combined vectors.
XsStatus galerkin_combine(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const WarmHistory& h,
                          bool use_ring, const float* const* extra, int n_extra, const float* rhs, float* out, const double* rhs_d = nullptr);
// The coarse-grid correction of a start residual r: h.correction =
// P A_c^-1 R r.  R r = (sum of the f^3 children) / f: the operator is the
// spacing-squared-scaled Laplacian, so the coarse system at spacing f h
// takes f^2 times the children's mean.  A_c is the same stencil on the
// coarse grid (boundary modes kept, no fixed values), solved by Jacobi-PCG
// to kCoarseTolerance; P is trilinear interpolation at the fine cell
// centres, clamped at the domain edges.  Grids without colliders only.
XsStatus coarse_correction(cudaStream_t st, const Grid& g, uint32_t anchor, const XsScalarBoundary& pb, const WarmHistory& h, const float* r,
                           uint32_t max_iterations = kCoarseMaxIterations);
// `sweeps` damped Jacobi sweeps from x (FP32 rhs with fixed values, or the
// FP64 adjoint rhs_d without), result in x_out; tmp is scratch (N).  x_out
// may not alias x or tmp.
XsStatus jacobi_sweeps(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const float* rhs,
                       const double* rhs_d, const float* x, float* tmp, float* x_out, int sweeps = kCoarsePreSweeps);
// Copies the coarse solve's iteration count into the fine solve's statistics.
XsStatus record_coarse_iterations(cudaStream_t st, const WarmHistory& h, void* fine_workspace, const Grid& g);
// One energy-optimal step along a direction d from x (in place allowed):
// x_out = x + c d, r -= c A d with c = (d . r) / (d . A d) minimising the
// A-norm of the error along d (0 when d . A d vanishes); r is the residual
// of x on entry and, with update_residual, of x_out on return (left as it
// was otherwise: a step whose residual nothing reads moves 8 bytes per cell
// less).  A d goes to h.extra_product.
XsStatus line_step(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const WarmHistory& h,
                   const float* d, const float* x, float* r, float* x_out, bool update_residual = true);
// Rounds of the start pipeline (sweeps + coarse-grid correction) before the
// forward and the adjoint fine solves.  Measured at 256^3 (plume, steps
// 185-205, exact coarse solve): the forward start leaves a relative residual
// of 2.8e-5 after one round (9 fine iterations) and 6.2e-6 after two (4):
// 203.5 against 211.0 steps/s.  With the learned correction after the
// rounds, one round and the network's step give 7 iterations, two rounds
// and the step 4: 193.1 against 185.8 steps/s.  The adjoint start's ring
// predicts far less (0.03-0.15 left, against 3e-3 forward), and each round
// takes a further factor of about 7: 133 / 38 / 7 / 3 fine iterations after
// 1 / 2 / 3 / 4 rounds.
constexpr int kForwardStartCycles = 2;
constexpr int kForwardStartCyclesLearned = 1;
constexpr int kAdjointStartCycles = 3;
constexpr uint32_t kMaxStartRounds = 8;
// Iteration cap of the coarse Jacobi-PCG (grids without the exact coarse
// solve) in rounds after the first: their residuals are rougher, and a
// solve to kCoarseTolerance took 60-260 iterations for little gain.
constexpr uint32_t kLaterCoarseIterations = 16;
// `cycles` rounds of: kCoarsePreSweeps Jacobi sweeps (kAdjointPreSweeps
// for an adjoint start, rhs_d given), the residual, the
// coarse-grid correction of it, one line step along that correction; from x
// (h.ring_start on entry), the rounds alternating between h.start and
// h.ring_start.  *out = the final start; with keep_residual h.residual = its
// residual (otherwise a scratch value: every round recomputes the residual
// after its sweeps).  Grids without colliders only.
XsStatus coarse_cycles(cudaStream_t st, const Grid& g, uint32_t anchor, const XsScalarBoundary& pb, const WarmHistory& h, const float* rhs,
                       const double* rhs_d, int cycles, const float** out, bool keep_residual = false);
// Trilinear interpolation of a cell-centred field on the grid coarsened f
// times (coarse) at the cell centres of `fine`, clamped at the edges.
XsStatus prolong_cells(cudaStream_t st, const Grid& fine, const Grid& coarse, uint32_t f, const float* ec, float* out);
// r = b + fixed boundary values - A x, or r = rhs_d - A x for the FP64
// adjoint right-hand side (no fixed values) when rhs_d is given
XsStatus start_residual(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const float* rhs,
                        const float* x, float* r, const double* rhs_d = nullptr);
// Stores a solution (FP32, or FP64 rounded to FP32) in the next ring slot,
// with its product by the operator.
XsStatus history_push(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const WarmHistory& h,
                      const float* pressure, const double* pressure64 = nullptr);
// Empties the ring.
XsStatus history_reset(cudaStream_t st, const WarmHistory& h);

}  // namespace xs
