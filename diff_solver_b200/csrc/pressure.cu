// Pressure Poisson solve on sm_100a.
//
// The system is the one the reference's red-black Gauss-Seidel iteration
// converges to (solvers/smoke/operators.cu:852-902): for every fluid cell i
// that is not the pressure anchor and has a non-zero diagonal,
//
//     diag_i p_i - sum_{connected j} p_j = rhs_i + sum_{fixed faces} value
//
// where diag_i counts connected fluid neighbours plus fixed-value boundary
// faces, Neumann faces drop out and periodic faces wrap.  Every other cell
// holds p = 0.  The matrix is symmetric positive definite on the active
// cells whenever every fluid region touches a fixed face or the anchor.
//
// Solvers (one cooperative persistent launch each, bounded grid barriers):
//   * Jacobi-PCG.  CG vectors are FP32 (z = r/diag, p ping-pong, q, e), all
//     reductions are FP64 and deterministic (block partials summed in fixed
//     order by the last block to arrive).  The solution is accumulated in an
//     FP64 iterate x64: each CG pass solves for an FP32 correction e, which
//     is folded into x64, after which the true residual b - A x64 is
//     recomputed in FP64 and, if still above tolerance, a further pass runs
//     on it.  FP32 storage of the pressure alone cannot reach a 1e-6
//     relative residual on large grids; this refinement can.
//   * Red-black Gauss-Seidel with a fixed sweep count, the reference's own
//     method (operators.cu:1004-1013), in FP32, for drop-in behaviour.
//   * The reverse of those sweeps (operators.cu:935-955, 1025-1028) in
//     gather form, for the reference-compatible VJP.
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "launch.cuh"
#include "pressure.cuh"

namespace xs {

// ------------------------------------------------------------------ layout
size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

PressureWorkspace carve_pressure_workspace(void* base, const Grid& g) {
    const size_t n = cell_count(g);
    PressureWorkspace w{};
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        void* r = p ? p + off : nullptr;
        off = align_up(off + bytes, 256);
        return r;
    };
    w.state = static_cast<SolverState*>(take(sizeof(SolverState)));
    w.partials = static_cast<double*>(take(sizeof(double) * kPartialSlots * kMaxPersistentBlocks));
    w.x64 = static_cast<double*>(take(sizeof(double) * n));
    w.z = static_cast<float*>(take(sizeof(float) * n));
    w.p0 = static_cast<float*>(take(sizeof(float) * n));
    w.p1 = static_cast<float*>(take(sizeof(float) * n));
    w.q = static_cast<float*>(take(sizeof(float) * n));
    w.e = static_cast<float*>(take(sizeof(float) * n));
    w.s = static_cast<float*>(take(sizeof(float) * n));
    w.y = static_cast<float*>(take(sizeof(float) * n));
    w.bytes = off;
    return w;
}

size_t pressure_workspace_bytes(const Grid& g) { return carve_pressure_workspace(nullptr, g).bytes; }

// ------------------------------------------------------------ the operator
struct Operator {
    Grid g;
    const uint32_t* mask;
    uint32_t anchor;
    XsScalarBoundary pb;
    bool use_fixed_values;
};

// Neighbour structure of cell (x,y,z) (operators.cu:852-873).  Returns
// whether the cell is an unknown of the system; nb[] holds the six
// neighbour indices (valid where bit d of conn is set).
struct CellStencil {
    uint64_t nb[6];
    unsigned conn;
    float diag;
    float fixed_sum;
};

__device__ __forceinline__ bool stencil(const Operator& op, int x, int y, int z, uint64_t i, CellStencil& s) {
    const Grid& g = op.g;
    s.conn = 0u;
    s.diag = 0.0f;
    s.fixed_sum = 0.0f;
    if (is_solid(op.mask, i)) return false;
    const uint64_t sx = 1, sy = static_cast<uint64_t>(g.nx), sz = static_cast<uint64_t>(g.nx) * g.ny;
    const int coord[3] = {x, y, z};
    const int size[3] = {g.nx, g.ny, g.nz};
    const uint64_t stride[3] = {sx, sy, sz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int dir = side ? 1 : -1;
            const int c = coord[d] + dir;
            const int face = 2 * d + side;
            uint64_t j;
            if (c < 0 || c >= size[d]) {
                if (periodic(op.pb, d)) {
                    j = side ? i - stride[d] * (size[d] - 1) : i + stride[d] * (size[d] - 1);
                } else {
                    if (op.pb.modes[face] == 0u) {
                        s.diag += 1.0f;
                        if (op.use_fixed_values) s.fixed_sum += op.pb.values[face];
                    }
                    continue;
                }
            } else {
                j = side ? i + stride[d] : i - stride[d];
            }
            if (!is_solid(op.mask, j)) {
                s.nb[face] = j;
                s.conn |= 1u << face;
                s.diag += 1.0f;
            }
        }
    }
    return i != op.anchor && s.diag > 0.0f;
}

// ------------------------------------------------------------- grid sync
// Arrive at the grid barrier with K block-summed values; the last block to
// arrive sums every block's partials in block order (deterministic), stores
// the totals and releases the others.  Waits are bounded: a wait that runs
// past kBarrierTimeoutCycles marks state->error and returns.  Returns false
// if any block has flagged an error.
constexpr long long kBarrierTimeoutCycles = 8000000000ll;  // ~4 s at 2 GHz

template <int K>
__device__ bool grid_reduce(SolverState* st, double* partials, double* v, double* red) {
    __shared__ unsigned s_last, s_gen;
    if (K > 0) {
        block_sum<K>(v, red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) partials[static_cast<size_t>(blockIdx.x) * kPartialSlots + k] = v[k];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = *reinterpret_cast<volatile unsigned*>(&st->gen);
        __threadfence();
        const unsigned prev = atomicAdd(&st->count, 1u);
        s_last = prev == gridDim.x - 1 ? 1u : 0u;
        s_gen = gen;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (K > 0) {
            double acc[K > 0 ? K : 1];
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] = 0.0;
            for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
                for (int k = 0; k < K; ++k) acc[k] += __ldcg(partials + static_cast<size_t>(b) * kPartialSlots + k);
            }
            block_sum<K>(acc, red);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int k = 0; k < K; ++k) st->sum[k] = acc[k];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            st->count = 0u;
            __threadfence();
            atomicExch(&st->gen, s_gen + 1u);
        }
    } else if (threadIdx.x == 0) {
        const long long t0 = clock64();
        while (*reinterpret_cast<volatile unsigned*>(&st->gen) == s_gen) {
            __nanosleep(64);
            if (clock64() - t0 > kBarrierTimeoutCycles) {
                atomicExch(&st->error, 1u);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = __ldcg(&st->sum[k]);
    return __ldcg(&st->error) == 0u;
}

__device__ __forceinline__ bool grid_barrier(SolverState* st, double* partials, double* red) {
    return grid_reduce<0>(st, partials, nullptr, red);
}

// --------------------------------------------------------------- PCG phases
struct PcgArgs {
    Operator op;
    const float* rhs_f;   // forward right-hand side (FP32), or
    const double* rhs_d;  // adjoint right-hand side (FP64)
    const float* guess;   // warm start or null
    uint32_t scale_guess; // start from alpha * guess, alpha = (g.b) / (g.A g)
    double* x64;
    float* z;
    float* p[2];
    float* q;
    float* e;
    float* s;             // smoothed residual (smooth != 0)
    float* y;             // smoothed correction (smooth != 0)
    float* pressure_out;  // FP32 copy of the solution (null: none)
    double* solution_out; // FP64 copy of the solution (null: none)
    double* partials;
    SolverState* st;
    double tol;
    uint32_t max_iterations;
    FastGeom fast;
    uint32_t use_fast;
    uint32_t smooth;      // minimal-residual smoothing of the iterates (warm starts)
    uint32_t fast_residual;  // residual_fast serves the residual phases (fast path, no anchor, no fixed values)
};

enum ResidualMode { kFromZero = 0, kFromGuess = 1, kFromX64 = 2 };

__device__ __forceinline__ double rhs_at(const PcgArgs& a, uint64_t i) {
    return a.rhs_d ? a.rhs_d[i] : static_cast<double>(a.rhs_f[i]);
}

// Partial sums v = {g.b, g.A g} of the guess g over the active cells, for the
// energy-optimal scale alpha = (g.b) / (g.A g) that minimises the A-norm of
// the error of alpha g.
__device__ void guess_energy_phase(const PcgArgs& a, double (&v)[2]) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    v[0] = v[1] = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        CellStencil s;
        if (!stencil(a.op, x, y, z, i, s)) continue;
        const double gi = a.guess[i];
        double ag = s.diag * gi;
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if ((s.conn >> f) & 1u) { const uint64_t j = s.nb[f]; if (j != a.op.anchor) ag -= static_cast<double>(a.guess[j]); }
        v[0] += gi * (rhs_at(a, i) + static_cast<double>(s.fixed_sum));
        v[1] += gi * ag;
    }
}

// r = b - A x in FP64; z = r/diag, p0 = z, e = 0; partial sums
// v = {||b||^2, ||r||^2, r.z}.  kFromGuess starts from scale * guess.
__device__ void residual_phase(const PcgArgs& a, int mode, double (&v)[3], double scale = 1.0) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    v[0] = v[1] = v[2] = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        CellStencil s;
        const bool act = stencil(a.op, x, y, z, i, s);
        if (!act) {
            a.z[i] = 0.0f; a.p[0][i] = 0.0f; a.e[i] = 0.0f;
            if (a.smooth) { a.s[i] = 0.0f; a.y[i] = 0.0f; }
            if (mode != kFromX64) a.x64[i] = 0.0;
            if (a.pressure_out) a.pressure_out[i] = 0.0f;
            if (a.solution_out) a.solution_out[i] = 0.0;
            continue;
        }
        const double b = rhs_at(a, i) + static_cast<double>(s.fixed_sum);
        double xi = 0.0, ax = 0.0;
        if (mode == kFromGuess) {
            xi = a.guess[i];
            ax = s.diag * xi;
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if ((s.conn >> f) & 1u) { const uint64_t j = s.nb[f]; if (j != a.op.anchor) ax -= static_cast<double>(a.guess[j]); }
            xi *= scale;
            ax *= scale;
            a.x64[i] = xi;
        } else if (mode == kFromX64) {
            xi = a.x64[i];
            ax = s.diag * xi;
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if ((s.conn >> f) & 1u) ax -= a.x64[s.nb[f]];
        } else {
            a.x64[i] = 0.0;
        }
        const double r = b - ax;
        const float zf = static_cast<float>(r / s.diag);
        a.z[i] = zf;
        a.p[0][i] = zf;
        a.e[i] = 0.0f;
        if (a.smooth) {  // the smoothed sequence starts at the pass' start
            a.s[i] = zf * s.diag;
            a.y[i] = 0.0f;
        }
        if (a.pressure_out) a.pressure_out[i] = static_cast<float>(xi);
        if (a.solution_out) a.solution_out[i] = xi;
        v[0] += b * b;
        v[1] += r * r;
        v[2] += r * static_cast<double>(zf);
    }
}

// Smoothing state of a CG pass: off, starting (this spmv begins the smoothed
// sequence at the current iterate), or active.
enum SmoothMode { kSmoothOff = 0, kSmoothStart = 1, kSmoothActive = 2 };

// Iteration k: p_k = z + beta p_{k-1} (k > 0), q = A p_k, e += alpha_{k-1} p_{k-1};
// partial p_k.q.
// With smoothing active (k > 0): s_k = s_{k-1} + eta (r_k - s_{k-1}) and
// y_k = y_{k-1} + eta (e_k - y_{k-1}), r_k = z_k diag, e_k the updated e;
// starting: s_k = r_k, y_k = e_k.
template <bool kSmooth>
__device__ void spmv_phase(const PcgArgs& a, int k, float beta, float alpha_prev, float eta, int smooth, double& pq) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    const float* pold = a.p[(k + 1) & 1];
    float* pnew = a.p[k & 1];
    pq = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        CellStencil s;
        const bool act = stencil(a.op, x, y, z, i, s);
        if (!act) {
            if (k > 0) pnew[i] = 0.0f;
            a.q[i] = 0.0f;
            continue;
        }
        float pc, acc;
        if (k == 0) {
            pc = pnew[i];
            acc = 0.0f;
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if ((s.conn >> f) & 1u) acc += pnew[s.nb[f]];
        } else {
            const float po = pold[i];
            const float zc = a.z[i];
            pc = zc + beta * po;
            acc = 0.0f;
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if ((s.conn >> f) & 1u) { const uint64_t j = s.nb[f]; acc += a.z[j] + beta * pold[j]; }
            pnew[i] = pc;
            const float en = a.e[i] + alpha_prev * po;
            a.e[i] = en;
            if (kSmooth && smooth == kSmoothActive) {
                const float sv = a.s[i], yv = a.y[i];
                a.s[i] = sv + eta * (zc * s.diag - sv);
                a.y[i] = yv + eta * (en - yv);
            } else if (kSmooth && smooth == kSmoothStart) {
                a.s[i] = zc * s.diag;
                a.y[i] = en;
            }
        }
        const float qv = s.diag * pc - acc;
        a.q[i] = qv;
        pq += static_cast<double>(pc) * static_cast<double>(qv);
    }
}

// z -= alpha q / diag; partial {r.z, r.r} with r = z diag.
// z -= alpha q / diag; partial {r.z, r.r, s.r, s.s} with r = z diag (the last
// two with smoothing only).
template <bool kSmooth>
__device__ void update_phase(const PcgArgs& a, float alpha, bool smooth, double (&v)[4]) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    v[0] = v[1] = v[2] = v[3] = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        CellStencil s;
        if (!stencil(a.op, x, y, z, i, s)) continue;
        const float zn = a.z[i] - alpha * a.q[i] / s.diag;
        a.z[i] = zn;
        const double r = static_cast<double>(zn) * s.diag;
        v[0] += r * static_cast<double>(zn);
        v[1] += r * r;
        if (kSmooth && smooth) {
            const double sv = a.s[i];
            v[2] += sv * r;
            v[3] += sv * sv;
        }
    }
}

// x64 += e + alpha p_k
__device__ void fold_phase(const PcgArgs& a, int k, float alpha) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    const float* pk = a.p[k & 1];
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        a.x64[i] += static_cast<double>(a.e[i]) + static_cast<double>(alpha) * static_cast<double>(pk[i]);
    }
}

// The smoothed iterate: x64 += y_k + eta (e_k + alpha p_k - y_k).
__device__ void fold_smoothed_phase(const PcgArgs& a, int k, float alpha, double eta) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    const float* pk = a.p[k & 1];
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double xk = static_cast<double>(a.e[i]) + static_cast<double>(alpha) * static_cast<double>(pk[i]);
        const double yk = a.y[i];
        a.x64[i] += yk + eta * (xk - yk);
    }
}

// ------------------------------------------------------------ fast path
// Grids without colliders whose x extent is a multiple of 4: each thread
// owns 4 consecutive cells of a row (float4 loads and stores), indices are
// 32-bit, and the operator's diagonal and neighbour offsets follow from the
// row's boundary flags instead of a per-cell stencil.

inline FastDiv make_fastdiv(uint32_t d) {
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    const uint32_t shift = 31 + l;
    return FastDiv{((1ull << shift) / d) + 1, shift};
}

__device__ __forceinline__ uint32_t fastdiv(uint32_t n, const FastDiv& f) {
    return static_cast<uint32_t>((static_cast<uint64_t>(n) * f.m) >> f.shift);
}

struct RowGeom {
    int32_t off[4];  // -y, +y, -z, +z neighbour offsets; 0 = no neighbour
    float dyz;       // diagonal share of the y and z directions
};

__device__ __forceinline__ RowGeom row_geom(const FastGeom& f, uint32_t y, uint32_t z) {
    RowGeom r;
    r.dyz = 0.0f;
    const int32_t sy = static_cast<int32_t>(f.nx), sz = static_cast<int32_t>(f.nx * f.ny);
    const uint32_t c[2] = {y, z};
    const uint32_t size[2] = {f.ny, f.nz};
    const int32_t stride[2] = {sy, sz};
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        // lower side
        if (c[d] > 0) { r.off[2 * d] = -stride[d]; r.dyz += 1.0f; }
        else if (f.kind[2 + 2 * d] == 2u) { r.off[2 * d] = stride[d] * static_cast<int32_t>(size[d] - 1); r.dyz += 1.0f; }
        else { r.off[2 * d] = 0; if (f.kind[2 + 2 * d] == 1u) r.dyz += 1.0f; }
        // upper side
        if (c[d] + 1 < size[d]) { r.off[2 * d + 1] = stride[d]; r.dyz += 1.0f; }
        else if (f.kind[3 + 2 * d] == 2u) { r.off[2 * d + 1] = -stride[d] * static_cast<int32_t>(size[d] - 1); r.dyz += 1.0f; }
        else { r.off[2 * d + 1] = 0; if (f.kind[3 + 2 * d] == 1u) r.dyz += 1.0f; }
    }
    return r;
}

// Offsets of the x neighbours of the group's first and last cell (0: none)
// and the diagonals of the four cells.
__device__ __forceinline__ void x_geom(const FastGeom& f, uint32_t x0, float dyz, int32_t& left, int32_t& right, float4& d) {
    d = make_float4(dyz + 2.0f, dyz + 2.0f, dyz + 2.0f, dyz + 2.0f);
    if (x0 > 0) left = -1;
    else if (f.kind[0] == 2u) left = static_cast<int32_t>(f.nx) - 1;
    else { left = 0; d.x -= f.kind[0] == 1u ? 0.0f : 1.0f; }
    if (x0 + 4 < f.nx) right = 4;
    else if (f.kind[1] == 2u) right = 4 - static_cast<int32_t>(f.nx);
    else { right = 0; d.w -= f.kind[1] == 1u ? 0.0f : 1.0f; }
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, const float4& v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 axpy4(const float4& a, float b, const float4& x) {
    return make_float4(fmaf(b, x.x, a.x), fmaf(b, x.y, a.y), fmaf(b, x.z, a.z), fmaf(b, x.w, a.w));
}

// spmv_phase for the fast path.  The centre vectors of the thread's next
// group are loaded before this group's stores (software prefetch, as in
// update_fast); the stores go to p_k, e, q, s and y, none of which this
// phase reads at another group.
template <bool kFirst, bool kSmooth>
__device__ void spmv_fast(const PcgArgs& a, const FastGeom& f, int k, float beta, float alpha_prev, float eta, int smooth, double& pq) {
    const float* zv = a.z;
    const float* pold = a.p[(k + 1) & 1];
    float* pnew = a.p[k & 1];
    pq = 0.0;
    auto value4 = [&](uint32_t j) -> float4 { return kFirst ? ld4(pnew + j) : axpy4(ld4(zv + j), beta, ld4(pold + j)); };
    auto value1 = [&](uint32_t j) -> float { return kFirst ? pnew[j] : fmaf(beta, pold[j], zv[j]); };
    const bool active = kSmooth && smooth == kSmoothActive;
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float4 pn = zero4, en_next = zero4, zn = zero4, sn = zero4, yn = zero4;  // the next group's centre values
    auto fetch = [&](uint32_t j) {
        if (kFirst) {
            pn = ld4(pnew + j);
        } else {
            pn = ld4(pold + j);
            en_next = ld4(a.e + j);
            zn = ld4(zv + j);
            if (active) {
                sn = ld4(a.s + j);
                yn = ld4(a.y + j);
            }
        }
    };
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < f.groups) fetch(4u * t);
    for (; t < f.groups; t += stride) {
        const uint32_t i = 4u * t;
        const float4 po = pn, ev = en_next, zc = zn, sv = sn, yv = yn;
        if (t + stride < f.groups) fetch(i + 4u * stride);
        const uint32_t row = fastdiv(i, f.dnx);
        const uint32_t x0 = i - row * f.nx;
        const uint32_t z = fastdiv(row, f.dny);
        const uint32_t y = row - z * f.ny;
        const RowGeom rg = row_geom(f, y, z);
        int32_t left, right;
        float4 d;
        x_geom(f, x0, rg.dyz, left, right, d);
        const float4 c = kFirst ? po : axpy4(zc, beta, po);
        float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (rg.off[q] != 0) {
                const float4 v = value4(static_cast<uint32_t>(static_cast<int32_t>(i) + rg.off[q]));
                s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
            }
        }
        const float l = left != 0 ? value1(static_cast<uint32_t>(static_cast<int32_t>(i) + left)) : 0.0f;
        const float r = right != 0 ? value1(static_cast<uint32_t>(static_cast<int32_t>(i) + right)) : 0.0f;
        float4 qv;
        qv.x = d.x * c.x - (s.x + l + c.y);
        qv.y = d.y * c.y - (s.y + c.x + c.z);
        qv.z = d.z * c.z - (s.z + c.y + c.w);
        qv.w = d.w * c.w - (s.w + c.z + r);
        if (f.anchor - i < 4u) {  // the anchor cell is not an unknown
            const uint32_t lane = f.anchor - i;
            if (lane == 0) qv.x = 0.0f; else if (lane == 1) qv.y = 0.0f; else if (lane == 2) qv.z = 0.0f; else qv.w = 0.0f;
        }
        if (!kFirst) {
            st4(pnew + i, c);
            const float4 en = axpy4(ev, alpha_prev, po);
            st4(a.e + i, en);
            if (active) {  // s += eta (z diag - s); y += eta (e - y)
                st4(a.s + i, make_float4(sv.x + eta * (zc.x * d.x - sv.x), sv.y + eta * (zc.y * d.y - sv.y), sv.z + eta * (zc.z * d.z - sv.z),
                                         sv.w + eta * (zc.w * d.w - sv.w)));
                st4(a.y + i, make_float4(yv.x + eta * (en.x - yv.x), yv.y + eta * (en.y - yv.y), yv.z + eta * (en.z - yv.z),
                                         yv.w + eta * (en.w - yv.w)));
            } else if (kSmooth && smooth == kSmoothStart) {  // s = z diag; y = e
                st4(a.s + i, make_float4(zc.x * d.x, zc.y * d.y, zc.z * d.z, zc.w * d.w));
                st4(a.y + i, en);
            }
        }
        st4(a.q + i, qv);
        pq += static_cast<double>(c.x) * qv.x + static_cast<double>(c.y) * qv.y + static_cast<double>(c.z) * qv.z +
              static_cast<double>(c.w) * qv.w;
    }
}

// update_phase for the fast path.  (Recomputing q = A p_k here instead of
// storing it saves 4 B/cell, but measured slower on B200: 183 vs 167 ms per
// 1329-iteration solve at 256^3, from the extra stencil loads and spills.)
// The loads of the thread's next group are issued before this group's
// stores (software prefetch): a thread then keeps two groups' vectors in
// flight, which the phase needs to cover HBM latency at 4 blocks per SM.
template <bool kSmooth>
__device__ void update_fast(const PcgArgs& a, const FastGeom& f, float alpha, bool smooth, double (&v)[4]) {
    v[0] = v[1] = v[2] = v[3] = 0.0;
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float4 zn = make_float4(0.0f, 0.0f, 0.0f, 0.0f), qn = zn, sn = zn;
    if (t < f.groups) {
        zn = ld4(a.z + 4u * t);
        qn = ld4(a.q + 4u * t);
        if (kSmooth && smooth) sn = ld4(a.s + 4u * t);
    }
    for (; t < f.groups; t += stride) {
        const uint32_t i = 4u * t;
        float4 zz = zn;
        const float4 q = qn, sv = sn;
        if (t + stride < f.groups) {
            const uint32_t j = i + 4u * stride;
            zn = ld4(a.z + j);
            qn = ld4(a.q + j);
            if (kSmooth && smooth) sn = ld4(a.s + j);
        }
        const uint32_t row = fastdiv(i, f.dnx);
        const uint32_t x0 = i - row * f.nx;
        const uint32_t z = fastdiv(row, f.dny);
        const uint32_t y = row - z * f.ny;
        const RowGeom rg = row_geom(f, y, z);
        int32_t left, right;
        float4 d;
        x_geom(f, x0, rg.dyz, left, right, d);
        zz.x -= alpha * q.x / d.x;
        zz.y -= alpha * q.y / d.y;
        zz.z -= alpha * q.z / d.z;
        zz.w -= alpha * q.w / d.w;
        st4(a.z + i, zz);
        const double r0 = static_cast<double>(zz.x) * d.x, r1 = static_cast<double>(zz.y) * d.y, r2 = static_cast<double>(zz.z) * d.z,
                     r3 = static_cast<double>(zz.w) * d.w;
        v[0] += r0 * zz.x + r1 * zz.y + r2 * zz.z + r3 * zz.w;
        v[1] += r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3;
        if (kSmooth && smooth) {
            v[2] += r0 * sv.x + r1 * sv.y + r2 * sv.z + r3 * sv.w;
            v[3] += static_cast<double>(sv.x) * sv.x + static_cast<double>(sv.y) * sv.y + static_cast<double>(sv.z) * sv.z +
                    static_cast<double>(sv.w) * sv.w;
        }
    }
}

// ------------------------------------------- stencil passes, fast path
// The warm start's passes outside the CG iteration (sweeps, residuals,
// operator products) on grids the fast path serves that also have no anchor
// cell and no non-zero fixed boundary values: A x for the 4 cells of a row
// a thread owns, accumulated in FP64 like the general path.  (For a smooth
// field A x is a small difference of large terms: accumulated in FP32, the
// stored products of the ring lost most of their digits and the Galerkin
// start measured 1.5-2x more CG iterations.)
struct Double4 {
    double x, y, z, w;
};

__device__ __forceinline__ Double4 apply4(const FastGeom& f, const float* __restrict__ x, uint32_t i, float4& c, float4& d) {
    const uint32_t row = fastdiv(i, f.dnx);
    const uint32_t x0 = i - row * f.nx;
    const uint32_t z = fastdiv(row, f.dny);
    const uint32_t y = row - z * f.ny;
    const RowGeom rg = row_geom(f, y, z);
    int32_t left, right;
    x_geom(f, x0, rg.dyz, left, right, d);
    c = ld4(x + i);
    Double4 q{static_cast<double>(d.x) * c.x, static_cast<double>(d.y) * c.y, static_cast<double>(d.z) * c.z,
              static_cast<double>(d.w) * c.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (rg.off[k] != 0) {
            const float4 v = ld4(x + static_cast<uint32_t>(static_cast<int32_t>(i) + rg.off[k]));
            q.x -= v.x; q.y -= v.y; q.z -= v.z; q.w -= v.w;
        }
    }
    if (left != 0) q.x -= x[static_cast<uint32_t>(static_cast<int32_t>(i) + left)];
    if (right != 0) q.w -= x[static_cast<uint32_t>(static_cast<int32_t>(i) + right)];
    q.x -= c.y;
    q.y -= static_cast<double>(c.x) + c.z;
    q.z -= static_cast<double>(c.y) + c.w;
    q.w -= c.z;
    return q;
}

// apply4 in FP32: the start pipeline's smoothing, residual and line-step
// passes (their results only shape the start; the solve's own residuals are
// FP64), without the float-to-double conversions that bound the FP64 form.
__device__ __forceinline__ float4 apply4f(const FastGeom& f, const float* __restrict__ x, uint32_t i, float4& c, float4& d) {
    const uint32_t row = fastdiv(i, f.dnx);
    const uint32_t x0 = i - row * f.nx;
    const uint32_t z = fastdiv(row, f.dny);
    const uint32_t y = row - z * f.ny;
    const RowGeom rg = row_geom(f, y, z);
    int32_t left, right;
    x_geom(f, x0, rg.dyz, left, right, d);
    c = ld4(x + i);
    float4 q = make_float4(d.x * c.x, d.y * c.y, d.z * c.z, d.w * c.w);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (rg.off[k] != 0) {
            const float4 v = ld4(x + static_cast<uint32_t>(static_cast<int32_t>(i) + rg.off[k]));
            q.x -= v.x; q.y -= v.y; q.z -= v.z; q.w -= v.w;
        }
    }
    if (left != 0) q.x -= x[static_cast<uint32_t>(static_cast<int32_t>(i) + left)];
    if (right != 0) q.w -= x[static_cast<uint32_t>(static_cast<int32_t>(i) + right)];
    q.x -= c.y;
    q.y -= c.x + c.z;
    q.z -= c.y + c.w;
    q.w -= c.z;
    return q;
}

__device__ __forceinline__ float4 round4(const Double4& v) {
    return make_float4(static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z), static_cast<float>(v.w));
}

__device__ __forceinline__ Double4 ld4_rhs(const float* p) {
    const float4 v = ld4(p);
    return Double4{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Double4 ld4_rhs(const double* p) {
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    return Double4{a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ float4 ld4_rhs_f(const float* p) { return ld4(p); }
__device__ __forceinline__ float4 ld4_rhs_f(const double* p) {
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    return make_float4(static_cast<float>(a.x), static_cast<float>(a.y), static_cast<float>(b.x), static_cast<float>(b.y));
}

enum FastPass { kPassJacobi = 0, kPassResidual = 1, kPassApply = 2 };

// kPassJacobi: out = x + omega (b - A x) / diag; kPassResidual: out = b - A x;
// kPassApply: out = A x.  FP32 arithmetic (apply4f): these passes build the
// start of a solve.
template <int kPass, class T>
__global__ void fast_pass_kernel(FastGeom f, const float* __restrict__ x, const T* __restrict__ rhs, float* __restrict__ out, float omega) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < f.groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        float4 c, d;
        const float4 q = apply4f(f, x, i, c, d);
        if (kPass == kPassApply) {
            st4(out + i, q);
        } else {
            const float4 b = ld4_rhs_f(rhs + i);
            const float4 r = make_float4(b.x - q.x, b.y - q.y, b.z - q.z, b.w - q.w);
            if (kPass == kPassResidual)
                st4(out + i, r);
            else  // damped Jacobi update
                st4(out + i, make_float4(fmaf(r.x, omega / d.x, c.x), fmaf(r.y, omega / d.y, c.y), fmaf(r.z, omega / d.z, c.z),
                                         fmaf(r.w, omega / d.w, c.w)));
        }
    }
}

// residual_phase on the fast path for grids without an anchor cell and with
// no non-zero fixed boundary values (then every cell is an unknown and b is
// the right-hand side alone): 4 cells of a row per thread, the same FP64
// arithmetic per cell.
__device__ __forceinline__ double rhs_at4(const PcgArgs& a, uint32_t i, int k) {
    return a.rhs_d ? a.rhs_d[i + k] : static_cast<double>(a.rhs_f[i + k]);
}

template <class T>
__device__ __forceinline__ void load_x4(const T* __restrict__ v, uint32_t i, double (&c)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = static_cast<double>(v[i + k]);
}

// A x for the 4 cells at i: x is the guess (FP32) or the FP64 iterate.
template <class T>
__device__ __forceinline__ void apply4_fp64(const FastGeom& f, const T* __restrict__ x, uint32_t i, double (&c)[4], double (&ax)[4],
                                            float4& d) {
    const uint32_t row = fastdiv(i, f.dnx);
    const uint32_t x0 = i - row * f.nx;
    const uint32_t z = fastdiv(row, f.dny);
    const uint32_t y = row - z * f.ny;
    const RowGeom rg = row_geom(f, y, z);
    int32_t left, right;
    x_geom(f, x0, rg.dyz, left, right, d);
    load_x4(x, i, c);
    const float dd[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) ax[k] = static_cast<double>(dd[k]) * c[k];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (rg.off[q] != 0) {
            double v[4];
            load_x4(x, static_cast<uint32_t>(static_cast<int32_t>(i) + rg.off[q]), v);
#pragma unroll
            for (int k = 0; k < 4; ++k) ax[k] -= v[k];
        }
    }
    if (left != 0) ax[0] -= static_cast<double>(x[static_cast<uint32_t>(static_cast<int32_t>(i) + left)]);
    if (right != 0) ax[3] -= static_cast<double>(x[static_cast<uint32_t>(static_cast<int32_t>(i) + right)]);
    ax[0] -= c[1];
    ax[1] -= c[0] + c[2];
    ax[2] -= c[1] + c[3];
    ax[3] -= c[2];
}

__device__ void residual_fast(const PcgArgs& a, const FastGeom& f, int mode, double (&v)[3], double scale = 1.0) {
    v[0] = v[1] = v[2] = 0.0;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < f.groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        double xi[4] = {0.0, 0.0, 0.0, 0.0}, ax[4] = {0.0, 0.0, 0.0, 0.0};
        float4 d4;
        if (mode == kFromGuess) {
            apply4_fp64(f, a.guess, i, xi, ax, d4);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                xi[k] *= scale;
                ax[k] *= scale;
            }
        } else if (mode == kFromX64) {
            apply4_fp64(f, a.x64, i, xi, ax, d4);
        } else {
            const uint32_t row = fastdiv(i, f.dnx);
            const uint32_t z = fastdiv(row, f.dny);
            const RowGeom rg = row_geom(f, row - z * f.ny, z);
            int32_t left, right;
            x_geom(f, i - row * f.nx, rg.dyz, left, right, d4);
        }
        const float dd[4] = {d4.x, d4.y, d4.z, d4.w};
        float zf[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double b = rhs_at4(a, i, k);
            const double r = b - ax[k];
            zf[k] = static_cast<float>(r / dd[k]);
            v[0] += b * b;
            v[1] += r * r;
            v[2] += r * static_cast<double>(zf[k]);
            if (mode != kFromX64) a.x64[i + k] = xi[k];
            if (a.solution_out) a.solution_out[i + k] = xi[k];
        }
        const float4 z4 = make_float4(zf[0], zf[1], zf[2], zf[3]);
        st4(a.z + i, z4);
        st4(a.p[0] + i, z4);
        st4(a.e + i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        if (a.smooth) {  // the smoothed sequence starts at the pass' start
            st4(a.s + i, make_float4(zf[0] * dd[0], zf[1] * dd[1], zf[2] * dd[2], zf[3] * dd[3]));
            st4(a.y + i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        }
        if (a.pressure_out)
            st4(a.pressure_out + i, make_float4(static_cast<float>(xi[0]), static_cast<float>(xi[1]), static_cast<float>(xi[2]),
                                                static_cast<float>(xi[3])));
    }
}

constexpr uint32_t kMaxRefinements = 4;

// Register caps measured at 256^3: the plain solve is fastest at 4 blocks
// per SM (64 registers); the smoothing specialisation carries five more
// vectors per group and spills at that cap, and runs 10 % faster at 3.
template <bool kFast, bool kSmooth>
__global__ void __launch_bounds__(kBlock, kSmooth ? 3 : 4) pcg_kernel(PcgArgs a) {
    __shared__ double red[4 * 32];
    SolverState* st = a.st;
    double v3[3];
    double scale = a.guess ? 1.0 : 0.0;
    if (a.guess && a.scale_guess) {
        double e2[2];
        guess_energy_phase(a, e2);
        if (!grid_reduce<2>(st, a.partials, e2, red)) return;
        scale = (e2[1] > 0.0 && isfinite(e2[0] / e2[1])) ? e2[0] / e2[1] : 0.0;
    }
    if (kFast && a.fast_residual) residual_fast(a, a.fast, a.guess ? kFromGuess : kFromZero, v3, scale);
    else residual_phase(a, a.guess ? kFromGuess : kFromZero, v3, scale);
    if (!grid_reduce<3>(st, a.partials, v3, red)) return;
    const double bb = v3[0];
    double rr = v3[1], rz = v3[2];
    uint32_t warm = a.guess ? 1u : 0u;
    if (a.guess && !(rr <= bb)) {  // the guess is worse than zero: fall back
        warm = 0u;
        scale = 0.0;
        if (kFast && a.fast_residual) residual_fast(a, a.fast, kFromZero, v3);
        else residual_phase(a, kFromZero, v3);
        if (!grid_reduce<3>(st, a.partials, v3, red)) return;
        rr = v3[1];
        rz = v3[2];
    }
    const double initial = bb > 0.0 ? sqrt(rr / bb) : 0.0;
    const double target2 = a.tol * a.tol * bb;
    // Smoothing pays off from a good start (relative residual below 0.1:
    // 2-4x fewer iterations measured at 128^3); from a poor one it saves a
    // few per cent of the iterations for 16 more bytes per cell and
    // iteration.  A dropped guess, or one no better than zero (an empty
    // history), makes this the plain solve.
    const bool smooth_run = kSmooth && warm != 0u && rr < 0.01 * bb;
    // The smoothed sequence begins once the CG residual is within 10x of the
    // tolerance: the plateau it cures lies below that, and the first
    // iterations of a pass then move 16 bytes per cell less (same iteration
    // count within 2 in FP64 experiments at 128^3).
    const double smooth_begin2 = 100.0 * target2;
    uint32_t iterations = 0, refinements = 0, smoothed_iterations = 0;
    uint32_t status = XS_OK;
    while (true) {
        if (!(rr <= target2)) {
            if (!isfinite(rr)) { status = XS_NUMERICAL_ERROR; break; }
            if (iterations >= a.max_iterations || refinements > kMaxRefinements) { status = XS_NOT_CONVERGED; break; }
        } else {
            status = XS_OK;
            break;
        }
        // one CG pass on the current residual (z, p0 set, e = 0; with smoothing
        // s = r, y = 0).  Minimal-residual smoothing (Schoenauer; Zhou and
        // Walker): y_k = y_{k-1} + eta_k (x_k - y_{k-1}) with eta_k minimising
        // the norm of s_k = b - A y_k.  From a warm start the CG residual
        // plateaus just above the tolerance for many iterations while the
        // smoothed residual crosses it far earlier; the pass ends when
        // either does and keeps the iterate whose residual did.
        int k = 0;
        float beta = 0.0f, alpha = 0.0f, eta = 0.0f;
        double eta_final = 0.0;
        bool broke = false, smoothed = false;
        // the residual phase set s = r, y = 0 for a pass that starts close enough
        int smode = smooth_run && rr < smooth_begin2 ? kSmoothActive : kSmoothOff;
        while (true) {
            double pq[1];
            if (kFast) {
                if (k == 0) spmv_fast<true, kSmooth>(a, a.fast, k, beta, alpha, eta, smode, pq[0]);
                else spmv_fast<false, kSmooth>(a, a.fast, k, beta, alpha, eta, smode, pq[0]);
            } else {
                spmv_phase<kSmooth>(a, k, beta, alpha, eta, smode, pq[0]);
            }
            if (!grid_reduce<1>(st, a.partials, pq, red)) return;
            if (!(pq[0] > 0.0) || !isfinite(pq[0])) { broke = true; break; }
            alpha = static_cast<float>(rz / pq[0]);
            double v4[4];
            if (kFast) update_fast<kSmooth>(a, a.fast, alpha, smode != kSmoothOff, v4);
            else update_phase<kSmooth>(a, alpha, smode != kSmoothOff, v4);
            if (!grid_reduce<4>(st, a.partials, v4, red)) return;
            ++iterations;
            if (smode != kSmoothOff) ++smoothed_iterations;
            beta = static_cast<float>(v4[0] / rz);
            rz = v4[0];
            if (!isfinite(v4[1])) { broke = true; break; }
            if (v4[1] <= target2 || iterations >= a.max_iterations) break;
            if (smode != kSmoothOff) {
                // s.s, s.r, r.r -> eta and the norm of the next smoothed residual
                const double den = v4[1] - 2.0 * v4[2] + v4[3];
                const double e = den > 0.0 ? (v4[3] - v4[2]) / den : 0.0;
                const double ss = v4[3] + 2.0 * e * (v4[2] - v4[3]) + e * e * den;
                eta = static_cast<float>(e);
                if (ss <= target2 && isfinite(ss)) {
                    smoothed = true;
                    eta_final = e;
                    break;
                }
                smode = kSmoothActive;
            } else if (smooth_run && v4[1] < smooth_begin2) {
                smode = kSmoothStart;
            }
            ++k;
        }
        if (broke) {
            status = XS_NUMERICAL_ERROR;
            break;
        }
        if (smoothed) fold_smoothed_phase(a, k, alpha, eta_final);
        else fold_phase(a, k, alpha);
        if (!grid_barrier(st, a.partials, red)) return;
        if (kFast && a.fast_residual) residual_fast(a, a.fast, kFromX64, v3);
        else residual_phase(a, kFromX64, v3);
        if (!grid_reduce<3>(st, a.partials, v3, red)) return;
        rr = v3[1];
        rz = v3[2];
        ++refinements;
    }
    if (status != XS_OK && rr <= target2) status = XS_OK;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->stats.iterations = iterations;
        st->stats.status = status;
        st->stats.refinements = refinements;
        st->stats.warm_start_used = warm;
        st->stats.rhs_norm = sqrt(bb);
        st->stats.initial_residual = initial;
        st->stats.final_residual = bb > 0.0 ? sqrt(rr / bb) : 0.0;
        st->stats.guess_scale = scale;
        st->stats.smoothed_iterations = smoothed_iterations;
    }
}

// -------------------------------------------------- red-black Gauss-Seidel
// operators.cu:885-902 applied to the cells of one parity.
__device__ void rbgs_phase(const Operator& op, int parity, const float* rhs, float* p) {
    const Grid& g = op.g;
    const uint64_t n = cell_count(g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        if (((x + y + z) & 1) != parity || is_solid(op.mask, i) || i == op.anchor) continue;
        // neighbour order of the reference: -x, +x, -y, +y, -z, +z
        float sum = rhs[i], diag = 0.0f;
        CellStencil s;
        stencil(op, x, y, z, i, s);
        const int coord[3] = {x, y, z};
        const int size[3] = {g.nx, g.ny, g.nz};
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if ((s.conn >> f) & 1u) {
                sum += p[s.nb[f]];
                diag += 1.0f;
            } else {
                const int d = f >> 1, dir = (f & 1) ? 1 : -1;
                const int c = coord[d] + dir;
                if ((c < 0 || c >= size[d]) && !periodic(op.pb, d) && op.pb.modes[f] == 0u) {
                    sum += op.pb.values[f];
                    diag += 1.0f;
                }
            }
        }
        p[i] = diag == 0.0f ? 0.0f : sum / diag;
    }
}

struct RbgsArgs {
    Operator op;
    const float* rhs;
    float* p;
    uint32_t sweeps;
    double* partials;
    SolverState* st;
};

__global__ void __launch_bounds__(kBlock) rbgs_kernel(RbgsArgs a) {
    __shared__ double red[4 * 32];
    for (uint32_t it = 0; it < a.sweeps; ++it) {
        rbgs_phase(a.op, 0, a.rhs, a.p);
        if (!grid_barrier(a.st, a.partials, red)) return;
        rbgs_phase(a.op, 1, a.rhs, a.p);
        if (!grid_barrier(a.st, a.partials, red)) return;
    }
    // report the relative residual reached, in FP64
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    double v[2] = {0.0, 0.0};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        CellStencil s;
        Operator op = a.op;
        op.use_fixed_values = true;
        if (!stencil(op, x, y, z, i, s)) continue;
        const double b = static_cast<double>(a.rhs[i]) + s.fixed_sum;
        double ax = s.diag * static_cast<double>(a.p[i]);
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if ((s.conn >> f) & 1u) { const uint64_t j = s.nb[f]; if (j != a.op.anchor) ax -= a.p[j]; }
        v[0] += b * b;
        v[1] += (b - ax) * (b - ax);
    }
    if (!grid_reduce<2>(a.st, a.partials, v, red)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->stats.iterations = a.sweeps;
        a.st->stats.status = XS_OK;
        a.st->stats.refinements = 0;
        a.st->stats.warm_start_used = 0;
        a.st->stats.rhs_norm = sqrt(v[0]);
        a.st->stats.initial_residual = 1.0;
        a.st->stats.final_residual = v[0] > 0.0 ? sqrt(v[1] / v[0]) : 0.0;
    }
}

// Reverse sweeps (operators.cu:935-955) in gather form: the cells of one
// parity hand lambda_p / diag to the right-hand-side adjoint and to their
// connected neighbours; a second phase gathers those contributions.
struct RbgsReverseArgs {
    Operator op;
    double* pressure_adjoint;
    double* rhs_adjoint;
    double* handoff;
    uint32_t sweeps;
    double* partials;
    SolverState* st;
};

__device__ void reverse_emit_phase(const RbgsReverseArgs& a, int parity) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        double out = 0.0;
        if (((x + y + z) & 1) == parity && !is_solid(a.op.mask, i) && i != a.op.anchor) {
            CellStencil s;
            stencil(a.op, x, y, z, i, s);
            const double adj = s.diag == 0.0f ? 0.0 : a.pressure_adjoint[i] / static_cast<double>(s.diag);
            a.pressure_adjoint[i] = 0.0;
            a.rhs_adjoint[i] += adj;
            out = adj;
        }
        a.handoff[i] = out;
    }
}

__device__ void reverse_gather_phase(const RbgsReverseArgs& a, int parity) {
    const Grid& g = a.op.g;
    const uint64_t n = cell_count(g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        if (is_solid(a.op.mask, i)) continue;
        CellStencil s;
        stencil(a.op, x, y, z, i, s);
        double acc = 0.0;
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if ((s.conn >> f) & 1u) {
                const uint64_t j = s.nb[f];
                int jx, jy, jz;
                decode(j, g.nx, g.ny, jx, jy, jz);
                if (((jx + jy + jz) & 1) == parity) acc += a.handoff[j];
            }
        if (acc != 0.0) a.pressure_adjoint[i] += acc;
    }
}

__global__ void __launch_bounds__(kBlock) rbgs_reverse_kernel(RbgsReverseArgs a) {
    __shared__ double red[4 * 32];
    for (uint32_t it = 0; it < a.sweeps; ++it) {
        for (int parity = 1; parity >= 0; --parity) {
            reverse_emit_phase(a, parity);
            if (!grid_barrier(a.st, a.partials, red)) return;
            reverse_gather_phase(a, parity);
            if (!grid_barrier(a.st, a.partials, red)) return;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->stats.iterations = a.sweeps;
        a.st->stats.status = XS_OK;
    }
}

// ------------------------------------------------------------ launching
namespace {

struct DeviceLimits {
    int sms = 0;
    int pcg_blocks_per_sm[2] = {0, 0};       // [smooth]
    int pcg_fast_blocks_per_sm[2] = {0, 0};  // [smooth]
    int rbgs_blocks_per_sm = 0;
    int rev_blocks_per_sm = 0;
};

XsStatus device_limits(DeviceLimits& out) {
    static std::mutex mu;
    static int cached_device = -1;
    static DeviceLimits cached;
    int dev;
    if (cudaGetDevice(&dev) != cudaSuccess) return XS_CUDA_ERROR;
    std::lock_guard<std::mutex> lock(mu);
    if (dev != cached_device) {
        DeviceLimits l;
        if (cudaDeviceGetAttribute(&l.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return XS_CUDA_ERROR;
        // each specialisation's cooperative grid is its own co-resident count
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&l.pcg_blocks_per_sm[0], pcg_kernel<false, false>, kBlock, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&l.pcg_blocks_per_sm[1], pcg_kernel<false, true>, kBlock, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&l.pcg_fast_blocks_per_sm[0], pcg_kernel<true, false>, kBlock, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&l.pcg_fast_blocks_per_sm[1], pcg_kernel<true, true>, kBlock, 0) != cudaSuccess)
            return XS_CUDA_ERROR;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&l.rbgs_blocks_per_sm, rbgs_kernel, kBlock, 0) != cudaSuccess) return XS_CUDA_ERROR;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&l.rev_blocks_per_sm, rbgs_reverse_kernel, kBlock, 0) != cudaSuccess)
            return XS_CUDA_ERROR;
        cached = l;
        cached_device = dev;
    }
    out = cached;
    return XS_OK;
}

unsigned persistent_blocks(int per_sm, int sms, uint64_t n) {
    uint64_t want = (n + kBlock - 1) / kBlock;
    uint64_t cap = static_cast<uint64_t>(per_sm) * sms;
    if (cap > kMaxPersistentBlocks) cap = kMaxPersistentBlocks;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return static_cast<unsigned>(want);
}

template <class Args>
XsStatus launch_cooperative(void (*kernel)(Args), unsigned blocks, Args& args, cudaStream_t stream) {
    void* params[] = {&args};
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kernel), dim3(blocks), dim3(kBlock), params, 0, stream);
    if (e != cudaSuccess) return check_cuda(e);
    return check_launch();
}

}  // namespace

namespace {

FastGeom fast_geom(const Grid& g, uint32_t anchor, const XsScalarBoundary& pb) {
    const uint64_t n = cell_count(g);
    FastGeom f{};
    f.nx = static_cast<uint32_t>(g.nx);
    f.ny = static_cast<uint32_t>(g.ny);
    f.nz = static_cast<uint32_t>(g.nz);
    f.n = static_cast<uint32_t>(n);
    f.groups = static_cast<uint32_t>(n / 4);
    f.dnx = make_fastdiv(f.nx);
    f.dny = make_fastdiv(f.ny);
    f.anchor = anchor < n ? anchor : static_cast<uint32_t>(n);
    for (int face = 0; face < 6; ++face) {
        const int d = face / 2;
        const bool per = pb.modes[2 * d] == 2u && pb.modes[2 * d + 1] == 2u;
        f.kind[face] = per ? 2u : (pb.modes[face] == 0u ? 1u : 0u);
    }
    return f;
}

// The stencil passes' fast path: the PCG's fast-path grids without an anchor
// cell and, where b carries them (fixed_values), without non-zero fixed
// boundary values.
bool fast_pass_ok(const Grid& g, const uint32_t* mask, uint32_t anchor, const XsScalarBoundary& pb, bool fixed_values) {
    const uint64_t n = cell_count(g);
    if (mask != nullptr || g.nx % 4 != 0 || n >= (1ull << 31) || anchor < n) return false;
    if (fixed_values)
        for (int face = 0; face < 6; ++face)
            if (pb.modes[face] == 0u && pb.values[face] != 0.0f) return false;
    return true;
}

unsigned fast_pass_blocks(const Grid& g) {
    return static_cast<unsigned>(std::min<uint64_t>((cell_count(g) / 4 + 255) / 256, 148 * 16));
}

}  // namespace

XsStatus solve_pressure(cudaStream_t stream, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                        const XsScalarBoundary& pb, const float* rhs_f, const double* rhs_d, float* pressure_out,
                        double* solution_out, void* workspace, PressureWorkspace* carved) {
    if (!workspace) return XS_INVALID_ARGUMENT;
    const PressureWorkspace w = carve_pressure_workspace(workspace, g);
    if (carved) *carved = w;
    DeviceLimits lim;
    XsStatus s = device_limits(lim);
    if (s != XS_OK) return s;
    if (cudaMemsetAsync(w.state, 0, sizeof(SolverState), stream) != cudaSuccess) return XS_CUDA_ERROR;
    Operator op{g, mask, anchor, pb, rhs_d == nullptr};
    if (solve.kind == XS_SOLVER_RED_BLACK_GAUSS_SEIDEL) {
        if (!rhs_f || !pressure_out) return XS_INVALID_ARGUMENT;
        if (cudaMemsetAsync(pressure_out, 0, sizeof(float) * cell_count(g), stream) != cudaSuccess) return XS_CUDA_ERROR;
        RbgsArgs a{op, rhs_f, pressure_out, solve.max_iterations, w.partials, w.state};
        return launch_cooperative(rbgs_kernel, persistent_blocks(lim.rbgs_blocks_per_sm, lim.sms, cell_count(g)), a, stream);
    }
    if (solve.kind != XS_SOLVER_JACOBI_PCG || !(solve.tolerance >= 0.0)) return XS_INVALID_ARGUMENT;
    PcgArgs a{};
    a.op = op;
    a.rhs_f = rhs_f;
    a.rhs_d = rhs_d;
    a.guess = solve.initial_guess;
    a.scale_guess = solve.scale_guess;
    // residual smoothing pays off from warm starts (2-4x fewer iterations at
    // 128^3); from zero it saves ~4 % of the iterations for 44 % more traffic
    a.smooth = solve.initial_guess != nullptr ? 1u : 0u;
    a.s = w.s;
    a.y = w.y;
    a.x64 = w.x64;
    a.z = w.z;
    a.p[0] = w.p0;
    a.p[1] = w.p1;
    a.q = w.q;
    a.e = w.e;
    a.pressure_out = pressure_out;
    a.solution_out = solution_out;
    a.partials = w.partials;
    a.st = w.state;
    a.tol = solve.tolerance;
    a.max_iterations = solve.max_iterations;
    const uint64_t n = cell_count(g);
    a.use_fast = (mask == nullptr && g.nx % 4 == 0 && n < (1ull << 31)) ? 1u : 0u;
    if (a.use_fast) a.fast = fast_geom(g, anchor, pb);
    a.fast_residual = (a.use_fast && fast_pass_ok(g, mask, anchor, pb, rhs_d == nullptr)) ? 1u : 0u;
    const unsigned fast_blocks = persistent_blocks(lim.pcg_fast_blocks_per_sm[a.smooth], lim.sms, n / 4);
    const unsigned blocks = persistent_blocks(lim.pcg_blocks_per_sm[a.smooth], lim.sms, n);
    if (a.use_fast)
        return a.smooth ? launch_cooperative(pcg_kernel<true, true>, fast_blocks, a, stream)
                        : launch_cooperative(pcg_kernel<true, false>, fast_blocks, a, stream);
    return a.smooth ? launch_cooperative(pcg_kernel<false, true>, blocks, a, stream) : launch_cooperative(pcg_kernel<false, false>, blocks, a, stream);
}

XsStatus reverse_rbgs(cudaStream_t stream, const Grid& g, uint32_t sweeps, uint32_t anchor, const uint32_t* mask,
                      const XsScalarBoundary& pb, double* pressure_adjoint, double* rhs_adjoint, void* workspace) {
    const PressureWorkspace w = carve_pressure_workspace(workspace, g);
    DeviceLimits lim;
    XsStatus s = device_limits(lim);
    if (s != XS_OK) return s;
    if (cudaMemsetAsync(w.state, 0, sizeof(SolverState), stream) != cudaSuccess) return XS_CUDA_ERROR;
    RbgsReverseArgs a{Operator{g, mask, anchor, pb, false}, pressure_adjoint, rhs_adjoint, w.x64, sweeps, w.partials, w.state};
    return launch_cooperative(rbgs_reverse_kernel, persistent_blocks(lim.rev_blocks_per_sm, lim.sms, cell_count(g)), a, stream);
}

// ------------------------------------------- warm-start subspace (Galerkin)
// Start vector x0 = sum_i a_i v_i minimising the A-norm of the error over the
// span of the vectors v_i: G a = c with G_ij = v_i . A v_j and c_i = v_i . b
// on the active cells, A v_j applied in FP64.  The vectors are the last
// forward solutions (a ring of `history` slots whose valid count and next
// slot live on the device) and optionally one extra vector (the learned
// guess).  Dependent vectors are dropped by an LDL^T of the Jacobi-scaled
// Gram matrix that skips pivots below kBasisPivot.
constexpr int kGramBlocks = 148 * 3;  // one wave at 3 blocks per SM (bases of 6 vectors run at 2)
constexpr double kBasisPivot = 1e-11;

template <int M>
struct BasisArgs {
    Operator op;
    const float* v[M];
    uint32_t history;      // the first `history` entries of v are ring slots
    const uint32_t* meta;  // [0] valid ring vectors, [1] next slot
    const float* rhs;      // forward right-hand side (fixed boundary values added), or
    const double* rhs_d;   // adjoint right-hand side (FP64, no fixed values)
    double* partials;      // [gridDim.x][M(M+1)/2 + M]
    const float* w[M];     // A v, zero on inactive cells
    uint32_t fixed_terms;  // the forward b has non-zero fixed boundary values
};

// The ring's vectors ordered newest first: ptr[j] for j < history is the j-th
// newest valid solution (null past the valid count); entries past the ring
// are the extra vectors.  The basis spans the same space but uses successive
// differences of the ring, b_0 = r_0, b_j = r_{j-1} - r_j: consecutive
// solutions are nearly collinear, their differences far less so, which keeps
// the scaled Gram matrix well conditioned.
template <int M>
__device__ __forceinline__ void basis_order(const BasisArgs<M>& a, const float* (&ptr)[M], uint32_t& count, const float* (*wptr)[M] = nullptr) {
    count = a.history > 0 ? min(a.meta[0], a.history) : 0u;
    const uint32_t head = a.history > 0 ? min(a.meta[1], a.history - 1) : 0u;
#pragma unroll
    for (int j = 0; j < M; ++j) {
        const bool ring = j < static_cast<int>(a.history);
        const uint32_t slot = ring ? (head + 2 * a.history - 1 - j) % a.history : static_cast<uint32_t>(j);
        const bool valid = ring ? static_cast<uint32_t>(j) < count : a.v[j] != nullptr;
        ptr[j] = valid ? a.v[slot] : nullptr;
        if (wptr) (*wptr)[j] = valid ? a.w[slot] : nullptr;
    }
}

// Fixed boundary values entering b at cell i (non-zero only next to a
// fixed-value face; the solver adds the same sum).
__device__ __forceinline__ double boundary_fixed_sum(const Operator& op, uint64_t i) {
    int x, y, z;
    decode(i, op.g.nx, op.g.ny, x, y, z);
    CellStencil s;
    stencil(op, x, y, z, i, s);
    return s.fixed_sum;
}

// Streams the vectors and their stored A products: no stencil work here.
template <int M>
__global__ void __launch_bounds__(256, M > 5 ? 2 : 3) basis_gram_kernel(BasisArgs<M> a) {
    constexpr int K = M * (M + 1) / 2 + M;
    __shared__ double red[K * 32];
    const float* ptr[M];
    const float* wptr[M];
    uint32_t count;
    basis_order(a, ptr, count, &wptr);
    const uint64_t n = cell_count(a.op.g);
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double b = a.rhs_d ? a.rhs_d[i] : static_cast<double>(a.rhs[i]);
        if (a.fixed_terms) b += boundary_fixed_sum(a.op, i);
        double rv[M], ar[M];  // raw vectors and their A products
#pragma unroll
        for (int j = 0; j < M; ++j) {
            rv[j] = ptr[j] ? static_cast<double>(__ldg(ptr[j] + i)) : 0.0;
            ar[j] = wptr[j] ? static_cast<double>(__ldg(wptr[j] + i)) : 0.0;
        }
        double vi[M], av[M];
#pragma unroll
        for (int j = 0; j < M; ++j) {
            const bool diff = j > 0 && j < static_cast<int>(a.history) && static_cast<uint32_t>(j) < count;
            vi[j] = diff ? rv[j - 1] - rv[j] : rv[j];
            av[j] = diff ? ar[j - 1] - ar[j] : ar[j];
        }
        int k = 0;
#pragma unroll
        for (int r = 0; r < M; ++r)
#pragma unroll
            for (int c = r; c < M; ++c) acc[k++] += vi[r] * av[c];
#pragma unroll
        for (int r = 0; r < M; ++r) acc[k++] += vi[r] * b;
    }
    block_sum<K>(acc, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) a.partials[static_cast<size_t>(blockIdx.x) * K + k] = acc[k];
}

// basis_gram_kernel on 4-cell groups (n a multiple of 4, no fixed boundary
// values in b): 16-byte loads, four times the bytes in flight per thread.
template <int M>
__global__ void __launch_bounds__(256, M > 3 ? 2 : 3) basis_gram4_kernel(BasisArgs<M> a, uint32_t groups) {
    constexpr int K = M * (M + 1) / 2 + M;
    __shared__ double red[K * 32];
    const float* ptr[M];
    const float* wptr[M];
    uint32_t count;
    basis_order(a, ptr, count, &wptr);
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        double b[4];
        if (a.rhs_d) {
            const double2 lo = *reinterpret_cast<const double2*>(a.rhs_d + i), hi = *reinterpret_cast<const double2*>(a.rhs_d + i + 2);
            b[0] = lo.x; b[1] = lo.y; b[2] = hi.x; b[3] = hi.y;
        } else {
            const float4 v = ld4(a.rhs + i);
            b[0] = v.x; b[1] = v.y; b[2] = v.z; b[3] = v.w;
        }
        float4 rv[M], ar[M];
#pragma unroll
        for (int j = 0; j < M; ++j) {
            rv[j] = ptr[j] ? ld4(ptr[j] + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            ar[j] = wptr[j] ? ld4(wptr[j] + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            double vi[M], av[M];
#pragma unroll
            for (int j = 0; j < M; ++j) {
                const float* r0 = reinterpret_cast<const float*>(&rv[j]);
                const float* a0 = reinterpret_cast<const float*>(&ar[j]);
                const bool diff = j > 0 && j < static_cast<int>(a.history) && static_cast<uint32_t>(j) < count;
                const float* r1 = reinterpret_cast<const float*>(&rv[j > 0 ? j - 1 : 0]);
                const float* a1 = reinterpret_cast<const float*>(&ar[j > 0 ? j - 1 : 0]);
                vi[j] = diff ? static_cast<double>(r1[e]) - static_cast<double>(r0[e]) : static_cast<double>(r0[e]);
                av[j] = diff ? static_cast<double>(a1[e]) - static_cast<double>(a0[e]) : static_cast<double>(a0[e]);
            }
            int k = 0;
#pragma unroll
            for (int r = 0; r < M; ++r)
#pragma unroll
                for (int c = r; c < M; ++c) acc[k++] += vi[r] * av[c];
#pragma unroll
            for (int r = 0; r < M; ++r) acc[k++] += vi[r] * b[e];
        }
    }
    block_sum<K>(acc, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) a.partials[static_cast<size_t>(blockIdx.x) * K + k] = acc[k];
}

// Sums the partials in block order and solves the scaled Gram system.
template <int M>
__global__ void basis_solve_kernel(const double* __restrict__ partials, uint32_t blocks, double* __restrict__ coef) {
    constexpr int K = M * (M + 1) / 2 + M;
    __shared__ double tot[K];
    if (threadIdx.x < K) {
        double s = 0.0;
        for (uint32_t b = 0; b < blocks; ++b) s += partials[static_cast<size_t>(b) * K + threadIdx.x];
        tot[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double G[M][M], c[M], d[M], L[M][M], D[M], y[M], a[M];
    bool keep[M];
    int k = 0;
    for (int r = 0; r < M; ++r)
        for (int col = r; col < M; ++col) G[r][col] = G[col][r] = tot[k++];
    for (int r = 0; r < M; ++r) c[r] = tot[k++];
    for (int i = 0; i < M; ++i) d[i] = G[i][i] > 0.0 && isfinite(G[i][i]) ? sqrt(G[i][i]) : 0.0;
    // LDL^T of the scaled matrix, skipping (nearly) dependent columns
    for (int j = 0; j < M; ++j) {
        keep[j] = d[j] > 0.0;
        for (int i = 0; i < M; ++i) L[i][j] = 0.0;
        D[j] = 0.0;
        if (!keep[j]) continue;
        double dj = 1.0;  // scaled diagonal
        for (int p = 0; p < j; ++p)
            if (keep[p]) dj -= L[j][p] * L[j][p] * D[p];
        if (!(dj > kBasisPivot)) { keep[j] = false; continue; }
        D[j] = dj;
        L[j][j] = 1.0;
        for (int i = j + 1; i < M; ++i) {
            if (!(d[i] > 0.0)) continue;
            double v = G[i][j] / (d[i] * d[j]);
            for (int p = 0; p < j; ++p)
                if (keep[p]) v -= L[i][p] * L[j][p] * D[p];
            L[i][j] = v / dj;
        }
    }
    for (int i = 0; i < M; ++i) {
        double v = keep[i] ? c[i] / d[i] : 0.0;
        for (int p = 0; p < i; ++p)
            if (keep[p]) v -= L[i][p] * y[p];
        y[i] = v;
    }
    for (int i = M - 1; i >= 0; --i) {
        double v = keep[i] ? y[i] / D[i] : 0.0;
        for (int p = i + 1; p < M; ++p)
            if (keep[p]) v -= L[p][i] * a[p];
        a[i] = keep[i] ? v : 0.0;
    }
    bool finite = true;
    for (int i = 0; i < M; ++i) finite = finite && isfinite(a[i]);
    for (int i = 0; i < M; ++i) coef[i] = (finite && keep[i]) ? a[i] / d[i] : 0.0;
}

template <int M>
__global__ void basis_combine_kernel(BasisArgs<M> a, const double* __restrict__ coef, float* __restrict__ x0) {
    const float* ptr[M];
    uint32_t count;
    basis_order(a, ptr, count);
    // coefficients of the raw vectors: sum_j w_j b_j with b_0 = r_0 and
    // b_j = r_{j-1} - r_j on the ring gives r_j the weight
    // (j == 0 ? w_0 : -w_j) + w_{j+1} (if b_{j+1} is a ring difference)
    double w[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
        if (ptr[j] == nullptr) { w[j] = 0.0; continue; }
        if (j >= static_cast<int>(a.history)) { w[j] = coef[j]; continue; }
        w[j] = (j == 0 ? coef[0] : -coef[j]) + (static_cast<uint32_t>(j + 1) < count ? coef[j + 1] : 0.0);
    }
    const uint64_t n = cell_count(a.op.g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < M; ++j)
            if (w[j] != 0.0) acc += w[j] * static_cast<double>(ptr[j][i]);
        x0[i] = static_cast<float>(acc);
    }
}

// basis_combine_kernel on 4-cell groups.
template <int M>
__global__ void __launch_bounds__(256) basis_combine4_kernel(BasisArgs<M> a, const double* __restrict__ coef, float* __restrict__ x0, uint32_t groups) {
    const float* ptr[M];
    uint32_t count;
    basis_order(a, ptr, count);
    double w[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
        if (ptr[j] == nullptr) { w[j] = 0.0; continue; }
        if (j >= static_cast<int>(a.history)) { w[j] = coef[j]; continue; }
        w[j] = (j == 0 ? coef[0] : -coef[j]) + (static_cast<uint32_t>(j + 1) < count ? coef[j + 1] : 0.0);
    }
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < M; ++j)
            if (w[j] != 0.0) {
                const float4 v = ld4(ptr[j] + i);
                acc[0] += w[j] * static_cast<double>(v.x);
                acc[1] += w[j] * static_cast<double>(v.y);
                acc[2] += w[j] * static_cast<double>(v.z);
                acc[3] += w[j] * static_cast<double>(v.w);
            }
        st4(x0 + i, make_float4(static_cast<float>(acc[0]), static_cast<float>(acc[1]), static_cast<float>(acc[2]), static_cast<float>(acc[3])));
    }
}

// r = b + fixed boundary values - A x on the active cells, 0 elsewhere
template <class T>
__global__ void start_residual_kernel(Operator op, const T* __restrict__ rhs, const float* __restrict__ x, float* __restrict__ r) {
    const Grid& g = op.g;
    const uint64_t n = cell_count(g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int cx, cy, cz;
        decode(i, g.nx, g.ny, cx, cy, cz);
        CellStencil s;
        if (!stencil(op, cx, cy, cz, i, s)) {
            r[i] = 0.0f;
            continue;
        }
        double ax = s.diag * static_cast<double>(x[i]);
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if ((s.conn >> f) & 1u) { const uint64_t nb = s.nb[f]; if (nb != op.anchor) ax -= static_cast<double>(x[nb]); }
        r[i] = static_cast<float>(static_cast<double>(rhs[i]) + static_cast<double>(s.fixed_sum) - ax);
    }
}

struct HistorySlots {
    float* s[kMaxBasis];
};

// (A u)_i of the FP32 rounding of u on the active cells, 0 elsewhere
template <class T>
__device__ __forceinline__ float apply_at(const Operator& op, const T* __restrict__ u, uint64_t i) {
    int x, y, z;
    decode(i, op.g.nx, op.g.ny, x, y, z);
    CellStencil s;
    if (!stencil(op, x, y, z, i, s)) return 0.0f;
    double q = s.diag * static_cast<double>(static_cast<float>(u[i]));
#pragma unroll
    for (int f = 0; f < 6; ++f)
        if ((s.conn >> f) & 1u) { const uint64_t nb = s.nb[f]; if (nb != op.anchor) q -= static_cast<double>(static_cast<float>(u[nb])); }
    return static_cast<float>(q);
}

// slot[meta[1]] = pressure (rounded to FP32), product[meta[1]] = A slot
template <class T>
__global__ void history_push_kernel(Operator op, const T* __restrict__ pressure, HistorySlots slots, HistorySlots products, uint32_t history,
                                    const uint32_t* meta) {
    const uint32_t k = min(meta[1], history - 1);
    float* dst = slots.s[k];
    float* prod = products.s[k];
    const uint64_t n = cell_count(op.g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        dst[i] = static_cast<float>(pressure[i]);
        prod[i] = apply_at(op, pressure, i);
    }
}

// history_push_kernel<float> on the stencil passes' fast path
__global__ void fast_push_kernel(FastGeom f, const float* __restrict__ pressure, HistorySlots slots, HistorySlots products, uint32_t history,
                                 const uint32_t* meta) {
    const uint32_t k = min(meta[1], history - 1);
    float* dst = slots.s[k];
    float* prod = products.s[k];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < f.groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        float4 c, d;
        const Double4 q = apply4(f, pressure, i, c, d);
        st4(dst + i, c);
        st4(prod + i, round4(q));
    }
}

// history_push_kernel<double> on the fast path (the adjoint ring: FP64
// solutions, their products by the operator applied in FP64)
__global__ void fast_push64_kernel(FastGeom f, const double* __restrict__ pressure, HistorySlots slots, HistorySlots products, uint32_t history,
                                   const uint32_t* meta) {
    const uint32_t k = min(meta[1], history - 1);
    float* dst = slots.s[k];
    float* prod = products.s[k];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < f.groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        double c[4], ax[4];
        float4 d;
        apply4_fp64(f, pressure, i, c, ax, d);
        st4(dst + i, make_float4(static_cast<float>(c[0]), static_cast<float>(c[1]), static_cast<float>(c[2]), static_cast<float>(c[3])));
        st4(prod + i, make_float4(static_cast<float>(ax[0]), static_cast<float>(ax[1]), static_cast<float>(ax[2]), static_cast<float>(ax[3])));
    }
}

__global__ void apply_operator_kernel(Operator op, const float* __restrict__ u, float* __restrict__ out) {
    const uint64_t n = cell_count(op.g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = apply_at(op, u, i);
}

__global__ void history_advance_kernel(uint32_t history, uint32_t* meta) {
    meta[1] = (min(meta[1], history - 1) + 1) % history;
    meta[0] = min(meta[0] + 1, history);
}

bool coarse_grid(const Grid& g, uint32_t coarsening, Grid& coarse) {
    if (coarsening < 2 || g.nx % static_cast<int>(coarsening) != 0 || g.ny % static_cast<int>(coarsening) != 0 ||
        g.nz % static_cast<int>(coarsening) != 0)
        return false;
    coarse = g;
    coarse.nx = g.nx / static_cast<int>(coarsening);
    coarse.ny = g.ny / static_cast<int>(coarsening);
    coarse.nz = g.nz / static_cast<int>(coarsening);
    coarse.h = g.h * static_cast<float>(coarsening);
    return true;
}

uint32_t second_coarsening(const Grid& coarse) {
    Grid c2;
    for (uint32_t f : {4u, 2u})
        if (coarse_grid(coarse, f, c2) && c2.nx >= 8 && c2.ny >= 8 && c2.nz >= 8) return f;
    return 0;
}

static bool spectral_fits(const Grid& c) { return c.nx <= kSpectralMax && c.ny <= kSpectralMax && c.nz <= kSpectralMax; }

size_t warm_history_bytes(const Grid& g, uint32_t history, uint32_t coarsening) {
    if (history == 0) return 0;
    const size_t n = cell_count(g);
    size_t bytes = align_up(256, 256) + (2 * history + 4) * align_up(n * 4, 256) +
                   align_up(sizeof(double) * kGramBlocks * (kMaxBasis * (kMaxBasis + 1) / 2 + kMaxBasis), 256) + 256;
    Grid c, c2;
    if (coarse_grid(g, coarsening, c)) {
        const size_t nc = cell_count(c);
        bytes += align_up(n * 4, 256) + align_up(nc * 8, 256) + align_up(nc * 4, 256) + align_up(pressure_workspace_bytes(c), 256);
        if (spectral_fits(c)) bytes += align_up(4 * 6 * kSpectralMax * kSpectralMax, 256) + align_up(4 * 3 * kSpectralMax, 256);
        const uint32_t f2 = second_coarsening(c);
        if (f2 && coarse_grid(c, f2, c2)) {
            const size_t nc2 = cell_count(c2);
            bytes += 5 * align_up(nc * 4, 256) + align_up(nc2 * 8, 256) + align_up(nc2 * 4, 256) + align_up(pressure_workspace_bytes(c2), 256);
        }
    }
    return bytes;
}

WarmHistory carve_warm_history(void* base, const Grid& g, uint32_t history, uint32_t coarsening) {
    WarmHistory h{};
    h.history = history;
    if (history == 0 || !base) return h;
    const size_t n = cell_count(g);
    char* p = static_cast<char*>(base);
    h.meta = reinterpret_cast<uint32_t*>(p);
    size_t off = 256;
    auto take = [&](size_t bytes) {
        char* r = p + off;
        off += align_up(bytes, 256);
        return r;
    };
    for (uint32_t i = 0; i < history; ++i) {
        h.slots[i] = reinterpret_cast<float*>(take(n * 4));
        h.products[i] = reinterpret_cast<float*>(take(n * 4));
    }
    h.extra_product = reinterpret_cast<float*>(take(n * 4));
    h.start = reinterpret_cast<float*>(take(n * 4));
    h.ring_start = reinterpret_cast<float*>(take(n * 4));
    h.residual = reinterpret_cast<float*>(take(n * 4));
    h.partials = reinterpret_cast<double*>(take(sizeof(double) * kGramBlocks * (kMaxBasis * (kMaxBasis + 1) / 2 + kMaxBasis)));
    h.coef = reinterpret_cast<double*>(take(256));
    if (coarse_grid(g, coarsening, h.coarse)) {
        const size_t nc = cell_count(h.coarse);
        h.coarsening = coarsening;
        h.correction = reinterpret_cast<float*>(take(n * 4));
        h.coarse_rhs = reinterpret_cast<double*>(take(nc * 8));
        h.coarse_solution = reinterpret_cast<float*>(take(nc * 4));
        h.coarse_solver = take(pressure_workspace_bytes(h.coarse));
        if (spectral_fits(h.coarse)) {
            h.spectral_basis = reinterpret_cast<float*>(take(4 * 6 * kSpectralMax * kSpectralMax));
            h.spectral_eigen = reinterpret_cast<float*>(take(4 * 3 * kSpectralMax));
        }
        const uint32_t f2 = second_coarsening(h.coarse);
        if (f2 && coarse_grid(h.coarse, f2, h.coarsest)) {
            const size_t nc2 = cell_count(h.coarsest);
            h.coarsening2 = f2;
            h.coarse_start = reinterpret_cast<float*>(take(nc * 4));
            h.coarse_tmp = reinterpret_cast<float*>(take(nc * 4));
            h.coarse_residual = reinterpret_cast<float*>(take(nc * 4));
            h.coarse_product = reinterpret_cast<float*>(take(nc * 4));
            h.coarse_correction = reinterpret_cast<float*>(take(nc * 4));
            h.coarsest_rhs = reinterpret_cast<double*>(take(nc2 * 8));
            h.coarsest_solution = reinterpret_cast<float*>(take(nc2 * 4));
            h.coarsest_solver = take(pressure_workspace_bytes(h.coarsest));
        }
    }
    return h;
}

template <int M>
XsStatus galerkin_m(cudaStream_t st, const Operator& op, const WarmHistory& h, uint32_t ring, const float* const* extra, int n_extra,
                    const float* rhs, const double* rhs_d, float* out) {
    BasisArgs<M> a{};
    a.op = op;
    for (uint32_t i = 0; i < ring; ++i) {
        a.v[i] = h.slots[i];
        a.w[i] = h.products[i];
    }
    const uint64_t n = cell_count(op.g);
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16));
    XsStatus s;
    for (int i = 0; i < n_extra; ++i) {  // at most one extra vector (one product buffer)
        a.v[ring + i] = extra[i];
        a.w[ring + i] = h.extra_product;
        apply_operator_kernel<<<grid, 256, 0, st>>>(op, extra[i], h.extra_product);
        if ((s = check_launch()) != XS_OK) return s;
    }
    a.history = ring;
    a.meta = h.meta;
    a.rhs = rhs;
    a.rhs_d = rhs_d;
    a.partials = h.partials;
    a.fixed_terms = 0u;
    if (!rhs_d)
        for (int f = 0; f < 6; ++f)
            if (op.pb.modes[f] == 0u && op.pb.values[f] != 0.0f) a.fixed_terms = 1u;
    // 4-cell groups when every group lies in the array and b has no fixed terms
    const bool vec = n % 4 == 0 && n < (1ull << 31) && !a.fixed_terms;
    const uint32_t groups = static_cast<uint32_t>(n / 4);
    // (the 4-cell form of a basis of 4 or more vectors runs 2 blocks per SM)
    const unsigned cap = vec && M > 3 ? 148u * 2u : static_cast<unsigned>(kGramBlocks);
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(((vec ? groups : n) + 255) / 256, cap));
    if (vec)
        basis_gram4_kernel<M><<<blocks, 256, 0, st>>>(a, groups);
    else
        basis_gram_kernel<M><<<blocks, 256, 0, st>>>(a);
    if ((s = check_launch()) != XS_OK) return s;
    basis_solve_kernel<M><<<1, 64, 0, st>>>(h.partials, blocks, h.coef);
    if ((s = check_launch()) != XS_OK) return s;
    if (vec)
        basis_combine4_kernel<M><<<static_cast<unsigned>(std::min<uint64_t>((groups + 255) / 256, 148 * 16)), 256, 0, st>>>(a, h.coef, out, groups);
    else
        basis_combine_kernel<M><<<static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16)), 256, 0, st>>>(a, h.coef, out);
    return check_launch();
}

XsStatus galerkin_combine(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const WarmHistory& h,
                          bool use_ring, const float* const* extra, int n_extra, const float* rhs, float* out, const double* rhs_d) {
    const uint32_t ring = use_ring ? h.history : 0u;
    const uint32_t m = ring + static_cast<uint32_t>(n_extra);
    if (m == 0 || m > static_cast<uint32_t>(kMaxBasis) || n_extra > 1 || !h.meta || !out || (!rhs && !rhs_d)) return XS_INVALID_ARGUMENT;
    const Operator op{g, mask, anchor, pb, rhs_d == nullptr};
    switch (m) {
        case 1: return galerkin_m<1>(st, op, h, ring, extra, n_extra, rhs, rhs_d, out);
        case 2: return galerkin_m<2>(st, op, h, ring, extra, n_extra, rhs, rhs_d, out);
        case 3: return galerkin_m<3>(st, op, h, ring, extra, n_extra, rhs, rhs_d, out);
        case 4: return galerkin_m<4>(st, op, h, ring, extra, n_extra, rhs, rhs_d, out);
        case 5: return galerkin_m<5>(st, op, h, ring, extra, n_extra, rhs, rhs_d, out);
        default: return galerkin_m<kMaxBasis>(st, op, h, ring, extra, n_extra, rhs, rhs_d, out);
    }
}

// ---------------------------------------------- coarse-grid correction
// One thread per coarse cell sums its f^3 children in a fixed order (a warp
// reads f consecutive floats per thread and fine row: coalesced).
__global__ void coarse_restrict_kernel(Grid g, Grid c, uint32_t f, const float* __restrict__ r, double* __restrict__ rc, double scale) {
    const uint64_t nc = cell_count(c);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nc; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, c.nx, c.ny, x, y, z);
        double acc = 0.0;
        for (uint32_t dz = 0; dz < f; ++dz)
            for (uint32_t dy = 0; dy < f; ++dy) {
                const uint64_t row = (static_cast<uint64_t>(z) * f + dz) * static_cast<uint64_t>(g.ny) + static_cast<uint64_t>(y) * f + dy;
                const float* src = r + row * static_cast<uint64_t>(g.nx) + static_cast<uint64_t>(x) * f;
                for (uint32_t dx = 0; dx < f; ++dx) acc += static_cast<double>(src[dx]);
            }
        rc[i] = acc * scale;
    }
}

// Trilinear interpolation of a cell-centred coarse field at the fine cell
// centres: coarse coordinate u = (i + 1/2) / f - 1/2 clamped to [0, n_c - 1].
__device__ __forceinline__ void coarse_axis(int i, int nc, float inv_f, int& i0, int& i1, float& w) {
    const float u = fminf(fmaxf((static_cast<float>(i) + 0.5f) * inv_f - 0.5f, 0.0f), static_cast<float>(nc - 1));
    i0 = min(static_cast<int>(u), nc - 1);
    i1 = min(i0 + 1, nc - 1);
    w = u - static_cast<float>(i0);
}

__global__ void coarse_prolong_kernel(Grid g, Grid c, float inv_f, const float* __restrict__ ec, float* __restrict__ out) {
    const uint64_t n = cell_count(g);
    const uint64_t sy = static_cast<uint64_t>(c.nx), sz = static_cast<uint64_t>(c.nx) * static_cast<uint64_t>(c.ny);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        int x0, x1, y0, y1, z0, z1;
        float wx, wy, wz;
        coarse_axis(x, c.nx, inv_f, x0, x1, wx);
        coarse_axis(y, c.ny, inv_f, y0, y1, wy);
        coarse_axis(z, c.nz, inv_f, z0, z1, wz);
        auto at = [&](int xx, int yy, int zz) { return __ldg(ec + static_cast<uint64_t>(zz) * sz + static_cast<uint64_t>(yy) * sy + static_cast<uint64_t>(xx)); };
        const float c00 = at(x0, y0, z0) * (1.0f - wx) + at(x1, y0, z0) * wx;
        const float c10 = at(x0, y1, z0) * (1.0f - wx) + at(x1, y1, z0) * wx;
        const float c01 = at(x0, y0, z1) * (1.0f - wx) + at(x1, y0, z1) * wx;
        const float c11 = at(x0, y1, z1) * (1.0f - wx) + at(x1, y1, z1) * wx;
        const float c0 = c00 * (1.0f - wy) + c10 * wy;
        const float c1 = c01 * (1.0f - wy) + c11 * wy;
        out[i] = c0 * (1.0f - wz) + c1 * wz;
    }
}

// coarse_prolong_kernel for 4 consecutive fine cells of a row per thread
// (nx a multiple of 4), rows and planes from the launch grid (32 x 8 threads
// per block: 8 rows): no index division, one 16-byte store.  The same
// arithmetic per cell.
__global__ void __launch_bounds__(256) coarse_prolong4_kernel(Grid g, Grid c, float inv_f, const float* __restrict__ ec, float* __restrict__ out) {
    const int x = 4 * static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y), z = static_cast<int>(blockIdx.z);
    if (x >= g.nx || y >= g.ny) return;
    int y0, y1, z0, z1;
    float wy, wz;
    coarse_axis(y, c.ny, inv_f, y0, y1, wy);
    coarse_axis(z, c.nz, inv_f, z0, z1, wz);
    const uint64_t sy = static_cast<uint64_t>(c.nx), sz = static_cast<uint64_t>(c.nx) * static_cast<uint64_t>(c.ny);
    const float* r00 = ec + static_cast<uint64_t>(z0) * sz + static_cast<uint64_t>(y0) * sy;
    const float* r10 = ec + static_cast<uint64_t>(z0) * sz + static_cast<uint64_t>(y1) * sy;
    const float* r01 = ec + static_cast<uint64_t>(z1) * sz + static_cast<uint64_t>(y0) * sy;
    const float* r11 = ec + static_cast<uint64_t>(z1) * sz + static_cast<uint64_t>(y1) * sy;
    float v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int x0, x1;
        float wx;
        coarse_axis(x + k, c.nx, inv_f, x0, x1, wx);
        const float c00 = __ldg(r00 + x0) * (1.0f - wx) + __ldg(r00 + x1) * wx;
        const float c10 = __ldg(r10 + x0) * (1.0f - wx) + __ldg(r10 + x1) * wx;
        const float c01 = __ldg(r01 + x0) * (1.0f - wx) + __ldg(r01 + x1) * wx;
        const float c11 = __ldg(r11 + x0) * (1.0f - wx) + __ldg(r11 + x1) * wx;
        const float c0 = c00 * (1.0f - wy) + c10 * wy;
        const float c1 = c01 * (1.0f - wy) + c11 * wy;
        v[k] = c0 * (1.0f - wz) + c1 * wz;
    }
    st4(out + (static_cast<uint64_t>(z) * g.ny + y) * g.nx + x, make_float4(v[0], v[1], v[2], v[3]));
}

namespace {

XsStatus restrict_to(cudaStream_t st, const Grid& fine, const Grid& coarse, uint32_t f, const float* r, double* rc) {
    const uint64_t nc = cell_count(coarse);
    coarse_restrict_kernel<<<static_cast<unsigned>(std::min<uint64_t>((nc + 255) / 256, 148 * 16)), 256, 0, st>>>(fine, coarse, f, r, rc,
                                                                                                                   1.0 / static_cast<double>(f));
    return check_launch();
}

XsStatus prolong_from(cudaStream_t st, const Grid& fine, const Grid& coarse, uint32_t f, const float* ec, float* out) {
    if (fine.nx % 4 == 0 && fine.nz <= 65535) {
        const dim3 grid(static_cast<unsigned>((fine.nx / 4 + 31) / 32), static_cast<unsigned>((fine.ny + 7) / 8), static_cast<unsigned>(fine.nz));
        coarse_prolong4_kernel<<<grid, dim3(32, 8), 0, st>>>(fine, coarse, 1.0f / static_cast<float>(f), ec, out);
        return check_launch();
    }
    const uint64_t n = cell_count(fine);
    coarse_prolong_kernel<<<static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16)), 256, 0, st>>>(
        fine, coarse, 1.0f / static_cast<float>(f), ec, out);
    return check_launch();
}

}  // namespace

XsStatus prolong_cells(cudaStream_t st, const Grid& fine, const Grid& coarse, uint32_t f, const float* ec, float* out) {
    return prolong_from(st, fine, coarse, f, ec, out);
}

namespace {

// the anchor moves to the coarse cell that contains it (n: none, on both grids)
uint32_t coarse_anchor(const Grid& g, uint32_t f, const Grid& c, uint32_t anchor) {
    const uint64_t n = cell_count(g);
    if (anchor >= n) return anchor;
    const uint64_t ax = anchor % static_cast<uint64_t>(g.nx), ay = (anchor / static_cast<uint64_t>(g.nx)) % static_cast<uint64_t>(g.ny),
                   az = anchor / (static_cast<uint64_t>(g.nx) * static_cast<uint64_t>(g.ny));
    return static_cast<uint32_t>(ax / f + static_cast<uint64_t>(c.nx) * (ay / f + static_cast<uint64_t>(c.ny) * (az / f)));
}

XsPressureSolve coarse_solve_settings(const float* guess, uint32_t max_iterations = kCoarseMaxIterations) {
    XsPressureSolve cs{};
    cs.kind = XS_SOLVER_JACOBI_PCG;
    cs.max_iterations = max_iterations;
    cs.tolerance = kCoarseTolerance;
    cs.initial_guess = guess;
    cs.scale_guess = 0u;
    return cs;
}

}  // namespace

XsStatus coarse_correction(cudaStream_t st, const Grid& g, uint32_t anchor, const XsScalarBoundary& pb, const WarmHistory& h, const float* r,
                           uint32_t max_iterations) {
    if (h.coarsening < 2 || !h.correction || !h.coarse_rhs || !h.coarse_solution || !h.coarse_solver || !r) return XS_INVALID_ARGUMENT;
    const Grid& c = h.coarse;
    const uint32_t f = h.coarsening;
    XsStatus s = restrict_to(st, g, c, f, r, h.coarse_rhs);
    if (s != XS_OK) return s;
    const uint32_t anchor_c = coarse_anchor(g, f, c, anchor);
    SpectralAxes ax;
    if (h.spectral_basis && spectral_axes(c, pb, anchor_c, ax)) {
        // the separable coarse operator: solved exactly (no CG iterations to report)
        if ((s = spectral_solve(st, c, ax, h.spectral_basis, h.spectral_eigen, h.coarse_rhs, h.coarse_solution)) != XS_OK) return s;
        const PressureWorkspace cw = carve_pressure_workspace(h.coarse_solver, c);
        if ((s = check_cuda(cudaMemsetAsync(&cw.state->stats.iterations, 0, sizeof(uint32_t), st))) != XS_OK) return s;
        return prolong_from(st, g, c, f, h.coarse_solution, h.correction);
    }
    const float* guess = nullptr;
    if (h.coarsening2) {
        // the coarse solve's own start, the same way one level down (from
        // zero: pre-sweeps, the coarsest grid's correction, one line step);
        // FP64 right-hand sides without fixed values on both levels
        const Grid& c2 = h.coarsest;
        const uint32_t f2 = h.coarsening2;
        const uint64_t nc = cell_count(c);
        if ((s = check_cuda(cudaMemsetAsync(h.coarse_product, 0, sizeof(float) * nc, st))) != XS_OK) return s;
        if ((s = jacobi_sweeps(st, c, anchor_c, nullptr, pb, nullptr, h.coarse_rhs, h.coarse_product, h.coarse_tmp, h.coarse_start)) != XS_OK)
            return s;
        if ((s = start_residual(st, c, anchor_c, nullptr, pb, nullptr, h.coarse_start, h.coarse_residual, h.coarse_rhs)) != XS_OK) return s;
        if ((s = restrict_to(st, c, c2, f2, h.coarse_residual, h.coarsest_rhs)) != XS_OK) return s;
        if ((s = solve_pressure(st, c2, coarse_solve_settings(nullptr), coarse_anchor(c, f2, c2, anchor_c), nullptr, pb, nullptr,
                                h.coarsest_rhs, h.coarsest_solution, nullptr, h.coarsest_solver, nullptr)) != XS_OK)
            return s;
        if ((s = prolong_from(st, c, c2, f2, h.coarsest_solution, h.coarse_correction)) != XS_OK) return s;
        WarmHistory level = h;
        level.extra_product = h.coarse_product;
        if ((s = line_step(st, c, anchor_c, nullptr, pb, level, h.coarse_correction, h.coarse_start, h.coarse_residual, h.coarse_start)) !=
            XS_OK)
            return s;
        guess = h.coarse_start;
    }
    if ((s = solve_pressure(st, c, coarse_solve_settings(guess, max_iterations), anchor_c, nullptr, pb, nullptr, h.coarse_rhs, h.coarse_solution, nullptr,
                            h.coarse_solver, nullptr)) != XS_OK)
        return s;
    return prolong_from(st, g, c, f, h.coarse_solution, h.correction);
}

XsStatus record_coarse_iterations(cudaStream_t st, const WarmHistory& h, void* fine_workspace, const Grid& g) {
    if (h.coarsening < 2 || !h.coarse_solver || !fine_workspace) return XS_OK;
    const PressureWorkspace fw = carve_pressure_workspace(fine_workspace, g);
    const PressureWorkspace cw = carve_pressure_workspace(h.coarse_solver, h.coarse);
    return check_cuda(cudaMemcpyAsync(&fw.state->stats.coarse_iterations, &cw.state->stats.iterations, sizeof(uint32_t),
                                      cudaMemcpyDeviceToDevice, st));
}

template <class T>
__global__ void jacobi_sweep_kernel(Operator op, const T* __restrict__ rhs, const float* __restrict__ x, float* __restrict__ x_out, float omega) {
    const Grid& g = op.g;
    const uint64_t n = cell_count(g);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int cx, cy, cz;
        decode(i, g.nx, g.ny, cx, cy, cz);
        CellStencil s;
        if (!stencil(op, cx, cy, cz, i, s)) {
            x_out[i] = 0.0f;
            continue;
        }
        const float xi = x[i];
        double ax = s.diag * static_cast<double>(xi);
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if ((s.conn >> f) & 1u) { const uint64_t nb = s.nb[f]; if (nb != op.anchor) ax -= static_cast<double>(x[nb]); }
        const double r = static_cast<double>(rhs[i]) + static_cast<double>(s.fixed_sum) - ax;
        x_out[i] = static_cast<float>(static_cast<double>(xi) + omega * r / s.diag);
    }
}

XsStatus jacobi_sweeps(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const float* rhs,
                       const double* rhs_d, const float* x, float* tmp, float* x_out, int sweeps) {
    if (!x || !tmp || !x_out || x_out == x || x_out == tmp || (!rhs && !rhs_d) || sweeps < 0) return XS_INVALID_ARGUMENT;
    const Operator op{g, mask, anchor, pb, rhs_d == nullptr};
    const uint64_t n = cell_count(g);
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16));
    const float omega = 2.0f / 3.0f;
    // ping-pong so that the last sweep writes x_out
    const bool fast = fast_pass_ok(g, mask, anchor, pb, rhs_d == nullptr);
    const FastGeom f = fast ? fast_geom(g, anchor, pb) : FastGeom{};
    const float* src = x;
    for (int k = 0; k < sweeps; ++k) {
        float* dst = ((sweeps - 1 - k) % 2 == 0) ? x_out : tmp;
        if (fast && rhs_d)
            fast_pass_kernel<kPassJacobi, double><<<fast_pass_blocks(g), 256, 0, st>>>(f, src, rhs_d, dst, omega);
        else if (fast)
            fast_pass_kernel<kPassJacobi, float><<<fast_pass_blocks(g), 256, 0, st>>>(f, src, rhs, dst, omega);
        else if (rhs_d)
            jacobi_sweep_kernel<double><<<blocks, 256, 0, st>>>(op, rhs_d, src, dst, omega);
        else
            jacobi_sweep_kernel<float><<<blocks, 256, 0, st>>>(op, rhs, src, dst, omega);
        const XsStatus s = check_launch();
        if (s != XS_OK) return s;
        src = dst;
    }
    if (sweeps == 0) return check_cuda(cudaMemcpyAsync(x_out, x, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    return XS_OK;
}

// ------------------------------------------------ energy-optimal line step
__global__ void line_update_kernel(uint64_t n, const double* __restrict__ coef, const float* __restrict__ d, const float* __restrict__ ad,
                                   const float* x, float* r, float* x_out) {
    const float c = static_cast<float>(coef[0]);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        x_out[i] = fmaf(c, d[i], x[i]);
        if (r) r[i] = fmaf(-c, ad[i], r[i]);
    }
}

// The same on 4-cell groups (n a multiple of 4).
__global__ void __launch_bounds__(256) line_update4_kernel(uint32_t groups, const double* __restrict__ coef, const float* __restrict__ d,
                                                           const float* __restrict__ ad, const float* x, float* r, float* x_out) {
    const float c = static_cast<float>(coef[0]);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        st4(x_out + i, axpy4(ld4(x + i), c, ld4(d + i)));
        if (r) st4(r + i, axpy4(ld4(r + i), -c, ld4(ad + i)));
    }
}

// A d of a line step's direction and the two products of its coefficient,
// d . A d and d . r, in one pass on the fast path's 4-cell groups: the same
// per-block partials as basis_gram_kernel<1> ([block][2]); FP32 products and
// per-thread sums (a few hundred terms), FP64 across the block.
__global__ void __launch_bounds__(256) line_gram_fast_kernel(FastGeom f, const float* __restrict__ d, const float* __restrict__ r,
                                                             float* __restrict__ ad, double* __restrict__ partials) {
    __shared__ double red[2 * 32];
    float s0 = 0.0f, s1 = 0.0f;  // a thread's own terms in FP32, the block's sums in FP64
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < f.groups; t += gridDim.x * blockDim.x) {
        const uint32_t i = 4u * t;
        float4 c, dg;
        const float4 q = apply4f(f, d, i, c, dg);
        st4(ad + i, q);
        const float4 rv = ld4(r + i);
        s0 = fmaf(c.x, q.x, fmaf(c.y, q.y, fmaf(c.z, q.z, fmaf(c.w, q.w, s0))));
        s1 = fmaf(c.x, rv.x, fmaf(c.y, rv.y, fmaf(c.z, rv.z, fmaf(c.w, rv.w, s1))));
    }
    double acc[2] = {s0, s1};
    block_sum<2>(acc, red);
    if (threadIdx.x == 0) {
        partials[2 * static_cast<size_t>(blockIdx.x)] = acc[0];
        partials[2 * static_cast<size_t>(blockIdx.x) + 1] = acc[1];
    }
}

XsStatus line_step(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const WarmHistory& h,
                   const float* d, const float* x, float* r, float* x_out, bool update_residual) {
    if (!h.meta || !h.extra_product || !d || !x || !r || !x_out) return XS_INVALID_ARGUMENT;
    const Operator op{g, mask, anchor, pb, true};
    const uint64_t n = cell_count(g);
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16));
    XsStatus s;
    if (fast_pass_ok(g, mask, anchor, pb, false)) {
        // A d with the coefficient's products in one pass, then the update
        const FastGeom f = fast_geom(g, anchor, pb);
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((f.groups + 255) / 256, kGramBlocks));
        line_gram_fast_kernel<<<blocks, 256, 0, st>>>(f, d, r, h.extra_product, h.partials);
        if ((s = check_launch()) != XS_OK) return s;
        basis_solve_kernel<1><<<1, 64, 0, st>>>(h.partials, blocks, h.coef);
        if ((s = check_launch()) != XS_OK) return s;
        line_update4_kernel<<<fast_pass_blocks(g), 256, 0, st>>>(f.groups, h.coef, d, h.extra_product, x, update_residual ? r : nullptr, x_out);
        return check_launch();
    }
    apply_operator_kernel<<<grid, 256, 0, st>>>(op, d, h.extra_product);
    if ((s = check_launch()) != XS_OK) return s;
    // the Galerkin machinery with the one vector d and b = r (r already holds
    // the fixed boundary values; r and A d vanish on inactive cells):
    // coef = (d . r) / (d . A d)
    BasisArgs<1> a{};
    a.op = op;
    a.v[0] = d;
    a.w[0] = h.extra_product;
    a.history = 0;
    a.meta = h.meta;
    a.rhs = r;
    a.rhs_d = nullptr;
    a.partials = h.partials;
    a.fixed_terms = 0u;
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, kGramBlocks));
    basis_gram_kernel<1><<<blocks, 256, 0, st>>>(a);
    if ((s = check_launch()) != XS_OK) return s;
    basis_solve_kernel<1><<<1, 64, 0, st>>>(h.partials, blocks, h.coef);
    if ((s = check_launch()) != XS_OK) return s;
    line_update_kernel<<<grid, 256, 0, st>>>(n, h.coef, d, h.extra_product, x, update_residual ? r : nullptr, x_out);
    return check_launch();
}

XsStatus coarse_cycles(cudaStream_t st, const Grid& g, uint32_t anchor, const XsScalarBoundary& pb, const WarmHistory& h, const float* rhs,
                       const double* rhs_d, int cycles, const float** out, bool keep_residual) {
    if (cycles < 1 || !out) return XS_INVALID_ARGUMENT;
    const float* x = h.ring_start;
    for (int c = 0; c < cycles; ++c) {
        float* dst = (c % 2 == 0) ? h.start : h.ring_start;  // never x
        XsStatus s;
        if ((s = jacobi_sweeps(st, g, anchor, nullptr, pb, rhs, rhs_d, x, h.extra_product, dst, rhs_d ? kAdjointPreSweeps : kCoarsePreSweeps)) !=
            XS_OK)
            return s;
        if ((s = start_residual(st, g, anchor, nullptr, pb, rhs, dst, h.residual, rhs_d)) != XS_OK) return s;
        if ((s = coarse_correction(st, g, anchor, pb, h, h.residual, c == 0 ? kCoarseMaxIterations : kLaterCoarseIterations)) != XS_OK) return s;
        if ((s = line_step(st, g, anchor, nullptr, pb, h, h.correction, dst, h.residual, dst, keep_residual && c == cycles - 1)) != XS_OK)
            return s;
        x = dst;
    }
    *out = x;
    return XS_OK;
}

XsStatus start_residual(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const float* rhs,
                        const float* x, float* r, const double* rhs_d) {
    const Operator op{g, mask, anchor, pb, rhs_d == nullptr};
    const uint64_t n = cell_count(g);
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16));
    if (fast_pass_ok(g, mask, anchor, pb, rhs_d == nullptr)) {
        const FastGeom f = fast_geom(g, anchor, pb);
        if (rhs_d)
            fast_pass_kernel<kPassResidual, double><<<fast_pass_blocks(g), 256, 0, st>>>(f, x, rhs_d, r, 0.0f);
        else
            fast_pass_kernel<kPassResidual, float><<<fast_pass_blocks(g), 256, 0, st>>>(f, x, rhs, r, 0.0f);
    } else if (rhs_d) {
        start_residual_kernel<double><<<blocks, 256, 0, st>>>(op, rhs_d, x, r);
    } else {
        start_residual_kernel<float><<<blocks, 256, 0, st>>>(op, rhs, x, r);
    }
    return check_launch();
}

XsStatus history_push(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsScalarBoundary& pb, const WarmHistory& h,
                      const float* pressure, const double* pressure64) {
    if (h.history == 0) return XS_OK;
    HistorySlots slots{}, products{};
    for (uint32_t i = 0; i < h.history; ++i) {
        slots.s[i] = h.slots[i];
        products.s[i] = h.products[i];
    }
    const Operator op{g, mask, anchor, pb, pressure64 == nullptr};
    const uint64_t n = cell_count(g);
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 148 * 16));
    if (pressure64 && fast_pass_ok(g, mask, anchor, pb, false))
        fast_push64_kernel<<<fast_pass_blocks(g), 256, 0, st>>>(fast_geom(g, anchor, pb), pressure64, slots, products, h.history, h.meta);
    else if (pressure64)
        history_push_kernel<double><<<blocks, 256, 0, st>>>(op, pressure64, slots, products, h.history, h.meta);
    else if (fast_pass_ok(g, mask, anchor, pb, false))
        fast_push_kernel<<<fast_pass_blocks(g), 256, 0, st>>>(fast_geom(g, anchor, pb), pressure, slots, products, h.history, h.meta);
    else
        history_push_kernel<float><<<blocks, 256, 0, st>>>(op, pressure, slots, products, h.history, h.meta);
    XsStatus s = check_launch();
    if (s != XS_OK) return s;
    history_advance_kernel<<<1, 1, 0, st>>>(h.history, h.meta);
    return check_launch();
}

XsStatus history_reset(cudaStream_t st, const WarmHistory& h) {
    if (h.history == 0 || !h.meta) return XS_OK;
    return check_cuda(cudaMemsetAsync(h.meta, 0, 2 * sizeof(uint32_t), st));
}

XsStatus read_solve_stats(cudaStream_t stream, const void* workspace, const Grid& g, XsSolveStats* out) {
    const PressureWorkspace w = carve_pressure_workspace(const_cast<void*>(workspace), g);
    SolverState host;
    if (cudaMemcpyAsync(&host, w.state, sizeof(SolverState), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return XS_CUDA_ERROR;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return XS_CUDA_ERROR;
    *out = host.stats;
    if (host.error) out->status = XS_TIMEOUT;
    return XS_OK;
}

}  // namespace xs

using namespace xs;

extern "C" {

size_t xs_projection_workspace_bytes(XsGrid grid) {
    if (!valid_grid(grid)) return 0;
    return pressure_workspace_bytes(make_grid(grid));
}

XsStatus xs_pressure_solve(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                           const uint32_t* cell_mask, XsScalarBoundary pressure_boundary, const float* rhs, float* pressure,
                           void* workspace) {
    if (!valid_grid(grid) || !solve || !rhs || !pressure || !workspace) return XS_INVALID_ARGUMENT;
    return solve_pressure(stream, make_grid(grid), *solve, pressure_anchor, cell_mask, pressure_boundary, rhs, nullptr, pressure,
                          nullptr, workspace, nullptr);
}

size_t xs_solve_stats_offset(void) { return offsetof(SolverState, stats); }

XsStatus xs_read_solve_stats(cudaStream_t stream, const void* workspace, XsSolveStats* host_stats) {
    if (!workspace || !host_stats) return XS_INVALID_ARGUMENT;
    const SolverState* st = static_cast<const SolverState*>(workspace);
    SolverState host;
    if (cudaMemcpyAsync(&host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return XS_CUDA_ERROR;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return XS_CUDA_ERROR;
    *host_stats = host.stats;
    if (host.error) host_stats->status = XS_TIMEOUT;
    return XS_OK;
}

}  // extern "C"
