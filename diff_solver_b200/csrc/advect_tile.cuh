// Tile staging for the semi-Lagrangian advection kernels (forward and
// adjoint) on grids without colliders.
//
// A CTA owns a box of TX x TY x TZ output positions (faces or cells with the
// same integer coordinates).  Every trilinear stencil those positions reach
// lies within the positions' box widened by H nodes on every side when the
// trace is shorter than H - 1/2 cells per step (a staggered component is
// sampled half a cell off its nodes); each field the kernel samples is
// copied once into shared memory over that box.  A staged node
// holds exactly the value the boundary-aware loads of the reference return
// for its integer coordinates (load_face / load_scalar: operators.cu:115-134):
// a node beyond the domain takes the fixed boundary value or its clamped /
// wrapped partner.  A stencil read from the box is therefore the stencil
// sample_face / sample_scalar read from global memory, and the samples are
// bit-identical; a stencil outside the box (a trace longer than the halo) is
// read from global memory by the out-of-line boundary-aware path.
//
// The adjoint kernels scatter the transposed trilinear weights into FP64
// accumulators over the same box (shared-memory atomics) and add each
// node's sum to global memory once, applying the reference's scatter rules
// per node (scatter_face / scatter_scalar: operators.cu:196-240): nodes on a
// constant boundary receive nothing, nodes beyond the domain go to their
// clamped / wrapped partner.
//
// Box strides are compile-time constants: a stencil is one base address and
// eight shared loads with immediate offsets.
#pragma once

#include "common.cuh"

namespace xs {
namespace tile {

template <int TX_, int TY_, int TZ_, int H_>
struct Shape {
    static constexpr int TX = TX_, TY = TY_, TZ = TZ_, kHalo = H_;
    static constexpr int kThreads = TX * TY;  // one thread per (x, y), looping over z
    static constexpr int SX = TX + 2 * kHalo, SY = TY + 2 * kHalo, SZ = TZ + 2 * kHalo;
    static constexpr int kNodes = SX * SY * SZ;
    static constexpr int kRows = SY * SZ;
    static constexpr int kRowPasses = (kRows + TY - 1) / TY;  // box rows per warp (the last pass partial)
    static constexpr int stride(int axis) { return axis == 0 ? 1 : (axis == 1 ? SX : SX * SY); }
    static_assert(TX == 32 && SX <= 64, "a box row is staged by one warp in two passes");
};

// Global coordinates of box node (0, 0, 0).
struct Origin {
    int x, y, z;
};

template <class S>
__device__ __forceinline__ Origin tile_origin() {
    return Origin{static_cast<int>(blockIdx.x) * S::TX - S::kHalo, static_cast<int>(blockIdx.y) * S::TY - S::kHalo,
                  static_cast<int>(blockIdx.z) * S::TZ - S::kHalo};
}

// Box offset of the position handled by this thread at z step kz.
template <class S>
__device__ __forceinline__ int local_index(int kz) {
    return (static_cast<int>(threadIdx.x) + S::kHalo) + S::SX * ((static_cast<int>(threadIdx.y) + S::kHalo) + S::SY * (kz + S::kHalo));
}

// Whether the box lies inside an array of the given extents (then every node
// is a plain element).
template <class S>
__device__ __forceinline__ bool box_inside(const Origin& o, int ex, int ey, int ez) {
    return o.x >= 0 && o.y >= 0 && o.z >= 0 && o.x + S::SX <= ex && o.y + S::SY <= ey && o.z + S::SZ <= ez;
}

__device__ __forceinline__ uint32_t index32(int x, int y, int z, int ex, int ey) {
    return static_cast<uint32_t>(x) + static_cast<uint32_t>(ex) * (static_cast<uint32_t>(y) + static_cast<uint32_t>(ey) * static_cast<uint32_t>(z));
}

// Asynchronous 4-byte global -> shared copy (no register round trip): every
// row of every box of a tile is in flight at once instead of one dependent
// load-store per row.  Completed by stage_wait() before the __syncthreads
// that publishes the boxes.
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Stages face component A over the box: one warp per box row (x-contiguous,
// coalesced), two passes for the row's SX nodes.  A box inside the array is
// copied asynchronously by a short unrolled loop; a box that crosses the
// domain edge (rolled loop, one copy of the boundary logic) copies its
// in-array nodes asynchronously and applies the boundary rules to the nodes
// beyond the edge only.  The caller runs stage_wait() and __syncthreads()
// before reading the box.
template <class S, int A>
__device__ __forceinline__ void stage_face(float* __restrict__ s, const float* __restrict__ v, const Origin& o, const Grid& g,
                                           const XsVelocityBoundary& b) {
    const int ex = extent(g, A, 0), ey = extent(g, A, 1), ez = extent(g, A, 2);
    // nodes that are plain elements: inside the array, and inside the wrap
    // period on a periodic axis (there the face at n is the face at 0)
    const int lx = periodic(b, 0) ? g.nx : ex, ly = periodic(b, 1) ? g.ny : ey, lz = periodic(b, 2) ? g.nz : ez;
    const int lane = threadIdx.x, warp = threadIdx.y;
    if (box_inside<S>(o, lx, ly, lz)) {
#pragma unroll
        for (int r = 0; r < S::kRowPasses; ++r) {
            const int row = warp + r * S::TY;
            if (S::kRows % S::TY != 0 && row >= S::kRows) break;
            const float* src = v + index32(o.x, o.y + row % S::SY, o.z + row / S::SY, ex, ey);
            float* dst = s + row * S::SX;
            cp_async4(dst + lane, src + lane);
            if (lane < S::SX - 32) cp_async4(dst + 32 + lane, src + 32 + lane);
        }
        return;
    }
#pragma unroll 1
    for (int row = warp; row < S::kRows; row += S::TY) {
        const int y = o.y + row % S::SY, z = o.z + row / S::SY;
        const bool row_in = static_cast<unsigned>(y) < static_cast<unsigned>(ly) && static_cast<unsigned>(z) < static_cast<unsigned>(lz);
        float* dst = s + row * S::SX;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int bx = lane + 32 * half;
            if (half == 1 && bx >= S::SX) break;
            const int x = o.x + bx;
            if (row_in && static_cast<unsigned>(x) < static_cast<unsigned>(lx))
                cp_async4(dst + bx, v + index32(x, y, z, ex, ey));
            else
                dst[bx] = load_face(v, A, x, y, z, g, b);
        }
    }
}

// The same for a cell-centred field.
template <class S>
__device__ __forceinline__ void stage_cells(float* __restrict__ s, const float* __restrict__ v, const Origin& o, const Grid& g,
                                            const XsScalarBoundary& b) {
    const int lane = threadIdx.x, warp = threadIdx.y;
    if (box_inside<S>(o, g.nx, g.ny, g.nz)) {
#pragma unroll
        for (int r = 0; r < S::kRowPasses; ++r) {
            const int row = warp + r * S::TY;
            if (S::kRows % S::TY != 0 && row >= S::kRows) break;
            const float* src = v + index32(o.x, o.y + row % S::SY, o.z + row / S::SY, g.nx, g.ny);
            float* dst = s + row * S::SX;
            cp_async4(dst + lane, src + lane);
            if (lane < S::SX - 32) cp_async4(dst + 32 + lane, src + 32 + lane);
        }
        return;
    }
#pragma unroll 1
    for (int row = warp; row < S::kRows; row += S::TY) {
        const int y = o.y + row % S::SY, z = o.z + row / S::SY;
        const bool row_in = static_cast<unsigned>(y) < static_cast<unsigned>(g.ny) && static_cast<unsigned>(z) < static_cast<unsigned>(g.nz);
        float* dst = s + row * S::SX;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int bx = lane + 32 * half;
            if (half == 1 && bx >= S::SX) break;
            const int x = o.x + bx;
            if (row_in && static_cast<unsigned>(x) < static_cast<unsigned>(g.nx))
                cp_async4(dst + bx, v + index32(x, y, z, g.nx, g.ny));
            else
                dst[bx] = load_scalar(v, x, y, z, g, b);
        }
    }
}

// Eight stencil nodes from the box, lower corner at box offset c.
template <class S>
__device__ __forceinline__ void box_stencil(const float* __restrict__ s, int c, float (&v8)[2][2][2]) {
    const float* p = s + c;
    v8[0][0][0] = p[0];
    v8[0][0][1] = p[1];
    v8[0][1][0] = p[S::SX];
    v8[0][1][1] = p[S::SX + 1];
    v8[1][0][0] = p[S::SX * S::SY];
    v8[1][0][1] = p[S::SX * S::SY + 1];
    v8[1][1][0] = p[S::SX * S::SY + S::SX];
    v8[1][1][1] = p[S::SX * S::SY + S::SX + 1];
}

// Box offset of a stencil's lower corner, or -1 when the stencil leaves the box.
template <class S>
__device__ __forceinline__ int box_corner(int x0, int y0, int z0, const Origin& o) {
    const unsigned lx = static_cast<unsigned>(x0 - o.x), ly = static_cast<unsigned>(y0 - o.y), lz = static_cast<unsigned>(z0 - o.z);
    if (lx >= static_cast<unsigned>(S::SX - 1) || ly >= static_cast<unsigned>(S::SY - 1) || lz >= static_cast<unsigned>(S::SZ - 1)) return -1;
    return static_cast<int>(lx + S::SX * (ly + S::SY * lz));
}

// Stencils that leave the box: sample_face's own global-memory path, out
// of line.  The tile kernels declare their grid and boundary parameters
// __grid_constant__: a kernel parameter passed out of line by reference
// would otherwise be copied to local memory, and every use of it on the
// common path would read that copy.
static __device__ __noinline__ Sample global_face_sample(const float* __restrict__ v, int axis, Vec3 p, const Grid& g,
                                                         const XsVelocityBoundary& b) {
    return sample_face<true>(v, axis, p, g, b);
}

static __device__ __noinline__ Sample global_scalar_sample(const float* __restrict__ v, Vec3 p, const Grid& g, const XsScalarBoundary& b) {
    return sample_scalar<true>(v, p, g, b);
}

// Per-thread constants of the tile kernels (power-of-two spacing).
struct TileConsts {
    float r;           // 1 / h, exact
    Vec3 extent;       // n h per axis (the trace's clamp)
    bool periodic[3];
};

__device__ __forceinline__ TileConsts tile_consts(const Grid& g, const XsVelocityBoundary& b) {
    return TileConsts{1.0f / g.h, Vec3{g.nx * g.h, g.ny * g.h, g.nz * g.h}, {periodic(b, 0), periodic(b, 1), periodic(b, 2)}};
}

// sample_face<kGradient> (operators.cu:166-194) of face component A with the
// stencil read from its staged box.
template <class S, int A, bool kGradient>
__device__ __forceinline__ Sample staged_face(const float* __restrict__ s, const float* __restrict__ v, const Vec3& p, const Origin& o,
                                              const TileConsts& k, const Grid& g, const XsVelocityBoundary& b) {
    float gx, gy, gz;
    grid_coordinates_pow2(p, k.r, A, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int c = box_corner<S>(x0, y0, z0, o);
    Sample r;
    if (c >= 0) {
        float v8[2][2][2];
        box_stencil<S>(s, c, v8);
        r = trilinear(v8, gx - x0, gy - y0, gz - z0, g.h);
    } else {
        r = global_face_sample(v, A, p, g, b);
    }
    if (kGradient) return r;
    return Sample{r.value, {0.0f, 0.0f, 0.0f}};
}

// sample_scalar<kGradient> (operators.cu:136-164) from a staged box.
template <class S, bool kGradient>
__device__ __forceinline__ Sample staged_scalar(const float* __restrict__ s, const float* __restrict__ v, const Vec3& p, const Origin& o,
                                                const TileConsts& k, const Grid& g, const XsScalarBoundary& b) {
    float gx, gy, gz;
    grid_coordinates_pow2(p, k.r, -1, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int c = box_corner<S>(x0, y0, z0, o);
    Sample r;
    if (c >= 0) {
        float v8[2][2][2];
        box_stencil<S>(s, c, v8);
        r = trilinear(v8, gx - x0, gy - y0, gz - z0, g.h);
    } else {
        r = global_scalar_sample(v, p, g, b);
    }
    if (kGradient) return r;
    return Sample{r.value, {0.0f, 0.0f, 0.0f}};
}

// The three staged face components of the velocity.
struct StagedVelocity {
    const float* s[3];  // boxes
    XsVector u;         // global arrays (stencils outside the boxes)
};

// sample_velocity (operators.cu:242-244) from the boxes, values or samples
// with gradients.
template <class S>
__device__ __forceinline__ Vec3 staged_velocity(const StagedVelocity& sv, const Vec3& p, const Origin& o, const TileConsts& k, const Grid& g,
                                                const XsVelocityBoundary& b) {
    return Vec3{staged_face<S, 0, false>(sv.s[0], sv.u.x, p, o, k, g, b).value, staged_face<S, 1, false>(sv.s[1], sv.u.y, p, o, k, g, b).value,
                staged_face<S, 2, false>(sv.s[2], sv.u.z, p, o, k, g, b).value};
}

// Velocity at the position of face A (integer coordinates at box offset li)
// for a power-of-two spacing, where the trilinear weights there are exact:
// component A is its own node; component B != A is the mean of four nodes
// (weights 1/2 along A and B, 0 / 1 along the third axis).  The non-zero
// terms are summed in the order of trilinear() (x fastest), each product
// 0.25 * v exact, so the value is bit-identical to sample_velocity's.
template <class S, int A, int B>
__device__ __forceinline__ float face_start_component(const float* __restrict__ s, int li) {
    if (A == B) return s[li];
    constexpr int lo = S::stride(A < B ? A : B), hi = S::stride(A < B ? B : A);
    const float* c = s + li - S::stride(A);
    float r = 0.25f * c[0];
    r = fmaf(0.25f, c[lo], r);
    r = fmaf(0.25f, c[hi], r);
    r = fmaf(0.25f, c[lo + hi], r);
    return r;
}

template <class S, int A>
__device__ __forceinline__ Vec3 face_start_velocity(const StagedVelocity& sv, int li) {
    return Vec3{face_start_component<S, A, 0>(sv.s[0], li), face_start_component<S, A, 1>(sv.s[1], li),
                face_start_component<S, A, 2>(sv.s[2], li)};
}

// Velocity at a cell centre (box offset li), power-of-two spacing: component
// B is the mean of the faces at li and li + e_B (weights 1/2, 1/2).
template <class S, int B>
__device__ __forceinline__ float cell_start_component(const float* __restrict__ s, int li) {
    const float r = 0.5f * s[li];
    return fmaf(0.5f, s[li + S::stride(B)], r);
}

template <class S>
__device__ __forceinline__ Vec3 cell_start_velocity(const StagedVelocity& sv, int li) {
    return Vec3{cell_start_component<S, 0>(sv.s[0], li), cell_start_component<S, 1>(sv.s[1], li), cell_start_component<S, 2>(sv.s[2], li)};
}

// The clamp of trace_rk2 (operators.cu:268-270): non-periodic axes clamp to
// the domain and zero that axis' derivative.  Branch-free: inside the domain
// the clamp returns the coordinate itself.
__device__ __forceinline__ float clamp_axis(float v, float hi, bool per, float& der) {
    const bool out = !per && (v < 0.0f || v > hi);
    der = out ? 0.0f : der;
    return per ? v : fminf(fmaxf(v, 0.0f), hi);
}

__device__ __forceinline__ void clamp_trace(Vec3& raw, Vec3& der, const TileConsts& k) {
    raw.x = clamp_axis(raw.x, k.extent.x, k.periodic[0], der.x);
    raw.y = clamp_axis(raw.y, k.extent.y, k.periodic[1], der.y);
    raw.z = clamp_axis(raw.z, k.extent.z, k.periodic[2], der.z);
}

// trace_rk2 (operators.cu:256-276) from the boxes for a domain without
// colliders (no bisection), given the velocity at the start.
template <class S>
__device__ __forceinline__ Vec3 staged_trace(const StagedVelocity& sv, const Vec3& s, const Vec3& v0, const Origin& o, const TileConsts& k,
                                             const Grid& g, const XsVelocityBoundary& b) {
    const Vec3 mid{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    const Vec3 v1 = staged_velocity<S>(sv, mid, o, k, g, b);
    Vec3 raw{s.x - g.dt * v1.x, s.y - g.dt * v1.y, s.z - g.dt * v1.z};
    Vec3 der{1.0f, 1.0f, 1.0f};
    clamp_trace(raw, der, k);
    return raw;
}

// ------------------------------------------------------------ adjoint side
// scatter_face (operators.cu:217-240) of one trilinear stencil into the FP64
// box of component B: the same products adj * wx * wy * wz; stencils outside
// the box go to global memory directly (with the reference's rules).
static __device__ __noinline__ void global_face_scatter(double* __restrict__ v, int axis, Vec3 p, double adj, const Grid& g,
                                                        const XsVelocityBoundary& b) {
    scatter_face(v, axis, p, adj, g, b);
}
static __device__ __noinline__ void global_scalar_scatter(double* __restrict__ v, Vec3 p, double adj, const Grid& g, const XsScalarBoundary& b) {
    scatter_scalar(v, p, adj, g, b);
}

// FP64 add to a shared-memory accumulator (a shared-window address: no
// generic-address resolution per access).
__device__ __forceinline__ void shared_add(double* p, double v) {
    asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))), "d"(v) : "memory");
}

template <class S>
__device__ __forceinline__ void box_scatter(double* __restrict__ acc, int c, double adj, float tx, float ty, float tz) {
    const double wx[2] = {1.0 - tx, static_cast<double>(tx)};
    const double wy[2] = {1.0 - ty, static_cast<double>(ty)};
    const double wz[2] = {1.0 - tz, static_cast<double>(tz)};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) shared_add(acc + c + dx + S::SX * (dy + S::SY * dz), adj * wx[dx] * wy[dy] * wz[dz]);
}

template <class S, int B>
__device__ __forceinline__ void staged_face_scatter(double* __restrict__ acc, double* __restrict__ v, const Vec3& p, double adj, const Origin& o,
                                                    const TileConsts& k, const Grid& g, const XsVelocityBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates_pow2(p, k.r, B, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int c = box_corner<S>(x0, y0, z0, o);
    if (c >= 0)
        box_scatter<S>(acc, c, adj, gx - x0, gy - y0, gz - z0);
    else
        global_face_scatter(v, B, p, adj, g, b);
}

template <class S>
__device__ __forceinline__ void staged_scalar_scatter(double* __restrict__ acc, double* __restrict__ v, const Vec3& p, double adj, const Origin& o,
                                                      const TileConsts& k, const Grid& g, const XsScalarBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates_pow2(p, k.r, -1, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int c = box_corner<S>(x0, y0, z0, o);
    if (c >= 0)
        box_scatter<S>(acc, c, adj, gx - x0, gy - y0, gz - z0);
    else
        global_scalar_scatter(v, p, adj, g, b);
}

// Transpose of face_start_component: scatter at the position of face A into
// component B with the exact weights there (1, or 1/4 on four nodes; the
// zero-weight nodes would receive exact zeros).
template <class S, int A, int B>
__device__ __forceinline__ void face_start_scatter(double* __restrict__ acc, int li, double adj) {
    if (adj == 0.0) return;
    if (A == B) {
        shared_add(acc + li, adj);
        return;
    }
    constexpr int lo = S::stride(A < B ? A : B), hi = S::stride(A < B ? B : A);
    double* c = acc + li - S::stride(A);
    const double w = adj * 0.5 * 0.5;
    shared_add(c, w);
    shared_add(c + lo, w);
    shared_add(c + hi, w);
    shared_add(c + lo + hi, w);
}

// Transpose of cell_start_component.
template <class S, int B>
__device__ __forceinline__ void cell_start_scatter(double* __restrict__ acc, int li, double adj) {
    if (adj == 0.0) return;
    const double w = adj * 0.5;
    shared_add(acc + li, w);
    shared_add(acc + li + S::stride(B), w);
}

template <class S>
__device__ __forceinline__ void zero_box(double* __restrict__ acc) {
    const int t = threadIdx.x + S::TX * threadIdx.y;
    for (int k = t; k < S::kNodes; k += S::kThreads) acc[k] = 0.0;
}

// Adds the box sums of face component A to global memory: one atomic per
// non-zero node; nodes beyond the domain follow scatter_face's rules.
template <class S, int A>
__device__ __forceinline__ void flush_face(const double* __restrict__ acc, double* __restrict__ v, const Origin& o, const Grid& g,
                                           const XsVelocityBoundary& b) {
    const int ex = extent(g, A, 0), ey = extent(g, A, 1), ez = extent(g, A, 2);
    // plain elements only inside the wrap period on a periodic axis (there the
    // face at n is the face at 0)
    const bool inside = box_inside<S>(o, periodic(b, 0) ? g.nx : ex, periodic(b, 1) ? g.ny : ey, periodic(b, 2) ? g.nz : ez);
    const int t = threadIdx.x + S::TX * threadIdx.y;
    for (int k = t; k < S::kNodes; k += S::kThreads) {
        const double s = acc[k];
        if (s == 0.0) continue;
        const int x = o.x + k % S::SX, y = o.y + (k / S::SX) % S::SY, z = o.z + k / (S::SX * S::SY);
        if (inside) {
            atomicAdd(v + index32(x, y, z, ex, ey), s);
            continue;
        }
        float unused;
        if (face_constant(A, x, y, z, g, b, unused)) continue;
        atomicAdd(v + mapped_face(x, y, z, g, A, b), s);
    }
}

// The same for a cell-centred field (scatter_scalar's rules, operators.cu:196-215).
template <class S>
__device__ __forceinline__ void flush_cells(const double* __restrict__ acc, double* __restrict__ v, const Origin& o, const Grid& g,
                                            const XsScalarBoundary& b) {
    const bool inside = box_inside<S>(o, g.nx, g.ny, g.nz);
    const int t = threadIdx.x + S::TX * threadIdx.y;
    for (int k = t; k < S::kNodes; k += S::kThreads) {
        const double s = acc[k];
        if (s == 0.0) continue;
        const int x = o.x + k % S::SX, y = o.y + (k / S::SX) % S::SY, z = o.z + k / (S::SX * S::SY);
        if (inside) {
            atomicAdd(v + index32(x, y, z, g.nx, g.ny), s);
            continue;
        }
        if ((x < 0 && b.modes[0] == 0u) || (beyond(x, g.nx) && b.modes[1] == 0u) || (y < 0 && b.modes[2] == 0u) ||
            (beyond(y, g.ny) && b.modes[3] == 0u) || (z < 0 && b.modes[4] == 0u) || (beyond(z, g.nz) && b.modes[5] == 0u))
            continue;
        atomicAdd(v + mapped_cell(x, y, z, g, periodic(b, 0), periodic(b, 1), periodic(b, 2)), s);
    }
}

// ------------------------------------------------ runtime face component
// The face component as a runtime value: the adjoint kernel loops over the
// three components with one copy of its per-face body (three unrolled
// copies of a body that large stall on instruction fetch).  The same
// arithmetic as the compile-time forms above.
template <class S>
__device__ __forceinline__ int stride_rt(int a) { return a == 0 ? 1 : (a == 1 ? S::SX : S::SX * S::SY); }

template <class S, int B>
__device__ __forceinline__ float face_start_component_rt(const float* __restrict__ s, int li, int A) {
    if (A == B) return s[li];
    const int lo = stride_rt<S>(A < B ? A : B), hi = stride_rt<S>(A < B ? B : A);
    const float* c = s + li - stride_rt<S>(A);
    float r = 0.25f * c[0];
    r = fmaf(0.25f, c[lo], r);
    r = fmaf(0.25f, c[hi], r);
    r = fmaf(0.25f, c[lo + hi], r);
    return r;
}

template <class S>
__device__ __forceinline__ Vec3 face_start_velocity_rt(const StagedVelocity& sv, int li, int A) {
    return Vec3{face_start_component_rt<S, 0>(sv.s[0], li, A), face_start_component_rt<S, 1>(sv.s[1], li, A),
                face_start_component_rt<S, 2>(sv.s[2], li, A)};
}

template <class S, int B>
__device__ __forceinline__ void face_start_scatter_rt(double* __restrict__ acc, int li, int A, double adj) {
    if (adj == 0.0) return;
    if (A == B) {
        shared_add(acc + li, adj);
        return;
    }
    const int lo = stride_rt<S>(A < B ? A : B), hi = stride_rt<S>(A < B ? B : A);
    double* c = acc + li - stride_rt<S>(A);
    const double w = adj * 0.5 * 0.5;
    shared_add(c, w);
    shared_add(c + lo, w);
    shared_add(c + hi, w);
    shared_add(c + lo + hi, w);
}

// staged_face<S, A, true> with A at run time
template <class S>
__device__ __forceinline__ Sample staged_face_rt(const float* __restrict__ s, const float* __restrict__ v, int A, const Vec3& p, const Origin& o,
                                                 const TileConsts& k, const Grid& g, const XsVelocityBoundary& b) {
    float gx, gy, gz;
    grid_coordinates_pow2(p, k.r, A, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int c = box_corner<S>(x0, y0, z0, o);
    if (c >= 0) {
        float v8[2][2][2];
        box_stencil<S>(s, c, v8);
        return trilinear(v8, gx - x0, gy - y0, gz - z0, g.h);
    }
    return global_face_sample(v, A, p, g, b);
}

// staged_face_scatter<S, B> with B at run time
template <class S>
__device__ __forceinline__ void staged_face_scatter_rt(double* __restrict__ acc, double* __restrict__ v, int B, const Vec3& p, double adj,
                                                       const Origin& o, const TileConsts& k, const Grid& g, const XsVelocityBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates_pow2(p, k.r, B, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int c = box_corner<S>(x0, y0, z0, o);
    if (c >= 0)
        box_scatter<S>(acc, c, adj, gx - x0, gy - y0, gz - z0);
    else
        global_face_scatter(v, B, p, adj, g, b);
}

// ------------------------------------------------------------ dispatch
// Whether the tile kernels apply: no collider mask (no bisection, no solid
// faces) and a power-of-two spacing (exact start weights).
inline bool tiled_advection(const Grid& g, const uint32_t* mask) {
    uint32_t bits;
    static_assert(sizeof(bits) == sizeof(g.h), "");
    __builtin_memcpy(&bits, &g.h, sizeof(bits));
    return mask == nullptr && (bits & 0x007FFFFFu) == 0u;
}

template <class S>
inline dim3 tile_grid(const Grid& g) {
    return dim3(static_cast<unsigned>((g.nx + S::TX - 1) / S::TX), static_cast<unsigned>((g.ny + S::TY - 1) / S::TY),
                static_cast<unsigned>((g.nz + S::TZ - 1) / S::TZ));
}

template <class S>
inline dim3 tile_block() {
    return dim3(S::TX, S::TY);
}

}  // namespace tile
}  // namespace xs
