// Shared device helpers of the smoke kernels: MAC-grid indexing, boundary
// handling, trilinear sampling and the RK2 backtrace.
//
// The semantics follow the reference helpers in solvers/smoke/operators.cu
// (cited per function); boundary modes and packing are the reference's
// (data.ixx:14-25, operators.cpp:85-105).  Everything here is header-only
// and __forceinline__ so each kernel specialises it.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "diff_smoke.h"

namespace xs {

constexpr int kBlock = 256;

// Launch accounting (read through xs_launch_count).
void count_launch();

struct Grid {
    int nx, ny, nz;
    float h, dt;
};

__host__ __device__ __forceinline__ Grid make_grid(const XsGrid& g) {
    return Grid{static_cast<int>(g.nx), static_cast<int>(g.ny), static_cast<int>(g.nz), g.cell_size, g.time_step};
}

struct Vec3 {
    float x, y, z;
};

struct Sample {
    float value;
    Vec3 gradient;
};

struct Trace {
    Vec3 position;
    Vec3 derivative;
};

__host__ __device__ __forceinline__ uint64_t cell_count(const Grid& g) {
    return static_cast<uint64_t>(g.nx) * g.ny * g.nz;
}

// operators.cu:36-39
__host__ __device__ __forceinline__ int extent(const Grid& g, int axis, int dim) {
    const int base = dim == 0 ? g.nx : (dim == 1 ? g.ny : g.nz);
    return base + (axis == dim ? 1 : 0);
}

// operators.cu:41-43
__host__ __device__ __forceinline__ uint64_t face_count(const Grid& g, int axis) {
    return static_cast<uint64_t>(extent(g, axis, 0)) * extent(g, axis, 1) * extent(g, axis, 2);
}

// operators.cu:45-47
__host__ __device__ __forceinline__ uint64_t idx3(int x, int y, int z, int nx, int ny) {
    return static_cast<uint64_t>(x) + static_cast<uint64_t>(nx) * (static_cast<uint64_t>(y) + static_cast<uint64_t>(ny) * z);
}

// operators.cu:49-54.  Every cell or face index of a valid grid is below
// 2^32 (the extents' product with +1 on each axis is checked on the host), so
// the divisions run in 32 bits (64-bit integer division is a long software
// sequence on the GPU).
__device__ __forceinline__ void decode(uint64_t i, int nx, int ny, int& x, int& y, int& z) {
    const uint32_t i32 = static_cast<uint32_t>(i);
    const uint32_t yz = i32 / static_cast<uint32_t>(nx);
    x = static_cast<int>(i32 - yz * static_cast<uint32_t>(nx));
    const uint32_t zz = yz / static_cast<uint32_t>(ny);
    y = static_cast<int>(yz - zz * static_cast<uint32_t>(ny));
    z = static_cast<int>(zz);
}

__device__ __forceinline__ bool in_grid(const Grid& g, int x, int y, int z) {
    return x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz;
}

template <class T>
__host__ __device__ __forceinline__ T* component(T* x, T* y, T* z, int axis) {
    return axis == 0 ? x : (axis == 1 ? y : z);
}

// operators.cu:80-86
__device__ __forceinline__ bool periodic(const XsVelocityBoundary& b, int d) {
    return b.modes[2 * d] == 3u && b.modes[2 * d + 1] == 3u;
}
__device__ __forceinline__ bool periodic(const XsScalarBoundary& b, int d) {
    return b.modes[2 * d] == 2u && b.modes[2 * d + 1] == 2u;
}

// operators.cu:88-96
__device__ __forceinline__ int wrap(int v, int p) {
    const int r = v % p;
    return r < 0 ? r + p : r;
}
__device__ __forceinline__ int map_coordinate(int v, int size, bool per, int period) {
    return per ? wrap(v, period) : max(0, min(size - 1, v));
}

__device__ __forceinline__ bool is_solid(const uint32_t* mask, uint64_t i) {
    return mask != nullptr && __ldg(mask + i) != 0u;
}

// operators.cu:98-103
__device__ __forceinline__ uint64_t mapped_cell(int x, int y, int z, const Grid& g, bool px, bool py, bool pz) {
    return idx3(map_coordinate(x, g.nx, px, g.nx), map_coordinate(y, g.ny, py, g.ny), map_coordinate(z, g.nz, pz, g.nz), g.nx, g.ny);
}

// operators.cu:105-113
__device__ __forceinline__ uint64_t mapped_face(int x, int y, int z, const Grid& g, int axis, const XsVelocityBoundary& b) {
    const int ex = extent(g, axis, 0), ey = extent(g, axis, 1), ez = extent(g, axis, 2);
    return idx3(map_coordinate(x, ex, periodic(b, 0), g.nx), map_coordinate(y, ey, periodic(b, 1), g.ny),
                map_coordinate(z, ez, periodic(b, 2), g.nz), ex, ey);
}

// The reference compares int coordinates with the grid's uint32_t extents
// (cuda_types.h:13-19): `x >= grid.nx` is then also true for x < 0, and
// `max(0, min(grid.nx - 1, x))` clamps as unsigned, sending x = -1 to nx - 1.
// Both behaviours are part of its results and are kept here.
__device__ __forceinline__ bool beyond(int c, int n) { return static_cast<unsigned>(c) >= static_cast<unsigned>(n); }
__device__ __forceinline__ int uclamp(int c, int n) { return static_cast<int>(umin(static_cast<unsigned>(c), static_cast<unsigned>(n - 1))); }

// operators.cu:115-123: value of a cell-centred field, boundary aware.
__device__ __forceinline__ float load_scalar(const float* __restrict__ v, int x, int y, int z, const Grid& g, const XsScalarBoundary& b) {
    if (x < 0 && b.modes[0] == 0u) return b.values[0];
    if (beyond(x, g.nx) && b.modes[1] == 0u) return b.values[1];
    if (y < 0 && b.modes[2] == 0u) return b.values[2];
    if (beyond(y, g.ny) && b.modes[3] == 0u) return b.values[3];
    if (z < 0 && b.modes[4] == 0u) return b.values[4];
    if (beyond(z, g.nz) && b.modes[5] == 0u) return b.values[5];
    return __ldg(v + mapped_cell(x, y, z, g, periodic(b, 0), periodic(b, 1), periodic(b, 2)));
}

// operators.cu:125-134: value of one face component, boundary aware.  A face
// outside the grid along a fixed-value face (or the normal component at a
// normal-fixed face) reads the boundary value of the first such dimension.
__device__ __forceinline__ bool face_constant(int axis, int x, int y, int z, const Grid& g, const XsVelocityBoundary& b, float& value) {
    const int c[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int size = extent(g, axis, d);
        if (c[d] >= 0 && c[d] < size) continue;
        const int face = 2 * d + (c[d] >= size);
        if (b.modes[face] == 0u || (b.modes[face] == 2u && axis == d)) {
            value = b.values[3 * face + axis];
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ float load_face(const float* __restrict__ v, int axis, int x, int y, int z, const Grid& g,
                                           const XsVelocityBoundary& b) {
    float value;
    if (face_constant(axis, x, y, z, g, b, value)) return value;
    return __ldg(v + mapped_face(x, y, z, g, axis, b));
}

// Division by the spacing h; for a power-of-two h the product with its exact
// reciprocal, which is the same IEEE result (see grid_coordinates below).
struct SpacingDivider {
    float h, r;
    bool pow2;
    __device__ __forceinline__ float operator()(float v) const { return pow2 ? v * r : v / h; }
};
__device__ __forceinline__ SpacingDivider spacing_divider(float h) {
    SpacingDivider d;
    d.h = h;
    d.r = 1.0f / h;
    d.pow2 = (__float_as_uint(h) & 0x007FFFFFu) == 0u;
    return d;
}

// Trilinear value and gradient of an 8-value cell (operators.cu:150-163).
__device__ __forceinline__ Sample trilinear(const float v[2][2][2], float tx, float ty, float tz, float h) {
    const float wx[2] = {1.0f - tx, tx}, wy[2] = {1.0f - ty, ty}, wz[2] = {1.0f - tz, tz};
    const SpacingDivider over_h = spacing_divider(h);
    Sample s{0.0f, {0.0f, 0.0f, 0.0f}};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) s.value += wx[dx] * wy[dy] * wz[dz] * v[dz][dy][dx];
            s.gradient.x += over_h(wy[dy] * wz[dz] * (v[dz][dy][1] - v[dz][dy][0]));
        }
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) s.gradient.y += over_h(wx[dx] * wz[dz] * (v[dz][1][dx] - v[dz][0][dx]));
    }
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) s.gradient.z += over_h(wx[dx] * wy[dy] * (v[1][dy][dx] - v[0][dy][dx]));
    return s;
}

// Grid coordinates of a sample point for a cell-centred field (offset 0.5
// on every axis) or face component `axis` (offset 0 along axis).
// A power-of-two spacing has an exact reciprocal, and both IEEE operations
// round the same exact quotient: p * (1/h) is then bit-identical to p / h at
// one multiply instead of a division sequence (the advection kernels issue
// 21 of these per face and are instruction-issue bound).  Other spacings
// divide.
// With the exact reciprocal r = 1/h of a power-of-two spacing given (the
// tile kernels compute it once per thread):
__device__ __forceinline__ void grid_coordinates_pow2(const Vec3& p, float r, int axis, float& gx, float& gy, float& gz) {
    const float x = p.x * r, y = p.y * r, z = p.z * r;
    gx = x - (axis == 0 ? 0.0f : 0.5f);
    gy = y - (axis == 1 ? 0.0f : 0.5f);
    gz = z - (axis == 2 ? 0.0f : 0.5f);
}

__device__ __forceinline__ void grid_coordinates(const Vec3& p, float h, int axis, float& gx, float& gy, float& gz) {
    if ((__float_as_uint(h) & 0x007FFFFFu) == 0u) {
        grid_coordinates_pow2(p, 1.0f / h, axis, gx, gy, gz);
        return;
    }
    const float x = p.x / h, y = p.y / h, z = p.z / h;
    gx = x - (axis == 0 ? 0.0f : 0.5f);
    gy = y - (axis == 1 ? 0.0f : 0.5f);
    gz = z - (axis == 2 ? 0.0f : 0.5f);
}

// True when the 2x2x2 stencil with lower corner (x0, y0, z0) lies inside an
// array whose rows run to lx, ly, lz with no boundary rule involved: then
// load_scalar / load_face return plain array elements, and the stencil is
// read with 32-bit offsets and no per-node boundary logic (the same values,
// so the same results).  lx etc. are the array extents, or the wrap period
// on a periodic axis.
__device__ __forceinline__ bool interior_stencil(int x0, int y0, int z0, int lx, int ly, int lz) {
    return static_cast<unsigned>(x0) + 1u < static_cast<unsigned>(lx) && static_cast<unsigned>(y0) + 1u < static_cast<unsigned>(ly) &&
           static_cast<unsigned>(z0) + 1u < static_cast<unsigned>(lz) && x0 >= 0 && y0 >= 0 && z0 >= 0;
}

__device__ __forceinline__ void load_stencil(const float* __restrict__ v, int x0, int y0, int z0, int ex, int ey, float (&v8)[2][2][2]) {
    const uint32_t sy = static_cast<uint32_t>(ex), sz = static_cast<uint32_t>(ex) * static_cast<uint32_t>(ey);
    const float* c = v + (static_cast<uint32_t>(x0) + sy * static_cast<uint32_t>(y0) + sz * static_cast<uint32_t>(z0));
    v8[0][0][0] = __ldg(c);
    v8[0][0][1] = __ldg(c + 1);
    v8[0][1][0] = __ldg(c + sy);
    v8[0][1][1] = __ldg(c + sy + 1);
    v8[1][0][0] = __ldg(c + sz);
    v8[1][0][1] = __ldg(c + sz + 1);
    v8[1][1][0] = __ldg(c + sz + sy);
    v8[1][1][1] = __ldg(c + sz + sy + 1);
}

// Boundary-aware samples (stencils that reach past the domain edge or wrap).
// Only samples near the edge take them; they stay out of line so that the
// gather loops of the advection kernels fit the instruction cache (inlined
// eight times per sample they made the kernels instruction-fetch bound).
// They return the whole sample by value: a stencil array passed out of line
// by reference would live in local memory on the interior path as well.  The
// kernels that reach them declare their grid and boundary parameters
// __grid_constant__, so the references here point into the parameter bank
// instead of forcing a local copy of those structs.
static __device__ __noinline__ Sample edge_scalar_sample(const float* __restrict__ v, int x0, int y0, int z0, float tx, float ty, float tz,
                                                         const Grid& g, const XsScalarBoundary& b) {
    float v8[2][2][2];
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) v8[dz][dy][dx] = load_scalar(v, x0 + dx, y0 + dy, z0 + dz, g, b);
    return trilinear(v8, tx, ty, tz, g.h);
}

static __device__ __noinline__ Sample edge_face_sample(const float* __restrict__ v, int axis, int x0, int y0, int z0, float tx, float ty,
                                                       float tz, const Grid& g, const XsVelocityBoundary& b) {
    float v8[2][2][2];
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) v8[dz][dy][dx] = load_face(v, axis, x0 + dx, y0 + dy, z0 + dz, g, b);
    return trilinear(v8, tx, ty, tz, g.h);
}

// operators.cu:136-164
template <bool kGradient>
__device__ __forceinline__ Sample sample_scalar(const float* __restrict__ v, const Vec3& p, const Grid& g, const XsScalarBoundary& b) {
    float gx, gy, gz;
    grid_coordinates(p, g.h, -1, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    Sample r;
    if (interior_stencil(x0, y0, z0, g.nx, g.ny, g.nz)) {
        float v8[2][2][2];
        load_stencil(v, x0, y0, z0, g.nx, g.ny, v8);
        r = trilinear(v8, gx - x0, gy - y0, gz - z0, g.h);
    } else {
        r = edge_scalar_sample(v, x0, y0, z0, gx - x0, gy - y0, gz - z0, g, b);
    }
    if (kGradient) return r;
    return Sample{r.value, {0.0f, 0.0f, 0.0f}};
}

// operators.cu:166-194
template <bool kGradient>
__device__ __forceinline__ Sample sample_face(const float* __restrict__ v, int axis, const Vec3& p, const Grid& g,
                                              const XsVelocityBoundary& b) {
    float gx, gy, gz;
    grid_coordinates(p, g.h, axis, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const int ex = extent(g, axis, 0), ey = extent(g, axis, 1), ez = extent(g, axis, 2);
    Sample r;
    if (interior_stencil(x0, y0, z0, periodic(b, 0) ? g.nx : ex, periodic(b, 1) ? g.ny : ey, periodic(b, 2) ? g.nz : ez)) {
        float v8[2][2][2];
        load_stencil(v, x0, y0, z0, ex, ey, v8);
        r = trilinear(v8, gx - x0, gy - y0, gz - z0, g.h);
    } else {
        r = edge_face_sample(v, axis, x0, y0, z0, gx - x0, gy - y0, gz - z0, g, b);
    }
    if (kGradient) return r;
    return Sample{r.value, {0.0f, 0.0f, 0.0f}};
}

// operators.cu:242-244
__device__ __forceinline__ Vec3 sample_velocity(const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
                                                const Vec3& p, const Grid& g, const XsVelocityBoundary& b) {
    return Vec3{sample_face<false>(ux, 0, p, g, b).value, sample_face<false>(uy, 1, p, g, b).value,
                sample_face<false>(uz, 2, p, g, b).value};
}

// operators.cu:246-254
__device__ __forceinline__ bool solid_at(Vec3 p, const uint32_t* mask, const Grid& g, const XsVelocityBoundary& b) {
    if (mask == nullptr) return false;
    if (periodic(b, 0)) p.x -= floorf(p.x / (g.nx * g.h)) * g.nx * g.h;
    if (periodic(b, 1)) p.y -= floorf(p.y / (g.ny * g.h)) * g.ny * g.h;
    if (periodic(b, 2)) p.z -= floorf(p.z / (g.nz * g.h)) * g.nz * g.h;
    const int x = uclamp(static_cast<int>(floorf(p.x / g.h)), g.nx);
    const int y = uclamp(static_cast<int>(floorf(p.y / g.h)), g.ny);
    const int z = uclamp(static_cast<int>(floorf(p.z / g.h)), g.nz);
    return __ldg(mask + idx3(x, y, z, g.nx, g.ny)) != 0u;
}

// operators.cu:256-276: RK2 midpoint backtrace.  Non-periodic axes clamp to
// the domain and zero that axis' derivative; a trace ending in a solid cell
// is bisected 8 times along the segment from the start.
__device__ __forceinline__ Trace trace_rk2(const Vec3& s, const float* __restrict__ ux, const float* __restrict__ uy,
                                           const float* __restrict__ uz, const uint32_t* mask, const Grid& g,
                                           const XsVelocityBoundary& b) {
    const Vec3 v0 = sample_velocity(ux, uy, uz, s, g, b);
    const Vec3 mid{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    const Vec3 v1 = sample_velocity(ux, uy, uz, mid, g, b);
    Vec3 raw{s.x - g.dt * v1.x, s.y - g.dt * v1.y, s.z - g.dt * v1.z};
    Vec3 der{1.0f, 1.0f, 1.0f};
    const Vec3 mx{g.nx * g.h, g.ny * g.h, g.nz * g.h};
    if (!periodic(b, 0) && (raw.x < 0.0f || raw.x > mx.x)) { raw.x = fminf(fmaxf(raw.x, 0.0f), mx.x); der.x = 0.0f; }
    if (!periodic(b, 1) && (raw.y < 0.0f || raw.y > mx.y)) { raw.y = fminf(fmaxf(raw.y, 0.0f), mx.y); der.y = 0.0f; }
    if (!periodic(b, 2) && (raw.z < 0.0f || raw.z > mx.z)) { raw.z = fminf(fmaxf(raw.z, 0.0f), mx.z); der.z = 0.0f; }
    if (!solid_at(raw, mask, g, b)) return Trace{raw, der};
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 8; ++it) {
        const float f = 0.5f * (lo + hi);
        const Vec3 t{s.x + f * (raw.x - s.x), s.y + f * (raw.y - s.y), s.z + f * (raw.z - s.z)};
        if (solid_at(t, mask, g, b)) hi = f; else lo = f;
    }
    return Trace{Vec3{s.x + lo * (raw.x - s.x), s.y + lo * (raw.y - s.y), s.z + lo * (raw.z - s.z)},
                 Vec3{lo * der.x, lo * der.y, lo * der.z}};
}

// operators.cu:278-284
__device__ __forceinline__ Vec3 face_position(int axis, int x, int y, int z, const Grid& g) {
    return Vec3{(x + (axis == 0 ? 0.0f : 0.5f)) * g.h, (y + (axis == 1 ? 0.0f : 0.5f)) * g.h, (z + (axis == 2 ? 0.0f : 0.5f)) * g.h};
}
__device__ __forceinline__ Vec3 cell_position(int x, int y, int z, const Grid& g) {
    return Vec3{(x + 0.5f) * g.h, (y + 0.5f) * g.h, (z + 0.5f) * g.h};
}

// Transposes of the trilinear gathers (FP64 atomics), the reference's
// scatter_scalar / scatter_face (operators.cu:196-240): nodes on a constant
// boundary receive nothing, nodes beyond the domain go to their clamped or
// wrapped partner.
__device__ __forceinline__ void scatter_scalar(double* v, const Vec3& p, double adj, const Grid& g, const XsScalarBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates(p, g.h, -1, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const double wx[2] = {1.0 - (gx - x0), static_cast<double>(gx - x0)};
    const double wy[2] = {1.0 - (gy - y0), static_cast<double>(gy - y0)};
    const double wz[2] = {1.0 - (gz - z0), static_cast<double>(gz - z0)};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = x0 + dx, y = y0 + dy, z = z0 + dz;
                if ((x < 0 && b.modes[0] == 0u) || (beyond(x, g.nx) && b.modes[1] == 0u) || (y < 0 && b.modes[2] == 0u) ||
                    (beyond(y, g.ny) && b.modes[3] == 0u) || (z < 0 && b.modes[4] == 0u) || (beyond(z, g.nz) && b.modes[5] == 0u))
                    continue;
                atomicAdd(v + mapped_cell(x, y, z, g, periodic(b, 0), periodic(b, 1), periodic(b, 2)), adj * wx[dx] * wy[dy] * wz[dz]);
            }
}

// operators.cu:217-240
__device__ __forceinline__ void scatter_face(double* v, int axis, const Vec3& p, double adj, const Grid& g, const XsVelocityBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates(p, g.h, axis, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const double wx[2] = {1.0 - (gx - x0), static_cast<double>(gx - x0)};
    const double wy[2] = {1.0 - (gy - y0), static_cast<double>(gy - y0)};
    const double wz[2] = {1.0 - (gz - z0), static_cast<double>(gz - z0)};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int c[3] = {x0 + dx, y0 + dy, z0 + dz};
                bool constant = false;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int size = extent(g, axis, d);
                    if (c[d] >= 0 && c[d] < size) continue;
                    const int face = 2 * d + (c[d] >= size);
                    if (b.modes[face] == 0u || (b.modes[face] == 2u && axis == d)) constant = true;
                }
                if (!constant) atomicAdd(v + mapped_face(c[0], c[1], c[2], g, axis, b), adj * wx[dx] * wy[dy] * wz[dz]);
            }
}

// Inflow spheres travel as a kernel parameter.
struct InflowSet {
    uint32_t count;
    XsInflow items[XS_MAX_INFLOWS];
};

// Index of the last inflow containing cell (x,y,z), or -1.
__device__ __forceinline__ int inflow_hit(const InflowSet& f, int x, int y, int z, const Grid& g) {
    if (f.count == 0) return -1;
    const Vec3 p = cell_position(x, y, z, g);
    int hit = -1;
    for (uint32_t k = 0; k < f.count; ++k) {
        const float dx = p.x - f.items[k].center[0], dy = p.y - f.items[k].center[1], dz = p.z - f.items[k].center[2];
        const float r = f.items[k].radius;
        if (dx * dx + dy * dy + dz * dz <= r * r) hit = static_cast<int>(k);
    }
    return hit;
}

// Zeroed copies of boundary values, for tangents (operators.cu:396-397, 516-519).
__device__ __forceinline__ XsVelocityBoundary zero_values(XsVelocityBoundary b) {
#pragma unroll
    for (int i = 0; i < 18; ++i) b.values[i] = 0.0f;
    return b;
}
__device__ __forceinline__ XsScalarBoundary zero_values(XsScalarBoundary b) {
#pragma unroll
    for (int i = 0; i < 6; ++i) b.values[i] = 0.0f;
    return b;
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of K (<= 4) doubles; the result is valid in every thread.
template <int K>
__device__ __forceinline__ void block_sum(double* v, double* smem /* [4][32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) smem[k * 32 + warp] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double t = lane < nw ? smem[k * 32 + lane] : 0.0;
        v[k] = warp_sum(t);
    }
    __syncthreads();
}

inline unsigned blocks_for(uint64_t n, int block = kBlock) {
    return static_cast<unsigned>((n + block - 1) / block);
}

}  // namespace xs
