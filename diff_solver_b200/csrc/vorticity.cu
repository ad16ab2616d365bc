// Vorticity confinement forward, tangent and adjoint
// (solvers/smoke/operators.cu:660-846, 973-1002).
//
// The cache is 11 consecutive N-float arrays: centred velocity (3),
// vorticity (3), |vorticity| (1), normal (3), normalizer (1).  The forward
// pass fuses the centred-velocity and curl kernels (the curl reads centred
// velocities at the six neighbours, recomputed from faces), and the adjoint
// is written in gather form: every cell pulls the contributions its
// neighbours would have scattered (operators.cu:669-674, 791-846), so no
// atomics are needed and results are deterministic.
#include "common.cuh"
#include "launch.cuh"
#include "ops.cuh"

namespace xs {

constexpr float kSmoothEpsilon = 1.0e-6f;

struct VortCache {
    float *cx, *cy, *cz, *wx, *wy, *wz, *mag, *nx, *ny, *nz, *norm;
};

__host__ __device__ inline VortCache vort_cache(float* base, uint64_t n) {
    return VortCache{base, base + n, base + 2 * n, base + 3 * n, base + 4 * n, base + 5 * n, base + 6 * n,
                     base + 7 * n, base + 8 * n, base + 9 * n, base + 10 * n};
}

// operators.cu:662-667: the reference's clamp mixes uint32_t and int, so a
// coordinate of -1 reads the far side (n - 1); see uclamp.
__device__ __forceinline__ uint64_t clamped(int x, int y, int z, const Grid& g) {
    return idx3(uclamp(x, g.nx), uclamp(y, g.ny), uclamp(z, g.nz), g.nx, g.ny);
}

// Sources of the transposed clamped central difference along axis d for
// cell m at coordinate c (extent n): a cell j reads uclamp(c_j + 1) with
// weight +1 and uclamp(c_j - 1) with weight -1.  Fills up to 4 (j, w).
__device__ __forceinline__ int difference_sources(int x, int y, int z, int d, const Grid& g, uint64_t (&j)[4], double (&w)[4]) {
    const int c = d == 0 ? x : (d == 1 ? y : z);
    const int n = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
    const int64_t stride = d == 0 ? 1 : (d == 1 ? static_cast<int64_t>(g.nx) : static_cast<int64_t>(g.nx) * g.ny);
    const int64_t m = static_cast<int64_t>(idx3(x, y, z, g.nx, g.ny));
    int k = 0;
    if (c >= 1) { j[k] = static_cast<uint64_t>(m - stride); w[k++] = 1.0; }
    if (c + 1 < n) { j[k] = static_cast<uint64_t>(m + stride); w[k++] = -1.0; }
    if (c == n - 1) {
        j[k] = static_cast<uint64_t>(m); w[k++] = 1.0;                    // c_j + 1 = n clamps back to n - 1
        j[k] = static_cast<uint64_t>(m - stride * c); w[k++] = -1.0;    // c_j - 1 = -1 lands on n - 1
    }
    return k;
}

// operators.cu:676-685
__global__ void centered_velocity_kernel(Grid g, const uint32_t* __restrict__ mask, XsVector u, float* __restrict__ cx,
                                         float* __restrict__ cy, float* __restrict__ cz) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { cx[i] = 0.0f; cy[i] = 0.0f; cz[i] = 0.0f; return; }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    cx[i] = 0.5f * (u.x[idx3(x, y, z, g.nx + 1, g.ny)] + u.x[idx3(x + 1, y, z, g.nx + 1, g.ny)]);
    cy[i] = 0.5f * (u.y[idx3(x, y, z, g.nx, g.ny + 1)] + u.y[idx3(x, y + 1, z, g.nx, g.ny + 1)]);
    cz[i] = 0.5f * (u.z[idx3(x, y, z, g.nx, g.ny)] + u.z[idx3(x, y, z + 1, g.nx, g.ny)]);
}

// operators.cu:687-701
__global__ void curl_magnitude_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ cx,
                                      const float* __restrict__ cy, const float* __restrict__ cz, float* __restrict__ wx,
                                      float* __restrict__ wy, float* __restrict__ wz, float* __restrict__ mag) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { wx[i] = 0.0f; wy[i] = 0.0f; wz[i] = 0.0f; mag[i] = kSmoothEpsilon; return; }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const float is = 0.5f / g.h;
    const float a = (__ldg(cz + clamped(x, y + 1, z, g)) - __ldg(cz + clamped(x, y - 1, z, g)) - __ldg(cy + clamped(x, y, z + 1, g)) +
                     __ldg(cy + clamped(x, y, z - 1, g))) * is;
    const float b = (__ldg(cx + clamped(x, y, z + 1, g)) - __ldg(cx + clamped(x, y, z - 1, g)) - __ldg(cz + clamped(x + 1, y, z, g)) +
                     __ldg(cz + clamped(x - 1, y, z, g))) * is;
    const float c = (__ldg(cy + clamped(x + 1, y, z, g)) - __ldg(cy + clamped(x - 1, y, z, g)) - __ldg(cx + clamped(x, y + 1, z, g)) +
                     __ldg(cx + clamped(x, y - 1, z, g))) * is;
    wx[i] = a; wy[i] = b; wz[i] = c;
    mag[i] = sqrtf(a * a + b * b + c * c + kSmoothEpsilon * kSmoothEpsilon);
}

// operators.cu:703-720
__global__ void vorticity_normal_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ mag, float* __restrict__ nx,
                                        float* __restrict__ ny, float* __restrict__ nz, float* __restrict__ norm) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { nx[i] = 0.0f; ny[i] = 0.0f; nz[i] = 0.0f; norm[i] = kSmoothEpsilon; return; }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const float is = 0.5f / g.h;
    const float gx = (__ldg(mag + clamped(x + 1, y, z, g)) - __ldg(mag + clamped(x - 1, y, z, g))) * is;
    const float gy = (__ldg(mag + clamped(x, y + 1, z, g)) - __ldg(mag + clamped(x, y - 1, z, g))) * is;
    const float gz = (__ldg(mag + clamped(x, y, z + 1, g)) - __ldg(mag + clamped(x, y, z - 1, g))) * is;
    const float len = sqrtf(gx * gx + gy * gy + gz * gz + kSmoothEpsilon * kSmoothEpsilon);
    nx[i] = gx / len; ny[i] = gy / len; nz[i] = gz / len; norm[i] = len;
}

// operators.cu:722-729
__global__ void add_vorticity_force_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, const float* __restrict__ conf,
                                           XsVector f) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g) || is_solid(mask, i)) return;
    const float s = __ldg(conf) * g.h;
    f.x[i] += s * (c.ny[i] * c.wz[i] - c.nz[i] * c.wy[i]);
    f.y[i] += s * (c.nz[i] * c.wx[i] - c.nx[i] * c.wz[i]);
    f.z[i] += s * (c.nx[i] * c.wy[i] - c.ny[i] * c.wx[i]);
}

// ------------------------------------------------------------- tangent
// operators.cu:731-735
__global__ void magnitude_tangent_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, VortCache t) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    t.mag[i] = !is_solid(mask, i) ? (c.wx[i] * t.wx[i] + c.wy[i] * t.wy[i] + c.wz[i] * t.wz[i]) / c.mag[i] : 0.0f;
}

// operators.cu:737-753
__global__ void normal_tangent_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, VortCache t) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { t.nx[i] = 0.0f; t.ny[i] = 0.0f; t.nz[i] = 0.0f; return; }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const float is = 0.5f / g.h;
    const float gx = (t.mag[clamped(x + 1, y, z, g)] - t.mag[clamped(x - 1, y, z, g)]) * is;
    const float gy = (t.mag[clamped(x, y + 1, z, g)] - t.mag[clamped(x, y - 1, z, g)]) * is;
    const float gz = (t.mag[clamped(x, y, z + 1, g)] - t.mag[clamped(x, y, z - 1, g)]) * is;
    const float pr = c.nx[i] * gx + c.ny[i] * gy + c.nz[i] * gz;
    t.nx[i] = (gx - c.nx[i] * pr) / c.norm[i];
    t.ny[i] = (gy - c.ny[i] * pr) / c.norm[i];
    t.nz[i] = (gz - c.nz[i] * pr) / c.norm[i];
}

// operators.cu:755-771
__global__ void vorticity_force_tangent_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, VortCache t,
                                               const float* __restrict__ conf, const float* __restrict__ conf_t, XsVector ft) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g) || is_solid(mask, i)) return;
    const float crx = c.ny[i] * c.wz[i] - c.nz[i] * c.wy[i];
    const float cry = c.nz[i] * c.wx[i] - c.nx[i] * c.wz[i];
    const float crz = c.nx[i] * c.wy[i] - c.ny[i] * c.wx[i];
    const float tx = t.ny[i] * c.wz[i] + c.ny[i] * t.wz[i] - t.nz[i] * c.wy[i] - c.nz[i] * t.wy[i];
    const float ty = t.nz[i] * c.wx[i] + c.nz[i] * t.wx[i] - t.nx[i] * c.wz[i] - c.nx[i] * t.wz[i];
    const float tz = t.nx[i] * c.wy[i] + c.nx[i] * t.wy[i] - t.ny[i] * c.wx[i] - c.ny[i] * t.wx[i];
    const float k = __ldg(conf), kt = __ldg(conf_t);
    ft.x[i] += g.h * (kt * crx + k * tx);
    ft.y[i] += g.h * (kt * cry + k * ty);
    ft.z[i] += g.h * (kt * crz + k * tz);
}

// ------------------------------------------------------------- adjoint
struct VortAdj {
    double *cx, *cy, *cz, *wx, *wy, *wz, *mag, *nx, *ny, *nz;
};

__host__ __device__ inline VortAdj vort_adj(double* base, uint64_t n) {
    return VortAdj{base, base + n, base + 2 * n, base + 3 * n, base + 4 * n, base + 5 * n, base + 6 * n, base + 7 * n, base + 8 * n, base + 9 * n};
}

// operators.cu:773-789: per-cell adjoints of normal and vorticity; the
// confinement adjoint is block-reduced (one atomic per block).
__global__ void vorticity_force_reverse_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, const float* __restrict__ conf,
                                               XsAdjointVector fa, VortAdj a, double* __restrict__ conf_adj) {
    __shared__ double red[4 * 32];
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double part[1] = {0.0};
    if (i < cell_count(g)) {
        if (is_solid(mask, i)) {
            a.nx[i] = 0.0; a.ny[i] = 0.0; a.nz[i] = 0.0; a.wx[i] = 0.0; a.wy[i] = 0.0; a.wz[i] = 0.0;
        } else {
            const float crx = c.ny[i] * c.wz[i] - c.nz[i] * c.wy[i];
            const float cry = c.nz[i] * c.wx[i] - c.nx[i] * c.wz[i];
            const float crz = c.nx[i] * c.wy[i] - c.ny[i] * c.wx[i];
            const double s = static_cast<double>(__ldg(conf)) * g.h;
            const double fx = fa.x[i], fy = fa.y[i], fz = fa.z[i];
            part[0] = g.h * (crx * fx + cry * fy + crz * fz);
            a.nx[i] = s * (c.wy[i] * fz - c.wz[i] * fy);
            a.ny[i] = s * (c.wz[i] * fx - c.wx[i] * fz);
            a.nz[i] = s * (c.wx[i] * fy - c.wy[i] * fx);
            a.wx[i] = s * (fy * c.nz[i] - fz * c.ny[i]);
            a.wy[i] = s * (fz * c.nx[i] - fx * c.nz[i]);
            a.wz[i] = s * (fx * c.ny[i] - fy * c.nx[i]);
        }
    }
    block_sum<1>(part, red);
    if (threadIdx.x == 0 && part[0] != 0.0) atomicAdd(conf_adj, part[0]);
}

// Gradient adjoint of cell j for the normal (operators.cu:796-799).
__device__ __forceinline__ void normal_gradient_adjoint(const VortCache& c, const VortAdj& a, uint64_t j, double& gx, double& gy, double& gz) {
    const double pr = c.nx[j] * a.nx[j] + c.ny[j] * a.ny[j] + c.nz[j] * a.nz[j];
    gx = (a.nx[j] - c.nx[j] * pr) / c.norm[j];
    gy = (a.ny[j] - c.ny[j] * pr) / c.norm[j];
    gz = (a.nz[j] - c.nz[j] * pr) / c.norm[j];
}

// operators.cu:791-807 gathered, then :809-816 applied: every fluid cell m
// collects the +-(0.5/h) gradient adjoints of the fluid cells whose clamped
// central difference reads m, then adds (mag_adj / mag) * vorticity to the
// vorticity adjoint.
__global__ void magnitude_gather_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, VortAdj a) {
    const uint64_t m = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (m >= cell_count(g)) return;
    int x, y, z;
    decode(m, g.nx, g.ny, x, y, z);
    const double s = 0.5 / g.h;
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        uint64_t j[4];
        double w[4];
        const int k = difference_sources(x, y, z, d, g, j, w);
        for (int q = 0; q < k; ++q) {
            if (is_solid(mask, j[q])) continue;
            double gx, gy, gz;
            normal_gradient_adjoint(c, a, j[q], gx, gy, gz);
            acc += s * w[q] * (d == 0 ? gx : (d == 1 ? gy : gz));
        }
    }
    a.mag[m] = acc;
}

// operators.cu:809-816 then the gather form of :818-833: centred-velocity
// adjoint of cell m from the vorticity adjoints of the cells whose clamped
// curl stencil reads m.
__global__ void magnitude_apply_kernel(Grid g, const uint32_t* __restrict__ mask, VortCache c, VortAdj a) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g) || is_solid(mask, i)) return;
    const double s = a.mag[i] / c.mag[i];
    a.wx[i] += s * c.wx[i];
    a.wy[i] += s * c.wy[i];
    a.wz[i] += s * c.wz[i];
}

// Sum over fluid cells j of coefficient * wa(j) where j's clamped stencil
// along axis d reads m: weight +1 for "plus" reads, -1 for "minus" reads.
__device__ __forceinline__ double gather_axis(const Grid& g, const uint32_t* mask, int x, int y, int z, int d, const double* wa) {
    uint64_t j[4];
    double w[4];
    const int k = difference_sources(x, y, z, d, g, j, w);
    double acc = 0.0;
    for (int q = 0; q < k; ++q)
        if (!is_solid(mask, j[q])) acc += w[q] * wa[j[q]];
    return acc;
}

// curl (operators.cu:694-696): wx = d_y cz - d_z cy, wy = d_z cx - d_x cz,
// wz = d_x cy - d_y cx with central differences (0.5/h).  Reverse:
// cx_adj = s (D_z^T wy_adj - D_y^T wz_adj), etc.
__global__ void curl_gather_kernel(Grid g, const uint32_t* __restrict__ mask, VortAdj a) {
    const uint64_t m = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (m >= cell_count(g)) return;
    int x, y, z;
    decode(m, g.nx, g.ny, x, y, z);
    const double s = 0.5 / g.h;
    a.cx[m] = s * (gather_axis(g, mask, x, y, z, 2, a.wy) - gather_axis(g, mask, x, y, z, 1, a.wz));
    a.cy[m] = s * (gather_axis(g, mask, x, y, z, 0, a.wz) - gather_axis(g, mask, x, y, z, 2, a.wx));
    a.cz[m] = s * (gather_axis(g, mask, x, y, z, 1, a.wx) - gather_axis(g, mask, x, y, z, 0, a.wy));
}

// operators.cu:835-846 in gather form: each face takes half of the centred
// adjoint of the fluid cells on either side.
__global__ void centered_velocity_gather_kernel(Grid g, const uint32_t* __restrict__ mask, VortAdj a, XsAdjointVector ua) {
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= f0 + f1 + f2) return;
    int axis;
    uint64_t local;
    if (i < f0) { axis = 0; local = i; } else if (i < f0 + f1) { axis = 1; local = i - f0; } else { axis = 2; local = i - f0 - f1; }
    int x, y, z;
    decode(local, extent(g, axis, 0), extent(g, axis, 1), x, y, z);
    const double* ca = axis == 0 ? a.cx : (axis == 1 ? a.cy : a.cz);
    double acc = 0.0;
    const int lx = x - (axis == 0), ly = y - (axis == 1), lz = z - (axis == 2);
    if (in_grid(g, lx, ly, lz)) { const uint64_t c = idx3(lx, ly, lz, g.nx, g.ny); if (!is_solid(mask, c)) acc += 0.5 * ca[c]; }
    if (in_grid(g, x, y, z)) { const uint64_t c = idx3(x, y, z, g.nx, g.ny); if (!is_solid(mask, c)) acc += 0.5 * ca[c]; }
    if (acc != 0.0) {
        double* out = axis == 0 ? ua.x : (axis == 1 ? ua.y : ua.z);
        out[local] += acc;
    }
}

XsStatus vorticity_forward(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const float* conf, float* cache,
                           const XsVector& force) {
    const uint64_t n = cell_count(g);
    const VortCache c = vort_cache(cache, n);
    const unsigned nb = blocks_for(n);
    centered_velocity_kernel<<<nb, kBlock, 0, st>>>(g, mask, u, c.cx, c.cy, c.cz);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    curl_magnitude_kernel<<<nb, kBlock, 0, st>>>(g, mask, c.cx, c.cy, c.cz, c.wx, c.wy, c.wz, c.mag);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    vorticity_normal_kernel<<<nb, kBlock, 0, st>>>(g, mask, c.mag, c.nx, c.ny, c.nz, c.norm);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    add_vorticity_force_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, conf, force);
    return check_launch();
}

XsStatus vorticity_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& ut, const float* conf, const float* conf_t,
                       const float* cache, const XsVector& force_t, float* scratch) {
    const uint64_t n = cell_count(g);
    const VortCache c = vort_cache(const_cast<float*>(cache), n);
    // scratch: centred (3), vorticity (3), magnitude (1), normal (3)
    VortCache t = vort_cache(scratch, n);
    t.norm = nullptr;
    const unsigned nb = blocks_for(n);
    centered_velocity_kernel<<<nb, kBlock, 0, st>>>(g, mask, ut, t.cx, t.cy, t.cz);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    curl_magnitude_kernel<<<nb, kBlock, 0, st>>>(g, mask, t.cx, t.cy, t.cz, t.wx, t.wy, t.wz, t.mag);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    magnitude_tangent_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, t);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    normal_tangent_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, t);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    vorticity_force_tangent_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, t, conf, conf_t, force_t);
    return check_launch();
}

XsStatus vorticity_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* conf, const float* cache, const XsAdjointVector& fa,
                       const XsAdjointVector& ua, double* conf_adj, double* scratch) {
    const uint64_t n = cell_count(g);
    const VortCache c = vort_cache(const_cast<float*>(cache), n);
    const VortAdj a = vort_adj(scratch, n);
    const unsigned nb = blocks_for(n);
    vorticity_force_reverse_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, conf, fa, a, conf_adj);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    magnitude_gather_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, a);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    magnitude_apply_kernel<<<nb, kBlock, 0, st>>>(g, mask, c, a);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    curl_gather_kernel<<<nb, kBlock, 0, st>>>(g, mask, a);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    const uint64_t F = face_count(g, 0) + face_count(g, 1) + face_count(g, 2);
    centered_velocity_gather_kernel<<<blocks_for(F), kBlock, 0, st>>>(g, mask, a, ua);
    return check_launch();
}

}  // namespace xs

using namespace xs;

extern "C" {

XsStatus xs_vorticity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, const float* confinement,
                              float* cache, XsVector force) {
    if (!valid_grid(grid) || !valid(velocity) || !confinement || !cache || !valid(force)) return XS_INVALID_ARGUMENT;
    return vorticity_forward(stream, make_grid(grid), cell_mask, velocity, confinement, cache, force);
}

XsStatus xs_vorticity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity_tangent, const float* confinement,
                          const float* confinement_tangent, const float* cache, XsVector force_tangent, float* scratch) {
    if (!valid_grid(grid) || !valid(velocity_tangent) || !confinement || !confinement_tangent || !cache || !valid(force_tangent) || !scratch)
        return XS_INVALID_ARGUMENT;
    return vorticity_jvp(stream, make_grid(grid), cell_mask, velocity_tangent, confinement, confinement_tangent, cache, force_tangent,
                         scratch);
}

XsStatus xs_vorticity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* confinement, const float* cache,
                          XsAdjointVector force_adjoint, XsAdjointVector velocity_adjoint, double* confinement_adjoint, double* scratch) {
    if (!valid_grid(grid) || !confinement || !cache || !valid(force_adjoint) || !valid(velocity_adjoint) || !confinement_adjoint || !scratch)
        return XS_INVALID_ARGUMENT;
    return vorticity_vjp(stream, make_grid(grid), cell_mask, confinement, cache, force_adjoint, velocity_adjoint, confinement_adjoint, scratch);
}

}  // extern "C"
