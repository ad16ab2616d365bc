// Exact solve of the coarse pressure system of the warm start when the
// operator separates by axis.
//
// Without colliders and without an anchor cell, the pressure operator of
// the reference (operators.cu:852-902: diagonal = connected neighbours +
// fixed-value faces, off-diagonals -1, periodic axes wrapped) is the
// Kronecker sum A = Tx (+) Ty (+) Tz of three 1D operators, each a
// tridiagonal (-1, 2, -1) whose end rows depend on that axis' boundary modes:
// a zero-gradient end drops its missing neighbour (diagonal 1), a
// fixed-value end keeps it as a constant (diagonal 2), a periodic axis
// wraps.  Their orthonormal eigenbases are closed-form cosine / sine
// families (DCT-II, DST-I, the half-shifted cosines of a mixed axis, the
// real Fourier basis), so
//
//     A^-1 b = (Qx (x) Qy (x) Qz) diag(1 / (lx_i + ly_j + lz_k)) (Qx (x) Qy (x) Qz)^T b,
//
// three forward line transforms, one scaling and three inverse transforms.
// Each transform is a dense product with the n x n basis held in shared
// memory (n <= 256 on the coarse grids this serves; above 128 in two column
// halves): O(n) flops per cell and axis instead of the coarse Jacobi-PCG's
// dozens of latency-bound iterations.  A mode whose eigenvalue sum vanishes (the constant of an
// all-zero-gradient box) is dropped: the pseudo-inverse.
#include <algorithm>

#include "launch.cuh"
#include "pressure.cuh"

namespace xs {

namespace {

enum AxisKind : int { kZeroZero = 0, kFixedFixed = 1, kZeroFixed = 2, kFixedZero = 3, kPeriodicAxis = 4 };

constexpr int kTransformThreads = 256;  // 8 warps

// Basis entry Q[j][k] (spatial index j, mode k) and eigenvalue of mode k of
// a 1D operator of length n, in FP64.
__device__ double basis_entry(int kind, int n, int j, int k) {
    const double dn = n;
    switch (kind) {
        case kZeroZero:  // cos(pi k (j + 1/2) / n): DCT-II
            return (k == 0 ? sqrt(1.0 / dn) : sqrt(2.0 / dn)) * cospi(k * (j + 0.5) / dn);
        case kFixedFixed:  // sin(pi (k + 1)(j + 1) / (n + 1)): DST-I
            return sqrt(2.0 / (dn + 1.0)) * sinpi((k + 1.0) * (j + 1.0) / (dn + 1.0));
        case kZeroFixed:  // v_{-1} = v_0, v_n = 0: cos(theta (j + 1/2)), theta (n + 1/2) = pi (k + 1/2)
            return 2.0 / sqrt(2.0 * dn + 1.0) * cospi((k + 0.5) * (j + 0.5) / (dn + 0.5));
        case kFixedZero:  // the mirror image
            return 2.0 / sqrt(2.0 * dn + 1.0) * cospi((k + 0.5) * (n - 1 - j + 0.5) / (dn + 0.5));
        default: {  // periodic: 1, then cos / sin pairs of frequency m, then (-1)^j for even n
            if (k == 0) return sqrt(1.0 / dn);
            const int m = (k + 1) / 2;
            if (2 * m == n) return cospi(static_cast<double>(j)) * sqrt(1.0 / dn);
            return sqrt(2.0 / dn) * ((k & 1) ? cospi(2.0 * m * j / dn) : sinpi(2.0 * m * j / dn));
        }
    }
}

__device__ double eigenvalue(int kind, int n, int k) {
    const double dn = n;
    switch (kind) {
        case kZeroZero: return 2.0 - 2.0 * cospi(k / dn);
        case kFixedFixed: return 2.0 - 2.0 * cospi((k + 1.0) / (dn + 1.0));
        case kZeroFixed:
        case kFixedZero: return 2.0 - 2.0 * cospi((k + 0.5) / (dn + 0.5));
        default: return 2.0 - 2.0 * cospi(2.0 * ((k + 1) / 2) / dn);
    }
}

// basis: per axis a, Q (row j, column k) at a * 2 P^2 and its transpose at
// a * 2 P^2 + P^2 (P = kSpectralMax; zero beyond n); eigen: 3 x P.
__global__ void spectral_basis_kernel(SpectralAxes ax, float* __restrict__ basis, float* __restrict__ eigen) {
    constexpr int P = kSpectralMax;
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= 3 * P * P) return;
    const int a = i / (P * P), j = (i / P) % P, k = i % P;
    const int n = ax.n[a];
    const float q = (j < n && k < n) ? static_cast<float>(basis_entry(ax.kind[a], n, j, k)) : 0.0f;
    basis[static_cast<size_t>(a) * 2 * P * P + j * P + k] = q;
    basis[static_cast<size_t>(a) * 2 * P * P + P * P + k * P + j] = q;
    if (j == 0) eigen[a * P + k] = k < n ? static_cast<float>(eigenvalue(ax.kind[a], n, k)) : 0.0f;
}

// The lines of one axis: line L starts at (L % inner) * s_in + (L / inner) *
// s_out, its elements `stride` apart.
struct LineSet {
    uint32_t lines;
    uint32_t inner;
    uint64_t s_in, s_out;
    uint64_t stride;
    int n;
    __device__ __forceinline__ uint64_t base(uint32_t L) const { return static_cast<uint64_t>(L % inner) * s_in + static_cast<uint64_t>(L / inner) * s_out; }
};

// Eigenvalue sums for the scaling of the last axis: line L holds modes
// (L % inner, L / inner) of the two axes transformed before.
struct LineScale {
    const float* lam_a;  // indexed by L % inner
    const float* lam_b;  // indexed by L / inner
    const float* lam_line;
    uint32_t inner;
};

constexpr int kWarpLines = 8;                                  // lines per warp
constexpr int kTileLines = kWarpLines * kTransformThreads / 32;  // 64 lines per tile
constexpr int pitch(int np) { return np + 4; }                 // 16-byte rows
constexpr size_t transform_smem(int np) { return sizeof(float) * static_cast<size_t>(np + kTileLines) * pitch(np); }

// Copies the tile of lines L0.. into d (row pitch R, zero beyond n and past
// the last line): kBatch loads in flight per thread; contiguous lines are
// read along the line, strided ones across lines (consecutive threads take
// consecutive lines, which are adjacent in memory).
template <int NP, class Tin>
__device__ __forceinline__ void load_tile(const Tin* in, const LineSet& ls, uint32_t L0, float* d, int t) {
    constexpr int R = pitch(NP);
    constexpr int kPer = kTileLines * NP / kTransformThreads;  // tile elements per thread
    constexpr int kBatch = 8;
    static_assert(kPer % kBatch == 0, "");
    const bool contiguous = ls.stride == 1;
    for (int b0 = 0; b0 < kPer; b0 += kBatch) {
        float v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int i = t + (b0 + u) * kTransformThreads;
            const int l = contiguous ? i / NP : i % kTileLines, j = contiguous ? i % NP : i / kTileLines;
            const uint32_t L = L0 + l;
            v[u] = (L < ls.lines && j < ls.n) ? static_cast<float>(in[ls.base(L) + static_cast<uint64_t>(j) * ls.stride]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int i = t + (b0 + u) * kTransformThreads;
            const int l = contiguous ? i / NP : i % kTileLines, j = contiguous ? i % NP : i / kTileLines;
            d[l * R + j] = v[u];
        }
    }
}

template <int NP>
__device__ __forceinline__ void store_tile(float* out, const LineSet& ls, uint32_t L0, const float* d, int t) {
    constexpr int R = pitch(NP);
    const bool contiguous = ls.stride == 1;
    for (int i = t; i < kTileLines * NP; i += kTransformThreads) {
        const int l = contiguous ? i / NP : i % kTileLines, j = contiguous ? i % NP : i / kTileLines;
        const uint32_t L = L0 + l;
        if (L < ls.lines && j < ls.n) out[ls.base(L) + static_cast<uint64_t>(j) * ls.stride] = d[l * R + j];
    }
}

// acc[i][c] += sum_j d[l0 + i][j] * M[j][4 lane + c] over j < NP: the warp's
// kWarpLines lines (16-byte broadcasts of the tile) against the lane's four
// consecutive columns of M (row pitch RM).
template <int NP, int RM>
__device__ __forceinline__ void accumulate_modes(const float* d, const float* ms, int l0, int lane, float (&acc)[kWarpLines][4]) {
    constexpr int R = pitch(NP);
#pragma unroll 2
    for (int j = 0; j < NP; j += 4) {
        float4 v[kWarpLines];
#pragma unroll
        for (int i = 0; i < kWarpLines; ++i) v[i] = *reinterpret_cast<const float4*>(d + (l0 + i) * R + j);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const float4 q = *reinterpret_cast<const float4*>(ms + (j + jj) * RM + 4 * lane);
#pragma unroll
            for (int i = 0; i < kWarpLines; ++i) {
                const float x = jj == 0 ? v[i].x : (jj == 1 ? v[i].y : (jj == 2 ? v[i].z : v[i].w));
                acc[i][0] = fmaf(x, q.x, acc[i][0]);
                acc[i][1] = fmaf(x, q.y, acc[i][1]);
                acc[i][2] = fmaf(x, q.z, acc[i][2]);
                acc[i][3] = fmaf(x, q.w, acc[i][3]);
            }
        }
    }
}

// Divides coefficient k of line L by its eigenvalue sum (zero for a
// vanishing sum: the pseudo-inverse; zero past n and past the last line).
__device__ __forceinline__ float scaled_mode(float v, const LineSet& ls, const LineScale& sc, uint32_t L, int k) {
    if (!(L < ls.lines && k < ls.n)) return 0.0f;
    const float lam = sc.lam_a[L % sc.inner] + sc.lam_b[L / sc.inner] + sc.lam_line[k];
    return lam > 0.0f ? v / lam : 0.0f;
}

// out_l[k] = sum_j M[j][k] in_l[j] for tiles of 64 lines: the tile and M in
// shared memory (16-byte rows), each warp 8 lines, each lane NP / 32
// consecutive outputs, both operands read as 16-byte vectors (the tile's
// as broadcasts).  M = Q gives the coefficients, M = Q^T (stored) the
// values back; with kScale the coefficients are divided by their
// eigenvalue sums (the last axis' forward pass).  In place: a tile is read
// completely before it is written.
template <int NP, bool kScale, class Tin>
__global__ void __launch_bounds__(kTransformThreads, 2) line_transform_kernel(const Tin* in, float* out, LineSet ls, const float* __restrict__ m,
                                                                            LineScale sc) {
    constexpr int R = pitch(NP);
    constexpr int OL = NP / 32;  // outputs per lane
    extern __shared__ __align__(16) float smem[];
    float* ms = smem;          // NP x R
    float* d = smem + NP * R;  // kTileLines x R
    const int t = static_cast<int>(threadIdx.x), lane = t & 31, l0 = (t >> 5) * kWarpLines;
    // the matrix: 16-byte asynchronous copies, all in flight at once
    for (int i = t; i < NP * NP / 4; i += kTransformThreads) {
        const int row = i / (NP / 4), col = 4 * (i % (NP / 4));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(ms + row * R + col))),
                     "l"(m + row * kSpectralMax + col)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    const uint32_t tiles = (ls.lines + kTileLines - 1) / kTileLines;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t L0 = tile * kTileLines;
        __syncthreads();  // the matrix is in place; the previous tile is written out
        load_tile<NP>(in, ls, L0, d, t);
        __syncthreads();
        float acc[kWarpLines][OL];
#pragma unroll
        for (int i = 0; i < kWarpLines; ++i)
#pragma unroll
            for (int c = 0; c < OL; ++c) acc[i][c] = 0.0f;
#pragma unroll 2
        for (int j = 0; j < NP; j += 4) {
            float4 v[kWarpLines];
#pragma unroll
            for (int i = 0; i < kWarpLines; ++i) v[i] = *reinterpret_cast<const float4*>(d + (l0 + i) * R + j);
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                float w[OL];
                if (OL == 4) {
                    const float4 q = *reinterpret_cast<const float4*>(ms + (j + jj) * R + 4 * lane);
                    w[0] = q.x; w[OL > 1 ? 1 : 0] = q.y; w[OL > 2 ? 2 : 0] = q.z; w[OL > 3 ? 3 : 0] = q.w;
                } else {
#pragma unroll
                    for (int c = 0; c < OL; ++c) w[c] = ms[(j + jj) * R + OL * lane + c];
                }
#pragma unroll
                for (int i = 0; i < kWarpLines; ++i) {
                    const float x = jj == 0 ? v[i].x : (jj == 1 ? v[i].y : (jj == 2 ? v[i].z : v[i].w));
#pragma unroll
                    for (int c = 0; c < OL; ++c) acc[i][c] = fmaf(x, w[c], acc[i][c]);
                }
            }
        }
        if (kScale) {
#pragma unroll
            for (int i = 0; i < kWarpLines; ++i) {
                const uint32_t L = L0 + l0 + i;
                const float lam_ab = L < ls.lines ? sc.lam_a[L % sc.inner] + sc.lam_b[L / sc.inner] : 0.0f;
#pragma unroll
                for (int c = 0; c < OL; ++c) {
                    const int k = OL * lane + c;
                    const float lam = lam_ab + (k < ls.n ? sc.lam_line[k] : 0.0f);
                    acc[i][c] = (L < ls.lines && k < ls.n && lam > 0.0f) ? acc[i][c] / lam : 0.0f;
                }
            }
        }
        __syncthreads();  // every warp has read its lines
#pragma unroll
        for (int i = 0; i < kWarpLines; ++i)
#pragma unroll
            for (int c = 0; c < OL; ++c) d[(l0 + i) * R + OL * lane + c] = acc[i][c];
        __syncthreads();
        store_tile<NP>(out, ls, L0, d, t);
    }
}

template <int NP, bool kScale, class Tin>
XsStatus launch_transform(cudaStream_t st, const Tin* in, float* out, const LineSet& ls, const float* m, const LineScale& sc) {
    static DeviceOnce configured;
    const size_t smem = transform_smem(NP);
    if (!configured.run([smem] {
            return cudaFuncSetAttribute(line_transform_kernel<NP, kScale, Tin>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        }))
        return XS_CUDA_ERROR;
    const uint32_t tiles = (ls.lines + kTileLines - 1) / kTileLines;
    const unsigned blocks = std::min<uint32_t>(tiles, 2u * 148u);
    line_transform_kernel<NP, kScale, Tin><<<blocks, kTransformThreads, smem, st>>>(in, out, ls, m, sc);
    return check_launch();
}

// Lines of 129-256 values.  A 256 x 256 basis (256 KB) does not fit in shared
// memory beside a tile, so each tile is multiplied by the basis' two column
// halves in turn (modes 0-127, then 128-255), each half copied in once the
// previous one is no longer read; every lane keeps both halves' sums in
// registers until the tile is written back, in place as above.  The halves
// come from L2 (the basis stays resident): 256 KB per tile of 64 lines,
// against 2 x 64 x 256 x 256 flop of products.  One CTA per SM.
constexpr int kWideLines = 256;
constexpr int kHalfModes = kWideLines / 2;
constexpr int kHalfPitch = kHalfModes + 4;  // 16-byte rows
constexpr size_t wide_transform_smem() {
    return sizeof(float) * (static_cast<size_t>(kTileLines) * pitch(kWideLines) + static_cast<size_t>(kWideLines) * kHalfPitch);
}

// Columns [h 128, h 128 + 128) of the basis into mh (row pitch kHalfPitch),
// 16-byte asynchronous copies; the caller waits.
__device__ __forceinline__ void copy_half(float* mh, const float* __restrict__ m, int h, int t) {
    constexpr int kChunks = kHalfModes / 4;  // per row
    for (int i = t; i < kWideLines * kChunks; i += kTransformThreads) {
        const int row = i / kChunks, col = 4 * (i % kChunks);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(mh + row * kHalfPitch + col))),
                     "l"(m + row * kSpectralMax + h * kHalfModes + col)
                     : "memory");
    }
}

template <bool kScale, class Tin>
__global__ void __launch_bounds__(kTransformThreads, 1) line_transform_wide_kernel(const Tin* in, float* out, LineSet ls, const float* __restrict__ m,
                                                                                 LineScale sc) {
    constexpr int NP = kWideLines;
    constexpr int R = pitch(NP);
    extern __shared__ __align__(16) float smem[];
    float* d = smem;                    // kTileLines x R
    float* mh = smem + kTileLines * R;  // NP x kHalfPitch: one column half of the basis
    const int t = static_cast<int>(threadIdx.x), lane = t & 31, l0 = (t >> 5) * kWarpLines;
    const uint32_t tiles = (ls.lines + kTileLines - 1) / kTileLines;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t L0 = tile * kTileLines;
        __syncthreads();  // the previous tile is written out and its second half no longer read
        copy_half(mh, m, 0, t);
        load_tile<NP>(in, ls, L0, d, t);
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        float acc[2][kWarpLines][4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 1) {
                __syncthreads();  // every warp is done with the first half
                copy_half(mh, m, 1, t);
                asm volatile("cp.async.wait_all;" ::: "memory");
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < kWarpLines; ++i)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[h][i][c] = 0.0f;
            accumulate_modes<NP, kHalfPitch>(d, mh, l0, lane, acc[h]);
        }
        if (kScale) {
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int i = 0; i < kWarpLines; ++i)
#pragma unroll
                    for (int c = 0; c < 4; ++c) acc[h][i][c] = scaled_mode(acc[h][i][c], ls, sc, L0 + l0 + i, h * kHalfModes + 4 * lane + c);
        }
        __syncthreads();  // every warp has read its lines
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int i = 0; i < kWarpLines; ++i)
                *reinterpret_cast<float4*>(d + (l0 + i) * R + h * kHalfModes + 4 * lane) =
                    make_float4(acc[h][i][0], acc[h][i][1], acc[h][i][2], acc[h][i][3]);
        __syncthreads();
        store_tile<NP>(out, ls, L0, d, t);
    }
}

template <bool kScale, class Tin>
XsStatus launch_wide_transform(cudaStream_t st, const Tin* in, float* out, const LineSet& ls, const float* m, const LineScale& sc) {
    static DeviceOnce configured;
    constexpr size_t smem = wide_transform_smem();
    if (!configured.run([] {
            return cudaFuncSetAttribute(line_transform_wide_kernel<kScale, Tin>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        }))
        return XS_CUDA_ERROR;
    const uint32_t tiles = (ls.lines + kTileLines - 1) / kTileLines;
    const unsigned blocks = std::min<uint32_t>(tiles, 148u);
    line_transform_wide_kernel<kScale, Tin><<<blocks, kTransformThreads, smem, st>>>(in, out, ls, m, sc);
    return check_launch();
}

template <bool kScale, class Tin>
XsStatus transform(cudaStream_t st, const Tin* in, float* out, const LineSet& ls, const float* m, const LineScale& sc) {
    if (ls.n <= 32) return launch_transform<32, kScale, Tin>(st, in, out, ls, m, sc);
    if (ls.n <= 64) return launch_transform<64, kScale, Tin>(st, in, out, ls, m, sc);
    if (ls.n <= 128) return launch_transform<128, kScale, Tin>(st, in, out, ls, m, sc);
    return launch_wide_transform<kScale, Tin>(st, in, out, ls, m, sc);
}

}  // namespace

bool spectral_axes(const Grid& c, const XsScalarBoundary& pb, uint32_t anchor, SpectralAxes& out) {
    if (anchor < cell_count(c)) return false;  // the anchored operator is not a Kronecker sum
    const int n[3] = {c.nx, c.ny, c.nz};
    for (int a = 0; a < 3; ++a) {
        if (n[a] < 4 || n[a] > kSpectralMax) return false;
        const uint32_t lo = pb.modes[2 * a], hi = pb.modes[2 * a + 1];
        out.n[a] = n[a];
        if (lo == 2u && hi == 2u) {
            out.kind[a] = kPeriodicAxis;
        } else {
            const bool flo = lo == 0u, fhi = hi == 0u;  // fixed value; anything else drops the missing neighbour
            out.kind[a] = flo ? (fhi ? kFixedFixed : kFixedZero) : (fhi ? kZeroFixed : kZeroZero);
        }
    }
    return true;
}

XsStatus spectral_solve(cudaStream_t st, const Grid& c, const SpectralAxes& ax, float* basis, float* eigen, const double* rhs, float* x) {
    if (!basis || !eigen || !rhs || !x) return XS_INVALID_ARGUMENT;
    constexpr int P = kSpectralMax;
    spectral_basis_kernel<<<(3 * P * P + 255) / 256, 256, 0, st>>>(ax, basis, eigen);
    XsStatus s = check_launch();
    if (s != XS_OK) return s;
    const uint64_t nx = c.nx, ny = c.ny, nz = c.nz;
    // x lines: L = y + ny z, contiguous; y lines: L = x + nx z; z lines: L = x + nx y
    const LineSet lx{static_cast<uint32_t>(ny * nz), 1u, 0u, nx, 1u, c.nx};
    const LineSet ly{static_cast<uint32_t>(nx * nz), static_cast<uint32_t>(nx), 1u, nx * ny, nx, c.ny};
    const LineSet lz{static_cast<uint32_t>(nx * ny), 1u, 0u, 1u, nx * ny, c.nz};
    auto q = [&](int a) { return basis + static_cast<size_t>(a) * 2 * P * P; };       // Q: forward
    auto qt = [&](int a) { return basis + static_cast<size_t>(a) * 2 * P * P + P * P; };  // Q^T: inverse
    const LineScale none{nullptr, nullptr, nullptr, 1u};
    const LineScale scale{eigen, eigen + P, eigen + 2 * P, static_cast<uint32_t>(nx)};
    if ((s = transform<false, double>(st, rhs, x, lx, q(0), none)) != XS_OK) return s;
    if ((s = transform<false, float>(st, x, x, ly, q(1), none)) != XS_OK) return s;
    if ((s = transform<true, float>(st, x, x, lz, q(2), scale)) != XS_OK) return s;
    if ((s = transform<false, float>(st, x, x, lz, qt(2), none)) != XS_OK) return s;
    if ((s = transform<false, float>(st, x, x, ly, qt(1), none)) != XS_OK) return s;
    return transform<false, float>(st, x, x, lx, qt(0), none);
}

}  // namespace xs

using namespace xs;

extern "C" {

size_t xs_separable_solve_scratch_bytes(void) { return sizeof(float) * (6 * kSpectralMax * kSpectralMax + 3 * kSpectralMax); }

XsStatus xs_separable_solve(cudaStream_t stream, XsGrid grid, XsScalarBoundary pressure_boundary, uint32_t pressure_anchor,
                            const double* rhs, float* x, void* scratch) {
    if (!valid_grid(grid) || !rhs || !x || !scratch) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    SpectralAxes ax;
    if (!spectral_axes(g, pressure_boundary, pressure_anchor, ax)) return XS_INVALID_ARGUMENT;
    float* basis = static_cast<float*>(scratch);
    return spectral_solve(stream, g, ax, basis, basis + 6 * kSpectralMax * kSpectralMax, rhs, x);
}

}  // extern "C"
