// Learned pressure warm start: a 4-level U-Net whose 3x3x3 convolutions run
// on tcgen05 (conv.cu), trained on the GPU by this file's own backward pass
// and Adam, and used to produce an initial guess for the pressure PCG.
//
// Network (channels 16/32/64/64 at levels 0..3, level l has 1/2^l of the
// resolution; BF16 activations, FP32 accumulation; no biases):
//
//   x0 --c0--> e0a --c1--> e0b ------------------------------------+ skip
//               pool -> p1 --c2--> e1a --c3--> e1b ------------+    |
//                      pool -> p2 --c4--> e2a --c5--> e2b --+  |    |
//                             pool -> p3 --c6--> ma --c7--> mb  |  |    |
//                                   u2 = up(mb) + e2b <---------+  |    |
//                                   d2 = c8(u2)                    |    |
//                             u1 = up(d2) + e1b <------------------+    |
//                             d1 = c9(u1)                               |
//                       u0 = up(d1) + e0b <------------------------------+
//                       d0 = c10(u0);  out = c11(d0)  (no ReLU)
//
// Every convolution but the last is followed by ReLU.  Input channel 0 is
// the right-hand side of the pressure system scaled to unit RMS per sample,
// channel 1 is 1 inside the domain (an offset for the first layer and a
// boundary signal through the zero padding), the other 14 are zero.  Output
// channel 0 is the predicted pressure in units of its own RMS (the solver
// rescales the guess by the energy-optimal factor, so only the shape
// matters); output channels 1..15 receive no gradient and stay unused.
//
// Training losses (xs_warm_start_set_loss):
//   0: mean over samples and voxels of (out_0 - p / rms(p))^2;
//   1: energy loss, mean over samples of 1 - (g.Ap)^2 / ((g.Ag)(p.Ap)) with
//      g = out_0 and A the pressure operator of the training grid: the
//      squared relative A-norm error of the energy-optimally scaled guess,
//      which is what PCG started from that guess has left to remove.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "launch.cuh"
#include "pressure.cuh"
#include "unet.cuh"

namespace xs {
namespace {

constexpr int kLayers = 12;
constexpr int kStatBlocks = 128;

struct LayerSpec {
    int cin, cout;
    bool relu;
};
constexpr LayerSpec kSpec[kLayers] = {{16, 16, true}, {16, 16, true}, {16, 32, true}, {32, 32, true}, {32, 64, true}, {64, 64, true},
                                      {64, 64, true}, {64, 64, true}, {64, 32, true}, {32, 16, true}, {16, 16, true}, {16, 16, false}};

enum Act { A_X0, A_E0A, A_E0B, A_P1, A_E1A, A_E1B, A_P2, A_E2A, A_E2B, A_P3, A_MA, A_MB, A_U2, A_D2, A_U1, A_D1, A_U0, A_D0, A_OUT, A_COUNT };
constexpr int kActLevel[A_COUNT] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 1, 1, 0, 0, 0};
constexpr int kActChannels[A_COUNT] = {16, 16, 16, 16, 32, 32, 32, 64, 64, 64, 64, 64, 64, 32, 32, 16, 16, 16, 16};

enum Grad { G_OUT, G_D0, G_U0, G_D1, G_U1, G_D2, G_U2, G_MB, G_MA, G_P3, G_E2A, G_P2, G_E1A, G_P1, G_E0A, G_COUNT };
constexpr int kGradLevel[G_COUNT] = {0, 0, 0, 1, 1, 2, 2, 3, 3, 3, 2, 2, 1, 1, 0};
constexpr int kGradChannels[G_COUNT] = {16, 16, 16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 32, 16, 16};

// input and output activation of each convolution
constexpr int kLayerIn[kLayers] = {A_X0, A_E0A, A_P1, A_E1A, A_P2, A_E2A, A_P3, A_MA, A_U2, A_U1, A_U0, A_D0};
constexpr int kLayerOut[kLayers] = {A_E0A, A_E0B, A_E1A, A_E1B, A_E2A, A_E2B, A_MA, A_MB, A_D2, A_D1, A_D0, A_OUT};
constexpr int kLayerLevel[kLayers] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 1, 0, 0};

constexpr size_t layer_weights(int l) { return 27u * static_cast<size_t>(kSpec[l].cin) * kSpec[l].cout; }

size_t layer_offset(int l) {
    size_t o = 0;
    for (int i = 0; i < l; ++i) o += layer_weights(i);
    return o;
}

size_t parameter_count() { return layer_offset(kLayers); }

unsigned grid_for(uint64_t n) {
    const uint64_t b = (n + 255) / 256;
    return static_cast<unsigned>(b < 148u * 16u ? (b > 0 ? b : 1) : 148u * 16u);
}

// ------------------------------------------------------------------ kernels
__device__ __forceinline__ void load8(const __nv_bfloat16* p, float (&v)[8]) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

__device__ __forceinline__ void store8(__nv_bfloat16* p, const float (&v)[8]) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(p) = u;
}

// Index of the parent (coarse) voxel of fine voxel v; dims are the fine ones.
__device__ __forceinline__ uint64_t parent_of(uint64_t v, uint32_t X, uint32_t Y, uint32_t Z) {
    const uint32_t x = static_cast<uint32_t>(v % X);
    uint64_t t = v / X;
    const uint32_t y = static_cast<uint32_t>(t % Y);
    t /= Y;
    const uint32_t z = static_cast<uint32_t>(t % Z);
    const uint64_t b = t / Z;
    return ((b * (Z / 2) + z / 2) * (Y / 2) + y / 2) * (X / 2) + x / 2;
}

// partial[b * gridDim.x + block] = sum of squares of the block's slice of sample b
__global__ void sumsq_kernel(const float* __restrict__ a, uint64_t per_sample, double* __restrict__ partial) {
    __shared__ double red[4 * 32];
    const float* s = a + static_cast<uint64_t>(blockIdx.y) * per_sample;
    double acc[1] = {0.0};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < per_sample; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double v = s[i];
        acc[0] += v * v;
    }
    block_sum<1>(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = acc[0];
}

// inv_rms[b] = 1 / sqrt(mean square of sample b) (0 for an all-zero sample)
__global__ void inv_rms_kernel(const double* __restrict__ partial, uint32_t blocks, uint64_t per_sample, uint32_t batch, float* inv_rms) {
    const uint32_t b = threadIdx.x;
    if (b >= batch) return;
    double s = 0.0;
    for (uint32_t i = 0; i < blocks; ++i) s += partial[b * blocks + i];
    inv_rms[b] = s > 0.0 ? static_cast<float>(1.0 / sqrt(s / static_cast<double>(per_sample))) : 0.0f;
}

// x0[v] = {rhs[v] * inv_rms[b], 1, 0, ..., 0}
__global__ void input_kernel(const float* __restrict__ rhs, uint64_t per_sample, uint64_t total, const float* __restrict__ inv_rms,
                             __nv_bfloat16* __restrict__ x0) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float v[8] = {rhs[i] * inv_rms[i / per_sample], 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        store8(x0 + i * 16, v);
        const float z[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        store8(x0 + i * 16 + 8, z);
    }
}

// 2x2x2 average pooling; fine dims X, Y, Z; C channels.
__global__ void pool_kernel(const __nv_bfloat16* __restrict__ fine, uint32_t X, uint32_t Y, uint32_t Z, uint32_t batch, uint32_t C,
                            __nv_bfloat16* __restrict__ coarse) {
    const uint32_t cx = X / 2, cy = Y / 2, cz = Z / 2, chunks = C / 8;
    const uint64_t total = static_cast<uint64_t>(cx) * cy * cz * batch * chunks;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(i % chunks);
        uint64_t c = i / chunks;
        const uint32_t x = static_cast<uint32_t>(c % cx);
        uint64_t t = c / cx;
        const uint32_t y = static_cast<uint32_t>(t % cy);
        t /= cy;
        const uint32_t z = static_cast<uint32_t>(t % cz);
        const uint64_t b = t / cz;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const uint64_t f = ((b * Z + 2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X + 2 * x + (d & 1);
            float v[8];
            load8(fine + f * C + 8 * k, v);
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] += v[j];
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] *= 0.125f;
        store8(coarse + c * C + 8 * k, acc);
    }
}

// d_fine[v] (+)= d_coarse[parent(v)] / 8
__global__ void pool_backward_kernel(const __nv_bfloat16* __restrict__ dcoarse, uint32_t X, uint32_t Y, uint32_t Z, uint32_t batch, uint32_t C,
                                     __nv_bfloat16* __restrict__ dfine, int accumulate) {
    const uint32_t chunks = C / 8;
    const uint64_t total = static_cast<uint64_t>(X) * Y * Z * batch * chunks;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(i % chunks);
        const uint64_t v = i / chunks;
        float g[8];
        load8(dcoarse + parent_of(v, X, Y, Z) * C + 8 * k, g);
        float o[8];
        if (accumulate) load8(dfine + v * C + 8 * k, o);
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = (accumulate ? o[j] : 0.0f) + 0.125f * g[j];
        store8(dfine + v * C + 8 * k, o);
    }
}

// out[v] = coarse[parent(v)] + skip[v]; fine dims X, Y, Z.
__global__ void upsample_add_kernel(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip, uint32_t X, uint32_t Y,
                                    uint32_t Z, uint32_t batch, uint32_t C, __nv_bfloat16* __restrict__ out) {
    const uint32_t chunks = C / 8;
    const uint64_t total = static_cast<uint64_t>(X) * Y * Z * batch * chunks;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(i % chunks);
        const uint64_t v = i / chunks;
        float a[8], s[8];
        load8(coarse + parent_of(v, X, Y, Z) * C + 8 * k, a);
        load8(skip + v * C + 8 * k, s);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] += s[j];
        store8(out + v * C + 8 * k, a);
    }
}

// d_coarse[c] = sum of d_out over the 8 children of c; fine dims X, Y, Z.
__global__ void upsample_backward_kernel(const __nv_bfloat16* __restrict__ dout, uint32_t X, uint32_t Y, uint32_t Z, uint32_t batch, uint32_t C,
                                         __nv_bfloat16* __restrict__ dcoarse) {
    const uint32_t cx = X / 2, cy = Y / 2, cz = Z / 2, chunks = C / 8;
    const uint64_t total = static_cast<uint64_t>(cx) * cy * cz * batch * chunks;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(i % chunks);
        const uint64_t c = i / chunks;
        const uint32_t x = static_cast<uint32_t>(c % cx);
        uint64_t t = c / cx;
        const uint32_t y = static_cast<uint32_t>(t % cy);
        t /= cy;
        const uint32_t z = static_cast<uint32_t>(t % cz);
        const uint64_t b = t / cz;
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const uint64_t f = ((b * Z + 2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X + 2 * x + (d & 1);
            float v[8];
            load8(dout + f * C + 8 * k, v);
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] += v[j];
        }
        store8(dcoarse + c * C + 8 * k, acc);
    }
}

// d = (y > 0) ? d : 0, in place; n elements (a multiple of 8)
__global__ void relu_backward_kernel(__nv_bfloat16* __restrict__ d, const __nv_bfloat16* __restrict__ y, uint64_t n) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n / 8; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float g[8], a[8];
        load8(d + 8 * i, g);
        load8(y + 8 * i, a);
#pragma unroll
        for (int j = 0; j < 8; ++j) g[j] = a[j] > 0.0f ? g[j] : 0.0f;
        store8(d + 8 * i, g);
    }
}

// Loss gradient: t = p * inv_rms[b]; e = out_0 - t; g_out[v] = {scale * e, 0, ...};
// partial[b * gridDim.x + block] = sum of e^2 over the block's slice.
__global__ void loss_kernel(const __nv_bfloat16* __restrict__ out, const float* __restrict__ p, const float* __restrict__ inv_rms,
                            uint64_t per_sample, float scale, __nv_bfloat16* __restrict__ g_out, double* __restrict__ partial) {
    __shared__ double red[4 * 32];
    const uint32_t b = blockIdx.y;
    const float s = inv_rms[b];
    double acc[1] = {0.0};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < per_sample; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t v = static_cast<uint64_t>(b) * per_sample + i;
        const float e = __bfloat162float(out[v * 16]) - p[v] * s;
        acc[0] += static_cast<double>(e) * e;
        float g[8] = {scale * e, 0, 0, 0, 0, 0, 0, 0};
        store8(g_out + v * 16, g);
        const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        store8(g_out + v * 16 + 8, z);
    }
    block_sum<1>(acc, red);
    if (threadIdx.x == 0) partial[b * gridDim.x + blockIdx.x] = acc[0];
}

__global__ void loss_final_kernel(const double* __restrict__ partial, uint32_t count, double denom, double* loss) {
    __shared__ double red[4 * 32];
    double acc[1] = {0.0};
    // fixed assignment of partials to threads: deterministic
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) acc[0] += partial[i];
    block_sum<1>(acc, red);
    if (threadIdx.x == 0) *loss = acc[0] / denom;
}

// ----------------------------------------------------- energy (A-norm) loss
// The pressure operator on the network grid (no solids): diag counts the
// in-domain or periodic neighbours plus the fixed-value boundary faces,
// zero-gradient faces drop out; (A u)_c = diag u_c - sum of neighbours.
template <class Load>
__device__ __forceinline__ float apply_operator(const Load& u, int x, int y, int z, int X, int Y, int Z, const XsScalarBoundary& pb) {
    const int c[3] = {x, y, z}, n[3] = {X, Y, Z};
    float diag = 0.0f, acc = 0.0f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            int q[3] = {c[0], c[1], c[2]};
            q[d] += side ? 1 : -1;
            if (q[d] < 0 || q[d] >= n[d]) {
                if (periodic(pb, d)) {
                    q[d] = side ? 0 : n[d] - 1;
                } else {
                    if (pb.modes[2 * d + side] == 0u) diag += 1.0f;
                    continue;
                }
            }
            acc += u(q[0], q[1], q[2]);
            diag += 1.0f;
        }
    }
    return diag * u(x, y, z) - acc;
}

struct EnergyArgs {
    const __nv_bfloat16* out;  // network output, channel 0 at stride 16
    const float* p;            // target pressure (any scale)
    int X, Y, Z;
    XsScalarBoundary pb;
    uint64_t per_sample;
};

// Per sample: S1 = g.At, S2 = g.Ag, S3 = t.At, as block partials.
__global__ void energy_sums_kernel(EnergyArgs a, double* __restrict__ partial) {
    __shared__ double red[4 * 32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.y) * a.per_sample;
    auto G = [&](int x, int y, int z) { return __bfloat162float(a.out[(base + (static_cast<uint64_t>(z) * a.Y + y) * a.X + x) * 16]); };
    auto T = [&](int x, int y, int z) { return a.p[base + (static_cast<uint64_t>(z) * a.Y + y) * a.X + x]; };
    double s[3] = {0.0, 0.0, 0.0};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < a.per_sample; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % a.X), y = static_cast<int>((i / a.X) % a.Y), z = static_cast<int>(i / (static_cast<uint64_t>(a.X) * a.Y));
        const double at = apply_operator(T, x, y, z, a.X, a.Y, a.Z, a.pb), ag = apply_operator(G, x, y, z, a.X, a.Y, a.Z, a.pb);
        const double g = G(x, y, z), t = T(x, y, z);
        s[0] += g * at;
        s[1] += g * ag;
        s[2] += t * at;
    }
    block_sum<3>(s, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; ++k) partial[(static_cast<uint64_t>(blockIdx.y) * gridDim.x + blockIdx.x) * 3 + k] = s[k];
}

// Per sample: alpha = S1/S2 (the energy-optimal scale of the guess), loss
// 1 - S1^2/(S2 S3) (the squared relative A-norm error of alpha g), gradient
// factor -2 alpha / (S3 batch).  coef[2b] = alpha, coef[2b+1] = factor.
__global__ void energy_final_kernel(const double* __restrict__ partial, uint32_t blocks, uint32_t batch, double* __restrict__ coef, double* loss) {
    __shared__ double lb[64];
    const uint32_t b = threadIdx.x;
    if (b < batch) {
        double s[3] = {0.0, 0.0, 0.0};
        for (uint32_t i = 0; i < blocks; ++i)
            for (int k = 0; k < 3; ++k) s[k] += partial[(static_cast<uint64_t>(b) * blocks + i) * 3 + k];
        const bool ok = s[1] > 0.0 && s[2] > 0.0;
        const double alpha = ok ? s[0] / s[1] : 0.0;
        coef[2 * b] = alpha;
        coef[2 * b + 1] = ok ? -2.0 * alpha / (s[2] * batch) : 0.0;
        lb[b] = ok ? 1.0 - s[0] * s[0] / (s[1] * s[2]) : 1.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (uint32_t i = 0; i < batch; ++i) acc += lb[i];
        *loss = acc / batch;
    }
}

// g_out[v] = {factor_b (A t - alpha_b A g)_v, 0, ..., 0}
__global__ void energy_grad_kernel(EnergyArgs a, uint32_t batch, const double* __restrict__ coef, __nv_bfloat16* __restrict__ g_out) {
    const uint64_t total = a.per_sample * batch;
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < total; v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t b = v / a.per_sample, i = v % a.per_sample;
        const uint64_t base = b * a.per_sample;
        auto G = [&](int x, int y, int z) { return __bfloat162float(a.out[(base + (static_cast<uint64_t>(z) * a.Y + y) * a.X + x) * 16]); };
        auto T = [&](int x, int y, int z) { return a.p[base + (static_cast<uint64_t>(z) * a.Y + y) * a.X + x]; };
        const int x = static_cast<int>(i % a.X), y = static_cast<int>((i / a.X) % a.Y), z = static_cast<int>(i / (static_cast<uint64_t>(a.X) * a.Y));
        const float at = apply_operator(T, x, y, z, a.X, a.Y, a.Z, a.pb), ag = apply_operator(G, x, y, z, a.X, a.Y, a.Z, a.pb);
        const float d = static_cast<float>(coef[2 * b + 1] * (static_cast<double>(at) - coef[2 * b] * static_cast<double>(ag)));
        float o[8] = {d, 0, 0, 0, 0, 0, 0, 0};
        store8(g_out + v * 16, o);
        const float z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        store8(g_out + v * 16 + 8, z8);
    }
}

struct LayerTable {
    uint32_t offset[kLayers + 1];
    uint16_t cin[kLayers], cout[kLayers];
};

// Adam on the FP32 master weights (update != 0), then the BF16 copies: w as
// [27][cout][cin] and the input-gradient weights [27][cin][cout] with the
// taps reversed.
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                            __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wf, LayerTable t, int update, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    const uint32_t total = t.offset[kLayers];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int l = 0;
        while (l + 1 < kLayers && i >= t.offset[l + 1]) ++l;
        float wi = w[i];
        if (update) {
            const float gi = g[i];
            const float mi = b1 * m[i] + (1.0f - b1) * gi;
            const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            wi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
            w[i] = wi;
        }
        const uint32_t local = i - t.offset[l], cin = t.cin[l], cout = t.cout[l];
        const uint32_t tap = local / (cin * cout), rem = local % (cin * cout);
        const uint32_t co = rem / cin, ci = rem % cin;
        const __nv_bfloat16 h = __float2bfloat16(wi);
        wb[i] = h;
        wf[t.offset[l] + ((26u - tap) * cin + ci) * cout + co] = h;
    }
}

// Sum of the f^3 fine cells of every coarse cell (one sample).
__global__ void restrict_kernel(const float* __restrict__ fine, uint32_t X, uint32_t Y, uint32_t Z, uint32_t f, float* __restrict__ coarse) {
    const uint32_t cx = X / f, cy = Y / f, cz = Z / f;
    const uint64_t total = static_cast<uint64_t>(cx) * cy * cz;
    for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < total; c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t x = static_cast<uint32_t>(c % cx), y = static_cast<uint32_t>((c / cx) % cy), z = static_cast<uint32_t>(c / (static_cast<uint64_t>(cx) * cy));
        float acc = 0.0f;
        for (uint32_t dz = 0; dz < f; ++dz)
            for (uint32_t dy = 0; dy < f; ++dy)
                for (uint32_t dx = 0; dx < f; ++dx)
                    acc += fine[(static_cast<uint64_t>(z * f + dz) * Y + y * f + dy) * X + x * f + dx];
        coarse[c] = acc;
    }
}

// Trilinear interpolation of output channel 0 (coarse cell centres) onto the
// fine cell centres, clamped at the domain edge.  Fine dims X, Y, Z = f x coarse.
__global__ void prolong_kernel(const __nv_bfloat16* __restrict__ out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t f, float* __restrict__ guess) {
    const uint32_t cx = X / f, cy = Y / f, cz = Z / f;
    const uint64_t total = static_cast<uint64_t>(X) * Y * Z;
    const float inv = 1.0f / static_cast<float>(f);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t x = static_cast<uint32_t>(i % X), y = static_cast<uint32_t>((i / X) % Y), z = static_cast<uint32_t>(i / (static_cast<uint64_t>(X) * Y));
        int i0[3], i1[3];
        float w[3];
        const uint32_t c[3] = {x, y, z}, n[3] = {cx, cy, cz};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            float u = (static_cast<float>(c[d]) + 0.5f) * inv - 0.5f;
            u = fminf(fmaxf(u, 0.0f), static_cast<float>(n[d] - 1));
            const int a = min(static_cast<int>(u), static_cast<int>(n[d]) - 1);
            i0[d] = a;
            i1[d] = min(a + 1, static_cast<int>(n[d]) - 1);
            w[d] = u - static_cast<float>(a);
        }
        auto at = [&](int xx, int yy, int zz) {
            return __bfloat162float(out[((static_cast<uint64_t>(zz) * cy + yy) * cx + xx) * 16]);
        };
        const float c00 = at(i0[0], i0[1], i0[2]) * (1 - w[0]) + at(i1[0], i0[1], i0[2]) * w[0];
        const float c10 = at(i0[0], i1[1], i0[2]) * (1 - w[0]) + at(i1[0], i1[1], i0[2]) * w[0];
        const float c01 = at(i0[0], i0[1], i1[2]) * (1 - w[0]) + at(i1[0], i0[1], i1[2]) * w[0];
        const float c11 = at(i0[0], i1[1], i1[2]) * (1 - w[0]) + at(i1[0], i1[1], i1[2]) * w[0];
        const float c0 = c00 * (1 - w[1]) + c10 * w[1], c1 = c01 * (1 - w[1]) + c11 * w[1];
        guess[i] = c0 * (1 - w[2]) + c1 * w[2];
    }
}

// guess[v] = out_0[v] (network grid, every sample)
__global__ void extract_kernel(const __nv_bfloat16* __restrict__ out, uint64_t total, float* __restrict__ guess) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        guess[i] = __bfloat162float(out[i * 16]);
}

// ------------------------------------------------------------------ host RNG
uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double normal(uint64_t& s) {
    const double u1 = (static_cast<double>(splitmix(s) >> 11) + 1.0) / 9007199254740993.0;
    const double u2 = static_cast<double>(splitmix(s) >> 11) / 9007199254740992.0;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

}  // namespace

// ------------------------------------------------------------------ the network
struct WarmStartNet {
    uint32_t max_batch = 0, factor = 1;
    VolumeShape level[4]{};  // batch field = max_batch
    void* block = nullptr;
    float *master = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
    __nv_bfloat16 *w = nullptr, *wflip = nullptr;
    __nv_bfloat16* act[A_COUNT]{};
    __nv_bfloat16* gbuf[G_COUNT]{};
    float* wgrad_scratch = nullptr;
    double* partial = nullptr;  // kStatBlocks * max_batch
    float* inv_rms_in = nullptr;
    float* inv_rms_p = nullptr;
    double* loss = nullptr;
    int* error = nullptr;
    float* coarse_rhs = nullptr;  // restriction of a fine right-hand side (factor > 1)
    float* fine_guess = nullptr;  // prolonged guess on the fine grid
    double* coef = nullptr;       // energy loss: per-sample alpha and gradient factor
    uint64_t adam_steps = 0;
    LayerTable table{};
    uint32_t loss_kind = 0;       // 0: normalised L2, 1: energy (A-norm)
    XsScalarBoundary loss_boundary{};
};

namespace {

VolumeShape at_level(const WarmStartNet& n, int l, uint32_t batch) {
    VolumeShape s = n.level[l];
    s.batch = batch;
    return s;
}

uint64_t voxels(const VolumeShape& s) { return static_cast<uint64_t>(s.x) * s.y * s.z * s.batch; }

XsStatus forward(WarmStartNet& n, cudaStream_t st, uint32_t batch) {
    XsStatus s;
    auto conv = [&](int l) {
        const VolumeShape sh = at_level(n, kLayerLevel[l], batch);
        return conv3_forward(st, sh, kSpec[l].cin, kSpec[l].cout, n.act[kLayerIn[l]], n.w + layer_offset(l), nullptr, n.act[kLayerOut[l]],
                             kSpec[l].relu, n.error);
    };
    auto pool = [&](int from, int to) {
        const VolumeShape f = at_level(n, kActLevel[from], batch);
        pool_kernel<<<grid_for(voxels(f) / 8 * kActChannels[from] / 8), 256, 0, st>>>(n.act[from], f.x, f.y, f.z, batch, kActChannels[from],
                                                                                      n.act[to]);
        return check_launch();
    };
    auto up = [&](int coarse, int skip, int to) {
        const VolumeShape f = at_level(n, kActLevel[to], batch);
        upsample_add_kernel<<<grid_for(voxels(f) * kActChannels[to] / 8), 256, 0, st>>>(n.act[coarse], n.act[skip], f.x, f.y, f.z, batch,
                                                                                        kActChannels[to], n.act[to]);
        return check_launch();
    };
    if ((s = conv(0)) != XS_OK || (s = conv(1)) != XS_OK || (s = pool(A_E0B, A_P1)) != XS_OK) return s;
    if ((s = conv(2)) != XS_OK || (s = conv(3)) != XS_OK || (s = pool(A_E1B, A_P2)) != XS_OK) return s;
    if ((s = conv(4)) != XS_OK || (s = conv(5)) != XS_OK || (s = pool(A_E2B, A_P3)) != XS_OK) return s;
    if ((s = conv(6)) != XS_OK || (s = conv(7)) != XS_OK || (s = up(A_MB, A_E2B, A_U2)) != XS_OK) return s;
    if ((s = conv(8)) != XS_OK || (s = up(A_D2, A_E1B, A_U1)) != XS_OK) return s;
    if ((s = conv(9)) != XS_OK || (s = up(A_D1, A_E0B, A_U0)) != XS_OK) return s;
    if ((s = conv(10)) != XS_OK || (s = conv(11)) != XS_OK) return s;
    return XS_OK;
}

XsStatus backward(WarmStartNet& n, cudaStream_t st, uint32_t batch) {
    XsStatus s;
    // layer l: d_out holds the gradient of its output; applies the ReLU mask,
    // accumulates the weight gradient and writes the input gradient (if any)
    auto layer = [&](int l, int d_out, int d_in) {
        const VolumeShape sh = at_level(n, kLayerLevel[l], batch);
        const uint64_t count = voxels(sh) * kSpec[l].cout;
        if (kSpec[l].relu) {
            relu_backward_kernel<<<grid_for(count / 8), 256, 0, st>>>(n.gbuf[d_out], n.act[kLayerOut[l]], count);
            XsStatus r = check_launch();
            if (r != XS_OK) return r;
        }
        XsStatus r = conv3_wgrad(st, sh, kSpec[l].cin, kSpec[l].cout, n.act[kLayerIn[l]], n.gbuf[d_out], n.wgrad_scratch, n.grad + layer_offset(l),
                                 false, n.error);
        if (r != XS_OK || d_in < 0) return r;
        return conv3_forward(st, sh, kSpec[l].cout, kSpec[l].cin, n.gbuf[d_out], n.wflip + layer_offset(l), nullptr, n.gbuf[d_in], false,
                             n.error);
    };
    auto up_back = [&](int d_fine, int d_coarse) {
        const VolumeShape f = at_level(n, kGradLevel[d_fine], batch);
        upsample_backward_kernel<<<grid_for(voxels(f) / 8 * kGradChannels[d_fine] / 8), 256, 0, st>>>(n.gbuf[d_fine], f.x, f.y, f.z, batch,
                                                                                                      kGradChannels[d_fine], n.gbuf[d_coarse]);
        return check_launch();
    };
    auto pool_back = [&](int d_coarse, int d_fine) {
        const VolumeShape f = at_level(n, kGradLevel[d_fine], batch);
        pool_backward_kernel<<<grid_for(voxels(f) * kGradChannels[d_fine] / 8), 256, 0, st>>>(n.gbuf[d_coarse], f.x, f.y, f.z, batch,
                                                                                              kGradChannels[d_fine], n.gbuf[d_fine], 1);
        return check_launch();
    };
    if ((s = layer(11, G_OUT, G_D0)) != XS_OK || (s = layer(10, G_D0, G_U0)) != XS_OK || (s = up_back(G_U0, G_D1)) != XS_OK) return s;
    if ((s = layer(9, G_D1, G_U1)) != XS_OK || (s = up_back(G_U1, G_D2)) != XS_OK) return s;
    if ((s = layer(8, G_D2, G_U2)) != XS_OK || (s = up_back(G_U2, G_MB)) != XS_OK) return s;
    if ((s = layer(7, G_MB, G_MA)) != XS_OK || (s = layer(6, G_MA, G_P3)) != XS_OK || (s = pool_back(G_P3, G_U2)) != XS_OK) return s;
    if ((s = layer(5, G_U2, G_E2A)) != XS_OK || (s = layer(4, G_E2A, G_P2)) != XS_OK || (s = pool_back(G_P2, G_U1)) != XS_OK) return s;
    if ((s = layer(3, G_U1, G_E1A)) != XS_OK || (s = layer(2, G_E1A, G_P1)) != XS_OK || (s = pool_back(G_P1, G_U0)) != XS_OK) return s;
    if ((s = layer(1, G_U0, G_E0A)) != XS_OK || (s = layer(0, G_E0A, -1)) != XS_OK) return s;
    return XS_OK;
}

// per-sample 1/rms of a [batch][per_sample] FP32 array into inv_rms
XsStatus sample_inv_rms(WarmStartNet& n, cudaStream_t st, const float* a, uint64_t per_sample, uint32_t batch, float* inv_rms) {
    sumsq_kernel<<<dim3(kStatBlocks, batch), 256, 0, st>>>(a, per_sample, n.partial);
    XsStatus s = check_launch();
    if (s != XS_OK) return s;
    inv_rms_kernel<<<1, 64, 0, st>>>(n.partial, kStatBlocks, per_sample, batch, inv_rms);
    return check_launch();
}

XsStatus prepare_input(WarmStartNet& n, cudaStream_t st, const float* rhs, uint32_t batch) {
    const uint64_t per = voxels(at_level(n, 0, 1));
    XsStatus s = sample_inv_rms(n, st, rhs, per, batch, n.inv_rms_in);
    if (s != XS_OK) return s;
    input_kernel<<<grid_for(per * batch), 256, 0, st>>>(rhs, per, per * batch, n.inv_rms_in, n.act[A_X0]);
    return check_launch();
}

XsStatus refresh_weights(WarmStartNet& n, cudaStream_t st, bool update, float lr, float b1, float b2, float eps) {
    float c1 = 1.0f, c2 = 1.0f;
    if (update) {
        ++n.adam_steps;
        c1 = static_cast<float>(1.0 - std::pow(static_cast<double>(b1), static_cast<double>(n.adam_steps)));
        c2 = static_cast<float>(1.0 - std::pow(static_cast<double>(b2), static_cast<double>(n.adam_steps)));
    }
    adam_kernel<<<grid_for(parameter_count()), 256, 0, st>>>(n.master, n.m, n.v, n.grad, n.w, n.wflip, n.table, update ? 1 : 0, lr, b1, b2, eps,
                                                            c1, c2);
    return check_launch();
}

bool valid_net_shape(uint32_t nx, uint32_t ny, uint32_t nz) {
    if (nx % 8 || ny % 8 || nz % 8 || nx == 0 || ny == 0 || nz == 0) return false;
    for (int l = 0; l < 4; ++l) {
        uint32_t bx, by, bz;
        if (!conv_tile(VolumeShape{nx >> l, ny >> l, nz >> l, 1}, bx, by, bz)) return false;
    }
    return true;
}

}  // namespace

XsStatus warm_start_guess(WarmStartNet* n, cudaStream_t st, const Grid& g, const float* rhs, float** guess) {
    if (!n || !rhs || !guess) return XS_INVALID_ARGUMENT;
    const uint32_t f = n->factor;
    const VolumeShape l0 = at_level(*n, 0, 1);
    if (static_cast<uint32_t>(g.nx) != l0.x * f || static_cast<uint32_t>(g.ny) != l0.y * f || static_cast<uint32_t>(g.nz) != l0.z * f)
        return XS_INVALID_ARGUMENT;
    const float* coarse = rhs;
    XsStatus s;
    if (f > 1) {
        restrict_kernel<<<grid_for(voxels(l0)), 256, 0, st>>>(rhs, g.nx, g.ny, g.nz, f, n->coarse_rhs);
        if ((s = check_launch()) != XS_OK) return s;
        coarse = n->coarse_rhs;
    }
    if ((s = prepare_input(*n, st, coarse, 1)) != XS_OK) return s;
    if ((s = forward(*n, st, 1)) != XS_OK) return s;
    if (f > 1 && g.nx % 4 == 0) {
        // the output channel into a compact FP32 array (the restricted
        // right-hand side is no longer needed), then the 4-wide trilinear
        // prolongation of the coarse-grid correction: the same arithmetic
        extract_kernel<<<grid_for(voxels(l0)), 256, 0, st>>>(n->act[A_OUT], voxels(l0), n->coarse_rhs);
        if ((s = check_launch()) != XS_OK) return s;
        const Grid c{static_cast<int>(l0.x), static_cast<int>(l0.y), static_cast<int>(l0.z), g.h * static_cast<float>(f), g.dt};
        if ((s = prolong_cells(st, g, c, f, n->coarse_rhs, n->fine_guess)) != XS_OK) return s;
    } else {
        prolong_kernel<<<grid_for(voxels(l0) * f * f * f), 256, 0, st>>>(n->act[A_OUT], g.nx, g.ny, g.nz, f, n->fine_guess);
        if ((s = check_launch()) != XS_OK) return s;
    }
    *guess = n->fine_guess;
    return XS_OK;
}

}  // namespace xs

using namespace xs;

extern "C" {

size_t xs_warm_start_parameter_count(void) { return parameter_count(); }

XsStatus xs_warm_start_create(XsWarmStartNet** out, uint32_t max_batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t factor) {
    if (!out || max_batch == 0 || max_batch > 64 || factor == 0 || factor > 4 || !valid_net_shape(nx, ny, nz)) return XS_INVALID_ARGUMENT;
    *out = nullptr;
    WarmStartNet* n = new (std::nothrow) WarmStartNet();
    if (!n) return XS_CUDA_ERROR;
    n->max_batch = max_batch;
    n->factor = factor;
    for (int l = 0; l < 4; ++l) n->level[l] = VolumeShape{nx >> l, ny >> l, nz >> l, max_batch};
    for (int l = 0; l <= kLayers; ++l) n->table.offset[l] = static_cast<uint32_t>(layer_offset(l));
    for (int l = 0; l < kLayers; ++l) {
        n->table.cin[l] = static_cast<uint16_t>(kSpec[l].cin);
        n->table.cout[l] = static_cast<uint16_t>(kSpec[l].cout);
    }
    // carve one allocation
    const size_t P = parameter_count();
    size_t scratch = 0;
    for (int l = 0; l < kLayers; ++l)
        scratch = std::max(scratch, wgrad_partial_floats(n->level[kLayerLevel[l]], kSpec[l].cin, kSpec[l].cout));
    const uint64_t fine_cells = voxels(at_level(*n, 0, 1)) * factor * factor * factor;
    size_t off = 0;
    std::vector<std::pair<void**, size_t>> plan;
    auto take = [&](void** p, size_t bytes) { plan.push_back({p, off}); off = (off + bytes + 255) / 256 * 256; };
    take(reinterpret_cast<void**>(&n->master), P * 4);
    take(reinterpret_cast<void**>(&n->m), P * 4);
    take(reinterpret_cast<void**>(&n->v), P * 4);
    take(reinterpret_cast<void**>(&n->grad), P * 4);
    take(reinterpret_cast<void**>(&n->w), P * 2);
    take(reinterpret_cast<void**>(&n->wflip), P * 2);
    for (int a = 0; a < A_COUNT; ++a) take(reinterpret_cast<void**>(&n->act[a]), voxels(n->level[kActLevel[a]]) * kActChannels[a] * 2);
    for (int g = 0; g < G_COUNT; ++g) take(reinterpret_cast<void**>(&n->gbuf[g]), voxels(n->level[kGradLevel[g]]) * kGradChannels[g] * 2);
    take(reinterpret_cast<void**>(&n->wgrad_scratch), scratch * 4);
    take(reinterpret_cast<void**>(&n->partial), sizeof(double) * 3 * kStatBlocks * max_batch);
    take(reinterpret_cast<void**>(&n->inv_rms_in), 4 * max_batch);
    take(reinterpret_cast<void**>(&n->inv_rms_p), 4 * max_batch);
    take(reinterpret_cast<void**>(&n->loss), sizeof(double));
    take(reinterpret_cast<void**>(&n->coef), sizeof(double) * 2 * max_batch);
    take(reinterpret_cast<void**>(&n->error), sizeof(int));
    take(reinterpret_cast<void**>(&n->coarse_rhs), voxels(at_level(*n, 0, 1)) * 4);
    take(reinterpret_cast<void**>(&n->fine_guess), fine_cells * 4);
    if (cudaMalloc(&n->block, off) != cudaSuccess) {
        check_cuda(cudaGetLastError());
        delete n;
        return XS_CUDA_ERROR;
    }
    for (auto& [p, o] : plan) *p = static_cast<char*>(n->block) + o;
    if (check_cuda(cudaMemset(n->block, 0, off)) != XS_OK) {
        cudaFree(n->block);
        delete n;
        return XS_CUDA_ERROR;
    }
    *out = reinterpret_cast<XsWarmStartNet*>(n);
    return XS_OK;
}

XsStatus xs_warm_start_destroy(XsWarmStartNet* net) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n) return XS_OK;
    const XsStatus s = check_cuda(cudaFree(n->block));
    delete n;
    return s;
}

XsStatus xs_warm_start_set_parameters(XsWarmStartNet* net, cudaStream_t stream, const float* parameters) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || !parameters) return XS_INVALID_ARGUMENT;
    const size_t P = parameter_count();
    XsStatus s = check_cuda(cudaMemcpyAsync(n->master, parameters, P * 4, cudaMemcpyHostToDevice, stream));
    if (s == XS_OK) s = check_cuda(cudaMemsetAsync(n->m, 0, P * 4, stream));
    if (s == XS_OK) s = check_cuda(cudaMemsetAsync(n->v, 0, P * 4, stream));
    if (s != XS_OK) return s;
    n->adam_steps = 0;
    s = refresh_weights(*n, stream, false, 0, 0, 0, 0);
    if (s != XS_OK) return s;
    return check_cuda(cudaStreamSynchronize(stream));
}

XsStatus xs_warm_start_get_parameters(XsWarmStartNet* net, cudaStream_t stream, float* parameters) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || !parameters) return XS_INVALID_ARGUMENT;
    XsStatus s = check_cuda(cudaMemcpyAsync(parameters, n->master, parameter_count() * 4, cudaMemcpyDeviceToHost, stream));
    if (s != XS_OK) return s;
    return check_cuda(cudaStreamSynchronize(stream));
}

XsStatus xs_warm_start_initialize(XsWarmStartNet* net, cudaStream_t stream, uint64_t seed) {
    if (!net) return XS_INVALID_ARGUMENT;
    std::vector<float> p(parameter_count(), 0.0f);
    uint64_t s = seed ^ 0x5DEECE66Dull;
    for (int l = 0; l < kLayers; ++l) {
        const int cin = kSpec[l].cin, cout = kSpec[l].cout;
        const int used_in = l == 0 ? 2 : cin, used_out = l == kLayers - 1 ? 1 : cout;
        const double std_dev = std::sqrt((l == kLayers - 1 ? 1.0 : 2.0) / (27.0 * used_in));
        float* w = p.data() + layer_offset(l);
        for (int tap = 0; tap < 27; ++tap)
            for (int co = 0; co < cout; ++co)
                for (int ci = 0; ci < cin; ++ci) {
                    const double r = normal(s);
                    w[(tap * cout + co) * cin + ci] = (ci < used_in && co < used_out) ? static_cast<float>(std_dev * r) : 0.0f;
                }
    }
    return xs_warm_start_set_parameters(net, stream, p.data());
}

XsStatus xs_warm_start_predict(XsWarmStartNet* net, cudaStream_t stream, uint32_t batch, const float* rhs, float* guess) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || !rhs || !guess || batch == 0 || batch > n->max_batch) return XS_INVALID_ARGUMENT;
    XsStatus s = prepare_input(*n, stream, rhs, batch);
    if (s == XS_OK) s = forward(*n, stream, batch);
    if (s != XS_OK) return s;
    const uint64_t total = voxels(at_level(*n, 0, batch));
    extract_kernel<<<grid_for(total), 256, 0, stream>>>(n->act[A_OUT], total, guess);
    return check_launch();
}

XsStatus xs_warm_start_gradient(XsWarmStartNet* net, cudaStream_t stream, uint32_t batch, const float* rhs, const float* pressure, float* gradient,
                                double* loss) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || !rhs || !pressure || batch == 0 || batch > n->max_batch) return XS_INVALID_ARGUMENT;
    const uint64_t per = voxels(at_level(*n, 0, 1));
    XsStatus s = prepare_input(*n, stream, rhs, batch);
    if (s == XS_OK) s = forward(*n, stream, batch);
    if (s != XS_OK) return s;
    if (n->loss_kind == 1) {
        const VolumeShape l0 = at_level(*n, 0, 1);
        EnergyArgs ea{n->act[A_OUT], pressure, static_cast<int>(l0.x), static_cast<int>(l0.y), static_cast<int>(l0.z), n->loss_boundary, per};
        energy_sums_kernel<<<dim3(kStatBlocks, batch), 256, 0, stream>>>(ea, n->partial);
        if ((s = check_launch()) != XS_OK) return s;
        energy_final_kernel<<<1, 64, 0, stream>>>(n->partial, kStatBlocks, batch, n->coef, loss ? loss : n->loss);
        if ((s = check_launch()) != XS_OK) return s;
        energy_grad_kernel<<<grid_for(per * batch), 256, 0, stream>>>(ea, batch, n->coef, n->gbuf[G_OUT]);
        if ((s = check_launch()) != XS_OK) return s;
    } else {
        if ((s = sample_inv_rms(*n, stream, pressure, per, batch, n->inv_rms_p)) != XS_OK) return s;
        const double denom = static_cast<double>(per) * batch;
        loss_kernel<<<dim3(kStatBlocks, batch), 256, 0, stream>>>(n->act[A_OUT], pressure, n->inv_rms_p, per, static_cast<float>(2.0 / denom),
                                                                 n->gbuf[G_OUT], n->partial);
        if ((s = check_launch()) != XS_OK) return s;
        loss_final_kernel<<<1, 256, 0, stream>>>(n->partial, kStatBlocks * batch, denom, loss ? loss : n->loss);
        if ((s = check_launch()) != XS_OK) return s;
    }
    if ((s = backward(*n, stream, batch)) != XS_OK) return s;
    if (gradient) return check_cuda(cudaMemcpyAsync(gradient, n->grad, parameter_count() * 4, cudaMemcpyDeviceToDevice, stream));
    return XS_OK;
}

XsStatus xs_warm_start_set_loss(XsWarmStartNet* net, uint32_t kind, XsScalarBoundary pressure_boundary) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || kind > 1) return XS_INVALID_ARGUMENT;
    for (int f = 0; f < 6; ++f)
        if (pressure_boundary.modes[f] > 2u) return XS_INVALID_ARGUMENT;
    n->loss_kind = kind;
    n->loss_boundary = pressure_boundary;
    return XS_OK;
}

XsStatus xs_warm_start_adam_step(XsWarmStartNet* net, cudaStream_t stream, float learning_rate, float beta1, float beta2, float epsilon) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || !(learning_rate >= 0.0f) || !(beta1 >= 0.0f && beta1 < 1.0f) || !(beta2 >= 0.0f && beta2 < 1.0f) || !(epsilon > 0.0f))
        return XS_INVALID_ARGUMENT;
    return refresh_weights(*n, stream, true, learning_rate, beta1, beta2, epsilon);
}

XsStatus xs_warm_start_train_step(XsWarmStartNet* net, cudaStream_t stream, uint32_t batch, const float* rhs, const float* pressure,
                                  float learning_rate, double* loss) {
    XsStatus s = xs_warm_start_gradient(net, stream, batch, rhs, pressure, nullptr, loss);
    if (s != XS_OK) return s;
    return xs_warm_start_adam_step(net, stream, learning_rate, 0.9f, 0.999f, 1e-8f);
}

XsStatus xs_warm_start_guess(XsWarmStartNet* net, cudaStream_t stream, XsGrid grid, const float* rhs, float* guess) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n || !guess || !valid_grid(grid)) return XS_INVALID_ARGUMENT;
    float* g = nullptr;
    XsStatus s = warm_start_guess(n, stream, make_grid(grid), rhs, &g);
    if (s != XS_OK) return s;
    const uint64_t cells = static_cast<uint64_t>(grid.nx) * grid.ny * grid.nz;
    return check_cuda(cudaMemcpyAsync(guess, g, cells * 4, cudaMemcpyDeviceToDevice, stream));
}

XsStatus xs_warm_start_status(XsWarmStartNet* net, cudaStream_t stream) {
    WarmStartNet* n = reinterpret_cast<WarmStartNet*>(net);
    if (!n) return XS_INVALID_ARGUMENT;
    int flag = 0;
    XsStatus s = check_cuda(cudaMemcpyAsync(&flag, n->error, sizeof(int), cudaMemcpyDeviceToHost, stream));
    if (s == XS_OK) s = check_cuda(cudaStreamSynchronize(stream));
    if (s != XS_OK) return s;
    return flag ? XS_TIMEOUT : XS_OK;
}

}  // extern "C"
