// 3x3x3 convolutions of the learned pressure warm start on the 5th-generation
// tensor cores (tcgen05), BF16 operands, FP32 accumulation in TMEM.
//
// Activations are NDHWC (channels innermost).  Forward (and the input
// gradient, which is the same convolution with flipped, transposed weights)
// is an implicit GEMM: M = 128 output voxels (a box of the x-y plane at one
// z), N = output channels, K = 27 taps x input channels.  Per tap one TMA
// load brings the shifted 128 x C_in activation box (out-of-range voxels are
// zero-filled by TMA: this is the convolution's zero padding) and one the
// C_out x C_in weight slice, both K-major with the swizzle matching their
// row width; a single thread issues the MMAs; four warps read the
// accumulator back (tcgen05.ld) and apply bias and ReLU.
//
// The weight gradient uses MN-major operands: D[(tap, ci)][co] =
// sum_v X[v + tap][ci] * dY[v][co], M = 128 rows = a group of 128 / C_in taps,
// N = C_out, K = voxels, accumulated in TMEM over a slice of the volume per
// CTA; per-CTA partial sums are reduced in a fixed order by a second kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstring>
#include <mutex>

#include "common.cuh"
#include "launch.cuh"
#include "tc.cuh"
#include "unet.cuh"

namespace xs {

// ------------------------------------------------------------------ TMA maps
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

CUtensorMapSwizzle swizzle_mode(uint32_t row_bytes) {
    return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : (row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}

}  // namespace

// Activation map [B][Z][Y][X][C] with a (C, bx, by, bz, 1) box.
bool make_activation_map(CUtensorMap* map, const void* base, const VolumeShape& s, uint32_t channels, uint32_t bx, uint32_t by, uint32_t bz) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[5] = {channels, s.x, s.y, s.z, s.batch};
    const cuuint64_t e = 2;
    const cuuint64_t strides[4] = {channels * e, s.x * channels * e, static_cast<cuuint64_t>(s.y) * s.x * channels * e,
                                   static_cast<cuuint64_t>(s.z) * s.y * s.x * channels * e};
    const cuuint32_t box[5] = {channels, bx, by, bz, 1};
    const cuuint32_t elem[5] = {1, 1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
              swizzle_mode(channels * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Weight map [27][rows][cols] with a (cols, rows, 1) box: one tap's slice.
bool make_weight_map(CUtensorMap* map, const void* base, uint32_t rows, uint32_t cols) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {cols, rows, 27};
    const cuuint64_t strides[2] = {cols * 2ull, static_cast<cuuint64_t>(rows) * cols * 2ull};
    const cuuint32_t box[3] = {cols, rows, 1};
    const cuuint32_t elem[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
              swizzle_mode(cols * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ------------------------------------------------------------------ forward
constexpr int kConvThreads = 128;
constexpr int kStages = 4;

template <int CIN, int COUT>
struct ConvSmem {
    static constexpr uint32_t a_bytes = 128u * CIN * 2u;
    static constexpr uint32_t b_bytes_raw = static_cast<uint32_t>(COUT) * CIN * 2u;
    static constexpr uint32_t b_bytes = (b_bytes_raw + 1023u) / 1024u * 1024u;
    static constexpr uint32_t stage_bytes = a_bytes + b_bytes;
    static constexpr uint32_t total = 1024u /*alignment slack*/ + kStages * stage_bytes + 256u /*barriers*/;
    static constexpr uint32_t tmem_cols = COUT <= 32 ? 32u : 64u;
};

struct ConvArgs {
    VolumeShape s;
    uint32_t bx, by, bz;  // output tile box
    const float* bias;
    __nv_bfloat16* out;
    int relu;
    int* error;
};

// One CTA = one tile of 128 output voxels (a bx * by * bz box of one batch).
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3_forward_kernel(const __grid_constant__ CUtensorMap act_map,
                                                                     const __grid_constant__ CUtensorMap w_map, ConvArgs a) {
    using L = ConvSmem<CIN, COUT>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) & ~uintptr_t(1023u));
    unsigned char* a_tiles = smem;
    unsigned char* b_tiles = smem + kStages * L::a_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * L::stage_bytes);
    uint64_t* empty = full + kStages;
    uint64_t* accum = empty + kStages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // tile coordinates
    const uint32_t tiles_x = a.s.x / a.bx, tiles_y = a.s.y / a.by, tiles_z = a.s.z / a.bz;
    uint32_t t = blockIdx.x;
    const uint32_t tx = t % tiles_x; t /= tiles_x;
    const uint32_t ty = t % tiles_y; t /= tiles_y;
    const uint32_t tz = t % tiles_z;
    const uint32_t b = t / tiles_z;
    const int x0 = static_cast<int>(tx * a.bx), y0 = static_cast<int>(ty * a.by), z0 = static_cast<int>(tz * a.bz);

    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        tc::mbar_init(accum, 1);
        tc::fence_barrier_init();
        tc::prefetch_map(&act_map);
        tc::prefetch_map(&w_map);
    }
    if (warp == 0) {
        tc::tmem_alloc(tmem_slot, L::tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0 && lane == 0) {
        // TMA producer: one stage per tap
        for (int tap = 0; tap < 27; ++tap) {
            const int s = tap % kStages, round = tap / kStages;
            if (tap >= kStages && !tc::mbar_wait(&empty[s], (round - 1) & 1)) { ok = false; break; }
            tc::mbar_expect_tx(&full[s], L::a_bytes + L::b_bytes_raw);
            const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
            tc::tma_load_5d(a_tiles + s * L::a_bytes, &act_map, &full[s], 0, x0 + dx, y0 + dy, z0 + dz, static_cast<int>(b));
            tc::tma_load_3d(b_tiles + s * L::b_bytes, &w_map, &full[s], 0, 0, tap);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = tc::idesc_bf16(128, COUT, false, false);
        constexpr uint32_t row = CIN * 2;
        constexpr uint32_t swz = tc::swizzle_for_row_bytes(row);
        for (int tap = 0; tap < 27; ++tap) {
            const int s = tap % kStages, round = tap / kStages;
            if (!tc::mbar_wait(&full[s], round & 1)) { ok = false; break; }
            tc::tc_fence_after();
            const uint32_t a_addr = tc::smem_u32(a_tiles + s * L::a_bytes), b_addr = tc::smem_u32(b_tiles + s * L::b_bytes);
#pragma unroll
            for (int k = 0; k < CIN / 16; ++k) {
                const uint64_t ad = tc::smem_desc(a_addr + 32u * k, 16u, 8u * row, swz);
                const uint64_t bd = tc::smem_desc(b_addr + 32u * k, 16u, 8u * row, swz);
                tc::mma_bf16(tmem, ad, bd, idesc, (tap > 0 || k > 0) ? 1u : 0u);
            }
            tc::mma_commit(&empty[s]);
        }
        tc::mma_commit(accum);
    }
    __syncwarp();
    // epilogue: every warp reads its 32 TMEM lanes (= voxels)
    const bool got = tc::mbar_wait(accum, 0);
    tc::tc_fence_after();
    if (got) {
        const int r = warp * 32 + lane;
        const int bxy = static_cast<int>(a.bx * a.by);
        const int x = x0 + r % static_cast<int>(a.bx), y = y0 + (r % bxy) / static_cast<int>(a.bx), z = z0 + r / bxy;
        const uint64_t voxel = ((static_cast<uint64_t>(b) * a.s.z + z) * a.s.y + y) * a.s.x + x;
        __nv_bfloat16* dst = a.out + voxel * COUT;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0), v);
            __align__(16) __nv_bfloat16 o[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float y_ = v[i] + (a.bias ? __ldg(a.bias + c0 + i) : 0.0f);
                if (a.relu) y_ = fmaxf(y_, 0.0f);
                o[i] = __float2bfloat16(y_);
            }
            reinterpret_cast<uint4*>(dst + c0)[0] = reinterpret_cast<const uint4*>(o)[0];
            reinterpret_cast<uint4*>(dst + c0)[1] = reinterpret_cast<const uint4*>(o)[1];
        }
    }
    if ((!ok || !got) && a.error) atomicExch(a.error, 1);
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, L::tmem_cols);
}

template <int CIN, int COUT>
XsStatus launch_conv_forward(cudaStream_t st, const VolumeShape& s, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                             __nv_bfloat16* out, bool relu, int* error) {
    uint32_t bx, by, bz;
    if (!conv_tile(s, bx, by, bz)) return XS_INVALID_ARGUMENT;
    CUtensorMap am, wm;
    if (!make_activation_map(&am, in, s, CIN, bx, by, bz) || !make_weight_map(&wm, w, COUT, CIN)) return XS_CUDA_ERROR;
    using L = ConvSmem<CIN, COUT>;
    static DeviceOnce configured;
    if (!configured.run([] { return cudaFuncSetAttribute(conv3_forward_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::total); }))
        return XS_CUDA_ERROR;
    ConvArgs args{s, bx, by, bz, bias, out, relu ? 1 : 0, error};
    const uint64_t tiles = static_cast<uint64_t>(s.batch) * (s.z / bz) * (s.y / by) * (s.x / bx);
    conv3_forward_kernel<CIN, COUT><<<static_cast<unsigned>(tiles), kConvThreads, L::total, st>>>(am, wm, args);
    return check_launch();
}

// The 128-voxel output tile: as wide in x as the volume allows (up to 128),
// then in y, then in z (for small volumes, several z planes per tile).
bool conv_tile(const VolumeShape& s, uint32_t& bx, uint32_t& by, uint32_t& bz) {
    bx = s.x < 128 ? s.x : 128;
    if (bx == 0 || 128 % bx != 0 || s.x % bx != 0) return false;
    by = 128 / bx < s.y ? 128 / bx : s.y;
    if (by == 0 || (128 / bx) % by != 0 || s.y % by != 0) return false;
    bz = 128 / (bx * by);
    return bz <= s.z && s.z % bz == 0;
}

XsStatus conv3_forward(cudaStream_t st, const VolumeShape& s, int cin, int cout, const __nv_bfloat16* in, const __nv_bfloat16* w,
                       const float* bias, __nv_bfloat16* out, bool relu, int* error) {
#define XS_CONV_CASE(CI, CO) \
    if (cin == CI && cout == CO) return launch_conv_forward<CI, CO>(st, s, in, w, bias, out, relu, error);
    XS_CONV_CASE(16, 16) XS_CONV_CASE(16, 32) XS_CONV_CASE(16, 64)
    XS_CONV_CASE(32, 16) XS_CONV_CASE(32, 32) XS_CONV_CASE(32, 64)
    XS_CONV_CASE(64, 16) XS_CONV_CASE(64, 32) XS_CONV_CASE(64, 64)
#undef XS_CONV_CASE
    return XS_INVALID_ARGUMENT;
}

// ------------------------------------------------------------------ weight gradient
// D[(tap, ci)][co] = sum over voxels v of X[v + tap][ci] * dY[v][co].
// Rows: a group of G = 128 / C_in taps (the G shifted activation boxes sit
// in consecutive tiles, one MN-major atom each); columns: C_out; K: the 128
// voxels of a tile.  A CTA owns a slice of the voxel tiles and a set of tap
// groups whose accumulators fit 256 TMEM columns.
template <int CIN, int COUT>
struct WgradLayout {
    static constexpr int G = 128 / CIN;
    static constexpr int groups = (27 + G - 1) / G;
    static constexpr int groups_per_set = 256 / COUT;
    static constexpr int sets = (groups + groups_per_set - 1) / groups_per_set;
    static constexpr uint32_t x_tile = 128u * CIN * 2u;
    static constexpr uint32_t y_bytes = 128u * COUT * 2u;
    static constexpr uint32_t y_padded = (y_bytes + 1023u) / 1024u * 1024u;
    static constexpr uint32_t stage_bytes = G * x_tile + y_padded;
    static constexpr int stages = 3;
    static constexpr uint32_t total = 1024u + stages * stage_bytes + 256u;
};

struct WgradArgs {
    VolumeShape s;
    uint32_t bx, by, bz;
    uint32_t tiles;
    float* partial;  // [gridDim.x][27][COUT][CIN]
    int* error;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3_wgrad_kernel(const __grid_constant__ CUtensorMap x_map,
                                                                   const __grid_constant__ CUtensorMap dy_map, WgradArgs a) {
    using L = WgradLayout<CIN, COUT>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) & ~uintptr_t(1023u));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::stages * L::stage_bytes);
    uint64_t* empty = full + L::stages;
    uint64_t* accum = empty + L::stages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    const uint32_t cx = blockIdx.x, nctas = gridDim.x;
    const uint32_t t_begin = static_cast<uint32_t>(static_cast<uint64_t>(a.tiles) * cx / nctas);
    const uint32_t t_end = static_cast<uint32_t>(static_cast<uint64_t>(a.tiles) * (cx + 1) / nctas);
    const int g_begin = static_cast<int>(blockIdx.y) * L::groups_per_set;
    const int g_count = min(L::groups_per_set, L::groups - g_begin);
    const uint32_t items = (t_end - t_begin) * static_cast<uint32_t>(g_count);

    if (threadIdx.x == 0) {
        for (int i = 0; i < L::stages; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        tc::mbar_init(accum, 1);
        tc::fence_barrier_init();
        tc::prefetch_map(&x_map);
        tc::prefetch_map(&dy_map);
    }
    if (warp == 0) {
        tc::tmem_alloc(tmem_slot, 256);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    const uint32_t tiles_x = a.s.x / a.bx, tiles_y = a.s.y / a.by, tiles_z = a.s.z / a.bz;

    if (warp == 0 && lane == 0) {
        for (uint32_t i = 0; i < items; ++i) {
            const int s = static_cast<int>(i % L::stages), round = static_cast<int>(i / L::stages);
            if (i >= static_cast<uint32_t>(L::stages) && !tc::mbar_wait(&empty[s], (round - 1) & 1)) { ok = false; break; }
            const uint32_t tile = t_begin + i / g_count;
            const int group = g_begin + static_cast<int>(i % g_count);
            uint32_t t = tile;
            const uint32_t tx = t % tiles_x; t /= tiles_x;
            const uint32_t ty = t % tiles_y; t /= tiles_y;
            const int z = static_cast<int>((t % tiles_z) * a.bz), b = static_cast<int>(t / tiles_z);
            const int x0 = static_cast<int>(tx * a.bx), y0 = static_cast<int>(ty * a.by);
            unsigned char* st = smem + s * L::stage_bytes;
            tc::mbar_expect_tx(&full[s], L::G * L::x_tile + L::y_bytes);
            for (int j = 0; j < L::G; ++j) {
                const int tap = group * L::G + j;
                if (tap < 27) {
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    tc::tma_load_5d(st + j * L::x_tile, &x_map, &full[s], 0, x0 + dx, y0 + dy, z + dz, b);
                } else {  // missing taps of the last group: a box far outside the volume reads zeros
                    tc::tma_load_5d(st + j * L::x_tile, &x_map, &full[s], 0, 0, 0, -static_cast<int>(2 * a.bz + 64), 0);
                }
            }
            tc::tma_load_5d(st + L::G * L::x_tile, &dy_map, &full[s], 0, x0, y0, z, b);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = tc::idesc_bf16(128, COUT, true, true);
        constexpr uint32_t a_row = CIN * 2, b_row = COUT * 2;
        for (uint32_t i = 0; i < items; ++i) {
            const int s = static_cast<int>(i % L::stages), round = static_cast<int>(i / L::stages);
            if (!tc::mbar_wait(&full[s], round & 1)) { ok = false; break; }
            tc::tc_fence_after();
            const uint32_t gl = i % g_count;
            const bool first_tile = (i / g_count) == 0;
            const uint32_t xa = tc::smem_u32(smem + s * L::stage_bytes);
            const uint32_t ya = xa + L::G * L::x_tile;
#pragma unroll
            for (int k = 0; k < 8; ++k) {  // 16 voxels per MMA: two 8-row atoms
                const uint64_t ad = tc::smem_desc(xa + k * 16u * a_row, L::x_tile, 8u * a_row, tc::swizzle_for_row_bytes(a_row));
                const uint64_t bd = tc::smem_desc(ya + k * 16u * b_row, L::y_padded, 8u * b_row, tc::swizzle_for_row_bytes(b_row));
                tc::mma_bf16(tmem + gl * COUT, ad, bd, idesc, (!first_tile || k > 0) ? 1u : 0u);
            }
            tc::mma_commit(&empty[s]);
        }
        tc::mma_commit(accum);
    }
    __syncwarp();
    const bool got = items == 0 ? true : tc::mbar_wait(accum, 0);
    tc::tc_fence_after();
    if (got && items > 0) {
        const int m = warp * 32 + lane;
        const int j = m / CIN, ci = m % CIN;
        for (int gl = 0; gl < g_count; ++gl) {
            const int tap = (g_begin + gl) * L::G + j;
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(gl * COUT + c0), v);
                if (tap < 27) {
                    float* dst = a.partial + ((static_cast<size_t>(cx) * 27 + tap) * COUT + c0) * CIN + ci;
#pragma unroll
                    for (int q = 0; q < 16; ++q) dst[static_cast<size_t>(q) * CIN] = v[q];
                }
            }
        }
    }
    if ((!ok || !got) && a.error) atomicExch(a.error, 1);
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// dW[i] (+)= sum over CTAs of partial[cta][i], in CTA order.
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, uint32_t ctas, uint32_t count, float* __restrict__ dw, int accumulate) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float acc = 0.0f;
    for (uint32_t c = 0; c < ctas; ++c) acc += partial[static_cast<size_t>(c) * count + i];
    dw[i] = accumulate ? dw[i] + acc : acc;
}

uint32_t wgrad_ctas(const VolumeShape& s) {
    uint32_t bx, by, bz;
    if (!conv_tile(s, bx, by, bz)) return 0;
    const uint64_t tiles = static_cast<uint64_t>(s.batch) * (s.z / bz) * (s.y / by) * (s.x / bx);
    return static_cast<uint32_t>(tiles < 148 ? tiles : 148);
}

size_t wgrad_partial_floats(const VolumeShape& s, int cin, int cout) {
    return static_cast<size_t>(wgrad_ctas(s)) * 27u * static_cast<size_t>(cin) * static_cast<size_t>(cout);
}

template <int CIN, int COUT>
XsStatus launch_wgrad(cudaStream_t st, const VolumeShape& s, const __nv_bfloat16* x, const __nv_bfloat16* dy, float* partial, float* dw,
                      bool accumulate, int* error) {
    using L = WgradLayout<CIN, COUT>;
    uint32_t bx, by, bz;
    if (!conv_tile(s, bx, by, bz)) return XS_INVALID_ARGUMENT;
    CUtensorMap xm, ym;
    if (!make_activation_map(&xm, x, s, CIN, bx, by, bz) || !make_activation_map(&ym, dy, s, COUT, bx, by, bz)) return XS_CUDA_ERROR;
    static DeviceOnce configured;
    if (!configured.run([] { return cudaFuncSetAttribute(conv3_wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::total); }))
        return XS_CUDA_ERROR;
    const uint32_t tiles = static_cast<uint32_t>(static_cast<uint64_t>(s.batch) * (s.z / bz) * (s.y / by) * (s.x / bx));
    const uint32_t ctas = wgrad_ctas(s);
    WgradArgs args{s, bx, by, bz, tiles, partial, error};
    conv3_wgrad_kernel<CIN, COUT><<<dim3(ctas, L::sets), kConvThreads, L::total, st>>>(xm, ym, args);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    const uint32_t count = 27u * CIN * COUT;
    wgrad_reduce_kernel<<<(count + 255) / 256, 256, 0, st>>>(partial, ctas, count, dw, accumulate ? 1 : 0);
    return check_launch();
}

XsStatus conv3_wgrad(cudaStream_t st, const VolumeShape& s, int cin, int cout, const __nv_bfloat16* x, const __nv_bfloat16* dy, float* partial,
                     float* dw, bool accumulate, int* error) {
#define XS_WGRAD_CASE(CI, CO) \
    if (cin == CI && cout == CO) return launch_wgrad<CI, CO>(st, s, x, dy, partial, dw, accumulate, error);
    XS_WGRAD_CASE(16, 16) XS_WGRAD_CASE(16, 32) XS_WGRAD_CASE(16, 64)
    XS_WGRAD_CASE(32, 16) XS_WGRAD_CASE(32, 32) XS_WGRAD_CASE(32, 64)
    XS_WGRAD_CASE(64, 16) XS_WGRAD_CASE(64, 32) XS_WGRAD_CASE(64, 64)
#undef XS_WGRAD_CASE
    return XS_INVALID_ARGUMENT;
}

}  // namespace xs

using namespace xs;

extern "C" XsStatus xs_conv3d_weight_grad_bf16(cudaStream_t stream, uint32_t batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t in_channels,
                                               uint32_t out_channels, const void* input, const void* output_grad, float* partial,
                                               float* weight_grad, uint32_t accumulate, int* error_flag) {
    if (!input || !output_grad || !partial || !weight_grad) return XS_INVALID_ARGUMENT;
    const VolumeShape s{nx, ny, nz, batch};
    return conv3_wgrad(stream, s, static_cast<int>(in_channels), static_cast<int>(out_channels), static_cast<const __nv_bfloat16*>(input),
                       static_cast<const __nv_bfloat16*>(output_grad), partial, weight_grad, accumulate != 0, error_flag);
}

extern "C" size_t xs_conv3d_weight_grad_scratch_floats(uint32_t batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t in_channels,
                                                       uint32_t out_channels) {
    const VolumeShape s{nx, ny, nz, batch};
    return wgrad_partial_floats(s, static_cast<int>(in_channels), static_cast<int>(out_channels));
}

extern "C" XsStatus xs_conv3d_bf16(cudaStream_t stream, uint32_t batch, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t in_channels,
                                   uint32_t out_channels, const void* input, const void* weights, const float* bias, void* output,
                                   uint32_t relu, int* error_flag) {
    if (!input || !weights || !output) return XS_INVALID_ARGUMENT;
    const VolumeShape s{nx, ny, nz, batch};
    return conv3_forward(stream, s, static_cast<int>(in_channels), static_cast<int>(out_channels), static_cast<const __nv_bfloat16*>(input),
                         static_cast<const __nv_bfloat16*>(weights), bias, static_cast<__nv_bfloat16*>(output), relu != 0, error_flag);
}
