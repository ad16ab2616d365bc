// Learned pressure warm start: shared declarations.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "diff_smoke.h"

namespace xs {

// A batch of volumes, NDHWC: index (((b * z + k) * y + j) * x + i) * C + c.
struct VolumeShape {
    uint32_t x, y, z, batch;
};

// Output tile of the convolutions: 128 voxels = bx * by of one x-y plane.
bool conv_tile(const VolumeShape& s, uint32_t& bx, uint32_t& by, uint32_t& bz);

bool make_activation_map(CUtensorMap* map, const void* base, const VolumeShape& s, uint32_t channels, uint32_t bx, uint32_t by,
                         uint32_t bz);
bool make_weight_map(CUtensorMap* map, const void* base, uint32_t rows, uint32_t cols);

// out = act(conv3x3x3(in, w) + bias); w is [27][cout][cin] BF16.
XsStatus conv3_forward(cudaStream_t st, const VolumeShape& s, int cin, int cout, const __nv_bfloat16* in, const __nv_bfloat16* w,
                       const float* bias, __nv_bfloat16* out, bool relu, int* error);

// dw[27][cout][cin] (+)= sum_v x[v + tap][cin] * dy[v][cout]; partial is
// scratch of wgrad_partial_floats(s, cin, cout) floats.
XsStatus conv3_wgrad(cudaStream_t st, const VolumeShape& s, int cin, int cout, const __nv_bfloat16* x, const __nv_bfloat16* dy, float* partial,
                     float* dw, bool accumulate, int* error);
size_t wgrad_partial_floats(const VolumeShape& s, int cin, int cout);

struct Grid;
struct WarmStartNet;
// Restricts a fine-grid right-hand side to the network grid, runs the
// network and prolongs its output to the fine grid; *guess points into the
// network's own storage.
XsStatus warm_start_guess(WarmStartNet* net, cudaStream_t st, const Grid& g, const float* rhs, float** guess);

}  // namespace xs
