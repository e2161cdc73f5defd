// Adjoint of the fused Model C step for batched instances (lg_adjoint.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lg_kernels.h"

namespace lg {
namespace adj {

// Geometry of a batch of instances: each instance is N0 x N1 cells in
// blocks of n0 x n1 (nb0 blocks per row, bpi per instance), block-major
// slabs of slab_stride elements, fields phi and u, ghost width 1.
struct Geo {
    int64_t ninst;
    int N0, N1, n0, n1, nb0, bpi;
    int64_t slab_stride;
    int tiles_x, tiles_y;  // set by the launchers
};

// Per-instance constants in the adjoint's arithmetic type.
template <class T>
struct AdjParams {
    T lambda, d_thermal, inv_h2_flux, ih0, ih1;
    T f_a_bar, f_ae, f_a12, f_tol;  // flux: a_bar, a_bar eps', a12, tol
    T c_a_bar, c_ae, c_tol;         // cell-centred anisotropy
};

size_t adj_params_size(int dtype);  // dtype: 0 FP64, 1 FP32
void adj_params(int dtype, const ModelCDev& m, void* out);

// the two forms of the step adjoint: warp strips (the default) and shared-
// memory tiles; both compute the same cotangents up to rounding
constexpr int kAdjointStrip = 0, kAdjointTile = 1;

int adjoint_tile_rows(int dtype);
int adjoint_strips(const Geo& g);
int adjoint_strip_rows(const Geo& g);
// work items (tiles or strip units); the accumulator holds 3 doubles per item
int64_t adjoint_items(int dtype, int kernel, const Geo& g);
int64_t loss_items(const Geo& g);                // tiles of the loss kernel; one double each

// cotangents of x_n from those of x_{n+1}; acc[3 item + k] += the step's
// dL/d(lambda, D, eps4) share of each work item.  work (strip form; may be
// null) is a device counter, zero before the first of a run of launches on
// one stream: each launch advances it by exactly adjoint_items, and base is
// its value when the launch starts (launches so far x adjoint_items).
cudaError_t launch_adjoint_step(int dtype, int kernel, const void* x, const void* lam_in, void* lam_out, const void* prm,
                                const Geo& g, double dt, double* acc, unsigned long long* work,
                                unsigned long long base, cudaStream_t s);
// lam = (2 (phi - target), 0), loss[tile] = that tile's sum of squares
cudaError_t launch_loss_seed(int dtype, const void* x, const double* target, void* lam, Geo g, double* loss,
                             cudaStream_t s);

}  // namespace adj
}  // namespace lg
