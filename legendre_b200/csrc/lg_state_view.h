// What code outside lg_abi.cu may read of a state: its current arena and the
// block-major slab layout (lg_abi.cu owns the state itself).
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/legendre_b200.h"

namespace lg {

struct StateView {
    lg_ctx* ctx;
    const void* arena;  // the arena holding the current state
    int dtype, esize, D, nfields;
    const int* ghosts;  // per field
    int64_t slab_stride;  // elements between consecutive slabs (block b, field f at (b * nfields + f) * slab_stride)
    int64_t nblocks;
    int64_t block[3], nb[3];  // cells per block and blocks per dimension (1 past D)
    double spacing[3];
    int periodic[3];
    void* arena_rw;       // the same arena, writable (for entry points that replace the state)
};

int abi_state_view(const lg_state* st, StateView* v);
int abi_fail(lg_ctx* ctx, int code, const std::string& msg);
cudaStream_t abi_stream(lg_ctx* ctx);
// the context's device error word (allocated and zeroed on first use; null
// if that fails): kernels with bounded waits set it when a wait gives up,
// and lg_sync / field downloads report it as LG_ERR_DEVICE
int* abi_device_flag(lg_ctx* ctx);
int abi_device(lg_ctx* ctx);
void abi_count_launch(lg_ctx* ctx, int64_t n);

}  // namespace lg
