// Shared device/host definitions of the legendre B200 library.
//
// Layout (the reference's `State`, src/core/state.rs:219-296): every field of
// every block owns one dense slab of (n_d + 2g) entries per dimension,
// dimension 0 fastest (src/geometry/cartesian.rs:8-11, linearize :189-204).
// On the device all slabs of one state live in a single arena, block-major:
// slab(b, f) starts at arena + (b * nfields + f) * slab_stride, with
// slab_stride the largest field's slab rounded up to 256 bytes, so each slab
// starts 256-byte aligned.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define LG_MAX_DIM 3

namespace lg {

// Per-grid topology as seen by kernels.  `nbr[(b * 3 + d) * 2 + side]` is the
// face neighbour of block b across dimension d (side 0 = low, 1 = high),
// already wrapped in periodic dimensions, or -1 at a physical (mirror)
// boundary -- CartesianGrid::face_neighbor (src/geometry/cartesian.rs:162-181).
struct CartTopo {
    int D;
    int n[LG_MAX_DIM];    // interior cells per block per dimension
    int nb[LG_MAX_DIM];   // blocks per dimension
    int nblocks;
    const int* nbr;       // device table, nblocks * 3 * 2 entries
};

// Slab addressing of one state arena.
struct SlabLayout {
    int nfields;
    int ghost;            // ghost width of the fields a kernel touches
    int64_t slab_stride;  // elements between consecutive slabs
    int64_t len;          // ghost-inclusive slab length of those fields
    int gdim[LG_MAX_DIM]; // n_d + 2g
};

// ------------------------------------------------------------------ rng ---
// Counter-based generator of the reference (src/util/rng.rs:13-49).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// mix_key(seed, [salt, stream, block]) -- the per-block key of the Wiener
// driver (src/core/driver.rs:139-158).
__host__ __device__ __forceinline__ uint64_t wiener_block_key(uint64_t seed, uint64_t salt, uint64_t stream,
                                                              uint64_t block) {
    uint64_t s = splitmix64(seed);
    s = splitmix64(s ^ salt);
    s = splitmix64(s ^ stream);
    return splitmix64(s ^ block);
}

__host__ __device__ __forceinline__ double unit_open(uint64_t bits) {
    return (double)((bits >> 11) + 1) * (1.0 / 9007199254740992.0);
}

constexpr double kTau = 6.283185307179586476925286766559;

// Box-Muller cosine branch from one key (src/util/rng.rs:43-49).  Device
// log/cos are within 2 ulp of glibc; the integer stream is exact.
__device__ __forceinline__ double standard_normal(uint64_t key) {
    uint64_t a = splitmix64(key);
    uint64_t b = splitmix64(a ^ 0xD1B54A32D192ED03ull);
    double u = unit_open(a);
    double v = unit_open(b);
    return sqrt(-2.0 * log(u)) * cos(kTau * v);
}

// Single-precision Gaussian from the same two uniforms, for the FP32 path.
__device__ __forceinline__ float standard_normal_f32(uint64_t key) {
    uint64_t a = splitmix64(key);
    uint64_t b = splitmix64(a ^ 0xD1B54A32D192ED03ull);
    float u = (float)unit_open(a);
    float v = (float)unit_open(b);
    return sqrtf(-2.0f * logf(u)) * cospif(2.0f * v);
}

// Wiener stream tag of driver index j: (1 << 32) | j (driver.rs:134-140).
constexpr uint64_t kWienerStream0 = (1ull << 32) | 0ull;

// Streaming multiprocessors of the current device, queried once per device
// ordinal; the grid-sizing heuristics scale with it.
inline int device_sm_count() {
    static int cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
    int v = dev < 64 ? cache[dev] : 0;
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 1;
    if (dev < 64) cache[dev] = v;
    return v;
}

}  // namespace lg
