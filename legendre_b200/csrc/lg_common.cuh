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

#include "lg_log_table.h"

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

// ln u for the Box-Muller radius, u in [2^-53, 1], within 3.5e-16 relative
// of the exact logarithm (the Gaussian is held to 1e-12 of glibc's).  A
// table-driven reduction (the method of Tang, ACM TOMS 16, 1990, with the
// table holding the logarithm of its own rounded reciprocals): u = 2^e f
// with f in [sqrt(1/2), sqrt(2)), F_j = 1 + j/128 the nearest centre
// (j = rint((f - 1) 128), f - 1 exact), r = f RN(1/F_j) - 1 by one fma
// (|r| <= 0.0055), and ln u = e ln 2 + L_j + log1p(r) with
// L_j = -ln RN(1/F_j) from lg_log_table.h and log1p by its Taylor series to
// r^7 (truncation below 2e-17 relative).  The centre F_0 = 1 makes r = f - 1
// exact next to u = 1, where ln u is tiny; ln 2 is split so that e ln2_hi
// is exact.  u = 1 gives exactly +0.
__device__ __forceinline__ double log_unit_interval(double u) {
    const long long bu = __double_as_longlong(u);
    int e = (int)((bu >> 52) & 0x7ff) - 1023;
    double f = __longlong_as_double((bu & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    if (f > 1.4142135623730951) {
        f = 0.5 * f;
        e += 1;
    }
    const int j = __double2int_rn((f - 1.0) * 128.0);
    const double2 E = __ldg(&kLogTable[j - kLogTableMin]);
    const double r = fma(f, E.x, -1.0);
    double q = 1.0 / 7.0;
    q = fma(q, r, -1.0 / 6.0);
    q = fma(q, r, 1.0 / 5.0);
    q = fma(q, r, -0.25);
    q = fma(q, r, 1.0 / 3.0);
    q = fma(q, r, -0.5);
    const double p = fma(r * r, q, r);
    const double ln2_hi = 0x1.62e42fefa3800p-1, ln2_lo = 0x1.ef35793c76730p-45;
    return fma((double)e, ln2_hi, E.y) + fma((double)e, ln2_lo, p);
}

// cos x for the Box-Muller angle, x = fl(2 pi v) in (0, 2 pi], to about
// 1e-15 relative also next to the zeros of cos: Cody-Waite reduction
// r = x - k pi/2 with pi/2 in three parts (the first two of 33 bits, so
// k C1 and k C2 are exact and the two leading subtractions cancel exactly),
// then the sine or cosine Taylor polynomial of r (|r| <= pi/4, truncated at
// r^15 / r^16) and the quadrant's sign.
__device__ __forceinline__ double cos_full_turn(double x) {
    const double t = x * 0x1.45f306dc9c883p-1;  // x 2/pi
    const double magic = 0x1.8p52;               // t + magic rounds t to an integer (ties to even)
    const double kq = t + magic;
    const int q = __double2loint(kq) & 3;
    const double kd = kq - magic;
    double r = fma(-kd, 0x1.921fb544p+0, x);
    r = fma(-kd, 0x1.0b4611a6p-34, r);
    r = fma(-kd, 0x1.3198a2e037073p-69, r);
    const double z = r * r;
    // both polynomials, then a select (the lanes of a warp draw random
    // quadrants, so a branch would run both anyway, in two halves)
    double sp = 1.0 / 1307674368000.0;  // r - r^3/3! + r^5/5! - ... to r^15
    sp = fma(sp, z, -1.0 / 6227020800.0);
    sp = fma(sp, z, 1.0 / 39916800.0);
    sp = fma(sp, z, -1.0 / 362880.0);
    sp = fma(sp, z, 1.0 / 5040.0);
    sp = fma(sp, z, -1.0 / 120.0);
    sp = fma(sp, z, 1.0 / 6.0);
    const double sv = fma(-(r * z), sp, r);
    double cp = 1.0 / 20922789888000.0;  // 1 - r^2/2! + r^4/4! - ... to r^16
    cp = fma(cp, z, -1.0 / 87178291200.0);
    cp = fma(cp, z, 1.0 / 479001600.0);
    cp = fma(cp, z, -1.0 / 3628800.0);
    cp = fma(cp, z, 1.0 / 40320.0);
    cp = fma(cp, z, -1.0 / 720.0);
    cp = fma(cp, z, 1.0 / 24.0);
    cp = fma(cp, z, -0.5);
    const double cv = fma(z, cp, 1.0);
    const double v = (q & 1) ? sv : cv;
    return (q == 1 || q == 2) ? -v : v;
}

// Box-Muller cosine branch from one key (src/util/rng.rs:43-49): the
// integer stream and the uniforms are exact; the transcendental factors
// (log_unit_interval, cos_full_turn and the square root) are within about
// 1e-15 of glibc's, the Gaussian within 1e-12 relative as required.
__device__ __forceinline__ double standard_normal(uint64_t key) {
    uint64_t a = splitmix64(key);
    uint64_t b = splitmix64(a ^ 0xD1B54A32D192ED03ull);
    double u = unit_open(a);
    double v = unit_open(b);
    return sqrt(-2.0 * log_unit_interval(u)) * cos_full_turn(kTau * v);
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
