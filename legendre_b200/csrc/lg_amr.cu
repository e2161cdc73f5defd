// 2-D AMR on the device: Berger-Oliger subcycling of Model C or the heat
// model on a patch hierarchy, with plan-driven ghost fill (exchange, mirror,
// time-interpolated bilinear prolongation), restriction, gradient tagging
// and per-level work-list step kernels.  The hierarchy and its plans are
// built on the host (lg_amr_host.cu); regrids (tag on the device, cluster
// and migrate on the host) happen at the policy's cadence.
//
// Compiled with -fmad=false: every kernel keeps the reference's operand
// order, so FP64 results are bit-identical to the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/legendre_b200.h"
#include "lg_amr_host.h"
#include "lg_kernels.h"
#include "lg_modelc_ops.cuh"

namespace lg {
// lg_abi.cu
int abi_fail(lg_ctx* ctx, int code, const std::string& msg);
cudaStream_t abi_stream(lg_ctx* ctx);
int abi_device(lg_ctx* ctx);
void abi_count_launch(lg_ctx* ctx, int64_t n);
int64_t abi_launches(lg_ctx* ctx);
void abi_set_launches(lg_ctx* ctx, int64_t n);
}  // namespace lg

namespace {

using lg::amr::BlockDesc;
using lg::amr::GhostOp;
using lg::amr::RestrictOp;
using lg::amr::Unit;

constexpr int kMaxDepth = 8;

// Substep time of one level: t_l = fma(s_l, dt_l, t_{l-1}) down the
// recursion from the level-0 time in the device slot (subcycling.rs:256).
struct TimeChain {
    int depth;
    int s[kMaxDepth];
    double dt[kMaxDepth];
};

__device__ __forceinline__ double chain_time(double t0, const TimeChain& c) {
    double t = t0;
    for (int k = 0; k < c.depth; ++k) t = fma((double)c.s[k], c.dt[k], t);
    return t;
}

// ------------------------------------------------------------ kernels ----
// The value of field f of one ghost entry (GhostOp): a copy of a same-level
// interior entry of `in`, or the bilinear fold acc + v w over coarse
// interior corners, blended in time as old (1 - alpha) + new alpha
// (intergrid.rs:183-223 / 358-408).  All loads of one op are independent.
__device__ __forceinline__ double ghost_value(const GhostOp& op, const double* in, const double* cnew,
                                              const double* cold, int interp, double alpha, int f) {
    if (op.n == 0) return in[op.src[0] + (int64_t)f * op.stride[0]];
    double acc = 0.0, old = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < op.n) {
            const int64_t o = op.src[k] + (int64_t)f * op.stride[k];
            acc = acc + cnew[o] * op.w[k];
            if (interp) old = old + cold[o] * op.w[k];
        }
    }
    return interp ? old * (1.0 - alpha) + acc * alpha : acc;
}

// Ghost entries of one level, written in place (no time blend).  A and Ac
// (the coarser level) may be the same arena: the kernel writes ghost
// entries only and reads interior entries only.
__global__ void amr_fill_kernel(double* A, const double* Ac, const GhostOp* __restrict__ ops, int64_t nops,
                                int nfields) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += (int64_t)gridDim.x * blockDim.x) {
        const GhostOp op = ops[i];
        for (int f = 0; f < nfields; ++f) A[op.dst + (int64_t)f * op.dst_stride] = ghost_value(op, A, Ac, Ac, 0, 0.0, f);
    }
}

// Covered coarse cells <- sum of r x r fine children (dimension 0 fastest,
// from zero) times 1/r^2 (intergrid.rs:110-150).
// C (coarse level) and F (fine level) may be the same arena (disjoint slabs).
__global__ void amr_restrict_kernel(double* C, const double* F, const RestrictOp* __restrict__ ops, int64_t nops,
                                    int r, double inv, int f0, int f1);

// GradientTagger::tag_level (adapt.rs:78-103): flag where
// max_d |(u(+e_d) - u(-e_d)) 0.5| > threshold; cells in level coordinates.
__global__ void amr_tag_kernel(const BlockDesc* __restrict__ blocks, const int64_t* __restrict__ lo,
                               const Unit* __restrict__ units, int64_t nunits, const double* __restrict__ A,
                               int field, double threshold, int64_t* __restrict__ out, int64_t cap,
                               unsigned long long* __restrict__ count) {
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const BlockDesc b = blocks[un.block];
        const double* v = A + b.off + field * b.stride;
        const int sy = b.nx + 2;
        for (int c = un.start + threadIdx.x; c < un.start + un.count; c += blockDim.x) {
            const int i = c % b.nx, j = c / b.nx;
            const int o = (i + 1) + (j + 1) * sy;
            double gmax = 0.0;
            gmax = fmax(gmax, fabs((v[o + 1] - v[o - 1]) * 0.5));
            gmax = fmax(gmax, fabs((v[o + sy] - v[o - sy]) * 0.5));
            if (gmax > threshold) {
                const unsigned long long k = atomicAdd(count, 1ull);
                if ((int64_t)k < cap) {
                    out[2 * k] = lo[2 * un.block] + i;
                    out[2 * k + 1] = lo[2 * un.block + 1] + j;
                }
            }
        }
    }
}

// One fused ghost-fill + Euler-Maruyama launch over the tiles of a level.
// `in` / `out` are the level's current and next buffers (whole arenas,
// offsets from the block table); `cnew` / `cold` the coarse level's current
// and pre-step buffers for the time-interpolated prolongation (the coarse
// level's ping-pong buffer from before its step is the reference's
// snapshot: nothing writes that level's slabs of it until its next step).
// ------------------------------------------- tagging without allocation --
// Static scratch of lg_amr_tag_level_static: word 0 is the flag counter,
// then one (x, y) pair per flagged cell.  It holds kStaticTagCells cells
// (4 MiB), and a level with more cells is rejected before any launch, so the
// compaction cannot overflow.  The array is file-scope and shared by every
// call in the process on a device: calls that overlap on the GPU race.
constexpr int64_t kStaticTagCells = int64_t(1) << 18;
__device__ __align__(256) int64_t g_tag_scratch[2 + 2 * kStaticTagCells];

// amr_tag_kernel with its output in the static scratch (count at word 0)
__global__ void amr_tag_static_kernel(const BlockDesc* __restrict__ blocks, const int64_t* __restrict__ lo,
                                      const Unit* __restrict__ units, int64_t nunits, const double* __restrict__ A,
                                      int field, double threshold, int64_t* __restrict__ scratch) {
    unsigned long long* count = (unsigned long long*)scratch;
    int64_t* out = scratch + 2;
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const BlockDesc b = blocks[un.block];
        const double* v = A + b.off + field * b.stride;
        const int sy = b.nx + 2;
        for (int c = un.start + threadIdx.x; c < un.start + un.count; c += blockDim.x) {
            const int i = c % b.nx, j = c / b.nx;
            const int o = (i + 1) + (j + 1) * sy;
            double gmax = 0.0;
            gmax = fmax(gmax, fabs((v[o + 1] - v[o - 1]) * 0.5));
            gmax = fmax(gmax, fabs((v[o + sy] - v[o - sy]) * 0.5));
            if (gmax > threshold) {
                const unsigned long long k = atomicAdd(count, 1ull);
                if ((int64_t)k < kStaticTagCells) {
                    out[2 * k] = lo[2 * un.block] + i;
                    out[2 * k + 1] = lo[2 * un.block + 1] + j;
                }
            }
        }
    }
}

struct TileArgs {
    const lg::amr::Tile* tiles;
    int64_t ntiles;
    const GhostOp* tfill;
    const double* in;
    double* out;
    const double* cnew;
    const double* cold;
    double alpha;
    int interp;
    double dt;
    double* tdev;
    int slot;
    int write_t;   // this launch advances the level-0 time slot
    double dt0;    // level-0 step (for that advance)
    TimeChain chain;
    uint64_t seed;
    double scale_amp;
};

constexpr int kWin = lg::amr::kTile + 2;

// Stage the (w + 2) x (h + 2) window of a tile for NF fields: block interior
// entries from `in`, block ghost entries from the tile's fill ops.
// `pre`, when not null, is this thread's first fill op of the tile
// (tfill[fill0 + threadIdx.x]), read before the launch's dependency wait.
template <int NF>
__device__ __forceinline__ void stage_tile(const TileArgs& a, const lg::amr::Tile& T, double* s0, double* s1,
                                           const GhostOp* pre) {
    const int P = T.w + 2, R = T.h + 2, sy = T.nx + 2;
    const double* g0 = a.in + T.off;
    for (int k = threadIdx.x; k < P * R; k += blockDim.x) {
        const int c = k % P, r = k / P;
        const int i = T.x0 + c - 1, j = T.y0 + r - 1;
        if (i < 0 || i >= T.nx || j < 0 || j >= T.ny) continue;  // a ghost of the block
        const int o = (i + 1) + (j + 1) * sy;
        s0[k] = g0[o];
        if (NF == 2) s1[k] = g0[T.stride + o];
    }
    int k = T.fill0 + (int)threadIdx.x;
    if (pre && k < T.fill1) {
        s0[pre->dst] = ghost_value(*pre, a.in, a.cnew, a.cold, a.interp, a.alpha, 0);
        if (NF == 2) s1[pre->dst] = ghost_value(*pre, a.in, a.cnew, a.cold, a.interp, a.alpha, 1);
        k += blockDim.x;
    }
    for (; k < T.fill1; k += blockDim.x) {
        const GhostOp op = a.tfill[k];
        s0[op.dst] = ghost_value(op, a.in, a.cnew, a.cold, a.interp, a.alpha, 0);
        if (NF == 2) s1[op.dst] = ghost_value(op, a.in, a.cnew, a.cold, a.interp, a.alpha, 1);
    }
    __syncthreads();
}

// The tables of a CTA's first tile -- its descriptor and this thread's first
// fill op -- are read-only between regrids, so they are read before the
// launch's dependency wait (programmatic dependent launch), while the
// previous launch of the chain drains.
struct TilePrefetch {
    lg::amr::Tile T;
    GhostOp op;
    bool have_tile, have_op;
    __device__ __forceinline__ void load(const TileArgs& a) {
        have_tile = (int64_t)blockIdx.x < a.ntiles;
        have_op = false;
        if (have_tile) {
            T = a.tiles[blockIdx.x];
            const int k = T.fill0 + (int)threadIdx.x;
            if (k < T.fill1) {
                op = a.tfill[k];
                have_op = true;
            }
        }
    }
};

// Model C Euler-Maruyama on the tiles of one level (the reference-order cell
// update of phasefield.rs:353-422 with the Time and Wiener drivers,
// state.rs:706-753).  Lanes are the tile's columns, each warp a run of rows;
// a face flux is computed once and shared by the two cells it separates
// (right faces by shuffle, top faces down the row loop), which is bitwise
// the reference's per-cell evaluation: the left face of cell i + 1 and the
// right face of cell i are the same expression of the same operands.
template <bool NOISE>
__device__ __forceinline__ void modelc_tile(const TileArgs& a, const lg::MC<double>& m, const lg::amr::Tile& T,
                                            double t, double* sp, double* su, const GhostOp* pre) {
    using Ops = lg::OpsExact<double>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    stage_tile<2>(a, T, sp, su, pre);
    const int P = T.w + 2;
    const int rpw = (T.h + nwarps - 1) / nwarps;
    const int r0 = warp * rpw, r1 = min(T.h, r0 + rpw);
    if (r0 < r1) {  // warp-uniform
        const int ci = min(lane, T.w - 1);  // idle lanes duplicate the last column
        uint64_t block_key = 0;
        if (NOISE)
            block_key = lg::wiener_block_key(a.seed, (uint64_t)__double_as_longlong(t), lg::kWienerStream0,
                                             (uint64_t)T.block);
        // left faces of column 0, one row per lane
        double jl0;
        {
            const double* q = sp + 1 + (r0 + min(lane, r1 - r0 - 1) + 1) * P;
            jl0 = Ops::xface(m, q[0] - q[-1], q[P] - q[-P], q[P - 1], q[-P - 1]);
        }
        double jb;
        {
            const double* q = sp + (ci + 1) + (r0 + 1) * P;
            jb = Ops::yface(m, q[0] - q[-P], q[1] - q[-1], q[1 - P], q[-1 - P]);
        }
        for (int cj = r0; cj < r1; ++cj) {
            const double* q = sp + (ci + 1) + (cj + 1) * P;
            const double* w = su + (ci + 1) + (cj + 1) * P;
            const double jt = Ops::yface(m, q[P] - q[0], q[P + 1] - q[P - 1], q[1], q[-1]);
            const double jr = Ops::xface(m, q[1] - q[0], q[P + 1] - q[1 - P], q[P], q[-P]);
            double jl = __shfl_up_sync(0xffffffffu, jr, 1);
            const double jlb = __shfl_sync(0xffffffffu, jl0, cj - r0);
            if (lane == 0) jl = jlb;
            double kphi, ku;
            Ops::cell(m, jr, jl, jt, jb, q[0], q[1] - q[-1], q[P] - q[-P], w[0], w[-1], w[1], w[P], w[-P], kphi, ku);
            jb = jt;
            if (lane < T.w) {
                const int i = T.x0 + ci, j = T.y0 + cj;
                double phin = Ops::axpy(a.dt, kphi, q[0]);
                if (NOISE)
                    phin = Ops::add_noise(phin, a.scale_amp,
                                          Ops::noise(lg::splitmix64(block_key ^ (uint64_t)(j * T.nx + i))));
                const int64_t o = T.off + (i + 1) + (int64_t)(j + 1) * (T.nx + 2);
                a.out[o] = phin;
                a.out[o + T.stride] = Ops::axpy(a.dt, ku, w[0]);
            }
        }
    }
    __syncthreads();
}

// Programmatic dependent launch: a step of the subcycling chain lets the
// next launch start as soon as every CTA of this one is running, and waits
// for its predecessor's completion (and memory) only before it reads data a
// predecessor writes; table loads (tile descriptors, ghost and restriction
// ops) are read-only and may precede the wait.  Without the launch
// attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <bool NOISE>
__global__ void __launch_bounds__(256) amr_modelc_tiles(TileArgs a, lg::MC<double> m) {
    __shared__ double sp[kWin * kWin], su[kWin * kWin];
    pdl_release();
    TilePrefetch pf;
    pf.load(a);
    pdl_wait();
    const double t0 = a.tdev[a.slot];
    if (a.write_t && blockIdx.x == 0 && threadIdx.x == 0) a.tdev[a.slot ^ 1] = t0 + a.dt0;
    const double t = NOISE ? chain_time(t0, a.chain) : 0.0;
    if (pf.have_tile) modelc_tile<NOISE>(a, m, pf.T, t, sp, su, pf.have_op ? &pf.op : nullptr);
    for (int64_t ti = (int64_t)blockIdx.x + gridDim.x; ti < a.ntiles; ti += gridDim.x)
        modelc_tile<NOISE>(a, m, a.tiles[ti], t, sp, su, nullptr);
}

// Heat on the tiles of one level: k = lap(u) kappa, u + dt k
// (tests/amr.rs:324-339, finite_difference.rs:49-67, euler.rs:51-53).
__device__ __forceinline__ void heat_tile(const TileArgs& a, double kappa, double ih0, double ih1,
                                          const lg::amr::Tile& T, double* sp, const GhostOp* pre) {
    stage_tile<1>(a, T, sp, nullptr, pre);
    const int P = T.w + 2;
    for (int k = threadIdx.x; k < T.w * T.h; k += blockDim.x) {
        const int ci = k % T.w, cj = k / T.w;
        const double* q = sp + (ci + 1) + (cj + 1) * P;
        const double center = q[0];
        double acc = 0.0;
        acc += ((q[1] - (center + center)) + q[-1]) * ih0;
        acc += ((q[P] - (center + center)) + q[-P]) * ih1;
        const double kk = acc * kappa;
        a.out[T.off + (T.x0 + ci + 1) + (int64_t)(T.y0 + cj + 1) * (T.nx + 2)] = center + a.dt * kk;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) amr_heat_tiles(TileArgs a, double kappa, double ih0, double ih1) {
    __shared__ double sp[kWin * kWin];
    pdl_release();
    TilePrefetch pf;
    pf.load(a);
    pdl_wait();
    const double t0 = a.tdev[a.slot];
    if (a.write_t && blockIdx.x == 0 && threadIdx.x == 0) a.tdev[a.slot ^ 1] = t0 + a.dt0;
    if (pf.have_tile) heat_tile(a, kappa, ih0, ih1, pf.T, sp, pf.have_op ? &pf.op : nullptr);
    for (int64_t ti = (int64_t)blockIdx.x + gridDim.x; ti < a.ntiles; ti += gridDim.x)
        heat_tile(a, kappa, ih0, ih1, a.tiles[ti], sp, nullptr);
}

// restriction body shared by the launch-per-phase and persistent paths
__device__ __forceinline__ void restrict_ops(double* C, const double* F, const RestrictOp* __restrict__ ops,
                                             int64_t nops, int r, double inv, int f0, int f1) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += (int64_t)gridDim.x * blockDim.x) {
        const RestrictOp op = ops[i];
        for (int f = f0; f < f1; ++f) {
            const double* src = F + op.f + (int64_t)f * op.fstride;
            double sum = 0.0;
            for (int ky = 0; ky < r; ++ky)
                for (int kx = 0; kx < r; ++kx) sum += src[kx + ky * op.fsy];
            C[op.c + (int64_t)f * op.cstride] = sum * inv;
        }
    }
}

__global__ void amr_restrict_kernel(double* C, const double* F, const RestrictOp* __restrict__ ops, int64_t nops,
                                    int r, double inv, int f0, int f1) {
    pdl_release();
    pdl_wait();
    restrict_ops(C, F, ops, nops, r, inv, f0, f1);
}

// launch with the programmatic-dependent-launch attribute (see pdl_release)
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// ------------------------------------------------- persistent coarse step --
// One phase of a coarse step: a fused fill + step of one level's tiles, or
// the restriction of one fine level, with its buffer indices resolved on the
// host (the Berger-Oliger recursion of subcycling.rs:195-267, flattened).
struct Phase {
    int kind;  // 0: step, 1: restrict
    int level;
    int in, cnew, cold;  // step: own buffer and the coarse level's current / pre-step; restrict: fine, coarse
    int interp, write_t, slot;
    int r, barrier;  // restrict ratio; a grid barrier follows this phase
    int64_t first, count;  // tiles of the level's list, or restrict ops
    double alpha, dt, dt0, scale_amp, inv;
    TimeChain chain;
};

struct PersistArgs {
    const Phase* phases;
    int nphases;
    const lg::amr::Tile* tiles0;  // level 0's list
    const GhostOp* tfill0;
    const lg::amr::Tile* tiles;  // refined levels' list
    const GhostOp* tfill;
    const RestrictOp* rops;
    double* arena0;
    double* arena1;
    double* tdev;
    uint64_t seed;
    int nfields;
    double kappa;
    lg::MC<double> mc[kMaxDepth];
    unsigned* bar;  // [arrivals, generation]
    int* err;       // set when a barrier wait gave up
    long long spin_limit;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of a cooperative launch: every CTA's writes before it
// are visible to every CTA after it.  The wait is bounded: after spin_limit
// polls (or once another CTA has given up) the CTA records the error and
// every thread of it returns false.
__device__ bool grid_sync(const PersistArgs& a, unsigned& target, int* s_abort) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int abort = 0;
        target += 1;
        __threadfence();
        const unsigned prev = atomicAdd(&a.bar[0], 1u);
        if (prev == gridDim.x - 1) {
            atomicExch(&a.bar[0], 0u);
            __threadfence();
            atomicExch(&a.bar[1], target);
        } else {
            long long it = 0;
            while (ld_acquire_u32(&a.bar[1]) != target) {
                if (++it > a.spin_limit || *(volatile int*)a.err) {
                    abort = 1;
                    atomicExch(a.err, 1);
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        *s_abort = abort;
    }
    __syncthreads();
    return *s_abort == 0;
}

// Every phase of one (or two) coarse steps in one cooperative launch.
template <int MODEL, bool NOISE>
__global__ void __launch_bounds__(256) amr_persistent(PersistArgs a) {
    __shared__ double sp[kWin * kWin], su[kWin * kWin];
    __shared__ int s_abort;
    // the phase table is read-only: the next phase's descriptor is fetched
    // into the other half of this buffer while the current phase runs
    __shared__ Phase s_ph[2];
    constexpr int kWords = (int)(sizeof(Phase) / sizeof(int));
    static_assert(sizeof(Phase) % sizeof(int) == 0, "Phase is copied as words");
    unsigned target = 0;
    if (threadIdx.x == 0) {
        s_abort = *(volatile int*)a.err;  // an earlier launch gave up: do nothing
        target = ld_acquire_u32(&a.bar[1]);
    }
    for (int k = threadIdx.x; k < kWords; k += blockDim.x)
        ((int*)&s_ph[0])[k] = ((const int*)&a.phases[0])[k];
    __syncthreads();
    if (s_abort) return;
    for (int p = 0; p < a.nphases; ++p) {
        const Phase& ph = s_ph[p & 1];
        if (p + 1 < a.nphases && threadIdx.x >= blockDim.x - 32)  // last warp prefetches
            for (int k = threadIdx.x - (blockDim.x - 32); k < kWords; k += 32)
                ((int*)&s_ph[(p + 1) & 1])[k] = ((const int*)&a.phases[p + 1])[k];
        if (ph.kind == 0) {
            TileArgs t{};
            t.tiles = (ph.level == 0 ? a.tiles0 : a.tiles) + ph.first;
            t.ntiles = ph.count;
            t.tfill = ph.level == 0 ? a.tfill0 : a.tfill;
            t.in = ph.in ? a.arena1 : a.arena0;
            t.out = ph.in ? a.arena0 : a.arena1;
            t.cnew = ph.cnew ? a.arena1 : a.arena0;
            t.cold = ph.cold ? a.arena1 : a.arena0;
            t.alpha = ph.alpha;
            t.interp = ph.interp;
            t.dt = ph.dt;
            t.seed = a.seed;
            t.scale_amp = ph.scale_amp;
            const double t0 = __ldcg(&a.tdev[ph.slot]);
            if (ph.write_t && blockIdx.x == 0 && threadIdx.x == 0) a.tdev[ph.slot ^ 1] = t0 + ph.dt0;
            const double tt = NOISE ? chain_time(t0, ph.chain) : 0.0;
            for (int64_t ti = blockIdx.x; ti < t.ntiles; ti += gridDim.x) {
                if (MODEL == LG_MODEL_C)
                    modelc_tile<NOISE>(t, a.mc[ph.level], t.tiles[ti], tt, sp, su, nullptr);
                else
                    heat_tile(t, a.kappa, a.mc[ph.level].ih0, a.mc[ph.level].ih1, t.tiles[ti], sp, nullptr);
            }
        } else {
            double* C = ph.cnew ? a.arena1 : a.arena0;
            const double* F = ph.in ? a.arena1 : a.arena0;
            restrict_ops(C, F, a.rops + ph.first, ph.count, ph.r, ph.inv, 0, a.nfields);
        }
        const bool sync = ph.barrier && p + 1 < a.nphases;
        if (sync) {
            if (!grid_sync(a, target, &s_abort)) return;
        } else {
            __syncthreads();  // the prefetched descriptor is complete before it is read
        }
    }
}

unsigned grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)lg::device_sm_count() * 32));
}

template <class T>
T* dev_upload(const std::vector<T>& v, cudaError_t* err) {
    T* p = nullptr;
    if (v.empty()) return nullptr;
    *err = cudaMalloc(&p, v.size() * sizeof(T));
    if (*err != cudaSuccess) return nullptr;
    *err = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
}

}  // namespace

namespace {
// the tile height of a level's plans and the rows each warp of a tile owns
struct TileShape {
    int rows, rows_per_warp;
};
// one blob on the device holding every table of a Plans
struct Tables {
    char* d = nullptr;
    size_t cap = 0;
    BlockDesc* blocks = nullptr;
    int64_t* lo = nullptr;
    GhostOp* fill = nullptr;
    RestrictOp* restrict_ops = nullptr;
    Unit* units = nullptr;
    lg::amr::Tile* tiles = nullptr;
    GhostOp* tfill = nullptr;
};
}  // namespace

struct lg_amr_sim {
    lg_ctx* ctx = nullptr;
    lg::amr::Layout layout;
    lg::amr::Plans plans;
    int model = LG_MODEL_C;
    lg_modelc_params mp{};
    double kappa = 0.0;
    int integrator = LG_AMR_SUBCYCLING;
    uint64_t seed = 0;
    bool has_policy = false;
    lg::amr::Policy policy;
    int nfields = 2;
    lg::amr::Plans plans0;  // level 0's ring, tiles and units: built once
    // device: two state arenas (ping-pong per level) of arena_cap elements,
    // and the plan tables (tab0 from plans0, uploaded once; tab from plans)
    double* arena[2] = {nullptr, nullptr};
    int64_t arena_cap = 0;
    Tables tab0, tab;
    int64_t* d_tags = nullptr;
    int64_t tag_cap = 0;
    unsigned long long* d_count = nullptr;
    double* d_t = nullptr;
    std::vector<int> cur;  // current buffer per level
    int tslot = 0;
    double t = 0.0;
    int64_t step_index = 0, epoch = 0;
    std::map<std::string, std::pair<cudaGraphExec_t, int64_t>> graphs;  // exec, launches
    // persistent path: phase tables per (epoch, dt, slot, buffers, steps),
    // the grid barrier's state and its error flag
    std::map<std::string, std::pair<void*, int>> phase_tabs;  // device table, phase count
    unsigned* d_bar = nullptr;
    int* d_err = nullptr;
    long long barrier_spin_limit = 4000000;  // polls of >= 128 ns: well over a second
    int coop_grid[2] = {0, 0};  // per model kind (noise-free / noisy) once measured
    std::vector<double> host_old, host_new;  // host staging of whole states (get/set)
    std::vector<TileShape> tile_shapes;      // per level
    // regrid migration on the device: the old state's image and the old
    // hierarchy's patch tables (grow-only)
    double* d_mig_old = nullptr;
    int64_t mig_old_cap = 0;
    char* d_mig_tab = nullptr;
    size_t mig_tab_cap = 0;
    int* d_mig_err = nullptr;
};

namespace {

int fail(lg_amr_sim* s, int code, const std::string& m) { return lg::abi_fail(s ? s->ctx : nullptr, code, m); }

#define AMR_CUDA(s, call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail((s), LG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void drop_graphs(lg_amr_sim* s) {
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second.first);
    s->graphs.clear();
    for (auto& kv : s->phase_tabs) cudaFree(kv.second.first);
    s->phase_tabs.clear();
}

void free_device(lg_amr_sim* s) {
    drop_graphs(s);
    for (double*& a : s->arena) {
        cudaFree(a);
        a = nullptr;
    }
    s->arena_cap = 0;
    for (Tables* t : {&s->tab0, &s->tab}) {
        cudaFree(t->d);
        *t = Tables{};
    }
}

// elements of the level-0 slabs, which lead every arena (the base tiling
// never changes, so this prefix is the same in every layout)
int64_t level0_elems(const lg_amr_sim* s) {
    const uint32_t b1 = s->layout.level_start[1];
    const BlockDesc& last = s->plans.blocks[b1 - 1];
    return last.off + last.stride * s->nfields;
}

// level l's slabs are contiguous in the arena: [off of its first block, end of its last)
std::pair<int64_t, int64_t> level_range(const lg_amr_sim* s, int level) {
    const uint32_t b0 = s->layout.level_start[level], b1 = s->layout.level_start[level + 1];
    if (b0 == b1) return {0, 0};
    const BlockDesc& last = s->plans.blocks[b1 - 1];
    return {s->plans.blocks[b0].off, last.off + last.stride * s->nfields};
}

// Tile shape per level.  A level with enough cells to fill the GPU several
// times over is throughput-bound: 32-row tiles, four rows per warp, so that
// each face flux is shared down a warp's rows.  A sparse fine level is
// latency-bound (its launch is one short wave): tiles of at most 8 rows with
// one row per warp, the tallest that still gives two tiles per SM.
std::vector<TileShape> choose_tile_shapes(const lg::amr::Layout& g) {
    const int kSMs = lg::device_sm_count();
    std::vector<TileShape> shapes(g.max_levels(), TileShape{lg::amr::kTile, 4});
    for (int l = 0; l < g.num_levels(); ++l) {
        int64_t cells = 0;
        for (uint32_t b = g.level_start[l]; b < g.level_start[l + 1]; ++b) cells += g.patches[b].bx.cells();
        if (cells >= (int64_t)kSMs * 2048) continue;
        for (int r : {8, 4, 2, 1}) {
            int64_t tiles = 0;
            for (uint32_t b = g.level_start[l]; b < g.level_start[l + 1]; ++b) {
                const auto& bx = g.patches[b].bx;
                tiles += ((bx.extent(0) + lg::amr::kTile - 1) / lg::amr::kTile) * ((bx.extent(1) + r - 1) / r);
            }
            shapes[l] = TileShape{r, 1};
            if (tiles >= 2 * kSMs) break;
        }
    }
    return shapes;
}
std::vector<int> rows_of(const std::vector<TileShape>& s) {
    std::vector<int> r;
    for (const auto& t : s) r.push_back(t.rows);
    return r;
}
int tile_threads(const TileShape& t) { return 32 * std::max(1, (t.rows + t.rows_per_warp - 1) / t.rows_per_warp); }

// pack every table of `P` into one blob and upload it into `T`
// (stream-ordered; the caller has synchronised the stream, so no kernel
// reads the old tables)
int upload_tables(lg_amr_sim* s, const lg::amr::Plans& P, const lg::amr::Layout& g, Tables& T) {
    std::vector<int64_t> lo;
    for (const auto& p : g.patches) {
        lo.push_back(p.bx.lo[0]);
        lo.push_back(p.bx.lo[1]);
    }
    size_t off = 0;
    auto reserve = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_blocks = reserve(P.blocks.size() * sizeof(BlockDesc));
    const size_t o_lo = reserve(lo.size() * sizeof(int64_t));
    const size_t o_fill = reserve(P.fill.size() * sizeof(GhostOp));
    const size_t o_restrict = reserve(P.restrict_ops.size() * sizeof(RestrictOp));
    const size_t o_units = reserve(P.units.size() * sizeof(Unit));
    const size_t o_tiles = reserve(P.tiles.size() * sizeof(lg::amr::Tile));
    const size_t o_tfill = reserve(P.tile_fill.size() * sizeof(GhostOp));
    std::vector<char> blob(std::max<size_t>(off, 256), 0);
    auto put = [&](size_t o, const void* src, size_t bytes) {
        if (bytes) std::memcpy(blob.data() + o, src, bytes);
    };
    put(o_blocks, P.blocks.data(), P.blocks.size() * sizeof(BlockDesc));
    put(o_lo, lo.data(), lo.size() * sizeof(int64_t));
    put(o_fill, P.fill.data(), P.fill.size() * sizeof(GhostOp));
    put(o_restrict, P.restrict_ops.data(), P.restrict_ops.size() * sizeof(RestrictOp));
    put(o_units, P.units.data(), P.units.size() * sizeof(Unit));
    put(o_tiles, P.tiles.data(), P.tiles.size() * sizeof(lg::amr::Tile));
    put(o_tfill, P.tile_fill.data(), P.tile_fill.size() * sizeof(GhostOp));
    if (blob.size() > T.cap) {
        cudaFree(T.d);
        T = Tables{};
        const size_t cap = blob.size() + blob.size() / 4;
        AMR_CUDA(s, cudaMalloc(&T.d, cap));
        T.cap = cap;
    }
    cudaStream_t st = lg::abi_stream(s->ctx);
    AMR_CUDA(s, cudaMemcpyAsync(T.d, blob.data(), blob.size(), cudaMemcpyHostToDevice, st));
    AMR_CUDA(s, cudaStreamSynchronize(st));
    T.blocks = (BlockDesc*)(T.d + o_blocks);
    T.lo = (int64_t*)(T.d + o_lo);
    T.fill = (GhostOp*)(T.d + o_fill);
    T.restrict_ops = (RestrictOp*)(T.d + o_restrict);
    T.units = (Unit*)(T.d + o_units);
    T.tiles = (lg::amr::Tile*)(T.d + o_tiles);
    T.tfill = (GhostOp*)(T.d + o_tfill);
    return LG_OK;
}

// the ring, tile and unit lists of a level: level 0's are built once
struct Lists {
    const lg::amr::Plans* P;
    const Tables* T;
};
Lists lists(const lg_amr_sim* s, int level) {
    return level == 0 ? Lists{&s->plans0, &s->tab0} : Lists{&s->plans, &s->tab};
}

// arenas of at least `need` elements; when they are reallocated, the first
// `keep` elements of the buffer `from` move to the new buffer 0 and the
// function returns 0 in *now, else *now = from
int ensure_arenas(lg_amr_sim* s, int64_t need, int64_t keep, int from, int* now) {
    *now = from;
    if (need <= s->arena_cap) return LG_OK;
    cudaStream_t st = lg::abi_stream(s->ctx);
    const int64_t cap = need + need / 4;
    const size_t bytes = (size_t)cap * sizeof(double);
    double* fresh[2] = {nullptr, nullptr};
    cudaError_t e = cudaMalloc(&fresh[0], bytes);
    if (e == cudaSuccess) e = cudaMalloc(&fresh[1], bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(fresh[0], 0, bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(fresh[1], 0, bytes, st);
    if (e == cudaSuccess && keep > 0 && s->arena[from])
        e = cudaMemcpyAsync(fresh[0], s->arena[from], (size_t)keep * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(fresh[0]);
        cudaFree(fresh[1]);
        return fail(s, LG_ERR_NOMEM, std::string("AMR arena allocation: ") + cudaGetErrorString(e));
    }
    drop_graphs(s);  // graphs hold the old arena pointers
    for (int k = 0; k < 2; ++k) {
        cudaFree(s->arena[k]);
        s->arena[k] = fresh[k];
    }
    s->arena_cap = cap;
    *now = 0;
    return LG_OK;
}

// plans, tables and zeroed arenas for a fresh simulation
int setup_device(lg_amr_sim* s) {
    lg::amr::Layout base;
    std::string err = lg::amr::build_layout(s->layout.base, s->layout.ratios, {}, &base);
    if (!err.empty()) return fail(s, LG_ERR_STATE, err);
    s->tile_shapes = choose_tile_shapes(s->layout);
    s->plans0 = lg::amr::build_plans(base, s->nfields, 1024, 0, rows_of(s->tile_shapes));
    s->plans = lg::amr::build_plans(s->layout, s->nfields, 1024, 1, rows_of(s->tile_shapes));
    if (!s->plans.error.empty()) return fail(s, LG_ERR_STATE, s->plans.error);
    int rc = upload_tables(s, s->plans0, base, s->tab0);
    if (rc == LG_OK) rc = upload_tables(s, s->plans, s->layout, s->tab);
    if (rc != LG_OK) return rc;
    int now = 0;
    rc = ensure_arenas(s, s->plans.arena_elems, 0, 0, &now);
    if (rc != LG_OK) return rc;
    s->cur.assign(s->layout.num_levels(), 0);
    return LG_OK;
}

// the whole state (each level's current buffer) into `host`, arena layout
int download_state(lg_amr_sim* s, std::vector<double>& host) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    host.resize((size_t)s->plans.arena_elems);
    for (int l = 0; l < s->layout.num_levels(); ++l) {
        const auto r = level_range(s, l);
        if (r.second > r.first)
            AMR_CUDA(s, cudaMemcpyAsync(host.data() + r.first, s->arena[s->cur[l]] + r.first,
                                        (size_t)(r.second - r.first) * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    AMR_CUDA(s, cudaStreamSynchronize(st));
    return LG_OK;
}

int upload_state(lg_amr_sim* s, const std::vector<double>& host) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    for (int l = 0; l < s->layout.num_levels(); ++l) {
        const auto r = level_range(s, l);
        if (r.second > r.first)
            AMR_CUDA(s, cudaMemcpyAsync(s->arena[s->cur[l]] + r.first, host.data() + r.first,
                                        (size_t)(r.second - r.first) * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    AMR_CUDA(s, cudaStreamSynchronize(st));
    return LG_OK;
}

int launch_fill(lg_amr_sim* s, int level) {
    const Lists L = lists(s, level);
    const int64_t a = L.P->fill_start[level], b = L.P->fill_start[level + 1];
    if (b == a) return LG_OK;
    const double* coarse = level > 0 ? s->arena[s->cur[level - 1]] : nullptr;
    amr_fill_kernel<<<grid_for(b - a, 256), 256, 0, lg::abi_stream(s->ctx)>>>(s->arena[s->cur[level]], coarse,
                                                                                L.T->fill + a, b - a, s->nfields);
    lg::abi_count_launch(s->ctx, 1);
    AMR_CUDA(s, cudaGetLastError());
    return LG_OK;
}

int launch_restrict(lg_amr_sim* s, int fine, int f0, int f1) {
    const int64_t a = s->plans.restrict_start[fine], b = s->plans.restrict_start[fine + 1];
    if (b == a) return LG_OK;
    const int r = (int)s->layout.ratios[fine - 1];
    const double inv = 1.0 / ((double)r * (double)r);
    AMR_CUDA(s, launch_pdl(amr_restrict_kernel, dim3(grid_for(b - a, 256)), dim3(256), lg::abi_stream(s->ctx),
                           s->arena[s->cur[fine - 1]], (const double*)s->arena[s->cur[fine]],
                           (const RestrictOp*)(s->tab.restrict_ops + a), (int64_t)(b - a), r, inv, f0, f1));
    lg::abi_count_launch(s->ctx, 1);
    AMR_CUDA(s, cudaGetLastError());
    return LG_OK;
}

lg::MC<double> level_mc(const lg_amr_sim* s, int level) {
    lg::ModelCDev m{};
    const lg_modelc_params* p = &s->mp;
    m.lambda = p->lambda;
    m.d_thermal = p->d_thermal;
    m.a_bar = std::fma(3.0, -p->eps4, 1.0);
    m.eps_prime = 3.0 * p->eps4 / m.a_bar;
    m.tol = p->anisotropy_tol;
    m.f_a_bar = std::fma(3.0, -p->eps4, 1.0);
    m.f_eps_prime = 3.0 * p->eps4 / m.f_a_bar;
    m.f_a12 = 4.0 * m.f_a_bar * m.f_eps_prime;
    m.f_tol = p->flux_tol;
    const auto& h = s->layout.level_spacing[level];
    m.inv_h2_flux = 1.0 / (h[0] * h[1]);
    m.inv_h2[0] = 1.0 / (h[0] * h[0]);
    m.inv_h2[1] = 1.0 / (h[1] * h[1]);
    return lg::to_mc<double>(m);
}

// one fused ghost fill + Euler-Maruyama update of level `level`, reading
// its current buffer and writing the other; the coarse source is the
// coarse level's current buffer, blended with its pre-step buffer when
// `interp`
int launch_level(lg_amr_sim* s, int level, bool interp, double alpha, double dt, const TimeChain& chain,
                 bool write_t, double dt0) {
    const Lists L = lists(s, level);
    const int64_t t0 = L.P->tile_start[level], t1 = L.P->tile_start[level + 1];
    if (t1 == t0) return LG_OK;
    TileArgs a{};
    a.tiles = L.T->tiles + t0;
    a.ntiles = t1 - t0;
    a.tfill = L.T->tfill;
    const int in = s->cur[level];
    a.in = s->arena[in];
    a.out = s->arena[in ^ 1];
    a.cnew = level > 0 ? s->arena[s->cur[level - 1]] : nullptr;
    a.cold = level > 0 ? s->arena[s->cur[level - 1] ^ 1] : nullptr;
    a.alpha = alpha;
    a.interp = interp ? 1 : 0;
    a.dt = dt;
    a.tdev = s->d_t;
    a.slot = s->tslot;
    a.write_t = write_t ? 1 : 0;
    a.dt0 = dt0;
    a.chain = chain;
    a.seed = s->seed;
    a.scale_amp = std::sqrt(dt) * s->mp.noise_amplitude;
    const unsigned g = (unsigned)std::min<int64_t>(t1 - t0, (int64_t)lg::device_sm_count() * 16);
    const int threads = tile_threads(s->tile_shapes[level]);
    cudaStream_t st = lg::abi_stream(s->ctx);
    if (s->model == LG_MODEL_C) {
        if (s->mp.noise_amplitude != 0.0)
            AMR_CUDA(s, launch_pdl(amr_modelc_tiles<true>, dim3(g), dim3(threads), st, a, level_mc(s, level)));
        else
            AMR_CUDA(s, launch_pdl(amr_modelc_tiles<false>, dim3(g), dim3(threads), st, a, level_mc(s, level)));
    } else {
        const auto& h = s->layout.level_spacing[level];
        AMR_CUDA(s, launch_pdl(amr_heat_tiles, dim3(g), dim3(threads), st, a, s->kappa, 1.0 / (h[0] * h[0]),
                               1.0 / (h[1] * h[1])));
    }
    lg::abi_count_launch(s->ctx, 1);
    AMR_CUDA(s, cudaGetLastError());
    return LG_OK;
}

double stable_dt_at(const lg_amr_sim* s, int level) {
    const auto& h = s->layout.level_spacing[level];
    const double hm = std::min(h[0], h[1]);
    if (s->model == LG_MODEL_C) return 0.2 * (hm * hm) / s->mp.d_thermal;  // phasefield.rs:446-449
    return 0.25 * (hm * hm) / s->kappa;                                     // tests/amr.rs:339-341
}

// Subcycle::advance (subcycling.rs:195-267): ghosts (coarse source
// interpolated in time) and the step of this level in one launch, then the
// next level subcycled and restricted
int advance(lg_amr_sim* s, int level, TimeChain chain, double dt, double alpha, bool first) {
    int rc = launch_level(s, level, level > 0, alpha, dt, chain, first, dt);
    if (rc != LG_OK) return rc;
    s->cur[level] ^= 1;
    const int child = level + 1;
    if (child < s->layout.num_levels()) {
        const double n_f = std::round(stable_dt_at(s, level) / stable_dt_at(s, child));
        const uint64_t n = (uint64_t)std::max(n_f, 1.0);
        const double dt_child = dt / (double)n;
        if (chain.depth >= kMaxDepth) return fail(s, LG_ERR_INVALID, "too many refinement levels");
        for (uint64_t k = 0; k < n; ++k) {
            TimeChain c = chain;
            c.s[c.depth] = (int)k;
            c.dt[c.depth] = dt_child;
            c.depth += 1;
            rc = advance(s, child, c, dt_child, (double)k / (double)n, false);
            if (rc != LG_OK) return rc;
        }
        rc = launch_restrict(s, child, 0, s->nfields);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

// The phases of Subcycle::advance from `level` down, recorded instead of
// launched: the same buffer bookkeeping as advance(), on copies.
void record_advance(const lg_amr_sim* s, int level, TimeChain chain, double dt, double alpha, bool first,
                    std::vector<int>& cur, int slot, std::vector<Phase>& out) {
    const Lists L = lists(s, level);
    Phase ph{};
    ph.kind = 0;
    ph.level = level;
    ph.in = cur[level];
    ph.cnew = level > 0 ? cur[level - 1] : 0;
    ph.cold = level > 0 ? cur[level - 1] ^ 1 : 0;
    ph.interp = level > 0 ? 1 : 0;
    ph.write_t = first ? 1 : 0;
    ph.slot = slot;
    ph.barrier = 1;
    ph.first = L.P->tile_start[level];
    ph.count = L.P->tile_start[level + 1] - ph.first;
    ph.alpha = alpha;
    ph.dt = dt;
    ph.dt0 = dt;
    ph.scale_amp = std::sqrt(dt) * s->mp.noise_amplitude;
    ph.chain = chain;
    out.push_back(ph);
    cur[level] ^= 1;
    const int child = level + 1;
    if (child < s->layout.num_levels()) {
        const double n_f = std::round(stable_dt_at(s, level) / stable_dt_at(s, child));
        const uint64_t n = (uint64_t)std::max(n_f, 1.0);
        const double dt_child = dt / (double)n;
        for (uint64_t k = 0; k < n; ++k) {
            TimeChain c = chain;
            c.s[c.depth] = (int)k;
            c.dt[c.depth] = dt_child;
            c.depth += 1;
            record_advance(s, child, c, dt_child, (double)k / (double)n, false, cur, slot, out);
        }
        Phase rp{};
        rp.kind = 1;
        rp.level = child;
        rp.in = cur[child];
        rp.cnew = cur[child - 1];
        rp.barrier = 1;
        rp.first = s->plans.restrict_start[child];
        rp.count = s->plans.restrict_start[child + 1] - rp.first;
        rp.r = (int)s->layout.ratios[child - 1];
        rp.inv = 1.0 / ((double)rp.r * (double)rp.r);
        if (rp.count > 0) out.push_back(rp);
    }
}

// one coarse step of either integrator, recorded
void record_coarse_step(const lg_amr_sim* s, double dt, std::vector<int>& cur, int slot, std::vector<Phase>& out) {
    TimeChain c{};
    if (s->integrator == LG_AMR_SUBCYCLING) {
        record_advance(s, 0, c, dt, 0.0, true, cur, slot, out);
        return;
    }
    for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
        Phase rp{};
        rp.kind = 1;
        rp.level = fine;
        rp.in = cur[fine];
        rp.cnew = cur[fine - 1];
        rp.barrier = 1;
        rp.first = s->plans.restrict_start[fine];
        rp.count = s->plans.restrict_start[fine + 1] - rp.first;
        rp.r = (int)s->layout.ratios[fine - 1];
        rp.inv = 1.0 / ((double)rp.r * (double)rp.r);
        if (rp.count > 0) out.push_back(rp);
    }
    // every level steps from the pre-step buffers: one phase, no barriers
    // between the levels' tile lists
    const int L = s->layout.num_levels();
    for (int l = 0; l < L; ++l) {
        const Lists lst = lists(s, l);
        Phase ph{};
        ph.kind = 0;
        ph.level = l;
        ph.in = cur[l];
        ph.cnew = l > 0 ? cur[l - 1] : 0;
        ph.cold = ph.cnew;
        ph.write_t = l == 0 ? 1 : 0;
        ph.slot = slot;
        ph.barrier = l == L - 1 ? 1 : 0;
        ph.first = lst.P->tile_start[l];
        ph.count = lst.P->tile_start[l + 1] - ph.first;
        ph.dt = dt;
        ph.dt0 = dt;
        ph.scale_amp = std::sqrt(dt) * s->mp.noise_amplitude;
        ph.chain = c;
        out.push_back(ph);
    }
    for (int l = 0; l < L; ++l) cur[l] ^= 1;
}

template <int MODEL, bool NOISE>
int launch_persistent_kernel(lg_amr_sim* s, const PersistArgs& a) {
    const int kind = NOISE ? 1 : 0;
    auto kernel = amr_persistent<MODEL, NOISE>;
    if (s->coop_grid[kind] == 0) {
        int per_sm = 0, sms = 0;
        AMR_CUDA(s, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0));
        AMR_CUDA(s, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, lg::abi_device(s->ctx)));
        if (per_sm < 1) return fail(s, LG_ERR_DEVICE, "persistent AMR kernel cannot be resident");
        s->coop_grid[kind] = per_sm * sms;
    }
    PersistArgs args = a;
    void* params[] = {&args};
    AMR_CUDA(s, cudaLaunchCooperativeKernel((const void*)kernel, dim3((unsigned)s->coop_grid[kind]), dim3(256), params,
                                            0, lg::abi_stream(s->ctx)));
    lg::abi_count_launch(s->ctx, 1);
    return LG_OK;
}

// `nsteps` (1 or 2) coarse steps in one cooperative launch
int run_persistent(lg_amr_sim* s, double dt, int nsteps) {
    char key[160];
    snprintf(key, sizeof key, "%lld|%a|%d|%d|", (long long)s->epoch, dt, s->tslot, nsteps);
    std::string k = key;
    for (int c : s->cur) k += c ? '1' : '0';
    std::vector<int> cur = s->cur;
    int slot = s->tslot;
    auto it = s->phase_tabs.find(k);
    if (it == s->phase_tabs.end()) {
        std::vector<Phase> ph;
        for (int n = 0; n < nsteps; ++n) {
            record_coarse_step(s, dt, cur, slot, ph);
            slot ^= 1;
        }
        void* d = nullptr;
        AMR_CUDA(s, cudaMalloc(&d, ph.size() * sizeof(Phase)));
        cudaStream_t st = lg::abi_stream(s->ctx);
        cudaError_t e = cudaMemcpyAsync(d, ph.data(), ph.size() * sizeof(Phase), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            cudaFree(d);
            return fail(s, LG_ERR_CUDA, std::string("phase table upload: ") + cudaGetErrorString(e));
        }
        it = s->phase_tabs.emplace(k, std::make_pair(d, (int)ph.size())).first;
    } else {
        std::vector<Phase> ph;
        for (int n = 0; n < nsteps; ++n) {  // the buffer bookkeeping only
            record_coarse_step(s, dt, cur, slot, ph);
            slot ^= 1;
        }
    }
    PersistArgs a{};
    a.phases = (const Phase*)it->second.first;
    a.nphases = it->second.second;
    a.tiles0 = s->tab0.tiles;
    a.tfill0 = s->tab0.tfill;
    a.tiles = s->tab.tiles;
    a.tfill = s->tab.tfill;
    a.rops = s->tab.restrict_ops;
    a.arena0 = s->arena[0];
    a.arena1 = s->arena[1];
    a.tdev = s->d_t;
    a.seed = s->seed;
    a.nfields = s->nfields;
    a.kappa = s->kappa;
    for (int l = 0; l < s->layout.num_levels() && l < kMaxDepth; ++l) {
        a.mc[l] = level_mc(s, l);
        if (s->model != LG_MODEL_C) {
            const auto& h = s->layout.level_spacing[l];
            a.mc[l].ih0 = 1.0 / (h[0] * h[0]);
            a.mc[l].ih1 = 1.0 / (h[1] * h[1]);
        }
    }
    a.bar = s->d_bar;
    a.err = s->d_err;
    a.spin_limit = s->barrier_spin_limit;
    int rc;
    if (s->model == LG_MODEL_C)
        rc = s->mp.noise_amplitude != 0.0 ? launch_persistent_kernel<LG_MODEL_C, true>(s, a)
                                          : launch_persistent_kernel<LG_MODEL_C, false>(s, a);
    else
        rc = launch_persistent_kernel<LG_MODEL_HEAT, false>(s, a);
    if (rc != LG_OK) return rc;
    s->cur = cur;
    s->tslot = slot;
    return LG_OK;
}

int one_coarse_step(lg_amr_sim* s, double dt) {
    TimeChain c{};
    if (s->integrator == LG_AMR_SUBCYCLING) {
        int rc = advance(s, 0, c, dt, 0.0, true);
        if (rc != LG_OK) return rc;
    } else {
        // the model's AMR fill_ghosts (phasefield.rs:454-467): restrict, then
        // every level filled and stepped together from the pre-step buffers
        for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
            int rc = launch_restrict(s, fine, 0, s->nfields);
            if (rc != LG_OK) return rc;
        }
        for (int l = 1; l < s->layout.num_levels(); ++l)
            if (s->cur[l] != s->cur[0]) return fail(s, LG_ERR_STATE, "level buffers out of step");
        for (int l = 0; l < s->layout.num_levels(); ++l) {
            int rc = launch_level(s, l, false, 0.0, dt, c, l == 0, dt);
            if (rc != LG_OK) return rc;
        }
        for (int l = 0; l < s->layout.num_levels(); ++l) s->cur[l] ^= 1;
    }
    s->tslot ^= 1;
    return LG_OK;
}

int tag_level(lg_amr_sim* s, int field, int level, double threshold, std::vector<std::array<int64_t, 2>>& cells) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    int64_t need = 0;
    for (uint32_t b = s->layout.level_start[level]; b < s->layout.level_start[level + 1]; ++b)
        need += (int64_t)s->plans.blocks[b].nx * s->plans.blocks[b].ny;
    if (need > s->tag_cap) {
        cudaFree(s->d_tags);
        s->d_tags = nullptr;
        AMR_CUDA(s, cudaMalloc(&s->d_tags, 2 * need * sizeof(int64_t)));
        s->tag_cap = need;
    }
    if (!s->d_count) AMR_CUDA(s, cudaMalloc(&s->d_count, sizeof(unsigned long long)));
    AMR_CUDA(s, cudaMemsetAsync(s->d_count, 0, sizeof(unsigned long long), st));
    const Lists L = lists(s, level);
    const int64_t u0 = L.P->unit_start[level], u1 = L.P->unit_start[level + 1];
    if (u1 > u0) {
        amr_tag_kernel<<<(unsigned)std::min<int64_t>(u1 - u0, 65535), 256, 0, st>>>(
            s->tab.blocks, s->tab.lo, L.T->units + u0, u1 - u0, s->arena[s->cur[level]], field, threshold, s->d_tags,
            s->tag_cap, s->d_count);
        lg::abi_count_launch(s->ctx, 1);
        AMR_CUDA(s, cudaGetLastError());
    }
    unsigned long long n = 0;
    AMR_CUDA(s, cudaMemcpyAsync(&n, s->d_count, sizeof n, cudaMemcpyDeviceToHost, st));
    AMR_CUDA(s, cudaStreamSynchronize(st));
    std::vector<int64_t> host(2 * n);
    if (n)
        AMR_CUDA(s, cudaMemcpyAsync(host.data(), s->d_tags, 2 * n * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    AMR_CUDA(s, cudaStreamSynchronize(st));
    cells.resize(n);
    for (unsigned long long k = 0; k < n; ++k) cells[k] = {host[2 * k], host[2 * k + 1]};
    return LG_OK;
}

// slab pointers of field f of every block of `g`, whose arena layout is
// `P`, inside the host arena image `base` (which starts at element `first`)
template <class Ptr, class Vec>
std::vector<Ptr> slab_ptrs(const lg::amr::Plans& P, Vec& base, int64_t first, int f) {
    std::vector<Ptr> out(P.blocks.size(), nullptr);
    for (size_t b = 0; b < P.blocks.size(); ++b)
        if (P.blocks[b].off >= first) out[b] = base.data() + (P.blocks[b].off - first) + f * P.blocks[b].stride;
    return out;
}

// ------------------------------------------------- migration on the device
// BergerOliger::migrate / sample (adapt.rs:323-402) evaluated for every
// interior cell of the new hierarchy's refined blocks, from an image of the
// old state: a cell covered by an old patch of its level takes that value;
// otherwise the bilinear fold, from zero and in corner order, of the four
// coarser cells around it (reflected into the coarser domain), each sampled
// the same way -- the recursion ends at level 0, which covers everything.
// The expressions and their order are the host restatement's (compiled
// without contraction), so the migrated state is the same bits.
struct MigPatch {
    int64_t lo[2], hi[2];
    int64_t off;     // field 0's slab in the old image
    int64_t stride;  // between fields
};
struct MigLevel {
    int64_t dom[2];       // the level's domain [0, dom)
    int64_t side, nbx;    // the old layout's bucket index of the level
    int64_t s0, i0;       // its bucket starts and items in the shared arrays
    double ratio_below;   // refinement ratio between this level and the next coarser one
};
struct MigBlock {  // one refined block of the new hierarchy
    int64_t lo[2];
    int nx, ny, level, pad;
    int64_t off, stride;  // its slabs in the new arena
};
struct MigArgs {
    const double* old;
    const MigPatch* patches;
    const MigLevel* levels;
    const uint32_t* starts;
    const uint32_t* items;
    int old_levels;
    const MigBlock* blocks;
    int nblocks;
    double* out;
    int nfields;
    int* err;  // set when a sample found no level-0 block (not expected)
};

__device__ __forceinline__ int mig_find(const MigArgs& a, int level, int64_t x, int64_t y) {
    if (level >= a.old_levels) return -1;
    const MigLevel& L = a.levels[level];
    if (x < 0 || y < 0 || x >= L.dom[0] || y >= L.dom[1]) return -1;
    const int64_t k = x / L.side + (y / L.side) * L.nbx;
    for (uint32_t q = a.starts[L.s0 + k]; q < a.starts[L.s0 + k + 1]; ++q) {
        const uint32_t b = a.items[L.i0 + q];
        const MigPatch& P = a.patches[b];
        if (P.lo[0] <= x && x < P.hi[0] && P.lo[1] <= y && y < P.hi[1]) return (int)b;
    }
    return -1;
}

__device__ __forceinline__ int64_t mig_reflect(int64_t c, int64_t lo, int64_t hi) {
    if (c < lo) return 2 * lo - 1 - c;
    if (c >= hi) return 2 * hi - 1 - c;
    return c;
}

template <int DEPTH>
__device__ double mig_sample(const MigArgs& a, int level, int64_t x, int64_t y, int f) {
    const int b = mig_find(a, level, x, y);
    if (b >= 0) {
        const MigPatch& P = a.patches[b];
        return a.old[P.off + (int64_t)f * P.stride + (x - P.lo[0] + 1) + (y - P.lo[1] + 1) * (P.hi[0] - P.lo[0] + 2)];
    }
    if constexpr (DEPTH == 0) {
        atomicExch(a.err, 1);
        return 0.0;
    } else {
        if (level == 0) {
            atomicExch(a.err, 1);
            return 0.0;
        }
        const double r = a.levels[level].ratio_below;
        const int64_t cdx = a.levels[level - 1].dom[0], cdy = a.levels[level - 1].dom[1];
        const int64_t cell[2] = {x, y};
        int64_t c0[2];
        double w[2];
        for (int d = 0; d < 2; ++d) {
            const double pc = ((double)cell[d] + 0.5) / r - 0.5;
            const double fl = floor(pc);
            c0[d] = (int64_t)fl;
            w[d] = pc - fl;
        }
        double acc = 0.0;
#pragma unroll 1
        for (unsigned corner = 0; corner < 4; ++corner) {
            int64_t cc[2] = {c0[0], c0[1]};
            double weight = 1.0;
            for (int d = 0; d < 2; ++d) {
                if ((corner >> d) & 1) {
                    cc[d] += 1;
                    weight *= w[d];
                } else {
                    weight *= 1.0 - w[d];
                }
            }
            if (weight == 0.0) continue;
            cc[0] = mig_reflect(cc[0], 0, cdx);
            cc[1] = mig_reflect(cc[1], 0, cdy);
            acc += mig_sample<DEPTH - 1>(a, level - 1, cc[0], cc[1], f) * weight;
        }
        return acc;
    }
}

__global__ void __launch_bounds__(256) amr_migrate_kernel(MigArgs a) {
    for (int bi = blockIdx.x; bi < a.nblocks; bi += gridDim.x) {
        const MigBlock B = a.blocks[bi];
        for (int c = threadIdx.x; c < B.nx * B.ny; c += blockDim.x) {
            const int i = c % B.nx, j = c / B.nx;
            const int64_t o = B.off + (i + 1) + (int64_t)(j + 1) * (B.nx + 2);
            for (int f = 0; f < a.nfields; ++f)
                a.out[o + (int64_t)f * B.stride] = mig_sample<kMaxDepth - 1>(a, B.level, B.lo[0] + i, B.lo[1] + j, f);
        }
    }
}

// Copy the old state into the migration image (each level's slabs from its
// current buffer, at the old plans' offsets) and upload the old hierarchy's
// patch tables and the new hierarchy's refined blocks; fills the kernel
// arguments but the output arena.
int prepare_migration(lg_amr_sim* s, const lg::amr::Layout& ng, const lg::amr::Plans& np, MigArgs* a) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    const lg::amr::Layout& g = s->layout;
    const int64_t elems = s->plans.arena_elems;
    if (elems > s->mig_old_cap) {
        cudaFree(s->d_mig_old);
        s->d_mig_old = nullptr;
        s->mig_old_cap = 0;
        const int64_t cap = elems + elems / 4;
        AMR_CUDA(s, cudaMalloc(&s->d_mig_old, (size_t)cap * sizeof(double)));
        s->mig_old_cap = cap;
    }
    for (int l = 0; l < g.num_levels(); ++l) {
        const auto r = level_range(s, l);
        if (r.second > r.first)
            AMR_CUDA(s, cudaMemcpyAsync(s->d_mig_old + r.first, s->arena[s->cur[l]] + r.first,
                                        (size_t)(r.second - r.first) * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    std::vector<MigPatch> patches((size_t)g.num_blocks());
    for (int b = 0; b < g.num_blocks(); ++b) {
        const auto& bx = g.patches[(size_t)b].bx;
        patches[(size_t)b] = MigPatch{{bx.lo[0], bx.lo[1]}, {bx.hi[0], bx.hi[1]}, s->plans.blocks[(size_t)b].off,
                                      s->plans.blocks[(size_t)b].stride};
    }
    // every level the hierarchy may hold (a regrid can add one): domains and
    // ratios for all, bucket indices for the old layout's levels
    std::vector<MigLevel> levels((size_t)g.max_levels());
    std::vector<uint32_t> starts, items;
    for (int l = 0; l < g.max_levels(); ++l) {
        const auto d = g.domain(l);
        MigLevel L{{d.hi[0], d.hi[1]}, 1, 0, 0, 0, l > 0 ? (double)g.ratios[(size_t)l - 1] : 1.0};
        if (l < g.num_levels()) {
            const auto& ix = g.index[(size_t)l];
            L.side = ix.side;
            L.nbx = ix.nbx;
            L.s0 = (int64_t)starts.size();
            L.i0 = (int64_t)items.size();
            starts.insert(starts.end(), ix.start.begin(), ix.start.end());
            items.insert(items.end(), ix.items.begin(), ix.items.end());
        }
        levels[(size_t)l] = L;
    }
    std::vector<MigBlock> blocks;
    for (uint32_t b = ng.num_levels() > 1 ? ng.level_start[1] : (uint32_t)ng.num_blocks(); b < (uint32_t)ng.num_blocks();
         ++b) {
        const auto& bx = ng.patches[b].bx;
        const auto& d = np.blocks[b];
        blocks.push_back(MigBlock{{bx.lo[0], bx.lo[1]}, d.nx, d.ny, ng.patches[b].level, 0, d.off, d.stride});
    }
    size_t off = 0;
    auto reserve = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_p = reserve(patches.size() * sizeof(MigPatch)), o_l = reserve(levels.size() * sizeof(MigLevel)),
                 o_s = reserve(starts.size() * sizeof(uint32_t)), o_i = reserve(std::max<size_t>(1, items.size()) * 4),
                 o_b = reserve(blocks.size() * sizeof(MigBlock));
    std::vector<char> blob(std::max<size_t>(off, 256), 0);
    if (!blocks.empty()) std::memcpy(blob.data() + o_b, blocks.data(), blocks.size() * sizeof(MigBlock));
    std::memcpy(blob.data() + o_p, patches.data(), patches.size() * sizeof(MigPatch));
    std::memcpy(blob.data() + o_l, levels.data(), levels.size() * sizeof(MigLevel));
    std::memcpy(blob.data() + o_s, starts.data(), starts.size() * sizeof(uint32_t));
    if (!items.empty()) std::memcpy(blob.data() + o_i, items.data(), items.size() * sizeof(uint32_t));
    if (blob.size() > s->mig_tab_cap) {
        cudaFree(s->d_mig_tab);
        s->d_mig_tab = nullptr;
        s->mig_tab_cap = 0;
        const size_t cap = blob.size() + blob.size() / 4;
        AMR_CUDA(s, cudaMalloc(&s->d_mig_tab, cap));
        s->mig_tab_cap = cap;
    }
    if (!s->d_mig_err) AMR_CUDA(s, cudaMalloc(&s->d_mig_err, sizeof(int)));
    AMR_CUDA(s, cudaMemsetAsync(s->d_mig_err, 0, sizeof(int), st));
    AMR_CUDA(s, cudaMemcpyAsync(s->d_mig_tab, blob.data(), blob.size(), cudaMemcpyHostToDevice, st));
    // the host blob must outlive the copy
    AMR_CUDA(s, cudaStreamSynchronize(st));
    a->old = s->d_mig_old;
    a->patches = (const MigPatch*)(s->d_mig_tab + o_p);
    a->levels = (const MigLevel*)(s->d_mig_tab + o_l);
    a->starts = (const uint32_t*)(s->d_mig_tab + o_s);
    a->items = (const uint32_t*)(s->d_mig_tab + o_i);
    a->old_levels = g.num_levels();
    a->blocks = (const MigBlock*)(s->d_mig_tab + o_b);
    a->nblocks = (int)blocks.size();
    a->nfields = s->nfields;
    a->err = s->d_mig_err;
    return LG_OK;
}

// BergerOliger::regrid (adapt.rs:152-237): prepare (restrict + fill of the
// tagged field), tag every level on the device, build boxes on the host,
// keep the hierarchy if acceptable, else rebuild and migrate.  The level-0
// slabs stay where they are (the base tiling never changes); the refined
// levels are sampled on the device from an image of the old state.
int maybe_regrid(lg_amr_sim* s) {
    if (!s->has_policy || s->step_index % s->policy.every != 0) return LG_OK;
    const int f = s->policy.field;
    for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
        int rc = launch_restrict(s, fine, f, f + 1);
        if (rc != LG_OK) return rc;
    }
    // the global fill writes every field's ghosts; ghosts are rewritten
    // before any other read, so the extra fields' ghost values are unobservable
    for (int level = 0; level < s->layout.num_levels(); ++level) {
        int rc = launch_fill(s, level);
        if (rc != LG_OK) return rc;
    }
    std::vector<std::vector<std::array<int64_t, 2>>> flags(s->layout.num_levels());
    for (int level = 0; level < s->layout.num_levels() && level < s->layout.max_levels() - 1; ++level) {
        int rc = tag_level(s, f, level, s->policy.threshold, flags[level]);
        if (rc != LG_OK) return rc;
    }
    auto proposed = lg::amr::propose(s->layout, flags, s->policy);
    if (lg::amr::acceptable(s->layout, proposed)) return LG_OK;
    lg::amr::Layout ng;
    std::string err = lg::amr::build_layout(s->layout.base, s->layout.ratios, proposed, &ng);
    if (!err.empty()) return fail(s, LG_ERR_STATE, "regrid produced an invalid hierarchy: " + err);
    std::vector<TileShape> shapes = choose_tile_shapes(ng);
    shapes[0] = s->tile_shapes[0];  // level 0's plans are kept
    lg::amr::Plans np = lg::amr::build_plans(ng, s->nfields, 1024, 1, rows_of(shapes));
    if (!np.error.empty()) return fail(s, LG_ERR_STATE, np.error);
    // the old state's image and tables, then the new arenas (level 0 keeps
    // its slabs), zeroed refined slabs and one migration launch
    MigArgs ma{};
    int rc = prepare_migration(s, ng, np, &ma);
    if (rc != LG_OK) return rc;
    const int64_t l0 = level0_elems(s);
    int keep = 0;
    rc = ensure_arenas(s, np.arena_elems, l0, s->cur[0], &keep);
    if (rc != LG_OK) return rc;
    if (np.arena_elems > l0) {
        cudaStream_t st = lg::abi_stream(s->ctx);
        AMR_CUDA(s, cudaMemsetAsync(s->arena[keep] + l0, 0, (size_t)(np.arena_elems - l0) * sizeof(double), st));
        ma.out = s->arena[keep];
        if (ma.nblocks > 0) {
            amr_migrate_kernel<<<(unsigned)std::min(ma.nblocks, 65535), 256, 0, st>>>(ma);
            lg::abi_count_launch(s->ctx, 1);
            AMR_CUDA(s, cudaGetLastError());
        }
        int merr = 0;
        AMR_CUDA(s, cudaMemcpyAsync(&merr, s->d_mig_err, sizeof merr, cudaMemcpyDeviceToHost, st));
        AMR_CUDA(s, cudaStreamSynchronize(st));
        if (merr) return fail(s, LG_ERR_STATE, "migration found a cell outside every level-0 block");
    }
    s->layout = std::move(ng);
    s->plans = std::move(np);
    s->tile_shapes = shapes;
    drop_graphs(s);
    rc = upload_tables(s, s->plans, s->layout, s->tab);
    if (rc != LG_OK) return rc;
    s->cur.assign(s->layout.num_levels(), keep);
    s->epoch += 1;
    return LG_OK;
}

}  // namespace

extern "C" {

int lg_amr_sim_create(lg_ctx* ctx, const int64_t* cells, const int64_t* block, const double* origin,
                      const double* spacing, const uint32_t* ratios, int nratios, const int64_t* patches,
                      int64_t npatches, int model, const lg_modelc_params* mp, double kappa, int integrator,
                      uint64_t seed, const lg_amr_policy* policy, lg_amr_sim** out) {
    if (!ctx || !out || !cells || !block || !origin || !spacing || (nratios > 0 && !ratios) ||
        (npatches > 0 && !patches))
        return lg::abi_fail(ctx, LG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (model != LG_MODEL_C && model != LG_MODEL_HEAT) return lg::abi_fail(ctx, LG_ERR_INVALID, "unknown model");
    if (model == LG_MODEL_C && !mp) return lg::abi_fail(ctx, LG_ERR_INVALID, "Model C needs parameters");
    if (integrator != LG_AMR_SUBCYCLING && integrator != LG_AMR_GLOBAL_DT)
        return lg::abi_fail(ctx, LG_ERR_INVALID, "unknown integrator");
    if (nratios + 1 > kMaxDepth) return lg::abi_fail(ctx, LG_ERR_INVALID, "too many refinement levels");
    lg::amr::Base base{};
    for (int d = 0; d < 2; ++d) {
        base.cells[d] = cells[d];
        base.block[d] = block[d];
        base.origin[d] = origin[d];
        base.spacing[d] = spacing[d];
        if (!(spacing[d] > 0.0) || !std::isfinite(spacing[d]))
            return lg::abi_fail(ctx, LG_ERR_INVALID, "invalid spacing");
    }
    std::vector<uint32_t> r(ratios, ratios + nratios);
    std::vector<std::vector<lg::amr::Box>> levels;
    for (int64_t i = 0; i < npatches; ++i) {
        const int64_t lv = patches[5 * i];
        if (lv < 1 || lv > nratios) return lg::abi_fail(ctx, LG_ERR_INVALID, "patch level out of range");
        if ((int64_t)levels.size() < lv) levels.resize(lv);
        lg::amr::Box b;
        b.lo[0] = patches[5 * i + 1];
        b.lo[1] = patches[5 * i + 2];
        b.hi[0] = patches[5 * i + 3];
        b.hi[1] = patches[5 * i + 4];
        levels[lv - 1].push_back(b);
    }
    lg_amr_sim* s = new lg_amr_sim();
    s->ctx = ctx;
    std::string err = lg::amr::build_layout(base, r, levels, &s->layout);
    if (!err.empty()) {
        delete s;
        return lg::abi_fail(ctx, LG_ERR_INVALID, "AmrGrid: " + err);
    }
    s->model = model;
    if (mp) s->mp = *mp;
    s->kappa = kappa;
    s->integrator = integrator;
    s->seed = seed;
    s->nfields = model == LG_MODEL_C ? 2 : 1;
    if (policy) {
        s->has_policy = true;
        s->policy.every = std::max<int64_t>(1, policy->every);
        s->policy.buffer = policy->buffer;
        s->policy.min_width = policy->min_width;
        s->policy.efficiency = policy->efficiency;
        s->policy.threshold = policy->threshold;
        s->policy.field = policy->field;
        if (policy->field < 0 || policy->field >= s->nfields) {
            delete s;
            return lg::abi_fail(ctx, LG_ERR_INVALID, "tagged field out of range");
        }
    }
    cudaSetDevice(lg::abi_device(ctx));
    int rc = setup_device(s);
    if (rc == LG_OK && cudaMalloc(&s->d_t, 2 * sizeof(double)) != cudaSuccess) rc = LG_ERR_NOMEM;
    if (rc == LG_OK && cudaMemset(s->d_t, 0, 2 * sizeof(double)) != cudaSuccess) rc = LG_ERR_CUDA;
    if (rc == LG_OK && cudaMalloc(&s->d_bar, 2 * sizeof(unsigned)) != cudaSuccess) rc = LG_ERR_NOMEM;
    if (rc == LG_OK && cudaMemset(s->d_bar, 0, 2 * sizeof(unsigned)) != cudaSuccess) rc = LG_ERR_CUDA;
    if (rc == LG_OK && cudaMalloc(&s->d_err, sizeof(int)) != cudaSuccess) rc = LG_ERR_NOMEM;
    if (rc == LG_OK && cudaMemset(s->d_err, 0, sizeof(int)) != cudaSuccess) rc = LG_ERR_CUDA;
    if (rc != LG_OK) {
        const std::string why = lg_last_error(ctx);
        free_device(s);
        cudaFree(s->d_t);
        cudaFree(s->d_bar);
        cudaFree(s->d_err);
        delete s;
        return lg::abi_fail(ctx, rc, "AMR state set-up failed: " + why);
    }
    *out = s;
    return LG_OK;
}

int lg_amr_sim_destroy(lg_amr_sim* s) {
    if (!s) return LG_ERR_INVALID;
    cudaSetDevice(lg::abi_device(s->ctx));
    cudaStreamSynchronize(lg::abi_stream(s->ctx));
    free_device(s);
    cudaFree(s->d_t);
    cudaFree(s->d_bar);
    cudaFree(s->d_err);
    cudaFree(s->d_tags);
    cudaFree(s->d_count);
    cudaFree(s->d_mig_old);
    cudaFree(s->d_mig_tab);
    cudaFree(s->d_mig_err);
    delete s;
    return LG_OK;
}

int lg_amr_sim_info(const lg_amr_sim* s, int64_t* num_blocks, int* num_levels, int64_t* epoch) {
    if (!s || !num_blocks || !num_levels || !epoch) return LG_ERR_INVALID;
    *num_blocks = s->layout.num_blocks();
    *num_levels = s->layout.num_levels();
    *epoch = s->epoch;
    return LG_OK;
}

int lg_amr_sim_patch(const lg_amr_sim* s, int64_t block, int64_t* out5) {
    if (!s || !out5 || block < 0 || block >= s->layout.num_blocks()) return LG_ERR_INVALID;
    const auto& p = s->layout.patches[block];
    out5[0] = p.level;
    out5[1] = p.bx.lo[0];
    out5[2] = p.bx.lo[1];
    out5[3] = p.bx.hi[0];
    out5[4] = p.bx.hi[1];
    return LG_OK;
}

int lg_amr_sim_field_len(const lg_amr_sim* s, int64_t* n) {
    if (!s || !n) return LG_ERR_INVALID;
    int64_t k = 0;
    for (const auto& b : s->plans.blocks) k += (int64_t)(b.nx + 2) * (b.ny + 2);
    *n = k;
    return LG_OK;
}

int lg_amr_sim_get_field(lg_amr_sim* s, int field, double* host, int64_t nelem) {
    if (!s || !host || field < 0 || field >= s->nfields) return fail(s, LG_ERR_INVALID, "bad field");
    int64_t n = 0;
    lg_amr_sim_field_len(s, &n);
    if (nelem != n) return fail(s, LG_ERR_INVALID, "element count must equal lg_amr_sim_field_len");
    cudaSetDevice(lg::abi_device(s->ctx));
    int rc = download_state(s, s->host_old);
    if (rc != LG_OK) return rc;
    for (const auto& b : s->plans.blocks) {
        const size_t len = (size_t)(b.nx + 2) * (b.ny + 2);
        std::memcpy(host, s->host_old.data() + b.off + field * b.stride, len * sizeof(double));
        host += len;
    }
    return LG_OK;
}

int lg_amr_sim_set_field(lg_amr_sim* s, int field, const double* host, int64_t nelem) {
    if (!s || !host || field < 0 || field >= s->nfields) return fail(s, LG_ERR_INVALID, "bad field");
    int64_t n = 0;
    lg_amr_sim_field_len(s, &n);
    if (nelem != n) return fail(s, LG_ERR_INVALID, "element count must equal lg_amr_sim_field_len");
    cudaSetDevice(lg::abi_device(s->ctx));
    int rc = download_state(s, s->host_old);  // the other fields and the padding stay as they are
    if (rc != LG_OK) return rc;
    for (const auto& b : s->plans.blocks) {
        const size_t len = (size_t)(b.nx + 2) * (b.ny + 2);
        std::memcpy(s->host_old.data() + b.off + field * b.stride, host, len * sizeof(double));
        host += len;
    }
    return upload_state(s, s->host_old);
}

int lg_amr_sim_time(const lg_amr_sim* s, double* t, int64_t* step_index) {
    if (!s || !t || !step_index) return LG_ERR_INVALID;
    *t = s->t;
    *step_index = s->step_index;
    return LG_OK;
}

int lg_amr_sim_suggested_dt(const lg_amr_sim* s, double* dt) {
    if (!s || !dt) return LG_ERR_INVALID;
    // Subcycling::suggested_dt: level 0; a global-dt scheme: the finest
    // level the ratios allow (integrators/mod.rs:218-223, subcycling.rs:54-61)
    *dt = stable_dt_at(s, s->integrator == LG_AMR_SUBCYCLING ? 0 : (int)s->layout.level_spacing.size() - 1);
    return LG_OK;
}

int lg_amr_sim_set_barrier_spin_limit(lg_amr_sim* s, int64_t polls) {
    if (!s || polls < 0) return fail(s, LG_ERR_INVALID, "the spin limit is a non-negative poll count");
    s->barrier_spin_limit = (long long)polls;
    return LG_OK;
}

int lg_amr_sim_step(lg_amr_sim* s, double dt, int64_t nsteps, uint32_t flags) {
    if (!s) return LG_ERR_INVALID;
    if (nsteps < 0) return fail(s, LG_ERR_INVALID, "negative step count");
    cudaSetDevice(lg::abi_device(s->ctx));
    cudaStream_t st = lg::abi_stream(s->ctx);
    AMR_CUDA(s, cudaMemcpyAsync(s->d_t + s->tslot, &s->t, sizeof(double), cudaMemcpyHostToDevice, st));
    AMR_CUDA(s, cudaStreamSynchronize(st));  // the source is a host scalar that changes below
    int64_t done = 0;
    while (done < nsteps) {
        int rc = maybe_regrid(s);
        if (rc != LG_OK) return rc;
        // steps until the next regrid point, in pairs through a CUDA graph
        int64_t run = nsteps - done;
        if (s->has_policy) {
            const int64_t next = (s->step_index / s->policy.every + 1) * s->policy.every;
            run = std::min(run, next - s->step_index);
        }
        int64_t k = 0;
        if (flags & LG_RUN_PERSISTENT) {
            for (; k < run; k += 2) {
                const int n = run - k >= 2 ? 2 : 1;
                int rc2 = run_persistent(s, dt, n);
                if (rc2 != LG_OK) return rc2;
                for (int r2 = 0; r2 < n; ++r2) {
                    s->t += dt;
                    s->step_index += 1;
                }
            }
            k = run;
        }
        if ((flags & LG_RUN_GRAPH) && run - k >= 2) {
            char key[160];
            snprintf(key, sizeof key, "%lld|%a|%d", (long long)s->epoch, dt, s->tslot);
            std::string gk = key;
            for (int c : s->cur) gk += c ? '1' : '0';
            auto it = s->graphs.find(gk);
            if (it == s->graphs.end()) {
                const std::vector<int> cur0 = s->cur;
                const int slot0 = s->tslot;
                const int64_t before = lg::abi_launches(s->ctx);
                cudaGraph_t graph = nullptr;
                AMR_CUDA(s, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                int rc2 = one_coarse_step(s, dt);
                if (rc2 == LG_OK) rc2 = one_coarse_step(s, dt);
                cudaError_t ec = cudaStreamEndCapture(st, &graph);
                const int64_t captured = lg::abi_launches(s->ctx) - before;
                lg::abi_set_launches(s->ctx, before);
                if (rc2 != LG_OK) {
                    if (graph) cudaGraphDestroy(graph);
                    return rc2;
                }
                AMR_CUDA(s, ec);
                if (s->cur != cur0 || s->tslot != slot0) {
                    cudaGraphDestroy(graph);
                    return fail(s, LG_ERR_STATE, "a captured pair of coarse steps must restore the buffer parity");
                }
                cudaGraphExec_t exec = nullptr;
                cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                AMR_CUDA(s, ei);
                it = s->graphs.emplace(gk, std::make_pair(exec, captured)).first;
            }
            for (; k + 2 <= run; k += 2) {
                AMR_CUDA(s, cudaGraphLaunch(it->second.first, st));
                lg::abi_count_launch(s->ctx, it->second.second);
                for (int r2 = 0; r2 < 2; ++r2) {
                    s->t += dt;
                    s->step_index += 1;
                }
            }
        }
        for (; k < run; ++k) {
            int rc2 = one_coarse_step(s, dt);
            if (rc2 != LG_OK) return rc2;
            s->t += dt;  // simulation.rs:285-286
            s->step_index += 1;
        }
        done += run;
    }
    if (flags & LG_RUN_PERSISTENT) {  // did a grid barrier give up?
        int err = 0;
        AMR_CUDA(s, cudaMemcpyAsync(&err, s->d_err, sizeof err, cudaMemcpyDeviceToHost, st));
        AMR_CUDA(s, cudaStreamSynchronize(st));
        if (err) {
            AMR_CUDA(s, cudaMemsetAsync(s->d_bar, 0, 2 * sizeof(unsigned), st));
            AMR_CUDA(s, cudaMemsetAsync(s->d_err, 0, sizeof(int), st));
            AMR_CUDA(s, cudaStreamSynchronize(st));
            return fail(s, LG_ERR_TIMEOUT, "a grid barrier of the persistent AMR kernel timed out; the state is invalid");
        }
    }
    return LG_OK;
}

int lg_amr_restrict(lg_amr_sim* s, int field) {
    if (!s || field < 0 || field >= s->nfields) return fail(s, LG_ERR_INVALID, "bad field");
    cudaSetDevice(lg::abi_device(s->ctx));
    for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
        int rc = launch_restrict(s, fine, field, field + 1);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

int lg_amr_fill_ghosts(lg_amr_sim* s) {
    if (!s) return LG_ERR_INVALID;
    cudaSetDevice(lg::abi_device(s->ctx));
    for (int level = 0; level < s->layout.num_levels(); ++level) {
        int rc = launch_fill(s, level);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

int lg_amr_tag_level(lg_amr_sim* s, int field, int level, double threshold, int64_t* cells_out, int64_t cap,
                     int64_t* count) {
    if (!s || !count || field < 0 || field >= s->nfields || level < 0 || level >= s->layout.num_levels())
        return fail(s, LG_ERR_INVALID, "bad tag arguments");
    cudaSetDevice(lg::abi_device(s->ctx));
    std::vector<std::array<int64_t, 2>> cells;
    int rc = tag_level(s, field, level, threshold, cells);
    if (rc != LG_OK) return rc;
    std::sort(cells.begin(), cells.end());
    *count = (int64_t)cells.size();
    for (int64_t k = 0; k < (int64_t)cells.size() && k < cap; ++k) {
        cells_out[2 * k] = cells[k][0];
        cells_out[2 * k + 1] = cells[k][1];
    }
    return LG_OK;
}

// A tagging entry point that allocates nothing on its success path (no
// cudaMalloc, cudaFree or allocating library call, no host heap; only its
// error reports build a message string): the flags are compacted into the
// file-scope static scratch above, whose address is resolved once per
// device, and sorted in place in the caller's buffer.  It
// serves callers that cannot allocate: a step loop whose device memory is
// all held by a caching allocator (a cudaMalloc there fails or forces the
// cache to be released), and latency-bound loops in which cudaMalloc /
// cudaFree, which synchronise the device, would stall the stream.
// Limits: the level has at most 2^18 cells; cells_out needs room for every
// flagged cell (cap >= *count), else nothing is copied and the call fails
// with *count set.  Calls that overlap on the GPU race on the scratch.  Every
// call waits for its stream (it reads the flag count back to the host), so
// no call may be made while that stream is being captured into a graph.  The
// scratch address cached per device is that of the device's current primary
// context: the library must not be used on a device after a cudaDeviceReset.
namespace {
std::mutex g_scratch_mutex;
int64_t* g_scratch_ptr[64] = {};
}  // namespace

int lg_amr_tag_level_static(lg_amr_sim* s, int field, int level, double threshold, int64_t* cells_out, int64_t cap,
                            int64_t* count) {
    if (!s || !count || (cap > 0 && !cells_out) || cap < 0 || field < 0 || field >= s->nfields || level < 0 ||
        level >= s->layout.num_levels())
        return fail(s, LG_ERR_INVALID, "bad tag arguments");
    const int dev = lg::abi_device(s->ctx);
    if (dev < 0 || dev >= 64) return fail(s, LG_ERR_INVALID, "device ordinal out of range for the static scratch");
    int64_t cells = 0;
    for (uint32_t b = s->layout.level_start[level]; b < s->layout.level_start[level + 1]; ++b)
        cells += (int64_t)s->plans.blocks[b].nx * s->plans.blocks[b].ny;
    if (cells > kStaticTagCells)
        return fail(s, LG_ERR_INVALID, "level " + std::to_string(level) + " has " + std::to_string(cells) +
                                           " cells; the static tag scratch holds at most " +
                                           std::to_string(kStaticTagCells));
    AMR_CUDA(s, cudaSetDevice(dev));
    int64_t* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_tag_scratch);
            if (e != cudaSuccess)
                return fail(s, LG_ERR_CUDA, std::string("cudaGetSymbolAddress(static tag scratch): ") +
                                                cudaGetErrorString(e));
            g_scratch_ptr[dev] = (int64_t*)p;
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t st = lg::abi_stream(s->ctx);
    AMR_CUDA(s, cudaMemsetAsync(scratch, 0, sizeof(int64_t), st));  // the counter starts at zero
    const Lists L = lists(s, level);
    const int64_t u0 = L.P->unit_start[level], u1 = L.P->unit_start[level + 1];
    if (u1 > u0) {
        amr_tag_static_kernel<<<(unsigned)std::min<int64_t>(u1 - u0, 65535), 256, 0, st>>>(
            s->tab.blocks, s->tab.lo, L.T->units + u0, u1 - u0, s->arena[s->cur[level]], field, threshold, scratch);
        lg::abi_count_launch(s->ctx, 1);
        AMR_CUDA(s, cudaGetLastError());
    }
    int64_t n = 0;
    AMR_CUDA(s, cudaMemcpyAsync(&n, scratch, sizeof n, cudaMemcpyDeviceToHost, st));
    AMR_CUDA(s, cudaStreamSynchronize(st));
    *count = n;
    if (n > cap)
        return fail(s, LG_ERR_INVALID, "cells_out holds " + std::to_string(cap) + " cells; " + std::to_string(n) +
                                           " were flagged");
    if (n > 0) {
        AMR_CUDA(s, cudaMemcpyAsync(cells_out, scratch + 2, (size_t)n * 2 * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                    st));
        AMR_CUDA(s, cudaStreamSynchronize(st));
        struct Cell2 {
            int64_t x, y;
            bool operator<(const Cell2& o) const { return x < o.x || (x == o.x && y < o.y); }
        };
        static_assert(sizeof(Cell2) == 2 * sizeof(int64_t), "cells are packed pairs");
        Cell2* c = reinterpret_cast<Cell2*>(cells_out);
        std::sort(c, c + n);  // in place
    }
    return LG_OK;
}

}  // extern "C"
