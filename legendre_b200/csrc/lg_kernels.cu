// Halo fill, heat and Model C step kernels of the legendre B200 library.
//
// This translation unit is compiled with -fmad=false: the reference is Rust,
// which never contracts a*b+c into a fused multiply-add, so every product
// and sum below rounds separately and `fma` appears exactly where the
// reference calls `f64::mul_add`.  That is what makes the FP64 path
// bit-identical to the reference's SerialScheduler.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "lg_common.cuh"
#include "lg_kernels.h"
#include "lg_modelc_ops.cuh"

namespace lg {
namespace {

// Offset of interior-relative index l inside a ghost-inclusive slab
// (cartesian.rs:189-204).
template <int D>
__device__ __forceinline__ int64_t lin(const SlabLayout& L, const int* l) {
    int64_t o = l[0] + L.ghost;
    if (D > 1) o += (int64_t)(l[1] + L.ghost) * L.gdim[0];
    if (D > 2) o += (int64_t)(l[2] + L.ghost) * L.gdim[0] * L.gdim[1];
    return o;
}

// Write the value of interior cell `l` of block `b` into every ghost entry
// whose source it is.  The reference fills ghosts by a dimension sweep
// (cartesian.rs:439-526); its result is separable per dimension -- ghost
// (x, y, ...) holds the interior value at (map_0(x), map_1(y), ...), each
// map being the identity inside the block, the face neighbour's interior
// (wrapped in periodic dimensions) or the mirror image at a physical
// boundary.  Pushing along the pre-images of that map writes every ghost
// entry exactly once, with no ordering between blocks.
template <int D, class T>
__device__ __forceinline__ void push_ghost_images(T* __restrict__ arena, const CartTopo& topo,
                                                  const SlabLayout& L, int field, int b, const int* l, T val) {
    const int g = L.ghost;
    int step[D][3], cl[D][3], nc[D];
    bool any = false;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const int n = topo.n[d];
        nc[d] = 1;
        step[d][0] = 0;
        cl[d][0] = l[d];
        if (l[d] < g) {
            int nb = topo.nbr[(b * 3 + d) * 2 + 0];
            step[d][nc[d]] = nb >= 0 ? -1 : 0;
            cl[d][nc[d]] = nb >= 0 ? n + l[d] : -1 - l[d];
            ++nc[d];
            any = true;
        }
        if (l[d] >= n - g) {
            int nb = topo.nbr[(b * 3 + d) * 2 + 1];
            step[d][nc[d]] = nb >= 0 ? 1 : 0;
            cl[d][nc[d]] = nb >= 0 ? l[d] - n : 2 * n - 1 - l[d];
            ++nc[d];
            any = true;
        }
    }
    if (!any) return;
    int c[3] = {0, 0, 0};
    for (;;) {
        // advance the mixed-radix counter; the all-zero combination is the
        // cell itself and is skipped
        int d = 0;
        while (d < D) {
            if (++c[d] < nc[d]) break;
            c[d] = 0;
            ++d;
        }
        if (d == D) break;
        int blk = b;
        int tl[3] = {0, 0, 0};
#pragma unroll
        for (int e = 0; e < D; ++e) {
            int st = step[e][c[e]];
            if (st != 0) blk = topo.nbr[(blk * 3 + e) * 2 + (st > 0 ? 1 : 0)];
            tl[e] = cl[e][c[e]];
        }
        arena[slab_base(L, blk, field) + lin<D>(L, tl)] = val;
    }
}

// ------------------------------------------------------------- halo (b) --
struct RingShape {
    int64_t strip[LG_MAX_DIM];  // cells in one strip normal to dimension d
    int64_t total;              // all ring cells of one block
};

// One thread per ghost entry.  Ring cells are enumerated as in the
// reference's for_each_ring_cell (src/geometry/amr/intergrid.rs:73-86): per
// dimension d, a low and a high strip of width g, spanning the grown range
// in earlier dimensions and the interior range in later ones.
template <class T>
__global__ void halo_fill_kernel(T* __restrict__ arena, CartTopo topo, SlabLayout L, int field, RingShape rs) {
    const int g = L.ghost;
    for (int b = blockIdx.y; b < topo.nblocks; b += gridDim.y)
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rs.total;
         r += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = r;
        int d = 0;
        while (rem >= 2 * rs.strip[d]) {
            rem -= 2 * rs.strip[d];
            ++d;
        }
        const int side = rem >= rs.strip[d] ? 1 : 0;
        int64_t pos = rem - side * rs.strip[d];
        int idx[3] = {0, 0, 0};
        for (int e = 0; e < topo.D; ++e) {
            int64_t ext = e < d ? topo.n[e] + 2 * g : (e == d ? g : topo.n[e]);
            int p = (int)(pos % ext);
            pos /= ext;
            if (e < d) idx[e] = p - g;
            else if (e == d) idx[e] = side ? topo.n[e] + p : p - g;
            else idx[e] = p;
        }
        // source of this ghost entry, dimension by dimension
        int src = b;
        int sl[3] = {idx[0], idx[1], idx[2]};
        for (int e = 0; e < topo.D; ++e) {
            const int n = topo.n[e];
            if (idx[e] < 0) {
                int nb = topo.nbr[(src * 3 + e) * 2 + 0];
                if (nb >= 0) { src = nb; sl[e] = n + idx[e]; }
                else sl[e] = -1 - idx[e];
            } else if (idx[e] >= n) {
                int nb = topo.nbr[(src * 3 + e) * 2 + 1];
                if (nb >= 0) { src = nb; sl[e] = idx[e] - n; }
                else sl[e] = 2 * n - 1 - idx[e];
            }
        }
        int64_t to = idx[0] + g, so = sl[0] + g, stride = L.gdim[0];
        for (int e = 1; e < topo.D; ++e) {
            to += (int64_t)(idx[e] + g) * stride;
            so += (int64_t)(sl[e] + g) * stride;
            stride *= L.gdim[e];
        }
        arena[slab_base(L, b, field) + to] = arena[slab_base(L, src, field) + so];
    }
}

// ------------------------------------------------------------- heat (d) --
// Heat<D>::vector_field_block (examples/heat3d.rs:63-79): the central
// Laplacian (finite_difference.rs:49-67) times kappa, then ForwardEuler's
// axpy (integrators/euler.rs:51-53).  One thread per interior cell.
template <int D>
__global__ void __launch_bounds__(256) heat_step_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                        CartTopo topo, SlabLayout L, int field, double kappa,
                                                        double dt, double ih0, double ih1, double ih2) {
    const int64_t cells = (int64_t)topo.n[0] * (D > 1 ? topo.n[1] : 1) * (D > 2 ? topo.n[2] : 1);
    const int64_t st1 = L.gdim[0];
    const int64_t st2 = (int64_t)L.gdim[0] * (D > 1 ? L.gdim[1] : 1);
    for (int b = blockIdx.y; b < topo.nblocks; b += gridDim.y) {
    const double* s = in + slab_base(L, b, field);
    double* o_slab = out + slab_base(L, b, field);
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cells;
         c += (int64_t)gridDim.x * blockDim.x) {
        int l[3] = {0, 0, 0};
        int64_t rem = c;
        l[0] = (int)(rem % topo.n[0]);
        rem /= topo.n[0];
        if (D > 1) { l[1] = (int)(rem % topo.n[1]); rem /= topo.n[1]; }
        if (D > 2) l[2] = (int)rem;
        const int64_t o = lin<D>(L, l);
        const double center = s[o];
        double acc = 0.0;
        acc += ((s[o + 1] - (center + center)) + s[o - 1]) * ih0;
        if (D > 1) acc += ((s[o + st1] - (center + center)) + s[o - st1]) * ih1;
        if (D > 2) acc += ((s[o + st2] - (center + center)) + s[o - st2]) * ih2;
        const double k = acc * kappa;
        const double v = center + dt * k;
        o_slab[o] = v;
        push_ghost_images<D, double>(out, topo, L, field, b, l, v);
    }
    }
}

// One stage of RungeKutta4 (rk4.rs:40-79) for the heat model, one thread
// per interior cell: k = kappa lap(in) as heat_step_kernel computes it, then
//   MODE 1: kout = k, out = y + c k          (y_tmp = y; y_tmp += c k_i)
//   MODE 2: out = (((y + s6 k1) + s3 k2) + s3 k3) + s6 k   (the four axpys)
// with the output's ghost images pushed for the next stage.
template <int D, int MODE>
__global__ void __launch_bounds__(256) heat_rk_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                      const double* __restrict__ y, double* __restrict__ kout,
                                                      const double* __restrict__ k1, const double* __restrict__ k2,
                                                      const double* __restrict__ k3, CartTopo topo, SlabLayout L,
                                                      int field, double kappa, double ih0, double ih1, double ih2,
                                                      double c, double s6, double s3) {
    const int64_t cells = (int64_t)topo.n[0] * (D > 1 ? topo.n[1] : 1) * (D > 2 ? topo.n[2] : 1);
    const int64_t st1 = L.gdim[0];
    const int64_t st2 = (int64_t)L.gdim[0] * (D > 1 ? L.gdim[1] : 1);
    for (int b = blockIdx.y; b < topo.nblocks; b += gridDim.y) {
        const int64_t base = slab_base(L, b, field);
        const double* s = in + base;
        for (int64_t cc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cc < cells;
             cc += (int64_t)gridDim.x * blockDim.x) {
            int l[3] = {0, 0, 0};
            int64_t rem = cc;
            l[0] = (int)(rem % topo.n[0]);
            rem /= topo.n[0];
            if (D > 1) { l[1] = (int)(rem % topo.n[1]); rem /= topo.n[1]; }
            if (D > 2) l[2] = (int)rem;
            const int64_t o = lin<D>(L, l);
            const double center = s[o];
            double acc = 0.0;
            acc += ((s[o + 1] - (center + center)) + s[o - 1]) * ih0;
            if (D > 1) acc += ((s[o + st1] - (center + center)) + s[o - st1]) * ih1;
            if (D > 2) acc += ((s[o + st2] - (center + center)) + s[o - st2]) * ih2;
            const double k = acc * kappa;
            const int64_t e = base + o;
            double v;
            if (MODE == 1) {
                kout[e] = k;
                v = y[e] + c * k;
            } else {
                v = y[e];
                v = v + s6 * k1[e];
                v = v + s3 * k2[e];
                v = v + s3 * k3[e];
                v = v + s6 * k;
            }
            out[e] = v;
            push_ghost_images<D, double>(out, topo, L, field, b, l, v);
        }
    }
}

// asynchronous 8-byte global -> shared copy (completes at cp_async_wait)
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 3-D heat step with halos pulled from the neighbour blocks' interiors
// (no ghost entries are read or written).  One CTA owns a z-range of ZC
// planes of one block, threads on the (x, y) plane.  It first stages the
// range with its one-cell face halo -- the z planes above and below and the
// x and y rings of every plane -- in shared memory, every load issued before
// any is used so that the whole range is in flight at once; halo values come
// from the face-neighbour blocks or, at a mirror boundary, repeat the edge
// cell (the zero-flux ghost, boundary.rs:63-80).  Then each thread updates
// its column from shared memory.  Arithmetic and operand order as
// heat_step_kernel, so the results are bit-identical.
__global__ void __launch_bounds__(1024) heat3d_pull_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                           CartTopo topo, SlabLayout L, int field, double kappa,
                                                           double dt, double ih0, double ih1, double ih2, int zc) {
    extern __shared__ double stage[];
    // programmatic dependent launch: the next step may launch now; this one
    // waits for the previous step's grid (and its writes) before staging
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int n0 = topo.n[0], n1 = topo.n[1], n2 = topo.n[2];
    const int X2 = n0 + 2, PZ = (n0 + 2) * (n1 + 2);
    const int x = threadIdx.x, y = threadIdx.y;
    const int64_t sy = L.gdim[0], sz = (int64_t)L.gdim[0] * L.gdim[1];
    const int nchunks = (n2 + zc - 1) / zc;
    const int64_t items = (int64_t)topo.nblocks * nchunks;
    auto off = [&](int xx, int yy, int zz) { return (int64_t)(xx + 1) + (yy + 1) * sy + (zz + 1) * sz; };
    for (int64_t item = blockIdx.x; item < items; item += gridDim.x) {
        const int b = (int)(item / nchunks);
        const int z0 = (int)(item - (int64_t)b * nchunks) * zc, nz = min(zc, n2 - z0);
        const int* nb = topo.nbr + b * 6;
        const double* s = in + slab_base(L, b, field);
        const double* sxl = nb[0] >= 0 ? in + slab_base(L, nb[0], field) : nullptr;
        const double* sxr = nb[1] >= 0 ? in + slab_base(L, nb[1], field) : nullptr;
        const double* syl = nb[2] >= 0 ? in + slab_base(L, nb[2], field) : nullptr;
        const double* syr = nb[3] >= 0 ? in + slab_base(L, nb[3], field) : nullptr;
        // plane r of the stage holds block plane z0 - 1 + r; every copy is
        // issued before any is waited for
        double* mine = stage + (x + 1) + (y + 1) * X2;
        for (int r = 0; r < nz + 2; ++r) {
            const int z = z0 - 1 + r;
            const double* src;
            if (z < 0)
                src = nb[4] >= 0 ? in + slab_base(L, nb[4], field) + off(x, y, n2 - 1) : s + off(x, y, 0);
            else if (z >= n2)
                src = nb[5] >= 0 ? in + slab_base(L, nb[5], field) + off(x, y, 0) : s + off(x, y, n2 - 1);
            else
                src = s + off(x, y, z);
            cp_async8(mine + r * PZ, src);
        }
        for (int r = 1; r <= nz; ++r) {
            const int z = z0 - 1 + r;
            double* pl = stage + r * PZ;
            if (x == 0) cp_async8(pl + (y + 1) * X2, sxl ? sxl + off(n0 - 1, y, z) : s + off(0, y, z));
            if (x == n0 - 1) cp_async8(pl + (n0 + 1) + (y + 1) * X2, sxr ? sxr + off(0, y, z) : s + off(n0 - 1, y, z));
            if (y == 0) cp_async8(pl + x + 1, syl ? syl + off(x, n1 - 1, z) : s + off(x, 0, z));
            if (y == n1 - 1) cp_async8(pl + (x + 1) + (n1 + 1) * X2, syr ? syr + off(x, 0, z) : s + off(x, n1 - 1, z));
        }
        cp_async_wait();
        __syncthreads();
        double* o = out + slab_base(L, b, field);
        for (int r = 1; r <= nz; ++r) {
            const double* q = mine + r * PZ;
            const double uc = q[0];
            double acc = 0.0;
            acc += ((q[1] - (uc + uc)) + q[-1]) * ih0;
            acc += ((q[X2] - (uc + uc)) + q[-X2]) * ih1;
            acc += ((q[PZ] - (uc + uc)) + q[-PZ]) * ih2;
            const double k = acc * kappa;
            o[off(x, y, z0 - 1 + r)] = uc + dt * k;
        }
        __syncthreads();
    }
}

// ------------------------------------------------- TMA-staged 3-D heat step
// shared-memory address of a generic pointer into this CTA's shared memory
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for phase `parity` of the barrier, at most `limit` polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long limit) {
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// one tiled tensor copy global -> shared of box `map` at (c0, c1, c2, c3),
// completing on `bar` (no cluster multicast: the map covers this GPU's
// memory only)
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// Tensor maps over one field of a 3-D state arena, all on the same 4-D
// tensor (x = slab column, y = slab row, z = slab plane, w = block), whose
// slabs keep their ghost ring: interior cell (i, j, k) of block b is at
// (i + 1, j + 1, k + 1, b).  Boxes: `main` the zc planes of a block's
// interior rows (every column of each row, the two ghost columns included:
// a row's interior starts 8 bytes in, and a box's first column must sit on a
// 16-byte boundary); `plane` one such plane (the z halos); `row` one row
// over zc planes (the y halos); `col` two columns over the interior rows of
// zc planes (the x halos; the wanted column is one of the two).
struct HeatMaps {
    CUtensorMap main, plane, row, col;
};

// 3-D heat step with every tile staged by the tensor-memory accelerator.
// One CTA owns a z-range of up to zc planes of one block, threads on the
// (x, y) plane.  Thread (0, 0) issues seven tensor copies onto one mbarrier:
// the range's interior rows, the z halo planes below and above, the y halo
// rows and the x halo columns of every plane of the range -- the halos from
// the face-neighbour blocks' interiors or, at a mirror boundary, the block's
// own edge cells (the zero-flux ghost, boundary.rs:63-80) -- so no ghost
// entry is read or written per step.  The wait for them is bounded: if it
// gives up, the CTA sets the context's error word, waits once more (bounded)
// for its copies to land and skips its update.  Each thread then walks its
// column through the range, reading from shared memory; arithmetic and
// operand order are heat_step_kernel's, so results are bit-identical.
// Stores are plain coalesced writes (an interior row starts 8 bytes into
// the slab row, which a tensor store cannot start on).
__global__ void __launch_bounds__(1024) heat3d_tma_kernel(const __grid_constant__ HeatMaps maps, double* __restrict__ out,
                                                          CartTopo topo, SlabLayout L, int field, double kappa,
                                                          double dt, double ih0, double ih1, double ih2, int zc,
                                                          int* err, long long spin_limit) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n0 = topo.n[0], n1 = topo.n[1], n2 = topo.n[2];
    const int W = n0 + 2;  // doubles per staged row
    // stage regions, each 128-byte aligned: S[zc][n1][W], ZL/ZH[n1][W],
    // YL/YH[zc][W], XL/XH[zc][n1][2], then the mbarrier
    auto up128 = [](size_t b) { return (b + 127) & ~size_t(127); };
    const size_t bS = up128((size_t)zc * n1 * W * 8), bZ = up128((size_t)n1 * W * 8), bY = up128((size_t)zc * W * 8),
                 bX = up128((size_t)zc * n1 * 2 * 8);
    double* S = reinterpret_cast<double*>(smem_raw);
    double* ZL = reinterpret_cast<double*>(smem_raw + bS);
    double* ZH = reinterpret_cast<double*>(smem_raw + bS + bZ);
    double* YL = reinterpret_cast<double*>(smem_raw + bS + 2 * bZ);
    double* YH = reinterpret_cast<double*>(smem_raw + bS + 2 * bZ + bY);
    double* XL = reinterpret_cast<double*>(smem_raw + bS + 2 * bZ + 2 * bY);
    double* XH = reinterpret_cast<double*>(smem_raw + bS + 2 * bZ + 2 * bY + bX);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + bS + 2 * bZ + 2 * bY + 2 * bX);
    const unsigned tx_bytes =
        (unsigned)(((size_t)zc * n1 * W + 2 * (size_t)n1 * W + 2 * (size_t)zc * W + 2 * (size_t)zc * n1 * 2) * 8);
    const int x = threadIdx.x, y = threadIdx.y;
    const bool leader = x == 0 && y == 0;
    if (leader) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // programmatic dependent launch: the next step may launch now; this one
    // waits for the previous step's grid (and its writes) before staging
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int64_t sy = L.gdim[0], sz = (int64_t)L.gdim[0] * L.gdim[1];
    const int nchunks = (n2 + zc - 1) / zc;
    const int64_t items = (int64_t)topo.nblocks * nchunks;
    unsigned parity = 0;
    for (int64_t item = blockIdx.x; item < items; item += gridDim.x) {
        const int b = (int)(item / nchunks);
        const int z0 = (int)(item - (int64_t)b * nchunks) * zc, nz = min(zc, n2 - z0);
        const int* nb = topo.nbr + b * 6;
        if (leader) {
            // source block and slab coordinate of each halo
            const int bxl = nb[0] >= 0 ? nb[0] : b, cxl = nb[0] >= 0 ? n0 : 1;  // left: the neighbour's last column
            const int bxh = nb[1] >= 0 ? nb[1] : b, cxh = nb[1] >= 0 ? 1 : n0;  // right: its first column
            const int byl = nb[2] >= 0 ? nb[2] : b, ryl = nb[2] >= 0 ? n1 : 1;
            const int byh = nb[3] >= 0 ? nb[3] : b, ryh = nb[3] >= 0 ? 1 : n1;
            int bzl = b, pzl = z0;                 // plane z0 - 1 of this block
            if (z0 == 0) { bzl = nb[4] >= 0 ? nb[4] : b; pzl = nb[4] >= 0 ? n2 : 1; }
            int bzh = b, pzh = z0 + nz + 1;        // plane z0 + nz of this block
            if (z0 + nz == n2) { bzh = nb[5] >= 0 ? nb[5] : b; pzh = nb[5] >= 0 ? 1 : n2; }
            mbar_arrive_expect_tx(bar, tx_bytes);
            tma_load_4d(S, &maps.main, 0, 1, z0 + 1, b, bar);
            tma_load_4d(ZL, &maps.plane, 0, 1, pzl, bzl, bar);
            tma_load_4d(ZH, &maps.plane, 0, 1, pzh, bzh, bar);
            tma_load_4d(YL, &maps.row, 0, ryl, z0 + 1, byl, bar);
            tma_load_4d(YH, &maps.row, 0, ryh, z0 + 1, byh, bar);
            tma_load_4d(XL, &maps.col, cxl & ~1, 1, z0 + 1, bxl, bar);
            tma_load_4d(XH, &maps.col, cxh & ~1, 1, z0 + 1, bxh, bar);
        }
        bool ok = mbar_wait_bounded(bar, parity, spin_limit);
        if (!ok) {
            if (leader) atomicExch(err, 1);
            mbar_wait_bounded(bar, parity, spin_limit);  // let the copies land before the stage is reused
        }
        parity ^= 1u;
        if (ok) {
            // slab columns the x halos came from: left = neighbour's n0 (or
            // own 1), right = neighbour's 1 (or own n0); index within the pair
            const int il = (nb[0] >= 0 ? n0 : 1) & 1, ih = (nb[1] >= 0 ? 1 : n0) & 1;
            // a thread walks its (x, y) column up the planes: the z
            // neighbours slide through registers (zm <- uc <- zp) and every
            // address advances by its stride, the arithmetic unchanged
            const int plane = n1 * W;
            const double* q = S + (size_t)y * W + (x + 1);
            const double* xl = XL + (size_t)y * 2 + il;
            const double* xh = XH + (size_t)y * 2 + ih;
            const double* yl = YL + (x + 1);
            const double* yh = YH + (x + 1);
            double* op = out + slab_base(L, b, field) + (int64_t)(x + 1) + (int64_t)(y + 1) * sy +
                         (int64_t)(z0 + 1) * sz;
            double zm = ZL[(size_t)y * W + x + 1];
            double uc = q[0];
            for (int r = 0; r < nz; ++r) {
                const double xm = x == 0 ? *xl : q[-1];
                const double xp = x == n0 - 1 ? *xh : q[1];
                const double ym = y == 0 ? *yl : q[-W];
                const double yp = y == n1 - 1 ? *yh : q[W];
                const double zp = r == nz - 1 ? ZH[(size_t)y * W + x + 1] : q[plane];
                double acc = 0.0;
                acc += ((xp - (uc + uc)) + xm) * ih0;
                acc += ((yp - (uc + uc)) + ym) * ih1;
                acc += ((zp - (uc + uc)) + zm) * ih2;
                const double k = acc * kappa;
                *op = uc + dt * k;
                // the row's ghost columns too, with the halo values at hand,
                // so that the warp's two rows cover whole 32-byte sectors (a
                // partly written sector costs the DRAM a read; 256^3: DRAM
                // reads 208 -> 164 MB a step): ghost entries are read by no
                // step of a run and refilled at its end.  Writing the ghost
                // rows and corners as well saved 3 MB more and ran slower.
                if (x == 0) op[-1] = xm;
                if (x == n0 - 1) op[1] = xp;
                zm = uc;
                uc = zp;
                q += plane;
                xl += 2 * n1;
                xh += 2 * n1;
                yl += W;
                yh += W;
                op += sz;
            }
        }
        // every thread is done with the stage before the next item's copies
        // (async proxy) overwrite it
        __syncthreads();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
}

// Reference-order Model C step, one thread per interior cell: the flux
// kernel (finite_volume.rs:258-283), the local terms (phasefield.rs:395-404),
// the u Laplacian and coupling (phasefield.rs:412-421), the Time driver
// axpy (driver.rs:210-216) and the Wiener increment (driver.rs:218-236).
template <class T>
__global__ void __launch_bounds__(256) modelc_step_ref_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                              CartTopo topo, SlabLayout L, MC<T> m, T dt,
                                                              double dt64, NoiseDev nz, T scale_amp, double* tdev,
                                                              int slot) {
    const int n0 = topo.n[0], n1 = topo.n[1];
    const int64_t sy = L.gdim[0];
    // Simulation::t lives on the device in two slots: this step reads
    // tdev[slot] (its bits are the Wiener salt, euler_maruyama.rs:73) and
    // writes t + dt to the other slot (simulation.rs:285), so a captured
    // sequence of steps needs no host-side time.
    const double t = tdev[slot];
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) tdev[slot ^ 1] = t + dt64;
    for (int b = blockIdx.y; b < topo.nblocks; b += gridDim.y) {
    const T* ph = in + slab_base(L, b, 0);
    const T* uu = in + slab_base(L, b, 1);
    T* phi_out = out + slab_base(L, b, 0);
    T* u_out = out + slab_base(L, b, 1);
    uint64_t block_key = 0;
    if (nz.on) block_key = wiener_block_key(nz.seed, (uint64_t)__double_as_longlong(t), kWienerStream0, (uint64_t)b);
    const T quarter = T(0.25), half = T(0.5);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n0 * n1; c += gridDim.x * blockDim.x) {
        const int i = c % n0, j = c / n0;
        const int64_t o = (int64_t)(i + 1) + (int64_t)(j + 1) * sy;
        auto P = [&](int di, int dj) { return ph[o + di + dj * sy]; };
        T derx_r = P(1, 0) - P(0, 0);
        T derx_l = P(0, 0) - P(-1, 0);
        T derx_t = quarter * (P(1, 1) - P(-1, 1) + P(1, 0) - P(-1, 0));
        T derx_b = quarter * (P(1, 0) - P(-1, 0) + P(1, -1) - P(-1, -1));
        T dery_t = P(0, 1) - P(0, 0);
        T dery_b = P(0, 0) - P(0, -1);
        T dery_r = quarter * (P(1, 1) - P(1, -1) + P(0, 1) - P(0, -1));
        T dery_l = quarter * (P(0, 1) - P(0, -1) + P(-1, 1) - P(-1, -1));
        T a_r, da_r, a_l, da_l, a_t, da_t, a_b, da_b;
        kr_face(m, derx_r, dery_r, a_r, da_r);
        kr_face(m, derx_l, dery_l, a_l, da_l);
        kr_face(m, derx_t, dery_t, a_t, da_t);
        kr_face(m, derx_b, dery_b, a_b, da_b);
        T j_r = a_r * (a_r * derx_r - da_r * dery_r);
        T j_l = a_l * (a_l * derx_l - da_l * dery_l);
        T j_t = a_t * (a_t * dery_t + da_t * derx_t);
        T j_b = a_b * (a_b * dery_b + da_b * derx_b);
        T flux = (j_r - j_l + j_t - j_b) * m.inv_h2_flux;

        T p = P(0, 0);
        T g_prime = fma_t(p * p, p, -p);
        T one_m_p2 = fma_t(p, -p, T(1));
        T p_prime = one_m_p2 * one_m_p2;
        // center_anisotropy (phasefield.rs:159-175)
        T cdx = half * (P(1, 0) - P(-1, 0));
        T cdy = half * (P(0, 1) - P(0, -1));
        T cdx2 = cdx * cdx;
        T cdy2 = cdy * cdy;
        T csum = cdx2 + cdy2;
        T cmag2 = csum * csum;
        T a = cmag2 <= m.tol ? m.a_bar : m.a_bar * (T(1) + m.eps_prime * (cdx2 * cdx2 + cdy2 * cdy2) / cmag2);
        T uc = uu[o];
        T kphi = fma_t(m.lambda * uc, -p_prime, flux - g_prime) / (a * a);

        T acc = T(0);
        acc += ((uu[o + 1] - (uc + uc)) + uu[o - 1]) * m.ih0;
        acc += ((uu[o + sy] - (uc + uc)) + uu[o - sy]) * m.ih1;
        T ku = fma_t(acc, m.d_thermal, half * kphi);

        T phin = p + dt * kphi;
        if (nz.on) {
            uint64_t key = splitmix64(block_key ^ (uint64_t)(i + j * n0));
            phin += scale_amp * normal_t(key, T(0));
        }
        T un = uc + dt * ku;
        phi_out[o] = phin;
        u_out[o] = un;
        int l[2] = {i, j};
        push_ghost_images<2, T>(out, topo, L, 0, b, l, phin);
        push_ghost_images<2, T>(out, topo, L, 1, b, l, un);
    }
    }
}

__global__ void standard_normal_kernel(const uint64_t* keys, double* out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = standard_normal(keys[i]);
}

int grid_x_for(int64_t cells, int threads) {
    int64_t gx = (cells + threads - 1) / threads;
    return (int)(gx < 1 ? 1 : (gx > 65535 ? 65535 : gx));
}

int grid_y_for(int nblocks) { return nblocks < 1 ? 1 : (nblocks > 65535 ? 65535 : nblocks); }

}  // namespace

cudaError_t launch_halo_fill(void* arena, int elem_size, const CartTopo& topo, const SlabLayout& L, int field,
                             cudaStream_t s) {
    if (L.ghost == 0) return cudaSuccess;
    RingShape rs{};
    rs.total = 0;
    for (int d = 0; d < topo.D; ++d) {
        int64_t c = L.ghost;
        for (int e = 0; e < topo.D; ++e) {
            if (e < d) c *= topo.n[e] + 2 * L.ghost;
            else if (e > d) c *= topo.n[e];
        }
        rs.strip[d] = c;
        rs.total += 2 * c;
    }
    dim3 grid(grid_x_for(rs.total, 256), grid_y_for(topo.nblocks));
    if (elem_size == 8)
        halo_fill_kernel<double><<<grid, 256, 0, s>>>(static_cast<double*>(arena), topo, L, field, rs);
    else
        halo_fill_kernel<float><<<grid, 256, 0, s>>>(static_cast<float*>(arena), topo, L, field, rs);
    return cudaGetLastError();
}

bool heat3d_pull_supported(const CartTopo& topo, const SlabLayout& L) {
    return topo.D == 3 && L.ghost == 1 && topo.n[0] >= 1 && topo.n[1] >= 1 && topo.n[2] >= 1 &&
           topo.n[0] * topo.n[1] <= 1024 && 3 * (topo.n[0] + 2) * (topo.n[1] + 2) * 8 <= 96 * 1024;
}

cudaError_t launch_heat3d_pull(const double* in, double* out, const CartTopo& topo, const SlabLayout& L, int field,
                               double kappa, double dt, const double inv_h2[3], cudaStream_t s) {
    // z-chunks per block: whole blocks when there are enough of them to fill
    // the GPU several times, else chunks of at least 4 planes
    // planes per CTA: at most 16 (and the stage at most 96 KB), fewer when
    // whole blocks would not fill the GPU several times over
    const int n2 = topo.n[2];
    const int64_t plane = (int64_t)(topo.n[0] + 2) * (topo.n[1] + 2) * sizeof(double);
    int zc = std::min(n2, 16);
    while (zc > 1 && (zc + 2) * plane > 96 * 1024) --zc;
    while (zc > 4 && (int64_t)topo.nblocks * ((n2 + zc - 1) / zc) < (int64_t)lg::device_sm_count() * 8) zc = (zc + 1) / 2;
    const int64_t items = (int64_t)topo.nblocks * ((n2 + zc - 1) / zc);
    const unsigned grid = (unsigned)std::min<int64_t>(items, (int64_t)1 << 30);
    const size_t smem = (size_t)(zc + 2) * plane;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(heat3d_pull_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             96 * 1024 + 2 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(topo.n[0], topo.n[1]);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, heat3d_pull_kernel, in, out, topo, L, field, kappa, dt, inv_h2[0], inv_h2[1],
                              inv_h2[2], zc);
}

// ---- TMA heat launcher: tensor maps are encoded on the host per launch
// (cheap; a captured graph keeps the parameters it was captured with)
namespace {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool encode_heat_map(CUtensorMap* m, const double* base, const CartTopo& topo, const SlabLayout& L, uint32_t bx,
                     uint32_t by, uint32_t bz) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)topo.n[0] + 2, (cuuint64_t)topo.n[1] + 2, (cuuint64_t)topo.n[2] + 2,
                                (cuuint64_t)topo.nblocks};
    const cuuint64_t strides[3] = {(cuuint64_t)(topo.n[0] + 2) * 8, (cuuint64_t)(topo.n[0] + 2) * (topo.n[1] + 2) * 8,
                                   (cuuint64_t)L.nfields * L.slab_stride * 8};
    const cuuint32_t box[4] = {bx, by, bz, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t heat_tma_smem(const CartTopo& topo, int zc) {
    auto up128 = [](size_t b) { return (b + 127) & ~size_t(127); };
    const size_t W = topo.n[0] + 2, n1 = topo.n[1];
    return up128(zc * n1 * W * 8) + 2 * up128(n1 * W * 8) + 2 * up128(zc * W * 8) + 2 * up128(zc * n1 * 2 * 8) + 16;
}
}  // namespace

bool heat3d_tma_supported(const CartTopo& topo, const SlabLayout& L) {
    // rows of an even number of doubles keep every stride a multiple of 16
    // bytes; a box edge is at most 256 elements; one thread per (x, y)
    return heat3d_pull_supported(topo, L) && topo.n[0] % 2 == 0 && topo.n[0] + 2 <= 256 && topo.n[1] <= 256 &&
           (L.slab_stride * 8) % 16 == 0 && heat_tma_smem(topo, 1) <= 200 * 1024 && tensor_map_encoder() != nullptr;
}

cudaError_t launch_heat3d_tma(const double* in, double* out, const CartTopo& topo, const SlabLayout& L, int field,
                              double kappa, double dt, const double inv_h2[3], int* err, cudaStream_t s) {
    // planes per CTA: at most 16 and the stage at most 200 KB, fewer when
    // whole blocks would not fill the GPU several times over
    const int n2 = topo.n[2];
    int zc = std::min(n2, 16);
    while (zc > 1 && heat_tma_smem(topo, zc) > 200 * 1024) --zc;
    while (zc > 4 && (int64_t)topo.nblocks * ((n2 + zc - 1) / zc) < (int64_t)lg::device_sm_count() * 8) zc = (zc + 1) / 2;
    HeatMaps maps;
    const double* base = in + (int64_t)field * L.slab_stride;
    const uint32_t W = (uint32_t)topo.n[0] + 2, n1 = (uint32_t)topo.n[1];
    if (!encode_heat_map(&maps.main, base, topo, L, W, n1, (uint32_t)zc) ||
        !encode_heat_map(&maps.plane, base, topo, L, W, n1, 1) ||
        !encode_heat_map(&maps.row, base, topo, L, W, 1, (uint32_t)zc) ||
        !encode_heat_map(&maps.col, base, topo, L, 2, n1, (uint32_t)zc))
        return cudaErrorInvalidValue;
    const int64_t items = (int64_t)topo.nblocks * ((n2 + zc - 1) / zc);
    const unsigned grid = (unsigned)std::min<int64_t>(items, (int64_t)1 << 30);
    const size_t smem = heat_tma_smem(topo, zc);
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(heat3d_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024 + 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(topo.n[0], topo.n[1]);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // ~20M polls of the barrier: well over a second before a copy counts as lost
    const long long spin_limit = 20000000;
    return cudaLaunchKernelEx(&cfg, heat3d_tma_kernel, maps, out, topo, L, field, kappa, dt, inv_h2[0], inv_h2[1],
                              inv_h2[2], zc, err, spin_limit);
}

cudaError_t launch_heat_rk_stage(int mode, const double* in, double* out, const double* y, double* kout,
                                 const double* k1, const double* k2, const double* k3, const CartTopo& topo,
                                 const SlabLayout& L, int field, double kappa, const double* inv_h2, double c,
                                 double s6, double s3, cudaStream_t s) {
    const int64_t cells = (int64_t)topo.n[0] * (topo.D > 1 ? topo.n[1] : 1) * (topo.D > 2 ? topo.n[2] : 1);
    const dim3 grid((unsigned)std::min<int64_t>((cells + 255) / 256, 1024), (unsigned)std::min(topo.nblocks, 65535));
#define LG_HRK(DD, MM)                                                                                             \
    heat_rk_kernel<DD, MM><<<grid, 256, 0, s>>>(in, out, y, kout, k1, k2, k3, topo, L, field, kappa, inv_h2[0],   \
                                                 inv_h2[1], inv_h2[2], c, s6, s3)
    if (mode == 1) {
        if (topo.D == 1) LG_HRK(1, 1);
        else if (topo.D == 2) LG_HRK(2, 1);
        else LG_HRK(3, 1);
    } else {
        if (topo.D == 1) LG_HRK(1, 2);
        else if (topo.D == 2) LG_HRK(2, 2);
        else LG_HRK(3, 2);
    }
#undef LG_HRK
    return cudaGetLastError();
}

cudaError_t launch_heat_step(const double* in, double* out, const CartTopo& topo, const SlabLayout& L, int field,
                             double kappa, double dt, const double inv_h2[3], cudaStream_t s) {
    int64_t cells = 1;
    for (int d = 0; d < topo.D; ++d) cells *= topo.n[d];
    dim3 grid(grid_x_for(cells, 256), grid_y_for(topo.nblocks));
    switch (topo.D) {
        case 1:
            heat_step_kernel<1><<<grid, 256, 0, s>>>(in, out, topo, L, field, kappa, dt, inv_h2[0], 0.0, 0.0);
            break;
        case 2:
            heat_step_kernel<2><<<grid, 256, 0, s>>>(in, out, topo, L, field, kappa, dt, inv_h2[0], inv_h2[1], 0.0);
            break;
        default:
            heat_step_kernel<3><<<grid, 256, 0, s>>>(in, out, topo, L, field, kappa, dt, inv_h2[0], inv_h2[1],
                                                     inv_h2[2]);
    }
    return cudaGetLastError();
}

cudaError_t launch_modelc_step_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int variant, cudaStream_t s) {
    (void)variant;
    dim3 grid(grid_x_for((int64_t)topo.n[0] * topo.n[1], 256), grid_y_for(topo.nblocks));
    double scale_amp = std::sqrt(dt) * nz.amp;
    modelc_step_ref_kernel<double><<<grid, 256, 0, s>>>(in, out, topo, L, to_mc<double>(m), dt, dt, nz, scale_amp,
                                                        tdev, slot);
    return cudaGetLastError();
}

cudaError_t launch_modelc_step_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int variant, cudaStream_t s) {
    (void)variant;
    dim3 grid(grid_x_for((int64_t)topo.n[0] * topo.n[1], 256), grid_y_for(topo.nblocks));
    float scale_amp = (float)std::sqrt(dt) * (float)nz.amp;
    modelc_step_ref_kernel<float><<<grid, 256, 0, s>>>(in, out, topo, L, to_mc<float>(m), (float)dt, dt, nz,
                                                       scale_amp, tdev, slot);
    return cudaGetLastError();
}

cudaError_t launch_standard_normal(const uint64_t* keys, double* out, int64_t n, cudaStream_t s) {
    standard_normal_kernel<<<grid_x_for(n, 256), 256, 0, s>>>(keys, out, n);
    return cudaGetLastError();
}

}  // namespace lg
