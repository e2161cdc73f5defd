// Column-tile Model C step kernel, generic over an arithmetic policy.
//
// One CTA owns a run of rows of one block; thread t owns column t and walks
// up the rows.  Every face flux of the Karma-Rappel divergence is computed
// once and shared by the two cells that touch it: the reference evaluates
// the right face of cell i and the left face of cell i+1 (and top of j /
// bottom of j+1) with the same expression in the same operand order
// (finite_volume.rs:261-280), so sharing is bit-exact and halves the face
// work.  x faces travel between threads through a double-buffered
// shared-memory row (one barrier per row); the y face below a cell is the y
// face above it in the previous row, carried in a register.
//
// The row loop is unrolled four times over a rotating window of four phi
// rows (j-1, j, j+1 and the prefetch of j+2) so no register moves are
// needed to slide it.
//
// Ops (the arithmetic policy) provides, for element type T:
//   xface(m, dn, d1, c, e)  flux A (A dn - A' dt) through an x face, with the
//                           normal difference dn and the transverse
//                           difference dt = 0.25 ((d1 + c) - e)
//   yface(m, dn, d1, c, e)  flux A (A dn + A' dt) through a y face
//   cell(...)               the cell's dphi/dt and du/dt from its four face
//                           fluxes, phi, the central differences and the
//                           five u values
//   axpy(dt, k, x)          x + dt k
//   add_noise(x, s, key)    x + s N(key)
// The operand lists keep the reference's evaluation order available to an
// exact policy.
#pragma once

#include <algorithm>

#include "lg_common.cuh"
#include "lg_kernels.h"
#include "lg_modelc_ops.cuh"

namespace lg {

struct TileArgs {
    CartTopo topo;
    SlabLayout L;
    double dt64;
    uint64_t seed;
    double* tdev;
    int slot;
    int rows;
};

template <class T>
struct Row3 {
    T a, b, c;  // columns t-1, t, t+1
};

// One row of the tile: x face left of column t, y face above cell (t, j),
// barrier, then the cell update.  W = rows j-1 (A), j (B), j+1 (C); D
// receives row j+2.  uA..uD are u at column t for the same rows.
template <class T, class Ops, bool NOISE, int PAR>
__device__ __forceinline__ void tile_row(const typename Ops::Params& m, const TileArgs& g, int j, int r0, int t,
                                         bool cell, int n0, int n1, const T* __restrict__ phc,
                                         const T* __restrict__ uuc, T* __restrict__ out, T* __restrict__ phi_o,
                                         T* __restrict__ u_o, const Nbr2& nb, uint64_t block_key, T* xf,
                                         const T* xlast, Row3<T>& A, Row3<T>& B, Row3<T>& C, Row3<T>& D, T& uA,
                                         T& uB, T& uC, T& uD, T& jin, T& jout, T dt, T scale_amp) {
    const int sy = g.L.gdim[0];
    const int64_t rj = (int64_t)(j - r0) * sy;  // row j relative to the thread's column pointer at row r0
    T ul = T(0), ur = T(0);
    if (cell) {
        if (j + 2 <= n1) {
            const T* q = phc + rj + 2 * sy;
            D.a = __ldg(q - 1);
            D.b = __ldg(q);
            D.c = __ldg(q + 1);
            uD = __ldg(uuc + rj + 2 * sy);
        }
        ul = __ldg(uuc + rj - 1);
        ur = __ldg(uuc + rj + 1);
    }
    T* xrow = xf + PAR * n0;
    T jt = T(0);
    if (cell) {
        xrow[t] = Ops::xface(m, B.b - B.a, C.b - A.b, C.a, A.a);
        jt = Ops::yface(m, C.b - B.b, C.c - C.a, B.c, B.a);
    }
    __syncthreads();
    if (cell) {
        const T jl = xrow[t];
        const T jr = t + 1 < n0 ? xrow[t + 1] : xlast[j - r0];
        T kphi, ku;
        Ops::cell(m, jr, jl, jt, jin, B.b, B.c - B.a, C.b - A.b, uB, ul, ur, uC, uA, kphi, ku);
        T phin = Ops::axpy(dt, kphi, B.b);
        if (NOISE) {
            const uint64_t key = splitmix64(block_key ^ (uint64_t)(t + j * n0));
            phin = Ops::add_noise(phin, scale_amp, key);
        }
        const T un = Ops::axpy(dt, ku, uB);
        phi_o[rj] = phin;
        u_o[rj] = un;
        push_ghosts_2d_g1(out, g.L, 0, nb, n0, n1, t, j, phin);
        push_ghosts_2d_g1(out, g.L, 1, nb, n0, n1, t, j, un);
        jout = jt;
    }
}

template <class T, class Ops, bool NOISE, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    modelc_tile_kernel(const T* __restrict__ in, T* __restrict__ out, TileArgs g, typename Ops::Params m, T dt,
                       T scale_amp) {
    extern __shared__ __align__(16) unsigned char lg_smem[];
    const CartTopo& topo = g.topo;
    const int n0 = topo.n[0], n1 = topo.n[1];
    T* xf = reinterpret_cast<T*>(lg_smem);  // 2 x n0 x-face fluxes (left faces of the columns)
    T* xlast = xf + 2 * n0;                 // right face of the last column, one per row of the chunk
    const int sy = g.L.gdim[0];
    const int t = threadIdx.x;
    const int nt = blockDim.x;
    const bool cell = t < n0;
    const int rows = g.rows;

    // Simulation::t lives on the device in two slots: this step reads
    // tdev[slot] (its bits are the Wiener salt, euler_maruyama.rs:128) and
    // writes t + dt to the other slot (simulation.rs:285), so a captured
    // sequence of steps needs no host-side time.
    const double tnow = g.tdev[g.slot];
    if (blockIdx.x == 0 && blockIdx.y == 0 && t == 0) g.tdev[g.slot ^ 1] = tnow + g.dt64;

    for (int b = blockIdx.y; b < topo.nblocks; b += gridDim.y) {
        const int r0 = blockIdx.x * rows;
        const int r1 = min(n1, r0 + rows);
        if (r0 >= n1) continue;  // uniform over the CTA
        const T* ph = in + slab_base(g.L, b, 0);
        const T* uu = in + slab_base(g.L, b, 1);
        Nbr2 nb;
        nb.load(topo, b);
        uint64_t block_key = 0;
        if (NOISE)
            block_key = wiener_block_key(g.seed, (uint64_t)__double_as_longlong(tnow), kWienerStream0, (uint64_t)b);

        // the x face between column n0-1 and the ghost column, every row of
        // the chunk, lanes across rows
        for (int r = r0 + t; r < r1; r += nt) {
            const T* q = ph + (n0 - 1 + 1) + (int64_t)(r + 1) * sy;  // (column n0-1, row r)
            const T c0m = __ldg(q - sy), c1m = __ldg(q - sy + 1);
            const T c00 = __ldg(q), c10 = __ldg(q + 1);
            const T c0p = __ldg(q + sy), c1p = __ldg(q + sy + 1);
            xlast[r - r0] = Ops::xface(m, c10 - c00, c1p - c1m, c0p, c0m);
        }

        // thread's column pointers at (column t, row r0)
        const int64_t o0 = (int64_t)(t + 1) + (int64_t)(r0 + 1) * sy;
        const T* phc = ph + o0;
        const T* uuc = uu + o0;
        T* phi_o = out + slab_base(g.L, b, 0) + o0;
        T* u_o = out + slab_base(g.L, b, 1) + o0;

        Row3<T> w0{}, w1{}, w2{}, w3{};
        T u0 = T(0), u1 = T(0), u2 = T(0), u3 = T(0);
        T ja = T(0), jb = T(0);
        if (cell) {
            w0 = {__ldg(phc - sy - 1), __ldg(phc - sy), __ldg(phc - sy + 1)};
            w1 = {__ldg(phc - 1), __ldg(phc), __ldg(phc + 1)};
            w2 = {__ldg(phc + sy - 1), __ldg(phc + sy), __ldg(phc + sy + 1)};
            u0 = __ldg(uuc - sy);
            u1 = __ldg(uuc);
            u2 = __ldg(uuc + sy);
            // y face below the first row (between r0-1 and r0)
            ja = Ops::yface(m, w1.b - w0.b, w1.c - w1.a, w0.c, w0.a);
        }
        int j = r0;
        for (; j + 3 < r1; j += 4) {
            tile_row<T, Ops, NOISE, 0>(m, g, j, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key, xf,
                                       xlast, w0, w1, w2, w3, u0, u1, u2, u3, ja, jb, dt, scale_amp);
            tile_row<T, Ops, NOISE, 1>(m, g, j + 1, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key,
                                       xf, xlast, w1, w2, w3, w0, u1, u2, u3, u0, jb, ja, dt, scale_amp);
            tile_row<T, Ops, NOISE, 0>(m, g, j + 2, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key,
                                       xf, xlast, w2, w3, w0, w1, u2, u3, u0, u1, ja, jb, dt, scale_amp);
            tile_row<T, Ops, NOISE, 1>(m, g, j + 3, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key,
                                       xf, xlast, w3, w0, w1, w2, u3, u0, u1, u2, jb, ja, dt, scale_amp);
        }
        if (j < r1)
            tile_row<T, Ops, NOISE, 0>(m, g, j, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key, xf,
                                       xlast, w0, w1, w2, w3, u0, u1, u2, u3, ja, jb, dt, scale_amp);
        if (j + 1 < r1)
            tile_row<T, Ops, NOISE, 1>(m, g, j + 1, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key,
                                       xf, xlast, w1, w2, w3, w0, u1, u2, u3, u0, jb, ja, dt, scale_amp);
        if (j + 2 < r1)
            tile_row<T, Ops, NOISE, 0>(m, g, j + 2, r0, t, cell, n0, n1, phc, uuc, out, phi_o, u_o, nb, block_key,
                                       xf, xlast, w2, w3, w0, w1, u2, u3, u0, u1, ja, jb, dt, scale_amp);
        __syncthreads();  // xf / xlast reuse by the next block of this CTA
    }
}

// Tile height and launch shape from the grid: enough CTAs for several waves
// on 148 SMs, at least 16 rows each (the y face under the first row is
// evaluated once more per CTA).
inline int tile_rows(const CartTopo& topo, int rows) {
    const int n1 = topo.n[1];
    if (rows <= 0) {
        const int64_t want = 148 * 8;
        const int chunks = (int)std::max<int64_t>(1, (want + topo.nblocks - 1) / topo.nblocks);
        rows = std::max(16, (n1 + chunks - 1) / chunks);
    }
    return std::min(rows, n1);
}

// MINB: CTAs of 256 threads per SM the compiler must fit (bounds registers)
template <class T, class Ops, bool NOISE, int MINB = 2>
cudaError_t launch_tile_ops(const T* in, T* out, TileArgs g, const typename Ops::Params& m, T dt, T scale_amp,
                            cudaStream_t s) {
    const int n0 = g.topo.n[0], n1 = g.topo.n[1];
    const int threads = (n0 + 31) / 32 * 32;
    g.rows = tile_rows(g.topo, g.rows);
    dim3 grid((n1 + g.rows - 1) / g.rows, std::min(g.topo.nblocks, 65535));
    const size_t smem = (2 * (size_t)n0 + g.rows) * sizeof(T);
    if (threads <= 256)
        modelc_tile_kernel<T, Ops, NOISE, 256, MINB><<<grid, threads, smem, s>>>(in, out, g, m, dt, scale_amp);
    else
        modelc_tile_kernel<T, Ops, NOISE, 1024, 1><<<grid, threads, smem, s>>>(in, out, g, m, dt, scale_amp);
    return cudaGetLastError();
}

}  // namespace lg
