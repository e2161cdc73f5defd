// Warp-strip Model C step kernel, generic over an arithmetic policy.
//
// Work unit: one warp owns a strip of 32 columns of one block over a run of
// rows and walks up the rows; lane l owns column 32 s + l.  Warps are
// independent -- no barriers, no shared memory.
//
// Every face flux of the Karma-Rappel divergence is computed once and
// shared by the two cells that touch it: the reference evaluates the right
// face of cell i and the left face of cell i+1 (and top of j / bottom of
// j+1) with the same expression in the same operand order
// (finite_volume.rs:261-280), so sharing is bit-exact and halves the face
// work.  Lane l computes the x face on the left of its column and receives
// its right face from lane l+1 by a shuffle; the strip's last lane takes it
// from a batch of 32 right-boundary faces that the warp evaluates with its
// lanes across rows (one extra face per 32 cells).  The y face below a cell
// is the y face above it in the previous row, carried in a register.
//
// The row loop is unrolled four times over a rotating window of four phi
// rows (j-1, j, j+1 and the prefetch of j+2) so no register moves slide it.
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
//   noise(key)              N(key), the Gaussian of one cell
//   add_noise(x, s, n)      x + s n
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
    int rows;     // rows per work unit
    int strips;   // 32-column strips per block
    int chunks;   // row chunks per block
    int64_t units;
};

template <class T>
struct Row3 {
    T a, b, c;  // columns c-1, c, c+1
};

constexpr unsigned kFull = 0xffffffffu;

// One row: x face left of the lane's column, y face above cell (c, j), the
// cell update, stores and ghost pushes.  A, B, C = phi rows j-1, j, j+1; D
// receives row j+2.  uA..uD = u at the lane's column for the same rows.
template <class T, class Ops, bool NOISE>
__device__ __forceinline__ void strip_row(const typename Ops::Params& m, const TileArgs& g, int j, int r0, int lane,
                                          int col, bool valid, int last_lane, int n0, int n1,
                                          const T* __restrict__ phc, const T* __restrict__ uuc, T* __restrict__ out,
                                          T* __restrict__ phi_o, T* __restrict__ u_o, const Nbr2& nb,
                                          uint64_t block_key, T bnd, Row3<T>& A, Row3<T>& B, Row3<T>& C,
                                          Row3<T>& D, T& uA, T& uB, T& uC, T& uD, T& jin, T& jout, T dt,
                                          T scale_amp) {
    const int sy = g.L.gdim[0];
    const int64_t rj = (int64_t)(j - r0) * sy;  // row j relative to the lane's column pointer at row r0
    T ul = T(0), ur = T(0);
    if (valid) {
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
    T nval = T(0);
    if (NOISE && valid) nval = Ops::noise(splitmix64(block_key ^ (uint64_t)(col + j * n0)));
    T fl = T(0), jt = T(0);
    if (valid) {
        fl = Ops::xface(m, B.b - B.a, C.b - A.b, C.a, A.a);
        jt = Ops::yface(m, C.b - B.b, C.c - C.a, B.c, B.a);
    }
    // right face: the next lane's left face, or the strip's boundary face of this row
    T fr = __shfl_down_sync(kFull, fl, 1);
    const T fb = __shfl_sync(kFull, bnd, (j - r0) & 31);
    if (lane == last_lane) fr = fb;
    if (valid) {
        T kphi, ku;
        Ops::cell(m, fr, fl, jt, jin, B.b, B.c - B.a, C.b - A.b, uB, ul, ur, uC, uA, kphi, ku);
        T phin = Ops::axpy(dt, kphi, B.b);
        if (NOISE) phin = Ops::add_noise(phin, scale_amp, nval);
        const T un = Ops::axpy(dt, ku, uB);
        phi_o[rj] = phin;
        u_o[rj] = un;
        push_ghosts_2d_g1(out, g.L, 0, nb, n0, n1, col, j, phin);
        push_ghosts_2d_g1(out, g.L, 1, nb, n0, n1, col, j, un);
        jout = jt;
    }
}

template <class T, class Ops, bool NOISE, int MINB>
__global__ void __launch_bounds__(256, MINB)
    modelc_strip_kernel(const T* __restrict__ in, T* __restrict__ out, TileArgs g, typename Ops::Params m, T dt,
                        T scale_amp) {
    const CartTopo& topo = g.topo;
    const int n0 = topo.n[0], n1 = topo.n[1];
    const int sy = g.L.gdim[0];
    const int lane = threadIdx.x & 31;
    const int wpc = blockDim.x >> 5;

    // Simulation::t lives on the device in two slots: this step reads
    // tdev[slot] (its bits are the Wiener salt, euler_maruyama.rs:128) and
    // writes t + dt to the other slot (simulation.rs:285), so a captured
    // sequence of steps needs no host-side time.
    const double tnow = g.tdev[g.slot];
    if (blockIdx.x == 0 && threadIdx.x == 0) g.tdev[g.slot ^ 1] = tnow + g.dt64;

    for (int64_t unit = (int64_t)blockIdx.x * wpc + (threadIdx.x >> 5); unit < g.units;
         unit += (int64_t)gridDim.x * wpc) {
        const int s = (int)(unit % g.strips);
        const int k = (int)((unit / g.strips) % g.chunks);
        const int b = (int)(unit / ((int64_t)g.strips * g.chunks));
        const int r0 = k * g.rows;
        const int r1 = min(n1, r0 + g.rows);
        const int c0 = s * 32;
        const int col = c0 + lane;
        const bool valid = col < n0;
        const int last_lane = min(31, n0 - 1 - c0);
        const int cr = c0 + last_lane;  // last column of the strip; its right face is the boundary face

        const T* ph = in + slab_base(g.L, b, 0);
        const T* uu = in + slab_base(g.L, b, 1);
        Nbr2 nb;
        nb.load(topo, b);
        uint64_t block_key = 0;
        if (NOISE)
            block_key = wiener_block_key(g.seed, (uint64_t)__double_as_longlong(tnow), kWienerStream0, (uint64_t)b);

        // the lane's column pointers at (col, r0)
        const int64_t o0 = (int64_t)(col + 1) + (int64_t)(r0 + 1) * sy;
        const T* phc = ph + o0;
        const T* uuc = uu + o0;
        T* phi_o = out + slab_base(g.L, b, 0) + o0;
        T* u_o = out + slab_base(g.L, b, 1) + o0;

        // right-boundary face of the strip for rows rb .. rb+31 (lane = row)
        auto boundary = [&](int rb) -> T {
            const int r = rb + lane;
            if (r >= r1) return T(0);
            const T* q = ph + (cr + 1) + (int64_t)(r + 1) * sy;  // (column cr, row r)
            const T c0m = __ldg(q - sy), c1m = __ldg(q - sy + 1);
            const T c00 = __ldg(q), c10 = __ldg(q + 1);
            const T c0p = __ldg(q + sy), c1p = __ldg(q + sy + 1);
            return Ops::xface(m, c10 - c00, c1p - c1m, c0p, c0m);
        };

        Row3<T> w0{}, w1{}, w2{}, w3{};
        T u0 = T(0), u1 = T(0), u2 = T(0), u3 = T(0);
        T ja = T(0), jb = T(0);
        if (valid) {
            w0 = {__ldg(phc - sy - 1), __ldg(phc - sy), __ldg(phc - sy + 1)};
            w1 = {__ldg(phc - 1), __ldg(phc), __ldg(phc + 1)};
            w2 = {__ldg(phc + sy - 1), __ldg(phc + sy), __ldg(phc + sy + 1)};
            u0 = __ldg(uuc - sy);
            u1 = __ldg(uuc);
            u2 = __ldg(uuc + sy);
            // y face below the first row (between r0-1 and r0)
            ja = Ops::yface(m, w1.b - w0.b, w1.c - w1.a, w0.c, w0.a);
        }
        T bnd = boundary(r0);
        int j = r0;
        for (; j + 3 < r1; j += 4) {
            if (j != r0 && ((j - r0) & 31) == 0) bnd = boundary(j);
            strip_row<T, Ops, NOISE>(m, g, j, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o, u_o, nb,
                                     block_key, bnd, w0, w1, w2, w3, u0, u1, u2, u3, ja, jb, dt, scale_amp);
            strip_row<T, Ops, NOISE>(m, g, j + 1, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o,
                                     u_o, nb, block_key, bnd, w1, w2, w3, w0, u1, u2, u3, u0, jb, ja, dt, scale_amp);
            strip_row<T, Ops, NOISE>(m, g, j + 2, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o,
                                     u_o, nb, block_key, bnd, w2, w3, w0, w1, u2, u3, u0, u1, ja, jb, dt, scale_amp);
            strip_row<T, Ops, NOISE>(m, g, j + 3, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o,
                                     u_o, nb, block_key, bnd, w3, w0, w1, w2, u3, u0, u1, u2, jb, ja, dt, scale_amp);
        }
        if (j < r1 && j != r0 && ((j - r0) & 31) == 0) bnd = boundary(j);
        if (j < r1)
            strip_row<T, Ops, NOISE>(m, g, j, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o, u_o, nb,
                                     block_key, bnd, w0, w1, w2, w3, u0, u1, u2, u3, ja, jb, dt, scale_amp);
        if (j + 1 < r1)
            strip_row<T, Ops, NOISE>(m, g, j + 1, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o,
                                     u_o, nb, block_key, bnd, w1, w2, w3, w0, u1, u2, u3, u0, jb, ja, dt, scale_amp);
        if (j + 2 < r1)
            strip_row<T, Ops, NOISE>(m, g, j + 2, r0, lane, col, valid, last_lane, n0, n1, phc, uuc, out, phi_o,
                                     u_o, nb, block_key, bnd, w2, w3, w0, w1, u2, u3, u0, u1, ja, jb, dt, scale_amp);
    }
}

// Rows per work unit: a multiple of 32 (boundary faces come in batches of
// 32 rows), chosen so the grid holds several waves of warps on 148 SMs.
inline int strip_rows(const CartTopo& topo, int strips, int rows) {
    const int n1 = topo.n[1];
    if (rows <= 0) {
        const int64_t want_units = (int64_t)148 * 48 * 4;
        const int64_t per_chunk = (int64_t)topo.nblocks * strips;
        const int chunks =
            (int)std::max<int64_t>(1, std::min<int64_t>(n1, (want_units + per_chunk - 1) / per_chunk));
        rows = (n1 + chunks - 1) / chunks;
        rows = std::max(32, (rows + 31) / 32 * 32);
    }
    return std::max(1, std::min(rows, n1));
}

template <class T, class Ops, bool NOISE, int MINB = 2>
cudaError_t launch_strip_ops(const T* in, T* out, TileArgs g, const typename Ops::Params& m, T dt, T scale_amp,
                             cudaStream_t s) {
    const int n0 = g.topo.n[0], n1 = g.topo.n[1];
    g.strips = (n0 + 31) / 32;
    g.rows = strip_rows(g.topo, g.strips, g.rows);
    g.chunks = (n1 + g.rows - 1) / g.rows;
    g.units = (int64_t)g.topo.nblocks * g.strips * g.chunks;
    const int wpc = 8;
    const int64_t ctas = std::min<int64_t>((g.units + wpc - 1) / wpc, (int64_t)1 << 30);
    modelc_strip_kernel<T, Ops, NOISE, MINB><<<(unsigned)ctas, wpc * 32, 0, s>>>(in, out, g, m, dt, scale_amp);
    return cudaGetLastError();
}

}  // namespace lg
