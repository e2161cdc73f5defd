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
// The row loop keeps a window of four phi rows (j-1, j, j+1 and the
// prefetch of j+2).  It keeps one copy of the row code and shifts the window
// by register moves; only the FP32 oriented form unrolls it four times, so
// that the window rotates with no moves.
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
//   oxface/oyface/ocell     the same in a cell's crystal frame (ORIENT)
// The operand lists keep the reference's evaluation order available to an
// exact policy.
//
// Template flags beside the arithmetic: ORIENT steps the multi-grain form
// (every face's anisotropy in its cell's crystal frame, cos/sin theta0 from a
// per-state table); MODE 0 is the Euler-Maruyama step, MODE 1 and 2 the
// RungeKutta4 stages (see RkArgs); BATCH serves ensembles; TAIL blocks lower
// than the row group.
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
    // persistent work list (null: a static grid-stride schedule): one wave
    // of CTAs, each warp taking its first unit by position and every further
    // one from work[slot]; the step clears work[slot ^ 1] for the next step
    unsigned* work;
};

// Batched instances (BATCH kernels): block b belongs to instance b / bpi,
// whose parameters are params[instance] (an Ops::Params array on the
// device) and whose Wiener seed is seeds[instance]; its noise keys use the
// instance-local block index b % bpi.
struct BatchArgs {
    const void* params;
    const uint64_t* seeds;
    int bpi;
};

// RungeKutta4 stages (MODE 1, 2; rk4.rs:40-79).  All arenas share the
// state's slab layout.  MODE 1: k receives the drift of the input, the output
// is y + c k (y_tmp = y; y_tmp += c k_i).  MODE 2: the output is
// (((y + s6 k1) + s3 k2) + s3 k3) + s6 k4, k4 the drift of the input.
template <class T>
struct RkArgs {
    const T* y;
    T* k;
    const T* k1;
    const T* k2;
    const T* k3;
    T c, s6, s3;
};

// Ghost images of a strip's x-edge cells (the block's columns 0 and n0 - 1)
// for the rows of one unit: lane k holds row r0 + k's phi and u of the left
// (l0, l1) and right (r0, r1) edge cells, gathered by shuffles as the rows
// are stepped and written once at the unit's end (rows 0 and n1 - 1, whose
// images include y ghosts and corners, are pushed in full as they go).
template <class T>
struct EdgeHold {
    T l0, l1, r0, r1;
};

// store the cell, and take care of its ghost images (see EdgeHold)
template <class T>
__device__ __forceinline__ void store_cell(T* __restrict__ out, T* __restrict__ po, T* __restrict__ uo, int off,
                                           T phin, T un, bool ok, bool live, bool edge_x, int j, int r0, int n0,
                                           int n1, int col, int lane, int last_lane, const SlabLayout& L,
                                           const Nbr2& nb, EdgeHold<T>& eh) {
    if (ok) {
        po[off] = phin;
        uo[off] = un;
    }
    if (j == 0 || j == n1 - 1) {  // warp-uniform
        if (ok) {
            push_ghosts_2d_g1(out, L, 0, nb, n0, n1, col, j, phin);
            push_ghosts_2d_g1(out, L, 1, nb, n0, n1, col, j, un);
        }
    } else if (edge_x) {  // warp-uniform: warps on a block's x edge collect their edge cells
        const T l0 = __shfl_sync(0xffffffffu, phin, 0), l1 = __shfl_sync(0xffffffffu, un, 0);
        const T rr0 = __shfl_sync(0xffffffffu, phin, last_lane), rr1 = __shfl_sync(0xffffffffu, un, last_lane);
        if (live && lane == ((j - r0) & 31)) {
            eh.l0 = l0;
            eh.l1 = l1;
            eh.r0 = rr0;
            eh.r1 = rr1;
        }
    }
}

// the collected x-edge images of a unit's rows (r0 .. r1-1, not 0 or n1-1):
// the left edge's into the left neighbour's ghost column n0 (or this block's
// mirror ghost column -1), the right edge's likewise (push_ghosts_2d_g1)
template <class T>
__device__ __forceinline__ void flush_edges(T* __restrict__ out, const SlabLayout& L, const Nbr2& nb, int n0, int n1,
                                            int r0, int r1, int lane, bool left, bool right, const EdgeHold<T>& eh,
                                            int rs = -1) {
    const int r = r0 + lane;
    if (r >= r1 || r < rs || r == 0 || r == n1 - 1) return;  // rows below rs: another unit's
    const int64_t row = (int64_t)(r + 1) * L.gdim[0];
    if (left) {
        const int tb = nb.l >= 0 ? nb.l : nb.b, ci = nb.l >= 0 ? n0 : -1;
        out[slab_base(L, tb, 0) + (ci + 1) + row] = eh.l0;
        out[slab_base(L, tb, 1) + (ci + 1) + row] = eh.l1;
    }
    if (right) {
        const int tb = nb.r >= 0 ? nb.r : nb.b, ci = nb.r >= 0 ? -1 : n0;
        out[slab_base(L, tb, 0) + (ci + 1) + row] = eh.r0;
        out[slab_base(L, tb, 1) + (ci + 1) + row] = eh.r1;
    }
}

// The new phi and u of a cell from its drift (kphi, ku): the Euler-Maruyama
// update (MODE 0) or a RungeKutta4 stage (MODE 1, 2); e0/e1 index the cell's
// phi/u entries in any arena of the state's layout.
template <class T, class Ops, bool NOISE, int MODE>
__device__ __forceinline__ void cell_update(const RkArgs<T>& rk, T dt, T scale_amp, T nval, T kphi, T ku, T p, T uc,
                                            int64_t e0, int64_t e1, bool ok, T& phin, T& un) {
    if constexpr (MODE == 0) {
        phin = Ops::axpy(dt, kphi, p);
        if (NOISE) phin = Ops::add_noise(phin, scale_amp, nval);
        un = Ops::axpy(dt, ku, uc);
    } else if constexpr (MODE == 1) {
        phin = un = T(0);  // cells that store nothing read nothing either
        if (ok) {
            rk.k[e0] = kphi;
            rk.k[e1] = ku;
            phin = rk.y[e0] + rk.c * kphi;
            un = rk.y[e1] + rk.c * ku;
        }
    } else {
        phin = un = T(0);
        if (!ok) return;
        phin = rk.y[e0];
        phin = phin + rk.s6 * rk.k1[e0];
        phin = phin + rk.s3 * rk.k2[e0];
        phin = phin + rk.s3 * rk.k3[e0];
        phin = phin + rk.s6 * kphi;
        un = rk.y[e1];
        un = un + rk.s6 * rk.k1[e1];
        un = un + rk.s3 * rk.k2[e1];
        un = un + rk.s3 * rk.k3[e1];
        un = un + rk.s6 * ku;
    }
}

// Multi-grain kernels (ORIENT): cos theta0 of every interior cell, blocks in
// order and each block's cells dimension-0-fastest, followed by sin theta0
// in the same order (ncells values each), in the kernel's element type.
struct OrientArgs {
    const void* trig;
    int64_t ncells;
};

template <class T>
struct Row3 {
    T a, b, c;  // columns c-1, c, c+1
};

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool same_bits(double a, double b) { return __double_as_longlong(a) == __double_as_longlong(b); }
__device__ __forceinline__ bool same_bits(float a, float b) { return __float_as_int(a) == __float_as_int(b); }

// One row: x face left of the lane's column, y face above cell (c, j), the
// cell update, stores and ghost pushes.  A, B, C = phi rows j-1, j, j+1 at
// columns c-1, c, c+1; UA, UB, UC = u at column c for the same rows; P / UP
// receive the prefetch of row j+1+PF.  `off` is the slab offset of (col, j); ph/uu/po/uo
// are the warp's slab bases.  NX > 0 fixes the block width (and the row
// stride) at compile time; FULL means every lane owns a column.
template <class T, class Ops, bool NOISE, int NX, bool FULL, int PF, bool TAIL, bool ORIENT, int MODE>
__device__ __forceinline__ void strip_row(const typename Ops::Params& m, const TileArgs& g, int j, int r0, int r1,
                                          int lane,
                                          int col, bool valid, int last_lane, int n0, int n1, int off,
                                          const T* __restrict__ ph, const T* __restrict__ uu, T* __restrict__ out,
                                          T* __restrict__ po, T* __restrict__ uo, const Nbr2& nb, bool edge_x,
                                          uint64_t block_key, T bnd, const Row3<T>& A, const Row3<T>& B,
                                          const Row3<T>& C, Row3<T>& P, T UA, T UB, T UC, T& UP, T& jb, T dt,
                                          T scale_amp, const T* __restrict__ trig_b, int64_t ncells, T& cprev,
                                          T& sprev, T& cnext, T& snext, const RkArgs<T>& rk, EdgeHold<T>& eh,
                                          int rs) {
    const int sy = NX > 0 ? NX + 2 : g.L.gdim[0];
    // lanes past the block's last column (valid false) run the same code on
    // a clamped column and only skip the stores: no branch splits the face,
    // noise and cell arithmetic.  Unit heights are whole groups of NB rows,
    // so the row loop has no separately unrolled tail; only blocks of fewer
    // than NB rows (TAIL) run rows past the unit's end, without stores.
    // rows below rs belong to the unit below (a block's last unit overlaps
    // it): computed for their faces, stored only by their own unit
    const bool live = (!TAIL || j < r1) && j >= rs;
    const bool ok = (FULL || valid) && live;
    if (j + 1 + PF <= n1) {
        const T* q = ph + off + (1 + PF) * sy;
        P.a = __ldg(q - 1);
        P.b = __ldg(q);
        P.c = __ldg(q + 1);
        UP = __ldg(uu + off + (1 + PF) * sy);
    }
    T ul = T(0), ur = T(0);
    if (live) {
        ul = __ldg(uu + off - 1);
        ur = __ldg(uu + off + 1);
    }
    T nval = T(0);
    if (NOISE) nval = Ops::noise(splitmix64(block_key ^ (uint64_t)(col + j * n0)));
    if constexpr (ORIENT) {
        // multi-grain: every face's anisotropy in the frame of the cell being
        // updated.  Within a grain two neighbours share theta0, and the
        // reference evaluates their common face from the same differences in
        // the same order, so it is computed once: the left face comes from
        // this lane, the right face from the next lane (or the strip's
        // boundary batch), the bottom face from the previous row.  Where the
        // neighbour's cos/sin theta0 differ (grain boundaries), the face is
        // evaluated again in this cell's frame.
        // this row's frame arrived with the previous row; fetch the next one
        const T c0 = cnext, s0 = snext;
        if (j + 1 < n1) {
            const int64_t ci = (int64_t)(j + 1) * n0 + (FULL ? col : min(col, n0 - 1));
            cnext = __ldg(trig_b + ci);
            snext = __ldg(trig_b + ncells + ci);
        }
        const T q = T(0.25);
        const T jl = Ops::oxface(m, c0, s0, B.b - B.a, q * (C.b - A.b + C.a - A.a));
        const T jt = Ops::oyface(m, c0, s0, q * (C.c - C.a + B.c - B.a), C.b - B.b);
        T jr = __shfl_down_sync(kFull, jl, 1);
        const T c0n = __shfl_down_sync(kFull, c0, 1), s0n = __shfl_down_sync(kFull, s0, 1);
        const T fb = __shfl_sync(kFull, bnd, (j - r0) & 31);
        if (lane == last_lane)
            jr = fb;
        else if (!(same_bits(c0n, c0) && same_bits(s0n, s0)))
            jr = Ops::oxface(m, c0, s0, B.c - B.b, q * (C.c - A.c + C.b - A.b));
        T jbot = jb;
        if (!(same_bits(cprev, c0) && same_bits(sprev, s0)))
            jbot = Ops::oyface(m, c0, s0, q * (B.c - B.a + A.c - A.a), B.b - A.b);
        T kphi, ku;
        Ops::ocell(m, jr, jl, jt, jbot, B.b, B.c - B.a, C.b - A.b, c0, s0, UB, ul, ur, UC, UA, kphi, ku);
        T phin, un;
        cell_update<T, Ops, NOISE, MODE>(rk, dt, scale_amp, nval, kphi, ku, B.b, UB, (po - out) + off,
                                         (uo - out) + off, ok, phin, un);
        store_cell(out, po, uo, off, phin, un, ok, live, edge_x, j, r0, n0, n1, col, lane, last_lane, g.L, nb, eh);
        jb = jt;
        cprev = c0;
        sprev = s0;
        return;
    }
    const T fl = Ops::xface(m, B.b - B.a, C.b - A.b, C.a, A.a);
    const T jt = Ops::yface(m, C.b - B.b, C.c - C.a, B.c, B.a);
    // right face: the next lane's left face, or the strip's boundary face of this row
    T fr = __shfl_down_sync(kFull, fl, 1);
    const T fb = __shfl_sync(kFull, bnd, (j - r0) & 31);
    if (lane == last_lane) fr = fb;
    T kphi, ku;
    Ops::cell(m, fr, fl, jt, jb, B.b, B.c - B.a, C.b - A.b, UB, ul, ur, UC, UA, kphi, ku);
    T phin, un;
    cell_update<T, Ops, NOISE, MODE>(rk, dt, scale_amp, nval, kphi, ku, B.b, UB, (po - out) + off, (uo - out) + off,
                                     ok, phin, un);
    store_cell(out, po, uo, off, phin, un, ok, live, edge_x, j, r0, n0, n1, col, lane, last_lane, g.L, nb, eh);
    jb = jt;
}

// One work unit of the strip kernel: the rows [r0, r1) of the 32-column
// strip at c0 of block b, with the parameter record m (the kernel parameter,
// or a batched instance's record) and the Wiener key of block key_block.
template <class T, class Ops, bool NOISE, int NX, bool FULL, int PF, bool TAIL, bool ORIENT, int MODE>
__device__ __forceinline__ void strip_unit(const typename Ops::Params& m, uint64_t seed, int key_block,
                                           const TileArgs& g, const T* __restrict__ ph, const T* __restrict__ uu,
                                           T* __restrict__ out, T* __restrict__ po, T* __restrict__ uo,
                                           const Nbr2& nb, int r0, int r1, int lane, int col, bool valid,
                                           int last_lane, int cr, bool edge_x, int n0, int n1, int sy, double tnow,
                                           T dt, T scale_amp, const T* __restrict__ trig_b, int64_t ncells, const RkArgs<T>& rk,
                                           int rs) {
    constexpr int NB = PF + 3;
    uint64_t block_key = 0;
    if (NOISE)
        block_key = wiener_block_key(seed, (uint64_t)__double_as_longlong(tnow), kWienerStream0,
                                     (uint64_t)key_block);

    // slab offset of (col, r0); a lane past the last column reads the last one
    int off = ((FULL ? col : min(col, n0 - 1)) + 1) + (r0 + 1) * sy;
    Row3<T> w[NB];
    T uw[NB];
    T jb = T(0);
    // window: rows r0-1 .. r0+PF in w[0..NB-2]; w[NB-1] is filled by the first row
#pragma unroll
    for (int q = 0; q < NB - 1; ++q) {
        w[q] = Row3<T>{};
        uw[q] = T(0);
        const int r = r0 - 1 + q;
        if (r <= n1) {
            const T* p = ph + off + (q - 1) * sy;
            w[q] = {__ldg(p - 1), __ldg(p), __ldg(p + 1)};
            uw[q] = __ldg(uu + off + (q - 1) * sy);
        }
    }
    w[NB - 1] = Row3<T>{};
    uw[NB - 1] = T(0);
    // right-boundary face of the strip for rows r0 .. r0+31 (lane = row)
    T bnd = T(0);
    if constexpr (!ORIENT) {
        const int r = r0 + lane;
        if (r < r1) {
            const T* q = ph + (cr + 1) + (r + 1) * sy;  // (column cr, row r)
            const T c0m = __ldg(q - sy), c1m = __ldg(q - sy + 1);
            const T c00 = __ldg(q), c10 = __ldg(q + 1);
            const T c0p = __ldg(q + sy), c1p = __ldg(q + sy + 1);
            bnd = Ops::xface(m, c10 - c00, c1p - c1m, c0p, c0m);
        }
    } else {  // the same faces in the frame of the strip's last cell of each row
        const int r = r0 + lane;
        if (r < r1) {
            const T* q = ph + (cr + 1) + (r + 1) * sy;
            const T c0m = __ldg(q - sy), c1m = __ldg(q - sy + 1);
            const T c00 = __ldg(q), c10 = __ldg(q + 1);
            const T c0p = __ldg(q + sy), c1p = __ldg(q + sy + 1);
            const int64_t ci = (int64_t)r * n0 + cr;
            bnd = Ops::oxface(m, __ldg(trig_b + ci), __ldg(trig_b + ncells + ci), c10 - c00,
                              T(0.25) * (c1p - c1m + c0p - c0m));
        }
    }
    // y face below the first row (between r0-1 and r0)
    T cpv = T(0), spv = T(0);  // cos/sin theta0 of the previous row's cell (multi-grain)
    T cnx = T(0), snx = T(0);  // and of the row about to be stepped
    if constexpr (!ORIENT) {
        jb = Ops::yface(m, w[1].b - w[0].b, w[1].c - w[1].a, w[0].c, w[0].a);
    } else {  // bottom face of the first row in its own frame
        const int64_t ci = (int64_t)r0 * n0 + (FULL ? col : min(col, n0 - 1));
        cpv = cnx = __ldg(trig_b + ci);
        spv = snx = __ldg(trig_b + ncells + ci);
        jb = Ops::oyface(m, cpv, spv, T(0.25) * (w[1].c - w[1].a + w[0].c - w[0].a), w[1].b - w[0].b);
    }

    EdgeHold<T> eh{T(0), T(0), T(0), T(0)};
#define LG_ROW(J, Q)                                                                                            \
    strip_row<T, Ops, NOISE, NX, FULL, PF, TAIL, ORIENT, MODE>(m, g, J, r0, r1, lane, col, valid, last_lane, n0, n1, off, ph, uu, out, po,  \
                                       uo, nb, edge_x, block_key, bnd, w[(Q) % NB], w[((Q) + 1) % NB],          \
                                       w[((Q) + 2) % NB], w[((Q) + 2 + PF) % NB], uw[(Q) % NB],                \
                                       uw[((Q) + 1) % NB], uw[((Q) + 2) % NB], uw[((Q) + 2 + PF) % NB], jb, dt, \
                                       scale_amp, trig_b, ncells, cpv, spv, cnx, snx, rk, eh, rs);                                                          \
    off += sy
    if constexpr (sizeof(T) == 8 || !ORIENT) {
        // one copy of the row code: the window shifts down by one row
        // through registers instead of rotating through NB unrolled copies,
        // which overflowed the instruction cache and spilled (FP64 4096^2:
        // 51.8 against 45.1 Gcell/s; 10080^2 with 1000 oriented grains: 33.7
        // against 25.3; FP32 4096^2: 100.1 against 94.2, and 3 CTAs per SM
        // without spills).  The FP32 oriented form is faster unrolled
        // (10080^2: 74.7 against 71.8).
#pragma unroll 1
        for (int j = r0; j < r1; ++j) {
            LG_ROW(j, 0);
#pragma unroll
            for (int q = 0; q + 1 < NB; ++q) {
                w[q] = w[q + 1];
                uw[q] = uw[q + 1];
            }
        }
    } else {
        for (int j = r0; j < r1; j += NB) {
#pragma unroll
            for (int q = 0; q < NB; ++q) { LG_ROW(j + q, q); }
        }
    }
#undef LG_ROW
    if (edge_x) flush_edges(out, g.L, nb, n0, n1, r0, r1, lane, col - lane == 0, cr == n0 - 1, eh, rs);
}

// The paired form of one work unit (Euler-Maruyama, axis-aligned, units of
// an even number of rows): each pass of the row loop steps rows j and j+1
// together, so every lane carries two independent cells -- four face fluxes,
// two Gaussians, two cell updates -- whose dependency chains the scheduler
// interleaves; the y face between the two rows is computed once.  Each pass
// reads its four phi and u rows j-1 .. j+2 from L1, where the previous pass
// prefetched them, instead of carrying a six-row window in registers: the
// unit needs fewer registers (no spills at 3 CTAs per SM) and no register
// moves to shift the window.  Units are a multiple of four rows ending at
// or before the ghost row n1, so every row read lies inside the slab.
// Same arithmetic per cell, in the same operand order, as strip_row.
//
// ORIENT: the multi-grain faces (strip_row's ORIENT branch, for two rows):
// each face in the frame of the cell being updated, shared with the
// neighbour only where the neighbour's cos/sin theta0 are the same bits,
// else evaluated again in this cell's frame.
template <class T, class Ops, bool NOISE, int NX, bool FULL, bool ORIENT = false>
__device__ __forceinline__ void strip_unit_pair(const typename Ops::Params& m, uint64_t seed, int key_block,
                                                const TileArgs& g, const T* __restrict__ ph,
                                                const T* __restrict__ uu, T* __restrict__ out, T* __restrict__ po,
                                                T* __restrict__ uo, const Nbr2& nb, int r0, int r1, int lane,
                                                int col, bool valid, int last_lane, int cr, bool edge_x, int n0,
                                                int n1, int sy, double tnow, T dt, T scale_amp, int rs,
                                                const T* __restrict__ trig_b = nullptr, int64_t ncells = 0) {
    uint64_t block_key = 0;
    if (NOISE)
        block_key = wiener_block_key(seed, (uint64_t)__double_as_longlong(tnow), kWienerStream0,
                                     (uint64_t)key_block);
    const bool ok = FULL || valid;
    // slab offset of (col, r0), fixed for the unit; `off` follows the row pair
    const int off0 = ((FULL ? col : min(col, n0 - 1)) + 1) + (r0 + 1) * sy;
    int off = off0;
    // phi (columns col-1, col, col+1) and u of row r, for -1 <= r <= n1 (row
    // n1 is the ghost row); rows past n1 read as zero and are never used
    auto load_row = [&](int r, Row3<T>& w, T& uw) {
        w = Row3<T>{};
        uw = T(0);
        if (r <= n1) {
            const T* q = ph + off0 + (r - r0) * sy;
            w = {__ldg(q - 1), __ldg(q), __ldg(q + 1)};
            uw = __ldg(uu + off0 + (r - r0) * sy);
        }
    };
    Row3<T> A, B, C, D;
    T UA, UB, UC, UD;
    load_row(r0 - 1, A, UA);
    load_row(r0, B, UB);
    T bnd = T(0);
    {
        const int r = r0 + lane;
        if (r < r1) {
            const T* q = ph + (cr + 1) + (r + 1) * sy;  // (column cr, row r)
            const T c0m = __ldg(q - sy), c1m = __ldg(q - sy + 1);
            const T c00 = __ldg(q), c10 = __ldg(q + 1);
            const T c0p = __ldg(q + sy), c1p = __ldg(q + sy + 1);
            if constexpr (ORIENT) {  // in the frame of the strip's last cell of the row
                const int64_t ci = (int64_t)r * n0 + cr;
                bnd = Ops::oxface(m, __ldg(trig_b + ci), __ldg(trig_b + ncells + ci), c10 - c00,
                                  T(0.25) * (c1p - c1m + c0p - c0m));
            } else {
                bnd = Ops::xface(m, c10 - c00, c1p - c1m, c0p, c0m);
            }
        }
    }
    const int ccol = FULL ? col : min(col, n0 - 1);
    T cprev = T(0), sprev = T(0);  // multi-grain: cos/sin theta0 of the row below the pass
    T jb;
    if constexpr (ORIENT) {  // the bottom face of the first row in its own frame
        const int64_t ci = (int64_t)r0 * n0 + ccol;
        cprev = __ldg(trig_b + ci);
        sprev = __ldg(trig_b + ncells + ci);
        jb = Ops::oyface(m, cprev, sprev, T(0.25) * (B.c - B.a + A.c - A.a), B.b - A.b);
    } else {
        jb = Ops::yface(m, B.b - A.b, B.c - B.a, A.c, A.a);
    }
    EdgeHold<T> eh{T(0), T(0), T(0), T(0)};
#pragma unroll 1
    for (int j = r0; j < r1; j += 2) {
        // the four rows of this pass (j-1 .. j+2 <= n1) from L1, and an L1
        // prefetch of the next pass's two new rows
        {
            const T* q = ph + off - sy;
            A = {__ldg(q - 1), __ldg(q), __ldg(q + 1)};
            B = {__ldg(q + sy - 1), __ldg(q + sy), __ldg(q + sy + 1)};
            C = {__ldg(q + 2 * sy - 1), __ldg(q + 2 * sy), __ldg(q + 2 * sy + 1)};
            D = {__ldg(q + 3 * sy - 1), __ldg(q + 3 * sy), __ldg(q + 3 * sy + 1)};
            const T* w = uu + off - sy;
            UA = __ldg(w);
            UB = __ldg(w + sy);
            UC = __ldg(w + 2 * sy);
            UD = __ldg(w + 3 * sy);
            const int64_t p3 = (int64_t)(min(j + 3, n1) - j) * sy, p4 = (int64_t)(min(j + 4, n1) - j) * sy;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(ph + off + p3));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(ph + off + p4));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(uu + off + p3));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(uu + off + p4));
        }
        const T ul0 = __ldg(uu + off - 1), ur0 = __ldg(uu + off + 1);
        const T ul1 = __ldg(uu + off + sy - 1), ur1 = __ldg(uu + off + sy + 1);
        T c0 = T(0), s0 = T(0), c1 = T(0), s1 = T(0);  // multi-grain: frames of rows j and j+1
        if constexpr (ORIENT) {
            const int64_t ci = (int64_t)j * n0 + ccol;
            c0 = __ldg(trig_b + ci);
            s0 = __ldg(trig_b + ncells + ci);
            c1 = __ldg(trig_b + ci + n0);
            s1 = __ldg(trig_b + ncells + ci + n0);
        }
        // the Gaussians of the pass, drawn as soon as its loads are issued:
        // their integer and FP64 chains fill the loads' latency and the
        // anisotropy tests that follow, and are needed only at the end
        T nv0 = T(0), nv1 = T(0);
        auto draw = [&]() {
            if (NOISE) {
                nv0 = Ops::noise(splitmix64(block_key ^ (uint64_t)(col + j * n0)));
                nv1 = Ops::noise(splitmix64(block_key ^ (uint64_t)(col + (j + 1) * n0)));
            }
        };
        draw();
        const T fb0 = __shfl_sync(kFull, bnd, (j - r0) & 31), fb1 = __shfl_sync(kFull, bnd, (j + 1 - r0) & 31);
        T phin0, phin1, un0, un1, jt1;
        if constexpr (ORIENT) {
            const T q = T(0.25);
            const T jl0 = Ops::oxface(m, c0, s0, B.b - B.a, q * (C.b - A.b + C.a - A.a));
            const T jt0 = Ops::oyface(m, c0, s0, q * (C.c - C.a + B.c - B.a), C.b - B.b);
            const T jl1 = Ops::oxface(m, c1, s1, C.b - C.a, q * (D.b - B.b + D.a - B.a));
            jt1 = Ops::oyface(m, c1, s1, q * (D.c - D.a + C.c - C.a), D.b - C.b);
            T jr0 = __shfl_down_sync(kFull, jl0, 1), jr1 = __shfl_down_sync(kFull, jl1, 1);
            const T c0n = __shfl_down_sync(kFull, c0, 1), s0n = __shfl_down_sync(kFull, s0, 1);
            const T c1n = __shfl_down_sync(kFull, c1, 1), s1n = __shfl_down_sync(kFull, s1, 1);
            if (lane == last_lane) {
                jr0 = fb0;
                jr1 = fb1;
            } else {
                if (!(same_bits(c0n, c0) && same_bits(s0n, s0)))
                    jr0 = Ops::oxface(m, c0, s0, B.c - B.b, q * (C.c - A.c + C.b - A.b));
                if (!(same_bits(c1n, c1) && same_bits(s1n, s1)))
                    jr1 = Ops::oxface(m, c1, s1, C.c - C.b, q * (D.c - B.c + D.b - B.b));
            }
            T jbot0 = jb, jbot1 = jt0;
            if (!(same_bits(cprev, c0) && same_bits(sprev, s0)))
                jbot0 = Ops::oyface(m, c0, s0, q * (B.c - B.a + A.c - A.a), B.b - A.b);
            if (!(same_bits(c0, c1) && same_bits(s0, s1)))
                jbot1 = Ops::oyface(m, c1, s1, q * (C.c - C.a + B.c - B.a), C.b - B.b);
            T kphi0, ku0, kphi1, ku1;
            Ops::ocell(m, jr0, jl0, jt0, jbot0, B.b, B.c - B.a, C.b - A.b, c0, s0, UB, ul0, ur0, UC, UA, kphi0, ku0);
            Ops::ocell(m, jr1, jl1, jt1, jbot1, C.b, C.c - C.a, D.b - B.b, c1, s1, UC, ul1, ur1, UD, UB, kphi1, ku1);
            phin0 = Ops::axpy(dt, kphi0, B.b);
            phin1 = Ops::axpy(dt, kphi1, C.b);
            if (NOISE) {
                phin0 = Ops::add_noise(phin0, scale_amp, nv0);
                phin1 = Ops::add_noise(phin1, scale_amp, nv1);
            }
            un0 = Ops::axpy(dt, ku0, UB);
            un1 = Ops::axpy(dt, ku1, UC);
            cprev = c1;
            sprev = s1;
        } else {
            T fl0, jt0, fl1;
            T kphi0, ku0, kphi1, ku1;
            bool far = false;
            if constexpr (Ops::kFarPass) {
                // the four faces' and two centres' anisotropy tests; where
                // they are all flat across the warp (the far field) the pass
                // runs without branches, the same expressions as the general
                // path
                const T xn0 = B.b - B.a, xt0 = Ops::quarter(C.b - A.b, C.a, A.a);
                const T yn0 = C.b - B.b, yt0 = Ops::quarter(C.c - C.a, B.c, B.a);
                const T xn1 = C.b - C.a, xt1 = Ops::quarter(D.b - B.b, D.a, B.a);
                const T yn1 = D.b - C.b, yt1 = Ops::quarter(D.c - D.a, C.c, C.a);
                const bool flat = Ops::face_flat(m, xn0, xt0) && Ops::face_flat(m, yt0, yn0) &&
                                  Ops::face_flat(m, xn1, xt1) && Ops::face_flat(m, yt1, yn1) &&
                                  Ops::center_flat(m, B.c - B.a, C.b - A.b) &&
                                  Ops::center_flat(m, C.c - C.a, D.b - B.b);
                far = __all_sync(kFull, flat);
                if (far) {
                    fl0 = Ops::xface_far(m, xn0, xt0);
                    jt0 = Ops::yface_far(m, yn0, yt0);
                    fl1 = Ops::xface_far(m, xn1, xt1);
                    jt1 = Ops::yface_far(m, yn1, yt1);
                    T fr0 = __shfl_down_sync(kFull, fl0, 1), fr1 = __shfl_down_sync(kFull, fl1, 1);
                    if (lane == last_lane) {
                        fr0 = fb0;
                        fr1 = fb1;
                    }
                    Ops::cell_far(m, fr0, fl0, jt0, jb, B.b, UB, ul0, ur0, UC, UA, kphi0, ku0);
                    Ops::cell_far(m, fr1, fl1, jt1, jt0, C.b, UC, ul1, ur1, UD, UB, kphi1, ku1);
                }
            }
            if (!far) {
                fl0 = Ops::xface(m, B.b - B.a, C.b - A.b, C.a, A.a);
                jt0 = Ops::yface(m, C.b - B.b, C.c - C.a, B.c, B.a);
                fl1 = Ops::xface(m, C.b - C.a, D.b - B.b, D.a, B.a);
                jt1 = Ops::yface(m, D.b - C.b, D.c - D.a, C.c, C.a);
                T fr0 = __shfl_down_sync(kFull, fl0, 1), fr1 = __shfl_down_sync(kFull, fl1, 1);
                if (lane == last_lane) {
                    fr0 = fb0;
                    fr1 = fb1;
                }
                Ops::cell(m, fr0, fl0, jt0, jb, B.b, B.c - B.a, C.b - A.b, UB, ul0, ur0, UC, UA, kphi0, ku0);
                Ops::cell(m, fr1, fl1, jt1, jt0, C.b, C.c - C.a, D.b - B.b, UC, ul1, ur1, UD, UB, kphi1, ku1);
            }
            phin0 = Ops::axpy(dt, kphi0, B.b);
            phin1 = Ops::axpy(dt, kphi1, C.b);
            if (NOISE) {
                phin0 = Ops::add_noise(phin0, scale_amp, nv0);
                phin1 = Ops::add_noise(phin1, scale_amp, nv1);
            }
            un0 = Ops::axpy(dt, ku0, UB);
            un1 = Ops::axpy(dt, ku1, UC);
        }
        // rows below rs belong to the unit below (a block's last unit
        // overlaps it): computed for their faces, stored only once
        const bool own0 = j >= rs, own1 = j + 1 >= rs;
        store_cell(out, po, uo, off, phin0, un0, ok && own0, own0, edge_x, j, r0, n0, n1, col, lane, last_lane, g.L,
                   nb, eh);
        store_cell(out, po, uo, off + sy, phin1, un1, ok && own1, own1, edge_x, j + 1, r0, n0, n1, col, lane,
                   last_lane, g.L, nb, eh);
        jb = jt1;
        off += 2 * sy;
    }
    if (edge_x) flush_edges(out, g.L, nb, n0, n1, r0, r1, lane, col - lane == 0, cr == n0 - 1, eh, rs);
}

// Rows per work unit are at most 32, so one batch of boundary faces (lanes
// across rows) serves the whole unit.
template <class T, class Ops, bool NOISE, int MINB, int NX, int PF, bool BATCH = false, bool TAIL = false,
          bool ORIENT = false, int MODE = 0, bool PAIR = false>
__global__ void __launch_bounds__(256, MINB)
    modelc_strip_kernel(const T* __restrict__ in, T* __restrict__ out, TileArgs g, typename Ops::Params m0, T dt,
                        T scale_amp, BatchArgs bt, OrientArgs oa, RkArgs<T> rk) {
    constexpr bool FULL = NX > 0 && NX % 32 == 0;
    const CartTopo& topo = g.topo;
    const int n0 = NX > 0 ? NX : topo.n[0];
    const int n1 = topo.n[1];
    const int sy = NX > 0 ? NX + 2 : g.L.gdim[0];
    const int lane = threadIdx.x & 31;
    const int wpc = blockDim.x >> 5;

    // Simulation::t lives on the device in two slots: this step reads
    // tdev[slot] (its bits are the Wiener salt, euler_maruyama.rs:73) and
    // writes t + dt to the other slot (simulation.rs:285), so a captured
    // sequence of steps needs no host-side time.
    const double tnow = g.tdev[g.slot];
    if (MODE != 1 && blockIdx.x == 0 && threadIdx.x == 0) {
        g.tdev[g.slot ^ 1] = tnow + g.dt64;
        if (g.work) g.work[g.slot ^ 1] = 0u;
    }

    const int64_t first_listed = (int64_t)gridDim.x * wpc;
    for (int64_t unit = (int64_t)blockIdx.x * wpc + (threadIdx.x >> 5); unit < g.units;) {
        const int s = (int)(unit % g.strips);
        const int k = (int)((unit / g.strips) % g.chunks);
        const int b = (int)(unit / ((int64_t)g.strips * g.chunks));
        // units are g.rows high (a multiple of NB unless TAIL); a block's
        // last unit ends on its last row and may overlap the one before it,
        // whose rows it then recomputes to the same bits
        int r0 = k * g.rows;
        const int rs = r0;  // the unit's own rows start here
        int r1 = r0 + g.rows;
        if (r1 > n1) {
            r1 = n1;
            if (!TAIL) r0 = n1 - g.rows;
        }
        const int c0 = s * 32;
        const int col = c0 + lane;
        const bool valid = FULL || col < n0;
        const int last_lane = min(31, n0 - 1 - c0);
        const int cr = c0 + last_lane;  // last column of the strip; its right face is the boundary face
        const bool edge_x = s == 0 || s == g.strips - 1;

        const T* ph = in + slab_base(g.L, b, 0);
        const T* uu = in + slab_base(g.L, b, 1);
        T* po = out + slab_base(g.L, b, 0);
        T* uo = out + slab_base(g.L, b, 1);
        Nbr2 nb;
        nb.load(topo, b);
        if constexpr (PAIR) {
            static_assert(MODE == 0 && !TAIL && !(ORIENT && BATCH), "the paired rows serve the Euler-Maruyama step");
            if constexpr (BATCH) {
                const int inst = b / bt.bpi;
                const typename Ops::Params mi = static_cast<const typename Ops::Params*>(bt.params)[inst];
                strip_unit_pair<T, Ops, NOISE, NX, FULL>(mi, bt.seeds[inst], b - inst * bt.bpi, g, ph, uu, out, po, uo,
                                                         nb, r0, r1, lane, col, valid, last_lane, cr, edge_x, n0, n1,
                                                         sy, tnow, dt, scale_amp, rs);
            } else {
                const T* trig_b = ORIENT ? static_cast<const T*>(oa.trig) + (int64_t)b * n0 * n1 : nullptr;
                strip_unit_pair<T, Ops, NOISE, NX, FULL, ORIENT>(m0, g.seed, b, g, ph, uu, out, po, uo, nb, r0, r1,
                                                                 lane, col, valid, last_lane, cr, edge_x, n0, n1, sy,
                                                                 tnow, dt, scale_amp, rs, trig_b, oa.ncells);
            }
        } else if constexpr (BATCH) {
            const int inst = b / bt.bpi;
            const typename Ops::Params mi = static_cast<const typename Ops::Params*>(bt.params)[inst];
            strip_unit<T, Ops, NOISE, NX, FULL, PF, TAIL, ORIENT, MODE>(
                mi, bt.seeds[inst], b - inst * bt.bpi, g, ph, uu, out, po, uo, nb, r0, r1, lane, col, valid, last_lane,
                cr, edge_x, n0, n1, sy, tnow, dt, scale_amp, nullptr, 0, rk, rs);
        } else {
            // multi-grain: this block's cos theta0 (sin theta0 follows ncells later)
            const T* trig_b = ORIENT ? static_cast<const T*>(oa.trig) + (int64_t)b * n0 * n1 : nullptr;
            strip_unit<T, Ops, NOISE, NX, FULL, PF, TAIL, ORIENT, MODE>(m0, g.seed, b, g, ph, uu, out, po, uo, nb,
                                                                        r0, r1, lane, col, valid, last_lane, cr,
                                                                        edge_x, n0, n1, sy, tnow, dt, scale_amp,
                                                                        trig_b, oa.ncells, rk, rs);
        }
        if (g.work) {  // the next unit of the list
            unsigned n = 0;
            if (lane == 0) n = atomicAdd(g.work + g.slot, 1u);
            unit = first_listed + (int64_t)__shfl_sync(kFull, n, 0);
        } else {
            unit += first_listed;
        }
    }
}

// Rows per work unit: at most 32 (one batch of boundary faces per unit),
// fewer only when the grid would otherwise hold too few warps, and a whole
// number of groups of nb rows (the row loop's unroll) when the block has at
// least nb rows.
inline int strip_rows(const CartTopo& topo, int strips, int rows, int nb) {
    const int n1 = topo.n[1];
    if (rows <= 0) {
        const int64_t want_units = (int64_t)device_sm_count() * 48 * 2;
        const int64_t per_chunk = (int64_t)topo.nblocks * strips;
        const int chunks =
            (int)std::max<int64_t>(1, std::min<int64_t>(n1, (want_units + per_chunk - 1) / per_chunk));
        rows = std::max(8, (n1 + chunks - 1) / chunks);
    }
    rows = std::max(1, std::min(std::min(rows, 32), n1));
    if (n1 >= nb) rows = std::max(nb, rows / nb * nb);
    return rows;
}

// work decomposition of a launch: units of (block, strip, row chunk); true
// when the block is lower than the row group (the TAIL kernels)
inline bool strip_plan(TileArgs& g, int nb) {
    const int n0 = g.topo.n[0], n1 = g.topo.n[1];
    g.strips = (n0 + 31) / 32;
    g.rows = strip_rows(g.topo, g.strips, g.rows, nb);
    g.chunks = (n1 + g.rows - 1) / g.rows;
    g.units = (int64_t)g.topo.nblocks * g.strips * g.chunks;
    return n1 < nb;
}

inline dim3 strip_ctas(const TileArgs& g) {
    const int wpc = 8;
    return dim3((unsigned)std::min<int64_t>((g.units + wpc - 1) / wpc, (int64_t)1 << 30));
}

// batched instances: block widths 64 (the ensemble configuration) and 32
// get a compile-time row stride
// PAIR: the paired rows (256 instances of 256^2, FP32: 102.5 against 79.8 Gcell/s)
template <class T, class Ops, bool NOISE, int MINB, bool PAIR = false>
cudaError_t launch_strip_batch(const T* in, T* out, TileArgs g, BatchArgs bt, T dt, T scale_amp, cudaStream_t s) {
    const bool tail = strip_plan(g, 1 + 3);
    const dim3 grid = strip_ctas(g), block(256);
    const typename Ops::Params m{};
    if (tail) {
        modelc_strip_kernel<T, Ops, NOISE, MINB, 0, 1, true, true><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, bt, OrientArgs{}, RkArgs<T>{});
        return cudaGetLastError();
    }
    switch (g.topo.n[0]) {
        case 32: modelc_strip_kernel<T, Ops, NOISE, MINB, 32, 1, true, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, bt, OrientArgs{}, RkArgs<T>{}); break;
        case 64: modelc_strip_kernel<T, Ops, NOISE, MINB, 64, 1, true, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, bt, OrientArgs{}, RkArgs<T>{}); break;
        default: modelc_strip_kernel<T, Ops, NOISE, MINB, 0, 1, true, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, bt, OrientArgs{}, RkArgs<T>{});
    }
    return cudaGetLastError();
}

template <class T, class Ops, bool NOISE, int MINB, int PF, bool PAIR = false>
cudaError_t launch_strip_minb(const T* in, T* out, TileArgs g, const typename Ops::Params& m, T dt, T scale_amp,
                              cudaStream_t s) {
    const bool tail = strip_plan(g, PF + 3);
    dim3 grid = strip_ctas(g);
    const dim3 block(256);
    if (g.work)  // the work list: one wave, MINB CTAs per SM
        grid.x = (unsigned)std::min<int64_t>(grid.x, (int64_t)device_sm_count() * MINB);
    if (tail) {  // blocks lower than the row group: single rows (the paired form needs whole groups)
        modelc_strip_kernel<T, Ops, NOISE, MINB, 0, PF, false, true><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, BatchArgs{}, OrientArgs{}, RkArgs<T>{});
        return cudaGetLastError();
    }
    const BatchArgs nob{};
    const OrientArgs noo{};
    const RkArgs<T> nork{};
    switch (g.topo.n[0]) {  // block widths of the shipped configurations get a compile-time row stride
        case 32: modelc_strip_kernel<T, Ops, NOISE, MINB, 32, PF, false, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, nob, noo, nork); break;
        case 64: modelc_strip_kernel<T, Ops, NOISE, MINB, 64, PF, false, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, nob, noo, nork); break;
        case 126: modelc_strip_kernel<T, Ops, NOISE, MINB, 126, PF, false, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, nob, noo, nork); break;
        case 128: modelc_strip_kernel<T, Ops, NOISE, MINB, 128, PF, false, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, nob, noo, nork); break;
        case 256: modelc_strip_kernel<T, Ops, NOISE, MINB, 256, PF, false, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, nob, noo, nork); break;
        default: modelc_strip_kernel<T, Ops, NOISE, MINB, 0, PF, false, false, false, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, nob, noo, nork);
    }
    return cudaGetLastError();
}

// the multi-grain step: block widths 126 (the 101.6M-cell configuration)
// and 256 get a compile-time row stride; PAIR: the paired rows (10080^2
// with 1000 grains: FP64 37.6 against 36.4, FP32 81.7 against 77.0
// Gcell/s)
template <class T, class Ops, bool NOISE, int MINB, bool PAIR = false>
cudaError_t launch_strip_oriented(const T* in, T* out, TileArgs g, const typename Ops::Params& m, T dt, T scale_amp,
                                  OrientArgs oa, cudaStream_t s) {
    const bool tail = strip_plan(g, 1 + 3);
    const dim3 grid = strip_ctas(g), block(256);
    if (tail) {  // blocks lower than the row group: single rows
        modelc_strip_kernel<T, Ops, NOISE, MINB, 0, 1, false, true, true><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, BatchArgs{}, oa, RkArgs<T>{});
        return cudaGetLastError();
    }
    switch (g.topo.n[0]) {
        case 126: modelc_strip_kernel<T, Ops, NOISE, MINB, 126, 1, false, false, true, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, BatchArgs{}, oa, RkArgs<T>{}); break;
        case 256: modelc_strip_kernel<T, Ops, NOISE, MINB, 256, 1, false, false, true, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, BatchArgs{}, oa, RkArgs<T>{}); break;
        default: modelc_strip_kernel<T, Ops, NOISE, MINB, 0, 1, false, false, true, 0, PAIR><<<grid, block, 0, s>>>(in, out, g, m, dt, scale_amp, BatchArgs{}, oa, RkArgs<T>{});
    }
    return cudaGetLastError();
}

// RungeKutta4 stages of Model C (deterministic: no noise), axis-aligned or
// multi-grain, any block width
template <class T, class Ops, int MODE, bool ORIENT>
cudaError_t launch_strip_rk(const T* in, T* out, TileArgs g, const typename Ops::Params& m, T dt, OrientArgs oa,
                            RkArgs<T> rk, cudaStream_t s) {
    const bool tail = strip_plan(g, 1 + 3);
    const dim3 grid = strip_ctas(g), block(256);
    if (tail)
        modelc_strip_kernel<T, Ops, false, 2, 0, 1, false, true, ORIENT, MODE><<<grid, block, 0, s>>>(in, out, g, m, dt, T(0), BatchArgs{}, oa, rk);
    else
        modelc_strip_kernel<T, Ops, false, 2, 0, 1, false, false, ORIENT, MODE><<<grid, block, 0, s>>>(in, out, g, m, dt, T(0), BatchArgs{}, oa, rk);
    return cudaGetLastError();
}

// kind 2/3/4: single rows, CTAs of 256 threads per SM the register
// allocation must allow (2: up to 128 registers, 3: 80, 4: 64); kind 5/6/7:
// the paired rows (strip_unit_pair) at 2/3/4 CTAs per SM.
// PF: rows of prefetch ahead of the row being computed
template <class T, class Ops, bool NOISE, int PF>
cudaError_t launch_strip_ops(const T* in, T* out, TileArgs g, const typename Ops::Params& m, T dt, T scale_amp,
                             int kind, cudaStream_t s) {
    switch (kind) {
        case 3: return launch_strip_minb<T, Ops, NOISE, 3, PF>(in, out, g, m, dt, scale_amp, s);
        case 4: return launch_strip_minb<T, Ops, NOISE, 4, PF>(in, out, g, m, dt, scale_amp, s);
        case 5: return launch_strip_minb<T, Ops, NOISE, 2, PF, true>(in, out, g, m, dt, scale_amp, s);
        case 6: return launch_strip_minb<T, Ops, NOISE, 3, PF, true>(in, out, g, m, dt, scale_amp, s);
        case 7: return launch_strip_minb<T, Ops, NOISE, 4, PF, true>(in, out, g, m, dt, scale_amp, s);
        default: return launch_strip_minb<T, Ops, NOISE, 2, PF>(in, out, g, m, dt, scale_amp, s);
    }
}

}  // namespace lg
