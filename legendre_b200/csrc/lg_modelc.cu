// Column-tile Model C step kernel.
//
// One CTA owns a run of rows of one block; thread t owns column t and walks
// up the rows with a 3x3 register window of phi (u keeps its column).  Every
// face flux of the Karma-Rappel divergence is computed once and shared by
// the two cells that touch it: the reference evaluates the right face of
// cell i and the left face of cell i+1 (and top of j / bottom of j+1) with
// the same expression in the same operand order (finite_volume.rs:261-280),
// so sharing is bit-exact and halves the face work.  x faces travel between
// threads through a double-buffered shared-memory row (one barrier per
// row); the y face below a cell is the y face above it in the previous row.
//
// Compiled with -fmad=false (bit-exact FP64; see lg_kernels.cu).
#include <algorithm>
#include <cmath>

#include "lg_common.cuh"
#include "lg_kernels.h"
#include "lg_modelc_ops.cuh"

namespace lg {
namespace {

template <class T, bool NOISE, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    modelc_tile_kernel(const T* __restrict__ in, T* __restrict__ out, CartTopo topo, SlabLayout L, MC<T> m, T dt,
                       double dt64, uint64_t seed, T scale_amp, double* tdev, int slot, int rows) {
    extern __shared__ __align__(16) unsigned char lg_smem[];
    const int n0 = topo.n[0], n1 = topo.n[1];
    T* xf = reinterpret_cast<T*>(lg_smem);  // 2 x n0 x-face fluxes (left faces of the columns)
    T* xlast = xf + 2 * n0;                 // right face of the last column, one per row of the chunk
    const int sy = L.gdim[0];
    const int t = threadIdx.x;
    const int nt = blockDim.x;
    const bool cell = t < n0;
    const T quarter = T(0.25), half = T(0.5);

    const double tnow = tdev[slot];
    if (blockIdx.x == 0 && blockIdx.y == 0 && t == 0) tdev[slot ^ 1] = tnow + dt64;

    for (int b = blockIdx.y; b < topo.nblocks; b += gridDim.y) {
        const int r0 = blockIdx.x * rows;
        const int r1 = min(n1, r0 + rows);
        if (r0 >= n1) continue;  // uniform over the CTA
        const T* ph = in + slab_base(L, b, 0);
        const T* uu = in + slab_base(L, b, 1);
        T* phi_out = out + slab_base(L, b, 0);
        T* u_out = out + slab_base(L, b, 1);
        Nbr2 nb;
        nb.load(topo, b);
        uint64_t block_key = 0;
        if (NOISE) block_key = wiener_block_key(seed, (uint64_t)__double_as_longlong(tnow), kWienerStream0, (uint64_t)b);

        // slab offset of interior-relative (column c, row r)
        auto at = [&](int c, int r) -> int64_t { return (int64_t)(c + 1) + (int64_t)(r + 1) * sy; };

        // the x face between column n0-1 and the ghost column, every row of
        // the chunk, lanes across rows
        for (int r = r0 + t; r < r1; r += nt) {
            const T c0m = __ldg(ph + at(n0 - 1, r - 1)), c1m = __ldg(ph + at(n0, r - 1));
            const T c00 = __ldg(ph + at(n0 - 1, r)), c10 = __ldg(ph + at(n0, r));
            const T c0p = __ldg(ph + at(n0 - 1, r + 1)), c1p = __ldg(ph + at(n0, r + 1));
            T dx = c10 - c00;
            T dy = quarter * (c1p - c1m + c0p - c0m);
            T a, da;
            kr_face(m, dx, dy, a, da);
            xlast[r - r0] = a * (a * dx - da * dy);
        }

        T pm[3], p0[3], pp[3];  // phi at rows j-1, j, j+1; columns t-1, t, t+1
        T um, u0c, up;          // u at column t, rows j-1, j, j+1
        if (cell) {
            pm[0] = __ldg(ph + at(t - 1, r0 - 1));
            pm[1] = __ldg(ph + at(t, r0 - 1));
            pm[2] = __ldg(ph + at(t + 1, r0 - 1));
            p0[0] = __ldg(ph + at(t - 1, r0));
            p0[1] = __ldg(ph + at(t, r0));
            p0[2] = __ldg(ph + at(t + 1, r0));
            pp[0] = __ldg(ph + at(t - 1, r0 + 1));
            pp[1] = __ldg(ph + at(t, r0 + 1));
            pp[2] = __ldg(ph + at(t + 1, r0 + 1));
            um = __ldg(uu + at(t, r0 - 1));
            u0c = __ldg(uu + at(t, r0));
            up = __ldg(uu + at(t, r0 + 1));
        }
        // y face below the first row (between r0-1 and r0)
        T jb = T(0);
        if (cell) {
            T dy = p0[1] - pm[1];
            T dx = quarter * (p0[2] - p0[0] + pm[2] - pm[0]);
            T a, da;
            kr_face(m, dx, dy, a, da);
            jb = a * (a * dy + da * dx);
        }
        int par = 0;
        for (int j = r0; j < r1; ++j) {
            // prefetch row j+2 (ghost row n1 is the last that exists)
            const bool more = j + 2 <= n1;
            T q0 = T(0), q1 = T(0), q2 = T(0), uq = T(0), ul = T(0), ur = T(0);
            if (cell) {
                if (more) {
                    q0 = __ldg(ph + at(t - 1, j + 2));
                    q1 = __ldg(ph + at(t, j + 2));
                    q2 = __ldg(ph + at(t + 1, j + 2));
                    uq = __ldg(uu + at(t, j + 2));
                }
                ul = __ldg(uu + at(t - 1, j));
                ur = __ldg(uu + at(t + 1, j));
            }
            // x face on the left of column t, row j (the reference's j_l of
            // cell t and j_r of cell t-1)
            T* xrow = xf + par * n0;
            if (cell) {
                T dx = p0[1] - p0[0];
                T dy = quarter * (pp[1] - pm[1] + pp[0] - pm[0]);
                T a, da;
                kr_face(m, dx, dy, a, da);
                xrow[t] = a * (a * dx - da * dy);
            }
            // y face above cell (t, j)
            T jt = T(0);
            if (cell) {
                T dy = pp[1] - p0[1];
                T dx = quarter * (pp[2] - pp[0] + p0[2] - p0[0]);
                T a, da;
                kr_face(m, dx, dy, a, da);
                jt = a * (a * dy + da * dx);
            }
            __syncthreads();
            if (cell) {
                const T jl = xrow[t], jr = t + 1 < n0 ? xrow[t + 1] : xlast[j - r0];
                const T flux = (jr - jl + jt - jb) * m.inv_h2_flux;
                const T p = p0[1];
                const T g_prime = fma_t(p * p, p, -p);
                const T one_m_p2 = fma_t(p, -p, T(1));
                const T p_prime = one_m_p2 * one_m_p2;
                const T a = center_anisotropy(m, half * (p0[2] - p0[0]), half * (pp[1] - pm[1]));
                const T kphi = fma_t(m.lambda * u0c, -p_prime, flux - g_prime) / (a * a);
                T acc = T(0);
                acc += ((ur - (u0c + u0c)) + ul) * m.ih0;
                acc += ((up - (u0c + u0c)) + um) * m.ih1;
                const T ku = fma_t(acc, m.d_thermal, half * kphi);
                T phin = p + dt * kphi;
                if (NOISE) {
                    const uint64_t key = splitmix64(block_key ^ (uint64_t)(t + j * n0));
                    phin += scale_amp * normal_t(key, T(0));
                }
                const T un = u0c + dt * ku;
                phi_out[at(t, j)] = phin;
                u_out[at(t, j)] = un;
                push_ghosts_2d_g1(out, L, 0, nb, n0, n1, t, j, phin);
                push_ghosts_2d_g1(out, L, 1, nb, n0, n1, t, j, un);
                jb = jt;
                um = u0c;
                u0c = up;
                up = uq;
            }
            pm[0] = p0[0]; pm[1] = p0[1]; pm[2] = p0[2];
            p0[0] = pp[0]; p0[1] = pp[1]; p0[2] = pp[2];
            pp[0] = q0; pp[1] = q1; pp[2] = q2;
            par ^= 1;
        }
        __syncthreads();  // xf reuse by the next block of this CTA
    }
}

template <class T, bool NOISE>
cudaError_t launch_tile(const T* in, T* out, const CartTopo& topo, const SlabLayout& L, const MC<T>& m, T dt,
                        double dt64, uint64_t seed, T scale_amp, double* tdev, int slot, int rows, cudaStream_t s) {
    const int n0 = topo.n[0], n1 = topo.n[1];
    const int threads = (n0 + 31) / 32 * 32;
    if (rows <= 0) {
        // enough CTAs for several waves on 148 SMs, at least 16 rows each
        // (the y face under the first row is evaluated once more per CTA)
        const int64_t want = 148 * 8;
        int chunks = (int)std::max<int64_t>(1, (want + topo.nblocks - 1) / topo.nblocks);
        rows = std::max(16, (n1 + chunks - 1) / chunks);
    }
    rows = std::min(rows, n1);
    dim3 grid((n1 + rows - 1) / rows, std::min(topo.nblocks, 65535));
    size_t smem = (2 * (size_t)n0 + rows) * sizeof(T);
    if (threads <= 256)
        modelc_tile_kernel<T, NOISE, 256, 2><<<grid, threads, smem, s>>>(in, out, topo, L, m, dt, dt64, seed,
                                                                          scale_amp, tdev, slot, rows);
    else
        modelc_tile_kernel<T, NOISE, 1024, 1><<<grid, threads, smem, s>>>(in, out, topo, L, m, dt, dt64, seed,
                                                                           scale_amp, tdev, slot, rows);
    return cudaGetLastError();
}

}  // namespace

bool modelc_tile_supported(const CartTopo& topo) { return topo.D == 2 && topo.n[0] >= 1 && topo.n[0] <= 1024; }

cudaError_t launch_modelc_tile_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, cudaStream_t s) {
    const MC<double> mc = to_mc<double>(m);
    const double scale_amp = std::sqrt(dt) * nz.amp;
    if (nz.on)
        return launch_tile<double, true>(in, out, topo, L, mc, dt, dt, nz.seed, scale_amp, tdev, slot, rows, s);
    return launch_tile<double, false>(in, out, topo, L, mc, dt, dt, nz.seed, scale_amp, tdev, slot, rows, s);
}

cudaError_t launch_modelc_tile_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, cudaStream_t s) {
    const MC<float> mc = to_mc<float>(m);
    const float scale_amp = (float)std::sqrt(dt) * (float)nz.amp;
    if (nz.on)
        return launch_tile<float, true>(in, out, topo, L, mc, (float)dt, dt, nz.seed, scale_amp, tdev, slot, rows, s);
    return launch_tile<float, false>(in, out, topo, L, mc, (float)dt, dt, nz.seed, scale_amp, tdev, slot, rows, s);
}

}  // namespace lg
