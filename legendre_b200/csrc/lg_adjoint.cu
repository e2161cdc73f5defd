// Hand-written adjoint of the fused Model C Euler-Maruyama step, and the
// terminal-loss kernel that seeds it, for batched instances (lg_ensemble.cu).
//
// One step maps x_n = (phi, u) to x_{n+1}:
//   phi' = phi + dt kphi + s xi,   u' = u + dt (D lap(u) + kphi / 2),
//   kphi = N / A_c^2,  N = -lambda u P'(phi) + flux - g'(phi),
//   flux = (J_R - J_L + J_T - J_B) / (hx hy),
// with the Karma-Rappel face fluxes J(dn, dt) of finite_volume.rs:129-142 /
// 248-285 and the centre anisotropy A_c of phasefield.rs:159-175.  The noise
// s xi does not depend on the state or the parameters, so it drops out of the
// adjoint; the forward states it needs are recomputed by the forward kernel,
// which replays the noise from its counter-based keys.
//
// Given the cotangents (phi', u')^ of x_{n+1}, the kernel returns those of
// x_n and adds the step's contribution to dL/dlambda, dL/dD and dL/deps4.
// Derivation (per interior cell c, mu = dt (phi'^ + u'^/2), nu = dt D u'^):
//   Nbar = mu / A_c^2,  Abar = -2 mu kphi / A_c,
//   face J between cells l (left/below) and r: Jbar = (Nbar_l - Nbar_r)/(hx hy),
//   phi^(p) = [p interior] (phi'^ + Nbar dN/dphi)
//           + sum over the faces whose stencil holds p of Jbar dJ/d(input p)
//           + sum over the neighbours c whose A_c reads p of Abar dA_c/d(input p),
//   u^(p)   = [p interior] (u'^ - Nbar lambda P' - 2 (1/hx^2 + 1/hy^2) nu)
//           + (nu(p-x) + nu(p+x))/hx^2 + (nu(p-y) + nu(p+y))/hy^2.
// Ghost entries are mirror copies of interior cells (zero-flux boundaries),
// so the cotangent of each ghost position is added to its source cell.
//
// Work item: a tile of 32 x TH cells of one instance, in instance-global
// coordinates; its window of (32 + 4) x (TH + 4) positions (two-cell halo)
// is staged in shared memory.  Parameter partial sums are accumulated in
// FP64 into a slot per tile (no atomics: the sums are reproducible).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "lg_adjoint.h"

namespace lg {
namespace adj {
namespace {

constexpr int TW = 32;

__device__ __forceinline__ double recip(double x) { return 1.0 / x; }
// single precision: the correctly rounded hardware reciprocal (the FP32
// adjoint is not matched bit for bit to anything)
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }

// a(x, y), da(x, y) of KarmaRappelFlux::face and their partial derivatives
// in x, y and eps4; x and y are the face's (derx, dery).
template <class T>
struct FaceDer {
    T a, da, ax, ay, dax, day, ae, dae;
};

template <class T>
__device__ __forceinline__ FaceDer<T> face_der(T x, T y, T a_bar, T ae, T a12, T tol) {
    FaceDer<T> f;
    const T x2 = x * x, y2 = y * y;
    const T s = x2 + y2;
    const T mag2 = s * s;
    if (mag2 <= tol) {
        f.a = a_bar;
        f.da = T(0);
        f.ax = f.ay = f.dax = f.day = T(0);
        f.ae = T(-3);  // a = 1 - 3 eps4
        f.dae = T(0);
        return f;
    }
    const T is = recip(s);
    const T is2 = is * is, is3 = is2 * is;
    const T R = (x2 * x2 + y2 * y2) * is2;
    f.a = a_bar + ae * R;  // a_bar (1 + eps' R)
    const T Rx = T(4) * x * y2 * (x2 - y2) * is3;
    const T Ry = T(4) * y * x2 * (y2 - x2) * is3;
    f.ax = ae * Rx;
    f.ay = ae * Ry;
    const T G = x * y * (x2 - y2);
    f.da = -a12 * G * is2;
    const T Gx = y * (T(3) * x2 - y2), Gy = x * (x2 - T(3) * y2);
    f.dax = -a12 * (Gx * is2 - T(4) * x * G * is3);
    f.day = -a12 * (Gy * is2 - T(4) * y * G * is3);
    f.ae = T(-3) + T(3) * R;   // a = (1 - 3 eps4) + 3 eps4 R
    f.dae = T(-12) * G * is2;  // a12 = 12 eps4
    return f;
}

// A_c(hx, hy) of ModelC::center_anisotropy and dA/dhx, dA/dhy, dA/deps4
template <class T>
struct CentreDer {
    T a, ax, ay, ae;
};

template <class T>
__device__ __forceinline__ CentreDer<T> centre_der(T x, T y, T a_bar, T ae, T tol) {
    CentreDer<T> c;
    const T x2 = x * x, y2 = y * y;
    const T s = x2 + y2;
    if (s * s <= tol) {
        c.a = a_bar;
        c.ax = c.ay = T(0);
        c.ae = T(-3);
        return c;
    }
    const T is = recip(s);
    const T is2 = is * is, is3 = is2 * is;
    const T R = (x2 * x2 + y2 * y2) * is2;
    const T k = T(4) * (x2 - y2) * is3 * ae;
    c.a = a_bar + ae * R;
    c.ax = k * x * y2;
    c.ay = -k * y * x2;
    c.ae = T(-3) + T(3) * R;
    return c;
}

template <class T, int TH>
struct Smem {
    static constexpr int W2 = TW + 4, H2 = TH + 4, N = W2 * H2;
    T ph[N], u[N];   // forward state x_n
    T pb[N], ub[N];  // cotangents of x_{n+1}, then the gathered cotangents
    T nb[N], ax[N], ay[N], nu[N];
    T xj[N], xn[N], xt[N], xe[N];  // x faces: J, dJ/ddn (then Jbar dJ/ddn), dJ/ddt (then Jbar ...), dJ/deps
    T yj[N], yn[N], yt[N], ye[N];
    unsigned char out[N];  // bit 0: outside the instance in x, bit 1: in y
    int64_t col[W2];       // offset terms of a window column / row (see stage)
    int64_t row[H2];
    unsigned char cout_[W2], rout[H2];
    double red[3][32];
};

__device__ __forceinline__ int reflect_clamp(int c, int n) {
    c = c < 0 ? -1 - c : (c >= n ? 2 * n - 1 - c : c);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// the column (x) and row (y) terms of cell_offset: offset = inst * bpi * 2 *
// slab_stride + col_term(X) + row_term(Y)
__device__ __forceinline__ int64_t col_term(const Geo& g, int X) {
    X = reflect_clamp(X, g.N0);
    const int bx = X / g.n0;
    return (int64_t)bx * 2 * g.slab_stride + (X - bx * g.n0 + 1);
}
__device__ __forceinline__ int64_t row_term(const Geo& g, int Y) {
    Y = reflect_clamp(Y, g.N1);
    const int by = Y / g.n1;
    return (int64_t)by * g.nb0 * 2 * g.slab_stride + (int64_t)(Y - by * g.n1 + 1) * (g.n0 + 2);
}

// slab offset of field 0 of instance-global cell (X, Y), mirrored into the
// instance when outside it
__device__ __forceinline__ int64_t cell_offset(const Geo& g, int inst, int X, int Y) {
    X = reflect_clamp(X, g.N0);
    Y = reflect_clamp(Y, g.N1);
    const int bx = X / g.n0, by = Y / g.n1;
    const int x = X - bx * g.n0, y = Y - by * g.n1;
    const int64_t b = (int64_t)inst * g.bpi + bx + by * g.nb0;
    return b * 2 * g.slab_stride + (x + 1) + (int64_t)(y + 1) * (g.n0 + 2);
}

__device__ __forceinline__ void block_sum3(double a, double b, double c, double (*red)[32], double* out3) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        red[0][w] = a;
        red[1][w] = b;
        red[2][w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            s0 += red[0][k];
            s1 += red[1][k];
            s2 += red[2][k];
        }
        out3[0] += s0;
        out3[1] += s1;
        out3[2] += s2;
    }
    __syncthreads();
}

template <class T, int TH>
__global__ void __launch_bounds__(256) adjoint_step_kernel(const T* __restrict__ x, const T* __restrict__ lam_in,
                                                           T* __restrict__ lam_out, const AdjParams<T>* __restrict__ prm,
                                                           Geo g, T dt, double* __restrict__ acc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<T, TH>& S = *reinterpret_cast<Smem<T, TH>*>(smem_raw);
    constexpr int W2 = Smem<T, TH>::W2, H2 = Smem<T, TH>::H2, N = Smem<T, TH>::N;
    const int tiles = g.tiles_x * g.tiles_y;
    for (int64_t item = blockIdx.x; item < (int64_t)g.ninst * tiles; item += gridDim.x) {
        const int inst = (int)(item / tiles);
        const int tile = (int)(item - (int64_t)inst * tiles);
        const int X0 = (tile % g.tiles_x) * TW, Y0 = (tile / g.tiles_x) * TH;
        const int w = min(TW, g.N0 - X0), h = min(TH, g.N1 - Y0);
        const AdjParams<T> m = prm[inst];
        auto is_tile = [&](int cx, int cy) { return cx >= 2 && cx < 2 + w && cy >= 2 && cy < 2 + h; };
        auto region1 = [&](int cx, int cy) { return cx >= 1 && cx < W2 - 1 && cy >= 1 && cy < H2 - 1; };

        // A. stage x_n on the window, the incoming cotangents on region 1;
        // the window's column and row offset terms are computed once
        const int64_t base = (int64_t)inst * g.bpi * 2 * g.slab_stride;
        if (threadIdx.x < W2) {
            const int X = X0 - 2 + (int)threadIdx.x;
            S.col[threadIdx.x] = col_term(g, X);
            S.cout_[threadIdx.x] = (X < 0 || X >= g.N0) ? 1 : 0;
        } else if (threadIdx.x < W2 + H2) {
            const int r = threadIdx.x - W2, Y = Y0 - 2 + r;
            S.row[r] = row_term(g, Y);
            S.rout[r] = (Y < 0 || Y >= g.N1) ? 2 : 0;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const int cx = k % W2, cy = k / W2;
            const int fl = S.cout_[cx] | S.rout[cy];
            S.out[k] = (unsigned char)fl;
            const int64_t o = base + S.col[cx] + S.row[cy];
            S.ph[k] = x[o];
            S.u[k] = x[o + g.slab_stride];
            const bool in = fl == 0 && region1(cx, cy);
            S.pb[k] = in ? lam_in[o] : T(0);
            S.ub[k] = in ? lam_in[o + g.slab_stride] : T(0);
            S.nb[k] = S.ax[k] = S.ay[k] = S.nu[k] = T(0);
        }
        __syncthreads();

        // B. face fluxes and their derivatives: x faces (fx, fy) between
        // window columns fx and fx + 1 (rows 1 .. H2-2), y faces (fx, fy)
        // between rows fy and fy + 1 (columns 1 .. W2-2)
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const int cx = k % W2, cy = k / W2;
            if (cx < W2 - 1 && cy >= 1 && cy < H2 - 1) {
                const T* p = S.ph + k;
                const T dn = p[1] - p[0];
                const T dtr = T(0.25) * ((p[1 + W2] - p[1 - W2]) + p[W2] - p[-W2]);
                const FaceDer<T> f = face_der(dn, dtr, m.f_a_bar, m.f_ae, m.f_a12, m.f_tol);
                S.xj[k] = f.a * (f.a * dn - f.da * dtr);
                S.xn[k] = T(2) * f.a * f.ax * dn + f.a * f.a - (f.ax * f.da + f.a * f.dax) * dtr;
                S.xt[k] = T(2) * f.a * f.ay * dn - (f.ay * f.da + f.a * f.day) * dtr - f.a * f.da;
                S.xe[k] = (T(2) * f.a * dn - f.da * dtr) * f.ae - f.a * dtr * f.dae;
            } else {
                S.xj[k] = S.xn[k] = S.xt[k] = S.xe[k] = T(0);
            }
            if (cy < H2 - 1 && cx >= 1 && cx < W2 - 1) {
                const T* p = S.ph + k;
                const T dn = p[W2] - p[0];
                const T dtr = T(0.25) * ((p[1 + W2] - p[-1 + W2]) + p[1] - p[-1]);
                // KarmaRappelFlux::face(derx = dtr, dery = dn)
                const FaceDer<T> f = face_der(dtr, dn, m.f_a_bar, m.f_ae, m.f_a12, m.f_tol);
                S.yj[k] = f.a * (f.a * dn + f.da * dtr);
                S.yn[k] = T(2) * f.a * f.ay * dn + f.a * f.a + (f.ay * f.da + f.a * f.day) * dtr;
                S.yt[k] = T(2) * f.a * f.ax * dn + (f.ax * f.da + f.a * f.dax) * dtr + f.a * f.da;
                S.ye[k] = (T(2) * f.a * dn + f.da * dtr) * f.ae + f.a * dtr * f.dae;
            } else {
                S.yj[k] = S.yn[k] = S.yt[k] = S.ye[k] = T(0);
            }
        }
        __syncthreads();

        // C. cells of region 1 inside the instance: the cotangent weights
        double acc_l = 0.0, acc_d = 0.0, acc_e = 0.0;
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const int cx = k % W2, cy = k / W2;
            if (!region1(cx, cy) || S.out[k]) continue;
            const T ph = S.ph[k], uc = S.u[k];
            const T flux = ((S.xj[k] - S.xj[k - 1]) + (S.yj[k] - S.yj[k - W2])) * m.inv_h2_flux;
            const T omp = T(1) - ph * ph;
            const T pp = omp * omp;
            const T gp = ph * ph * ph - ph;
            const T Nn = -m.lambda * uc * pp + (flux - gp);
            const T cdx = S.ph[k + 1] - S.ph[k - 1], cdy = S.ph[k + W2] - S.ph[k - W2];
            const CentreDer<T> c = centre_der(T(0.5) * cdx, T(0.5) * cdy, m.c_a_bar, m.c_ae, m.c_tol);
            const T A = c.a;
            const T ia = recip(A);
            const T iq = ia * ia;
            const T kphi = Nn * iq;
            const T mu = dt * (S.pb[k] + T(0.5) * S.ub[k]);
            const T nbar = mu * iq;
            const T abar = T(-2) * mu * kphi * ia;
            S.nb[k] = nbar;
            S.ax[k] = abar * T(0.5) * c.ax;
            S.ay[k] = abar * T(0.5) * c.ay;
            S.nu[k] = dt * m.d_thermal * S.ub[k];
            if (is_tile(cx, cy)) {
                const T lap = ((S.u[k + 1] - T(2) * uc) + S.u[k - 1]) * m.ih0 +
                              ((S.u[k + W2] - T(2) * uc) + S.u[k - W2]) * m.ih1;
                acc_l += (double)(nbar * (-uc * pp));
                acc_d += (double)(dt * S.ub[k] * lap);
                acc_e += (double)(abar * c.ae);
            }
        }
        __syncthreads();

        // D. face cotangents Jbar; owned faces add their eps4 term
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const int cx = k % W2, cy = k / W2;
            if (cx < W2 - 1 && cy >= 1 && cy < H2 - 1) {
                const T jb = (S.nb[k] - S.nb[k + 1]) * m.inv_h2_flux;
                if (is_tile(cx + 1, cy) || (is_tile(cx, cy) && (S.out[k + 1] & 1))) acc_e += (double)(jb * S.xe[k]);
                S.xn[k] *= jb;
                S.xt[k] *= jb;
            }
            if (cy < H2 - 1 && cx >= 1 && cx < W2 - 1) {
                const T jb = (S.nb[k] - S.nb[k + W2]) * m.inv_h2_flux;
                if (is_tile(cx, cy + 1) || (is_tile(cx, cy) && (S.out[k + W2] & 2))) acc_e += (double)(jb * S.ye[k]);
                S.yn[k] *= jb;
                S.yt[k] *= jb;
            }
        }
        __syncthreads();

        // E. gather the cotangent of every region-1 position (interior cells
        // and the ghost positions that fold into them)
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const int cx = k % W2, cy = k / W2;
            if (!region1(cx, cy)) continue;
            const bool in = S.out[k] == 0;
            T pbar = T(0), ubar = T(0);
            if (in) {
                const T ph = S.ph[k], uc = S.u[k];
                const T omp = T(1) - ph * ph;
                const T dndphi = T(4) * m.lambda * uc * ph * omp + (T(1) - T(3) * ph * ph);
                pbar = S.pb[k] + S.nb[k] * dndphi;
                ubar = S.ub[k] - S.nb[k] * m.lambda * omp * omp - T(2) * (m.ih0 + m.ih1) * S.nu[k];
            }
            // x faces: normal difference, then the transverse quarter sums
            pbar += S.xn[k - 1] - S.xn[k];
            pbar += T(0.25) * ((S.xt[k - W2] - S.xt[k + W2]) + (S.xt[k - 1 - W2] - S.xt[k - 1 + W2]));
            // y faces
            pbar += S.yn[k - W2] - S.yn[k];
            pbar += T(0.25) * ((S.yt[k - 1] - S.yt[k + 1]) + (S.yt[k - 1 - W2] - S.yt[k + 1 - W2]));
            // centre anisotropy of the four neighbours
            pbar += (S.ax[k - 1] - S.ax[k + 1]) + (S.ay[k - W2] - S.ay[k + W2]);
            // Laplacian of u
            ubar += (S.nu[k - 1] + S.nu[k + 1]) * m.ih0 + (S.nu[k - W2] + S.nu[k + W2]) * m.ih1;
            S.pb[k] = pbar;
            S.ub[k] = ubar;
        }
        __syncthreads();

        // F. fold the ghost positions into their source cells (tiles on an
        // instance edge only) and store
        const bool edge = X0 == 0 || Y0 == 0 || X0 + w == g.N0 || Y0 + h == g.N1;
        for (int k = threadIdx.x; k < TW * TH; k += blockDim.x) {
            const int tx = k % TW, ty = k / TW;
            if (tx >= w || ty >= h) continue;
            const int cx = tx + 2, cy = ty + 2, q0 = cx + cy * W2;
            T pbar = S.pb[q0], ubar = S.ub[q0];
            if (edge) {
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0) continue;
                        const int q = q0 + dx + dy * W2;
                        if ((dx == 0 || (S.out[q] & 1)) && (dy == 0 || (S.out[q] & 2))) {
                            pbar += S.pb[q];
                            ubar += S.ub[q];
                        }
                    }
            }
            const int64_t o = base + S.col[cx] + S.row[cy];
            lam_out[o] = pbar;
            lam_out[o + g.slab_stride] = ubar;
        }
        block_sum3(acc_l, acc_d, acc_e, S.red, acc + 3 * item);
    }
}

// Seeds the backward sweep from L = sum (phi_T - target)^2 per instance:
// phi^ = 2 (phi_T - target), u^ = 0 on the interiors; the tile's share of
// the loss goes to loss[item].
template <class T>
__global__ void __launch_bounds__(256) loss_seed_kernel(const T* __restrict__ x, const double* __restrict__ target,
                                                        T* __restrict__ lam, Geo g, double* __restrict__ loss) {
    __shared__ double red[32];
    const int tiles = g.tiles_x * g.tiles_y;
    constexpr int TH = 8;
    for (int64_t item = blockIdx.x; item < (int64_t)g.ninst * tiles; item += gridDim.x) {
        const int inst = (int)(item / tiles);
        const int tile = (int)(item - (int64_t)inst * tiles);
        const int X0 = (tile % g.tiles_x) * TW, Y0 = (tile / g.tiles_x) * TH;
        double part = 0.0;
        for (int k = threadIdx.x; k < TW * TH; k += blockDim.x) {
            const int X = X0 + k % TW, Y = Y0 + k / TW;
            if (X >= g.N0 || Y >= g.N1) continue;
            const int64_t o = cell_offset(g, inst, X, Y);
            const double d = (double)x[o] - target[((int64_t)inst * g.N1 + Y) * g.N0 + X];
            part += d * d;
            lam[o] = (T)(2.0 * d);
            lam[o + g.slab_stride] = T(0);
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
            loss[item] = s;
        }
        __syncthreads();
    }
}

template <class T, int TH>
cudaError_t launch_adjoint(const T* x, const T* lam_in, T* lam_out, const void* prm, Geo g, double dt, double* acc,
                           cudaStream_t s) {
    g.tiles_x = (g.N0 + TW - 1) / TW;
    g.tiles_y = (g.N1 + TH - 1) / TH;
    const size_t smem = sizeof(Smem<T, TH>);
    auto kernel = adjoint_step_kernel<T, TH>;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int64_t items = (int64_t)g.ninst * g.tiles_x * g.tiles_y;
    const unsigned grid = (unsigned)std::min<int64_t>(items, (int64_t)148 * 32);
    kernel<<<grid, 256, smem, s>>>(x, lam_in, lam_out, static_cast<const AdjParams<T>*>(prm), g, (T)dt, acc);
    return cudaGetLastError();
}

}  // namespace

int adjoint_tile_rows(int dtype) { return dtype == 0 ? 8 : 16; }

cudaError_t launch_adjoint_step(int dtype, const void* x, const void* lam_in, void* lam_out, const void* prm,
                                const Geo& g, double dt, double* acc, cudaStream_t s) {
    if (dtype == 0)
        return launch_adjoint<double, 8>((const double*)x, (const double*)lam_in, (double*)lam_out, prm, g, dt, acc,
                                         s);
    return launch_adjoint<float, 16>((const float*)x, (const float*)lam_in, (float*)lam_out, prm, g, dt, acc, s);
}

cudaError_t launch_loss_seed(int dtype, const void* x, const double* target, void* lam, Geo g, double* loss,
                             cudaStream_t s) {
    g.tiles_x = (g.N0 + TW - 1) / TW;
    g.tiles_y = (g.N1 + 8 - 1) / 8;
    const int64_t items = (int64_t)g.ninst * g.tiles_x * g.tiles_y;
    const unsigned grid = (unsigned)std::min<int64_t>(items, (int64_t)148 * 32);
    if (dtype == 0)
        loss_seed_kernel<double><<<grid, 256, 0, s>>>((const double*)x, target, (double*)lam, g, loss);
    else
        loss_seed_kernel<float><<<grid, 256, 0, s>>>((const float*)x, target, (float*)lam, g, loss);
    return cudaGetLastError();
}

int64_t loss_items(const Geo& g) { return (int64_t)g.ninst * ((g.N0 + TW - 1) / TW) * ((g.N1 + 7) / 8); }

int64_t adjoint_items(int dtype, const Geo& g) {
    const int th = adjoint_tile_rows(dtype);
    return (int64_t)g.ninst * ((g.N0 + TW - 1) / TW) * ((g.N1 + th - 1) / th);
}

size_t adj_params_size(int dtype) { return dtype == 0 ? sizeof(AdjParams<double>) : sizeof(AdjParams<float>); }

void adj_params(int dtype, const ModelCDev& m, void* out) {
    auto fill = [&](auto* p) {
        using T = std::remove_reference_t<decltype(p->lambda)>;
        p->lambda = (T)m.lambda;
        p->d_thermal = (T)m.d_thermal;
        p->inv_h2_flux = (T)m.inv_h2_flux;
        p->ih0 = (T)m.inv_h2[0];
        p->ih1 = (T)m.inv_h2[1];
        p->f_a_bar = (T)m.f_a_bar;
        p->f_ae = (T)(m.f_a_bar * m.f_eps_prime);
        p->f_a12 = (T)m.f_a12;
        p->f_tol = (T)m.f_tol;
        p->c_a_bar = (T)m.a_bar;
        p->c_ae = (T)(m.a_bar * m.eps_prime);
        p->c_tol = (T)m.tol;
    };
    if (dtype == 0)
        fill(static_cast<AdjParams<double>*>(out));
    else
        fill(static_cast<AdjParams<float>*>(out));
}

}  // namespace adj
}  // namespace lg
