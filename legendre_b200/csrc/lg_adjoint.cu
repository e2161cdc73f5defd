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
// single precision: the hardware's approximate reciprocal (PTX rcp.approx,
// within one ulp; the FP32 adjoint is not matched bit for bit to anything)
__device__ __forceinline__ float recip(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <class T>
__device__ __forceinline__ T fma_(T a, T b, T c) { return fma(a, b, c); }

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
    const T is2 = is * is;
    const T d = x2 - y2;
    const T R = (x2 * x2 + y2 * y2) * is2;
    f.a = a_bar + ae * R;  // a_bar (1 + eps' R)
    // Rx = 4 x y^2 d / s^3, Ry = -4 y x^2 d / s^3: one shared factor
    const T k = ae * (T(4) * d) * (is2 * is);
    f.ax = k * (x * y2);
    f.ay = -k * (y * x2);
    const T G = x * y * d, Gs = G * is2;  // G / s^2
    f.da = -a12 * Gs;
    // dax = -a12 (Gx - 4 x G / s) / s^2, day likewise
    const T m4 = T(-4) * G * is, na = -a12 * is2;
    f.dax = na * fma_(m4, x, y * (T(3) * x2 - y2));
    f.day = na * fma_(m4, y, x * (x2 - T(3) * y2));
    f.ae = T(-3) + T(3) * R;  // a = (1 - 3 eps4) + 3 eps4 R
    f.dae = T(-12) * Gs;      // a12 = 12 eps4
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

// ------------------------------------------------------------ strip form --
// The same step adjoint with one warp per work unit and no shared memory:
// the warp owns 32 adjacent columns of one instance (lane l at column
// X = 29 s - 1 + l) and walks up a run of rows.  Lanes 1..29 produce the
// cotangents of their columns; lanes 0, 30 and 31 are the halo the
// derivation needs (the cell-centred N^ and A^ of the neighbours of an
// output cell, and the faces between them), so every face derivative is
// evaluated once per lane and row and reaches the neighbouring lanes by
// shuffles.
//
// Step r of the walk "completes" row r -- the x face left of each lane's
// cell, the y face above it, the cell's N^, A^ and nu, and the face
// cotangents that those make final -- and then gathers the cotangent of row
// r - 1, whose stencil (rows r-2 .. r) is complete.  A unit that starts at
// the instance's first row also gathers the ghost row below it, and one that
// ends at the last row the ghost row above it; both fold into the adjacent
// interior row, as the ghost columns X = -1 and X = N0 fold into columns 0
// and N0 - 1 across lanes.  Quantities of cells outside the instance are
// zero (selected, so that no value of a halo lane leaks in).
//
// A lane sums its share of the unit's parameter partials in the adjoint's
// arithmetic type and the warp adds the lanes in FP64 into the unit's slot,
// so the sums do not depend on which warp ran the unit.  Units past the
// grid's first wave come from a work list (see launch_adjoint_strip).
constexpr int SW = 29;  // output columns per strip

// Slab-offset row terms of consecutive rows: the division by the block
// height happens only when the walk crosses a block edge or the instance
// edge (where rows are mirrored).
struct RowWalk {
    int Y, yl;
    int64_t term;
    __device__ void init(const Geo& g, int y) {
        Y = y;
        term = row_term(g, y);
        const int yc = reflect_clamp(y, g.N1);
        yl = yc - (yc / g.n1) * g.n1;
    }
    __device__ void next(const Geo& g) {
        ++Y;
        ++yl;
        if (Y <= 0 || Y >= g.N1 || yl == g.n1)
            init(g, Y);
        else
            term += g.n0 + 2;
    }
};

template <class T>
__device__ __forceinline__ T shfl_up1(T v) {
    return __shfl_up_sync(0xffffffffu, v, 1);
}
template <class T>
__device__ __forceinline__ T shfl_dn1(T v) {
    return __shfl_down_sync(0xffffffffu, v, 1);
}

template <class T>
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class T>
__global__ void __launch_bounds__(256) adjoint_strip_kernel(const T* __restrict__ x, const T* __restrict__ lam_in,
                                                            T* __restrict__ lam_out,
                                                            const AdjParams<T>* __restrict__ prm, Geo g, T dt,
                                                            double* __restrict__ acc, int rows, int strips,
                                                            int chunks, unsigned long long* __restrict__ work,
                                                            unsigned long long work_base) {
    const int lane = threadIdx.x & 31;
    const int64_t units = g.ninst * strips * chunks;
    const int64_t first_listed = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t unit = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; unit < units;) {
        const int s = (int)(unit % strips);
        const int k = (int)((unit / strips) % chunks);
        const int64_t inst = unit / ((int64_t)strips * chunks);
        const AdjParams<T> m = prm[inst];
        const int X = s * SW - 1 + lane;
        const bool xin = X >= 0 && X < g.N0;
        const bool xo = xin && lane >= 1 && lane <= SW;  // this lane's column is an output of the unit
        const int Y0 = k * rows, Y1 = min(g.N1, Y0 + rows);
        const int gs = Y0 == 0 ? -1 : Y0;         // first gathered row (the ghost row below the instance)
        const int ge = Y1 == g.N1 ? g.N1 : Y1 - 1;  // last gathered row (the ghost row above)
        const int64_t base = inst * g.bpi * 2 * g.slab_stride;
        const int64_t cC = base + col_term(g, X), cL = base + col_term(g, X - 1);
        const int64_t ss = g.slab_stride;

        // window rows r-1 (m), r (0), r+1 (p) at X-1 (a), X (b); X+1 by shuffle
        // loads run one row ahead: step r reads the state of row r + 2 and
        // the incoming cotangents of row r + 1
        T pma, pmb, p0a, p0b, ppa, ppb, um, u0, up;
        RowWalk rw;  // the last state row loaded
        const int cs = gs - 1;
        rw.init(g, cs - 1);
        pma = x[cL + rw.term];
        pmb = x[cC + rw.term];
        um = x[cC + rw.term + ss];
        const int64_t t_m = rw.term;
        rw.next(g);
        p0a = x[cL + rw.term];
        p0b = x[cC + rw.term];
        u0 = x[cC + rw.term + ss];
        const int64_t t_0 = rw.term;
        rw.next(g);
        T nxa = x[cL + rw.term], nxb = x[cC + rw.term], nxu = x[cC + rw.term + ss];  // row cs + 1
        T npb = T(0), nub = T(0);  // cotangents of row cs
        if (xin && cs >= 0 && cs < g.N1) {
            npb = lam_in[cC + t_0];
            nub = lam_in[cC + t_0 + ss];
        }
        // y face (cs - 1, cs): its flux value for row cs
        T yJ_prev;
        {
            const T mc = shfl_dn1(pmb), c0 = shfl_dn1(p0b);
            const T dn = p0b - pmb;
            const T dtr = T(0.25) * (((c0 - p0a) + mc) - pma);
            const FaceDer<T> f = face_der(dtr, dn, m.f_a_bar, m.f_ae, m.f_a12, m.f_tol);
            yJ_prev = f.a * (f.a * dn + f.da * dtr);
        }
        T yn_raw_prev = T(0), yt_raw_prev = T(0), ye_raw_prev = T(0);  // y face (r-1, r) before its cotangent
        T nb_prev = T(0), pb_prev = T(0), ub_prev = T(0);                // row r-1
        T xn_prev = T(0), xt_pm = T(0), xt_prev = T(0);  // xn of row r-1; xt of rows r-2, r-1
        T yn_pm = T(0), yt_pm = T(0);                     // y face (r-2, r-1) with its cotangent
        T ax_prev = T(0), ay_pm = T(0), ay_prev = T(0), nu_pm = T(0), nu_prev = T(0);
        T gm_p = T(0), gm_u = T(0), gt_p = T(0), gt_u = T(0);  // ghost-row gathers below / the top row's gather
        // neighbour-lane copies kept for the next rows: xt of the right lane
        // (rows r-2, r-1), yt of the face (r-2, r-1) of both neighbours
        T xtR_pm = T(0), xtR_prev = T(0), ytL_pm = T(0), ytR_pm = T(0);
        // the parameter partials of the unit, per lane, in the adjoint's
        // arithmetic type (one FP64 sum per unit below)
        T acc_l = T(0), acc_d = T(0), acc_e = T(0);
        // row terms of rows r - 1, r and r + 1 (mirrored outside the instance,
        // where no cotangent is loaded or stored)
        int64_t rt_m = t_m, rt_0 = t_0, rt_p = rw.term;

        for (int r = cs; r <= ge + 1; ++r) {
            // ---- complete row r: row r + 1 arrived in the previous step;
            // start the loads of the next one
            ppa = nxa;
            ppb = nxb;
            up = nxu;
            const T pb = npb, ub = nub;
            rw.next(g);
            nxa = x[cL + rw.term];
            nxb = x[cC + rw.term];
            nxu = x[cC + rw.term + ss];
            npb = nub = T(0);
            if (xin && r + 1 >= 0 && r + 1 < g.N1) {
                npb = lam_in[cC + rt_p];
                nub = lam_in[cC + rt_p + ss];
            }
            const bool rin = r >= 0 && r < g.N1;
            const bool cin = rin && xin;
            const bool orow = r >= Y0 && r < Y1;
            const T p0c = shfl_dn1(p0b), ppc = shfl_dn1(ppb);
            // the x face left of X and the y face above X in row r, and the
            // centre anisotropy's derivatives.  Where all three are flat across
            // the warp (the far field) their derivatives are constants: the
            // branch-free body below gives the general path's values.
            const T dnx = p0b - p0a, dtx = T(0.25) * (((ppb - pmb) + ppa) - pma);
            const T dny = ppb - p0b, dty = T(0.25) * (((ppc - ppa) + p0c) - p0a);
            const T chx = T(0.5) * (p0c - p0a), chy = T(0.5) * (ppb - pmb);
            T xJ, xn_raw, xt_raw, xe_raw, yJ, yn_raw, yt_raw, ye_raw;
            CentreDer<T> c;
            {
                auto mag2 = [](T a, T b) {
                    const T sq = a * a + b * b;
                    return sq * sq;
                };
                const bool flat = mag2(dnx, dtx) <= m.f_tol && mag2(dty, dny) <= m.f_tol && mag2(chx, chy) <= m.c_tol;
                if (__all_sync(0xffffffffu, flat)) {
                    const T a = m.f_a_bar;
                    xJ = a * (a * dnx);
                    xn_raw = a * a;
                    xt_raw = T(0);
                    xe_raw = T(-6) * a * dnx;  // (2 a dn - da dt) ae - a dt dae, da = dae = 0, ae = -3
                    yJ = a * (a * dny);
                    yn_raw = a * a;
                    yt_raw = T(0);
                    ye_raw = T(-6) * a * dny;
                    c.a = m.c_a_bar;
                    c.ax = c.ay = T(0);
                    c.ae = T(-3);
                } else {
                    {
                        const FaceDer<T> f = face_der(dnx, dtx, m.f_a_bar, m.f_ae, m.f_a12, m.f_tol);
                        xJ = f.a * (f.a * dnx - f.da * dtx);
                        xn_raw = T(2) * f.a * f.ax * dnx + f.a * f.a - (f.ax * f.da + f.a * f.dax) * dtx;
                        xt_raw = T(2) * f.a * f.ay * dnx - (f.ay * f.da + f.a * f.day) * dtx - f.a * f.da;
                        xe_raw = (T(2) * f.a * dnx - f.da * dtx) * f.ae - f.a * dtx * f.dae;
                    }
                    {
                        const FaceDer<T> f = face_der(dty, dny, m.f_a_bar, m.f_ae, m.f_a12, m.f_tol);
                        yJ = f.a * (f.a * dny + f.da * dty);
                        yn_raw = T(2) * f.a * f.ay * dny + f.a * f.a + (f.ay * f.da + f.a * f.day) * dty;
                        yt_raw = T(2) * f.a * f.ax * dny + (f.ax * f.da + f.a * f.dax) * dty + f.a * f.da;
                        ye_raw = (T(2) * f.a * dny + f.da * dty) * f.ae + f.a * dty * f.dae;
                    }
                    c = centre_der(chx, chy, m.c_a_bar, m.c_ae, m.c_tol);
                }
            }
            // cell (X, r): N^, A^ and nu
            const T xJr = shfl_dn1(xJ);
            T nb, ax, ay, nu;
            {
                const T ph = p0b, uc = u0;
                const T flux = ((xJr - xJ) + (yJ - yJ_prev)) * m.inv_h2_flux;
                const T omp = T(1) - ph * ph;
                const T pp = omp * omp;
                const T gp = ph * ph * ph - ph;
                const T Nn = -m.lambda * uc * pp + (flux - gp);
                const T ia = recip(c.a);
                const T iq = ia * ia;
                const T kphi = Nn * iq;
                const T mu = dt * (pb + T(0.5) * ub);
                const T nbar = mu * iq;
                const T abar = T(-2) * mu * kphi * ia;
                nb = cin ? nbar : T(0);
                ax = cin ? abar * T(0.5) * c.ax : T(0);
                ay = cin ? abar * T(0.5) * c.ay : T(0);
                nu = cin ? dt * m.d_thermal * ub : T(0);
                const T uL = shfl_up1(u0), uR = shfl_dn1(u0);
                if (xo && orow) {
                    const T lap = ((uR - T(2) * uc) + uL) * m.ih0 + ((up - T(2) * uc) + um) * m.ih1;
                    acc_l += nbar * (-uc * pp);
                    acc_d += dt * ub * lap;
                    acc_e += abar * c.ae;
                }
            }
            // cotangent of the x face left of X (cells X-1 and X of row r)
            T nbl = shfl_up1(nb);
            if (lane == 0) nbl = T(0);  // lane 0 is a halo lane; its left face matters only outside the instance
            const T jbx = (nbl - nb) * m.inv_h2_flux;
            const T xn = xn_raw * jbx, xt = xt_raw * jbx;
            // the face is counted by the cell on its right, or by the last cell for the face into the ghost column
            if (orow && ((xo) || (X == g.N0 && lane >= 2 && lane <= SW + 1))) acc_e += jbx * xe_raw;
            // cotangent of the y face (r-1, r)
            const T jby = (nb_prev - nb) * m.inv_h2_flux;
            const T yn_f = yn_raw_prev * jby, yt_f = yt_raw_prev * jby;
            if (xo && (orow || (r == g.N1 && r - 1 >= Y0 && r - 1 < Y1))) acc_e += jby * ye_raw_prev;

            // neighbour copies of this row's face terms (used now and by the next two gathers)
            const T xtR = shfl_dn1(xt);
            T ytL = shfl_up1(yt_f);
            const T ytR = shfl_dn1(yt_f);
            if (lane == 0) ytL = T(0);  // column X-2: outside whenever lane 0 is gathered

            // ---- gather row q = r - 1 (its stencil rows q-1 .. q+1 are complete)
            const int q = r - 1;
            if (q >= gs) {
                const bool qin = q >= 0 && q < g.N1;
                T pbar = T(0), ubar = T(0);
                if (qin && xin) {
                    const T ph = pmb, uc = um;
                    const T omp = T(1) - ph * ph;
                    const T dndphi = T(4) * m.lambda * uc * ph * omp + (T(1) - T(3) * ph * ph);
                    pbar = pb_prev + nb_prev * dndphi;
                    ubar = ub_prev - nb_prev * m.lambda * omp * omp - T(2) * (m.ih0 + m.ih1) * nu_prev;
                }
                const T xnR = shfl_dn1(xn_prev);
                pbar += xn_prev - xnR;
                pbar += T(0.25) * ((xtR_pm - xtR) + (xt_pm - xt));
                pbar += yn_pm - yn_f;
                T axL = shfl_up1(ax_prev), nuL = shfl_up1(nu_prev);
                if (lane == 0) axL = nuL = T(0);
                const T axR = shfl_dn1(ax_prev), nuR = shfl_dn1(nu_prev);
                const T ytL_m = ytL_pm, ytR_m = ytR_pm;
                pbar += T(0.25) * ((ytL - ytR) + (ytL_m - ytR_m));
                pbar += (axL - axR) + (ay_pm - ay);
                ubar += (nuL + nuR) * m.ih0 + (nu_pm + nu) * m.ih1;
                // fold the ghost columns into columns 0 and N0 - 1
                const T gpl = shfl_up1(pbar), gul = shfl_up1(ubar), gpr = shfl_dn1(pbar), gur = shfl_dn1(ubar);
                if (X == 0 && lane >= 1) {
                    pbar += gpl;
                    ubar += gul;
                }
                if (X == g.N0 - 1 && lane <= 30) {
                    pbar += gpr;
                    ubar += gur;
                }
                // fold the ghost rows; store row q, or the top row once its ghost row is in
                if (q == -1) {
                    gm_p = pbar;
                    gm_u = ubar;
                } else if (q == g.N1) {
                    if (xo) {
                        const int64_t o = cC + row_term(g, g.N1 - 1);
                        lam_out[o] = gt_p + pbar;
                        lam_out[o + ss] = gt_u + ubar;
                    }
                } else {
                    if (q == 0 && gs == -1) {
                        pbar += gm_p;
                        ubar += gm_u;
                    }
                    if (q == g.N1 - 1) {
                        gt_p = pbar;
                        gt_u = ubar;
                    } else if (xo) {
                        lam_out[cC + rt_m] = pbar;
                        lam_out[cC + rt_m + ss] = ubar;
                    }
                }
            }

            // ---- shift the window
            rt_m = rt_0;
            rt_0 = rt_p;
            rt_p = rw.term;
            pma = p0a;
            pmb = p0b;
            p0a = ppa;
            p0b = ppb;
            um = u0;
            u0 = up;
            yJ_prev = yJ;
            yn_raw_prev = yn_raw;
            yt_raw_prev = yt_raw;
            ye_raw_prev = ye_raw;
            nb_prev = nb;
            pb_prev = pb;
            ub_prev = ub;
            xn_prev = xn;
            xt_pm = xt_prev;
            xt_prev = xt;
            xtR_pm = xtR_prev;
            xtR_prev = xtR;
            ytL_pm = ytL;
            ytR_pm = ytR;
            yn_pm = yn_f;
            yt_pm = yt_f;
            ax_prev = ax;
            ay_pm = ay_prev;
            ay_prev = ay;
            nu_pm = nu_prev;
            nu_prev = nu;
        }
        const double sl = warp_sum<T>((double)acc_l), sd = warp_sum<T>((double)acc_d),
                     se = warp_sum<T>((double)acc_e);
        if (lane == 0) {
            acc[3 * unit + 0] += sl;
            acc[3 * unit + 1] += sd;
            acc[3 * unit + 2] += se;
        }
        // the next unit: from the work list (units past the grid's first
        // wave, in order, to whichever warp is free), or the grid stride
        if (work) {
            unsigned long long n = 0;
            if (lane == 0) n = atomicAdd(work, 1ull) - work_base;
            n = __shfl_sync(0xffffffffu, n, 0);
            unit = n < (unsigned long long)units ? first_listed + (int64_t)n : units;  // no wrapped value runs
        } else {
            unit += first_listed;
        }
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
    const unsigned grid = (unsigned)std::min<int64_t>(items, (int64_t)lg::device_sm_count() * 32);
    kernel<<<grid, 256, smem, s>>>(x, lam_in, lam_out, static_cast<const AdjParams<T>*>(prm), g, (T)dt, acc);
    return cudaGetLastError();
}


// With a work list the grid is one wave of resident CTAs and each warp
// takes its next unit from the counter when it finishes one, so the strips
// that cross an interface (the general derivative path) and the flat ones
// (the far-field body, about a quarter of the instructions fewer) share the
// SMs evenly; without one every warp runs one unit and a CTA holds its SM
// slot until its slowest warp is done.
template <class T>
cudaError_t launch_adjoint_strip(const T* x, const T* lam_in, T* lam_out, const void* prm, const Geo& g, double dt,
                                 double* acc, unsigned long long* work, unsigned long long base, cudaStream_t s) {
    const int strips = adjoint_strips(g), rows = adjoint_strip_rows(g);
    const int chunks = (g.N1 + rows - 1) / rows;
    const int64_t units = g.ninst * strips * chunks;
    int64_t grid = std::min<int64_t>((units + 7) / 8, (int64_t)1 << 30);
    if (work) {
        static const int per_sm = [] {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjoint_strip_kernel<T>, 256, 0) != cudaSuccess)
                n = 1;
            return std::max(n, 1);
        }();
        grid = std::min<int64_t>(grid, (int64_t)lg::device_sm_count() * per_sm);
    }
    adjoint_strip_kernel<T><<<(unsigned)grid, 256, 0, s>>>(x, lam_in, lam_out, static_cast<const AdjParams<T>*>(prm),
                                                           g, (T)dt, acc, rows, strips, chunks, work, base);
    return cudaGetLastError();
}

}  // namespace

int adjoint_tile_rows(int dtype) { return dtype == 0 ? 8 : 16; }

int adjoint_strips(const Geo& g) { return (g.N0 + SW - 1) / SW; }

// rows per strip unit: the whole instance height, halved while the launch
// would hold fewer units than 15 warps per SM, most of one wave of 16 (down
// to 16 rows).  Each unit completes two rows beyond the ones it gathers, so
// tall units waste least; the work list evens out the rest (on 256
// instances of 256^2, 9 x 256 = 2304 units of the whole height, 97 % of a
// wave, ran the gradient 0.5 % faster than 128-row units, which ran it
// 1.6 % faster than 64-row ones)
int adjoint_strip_rows(const Geo& g) {
    const int strips = adjoint_strips(g);
    const int64_t wave = (int64_t)lg::device_sm_count() * 15;
    int rows = std::max(1, g.N1);
    while (rows > 16 && g.ninst * strips * ((g.N1 + rows - 1) / rows) < wave) rows = (rows + 1) / 2;
    return rows;
}

cudaError_t launch_adjoint_step(int dtype, int kernel, const void* x, const void* lam_in, void* lam_out,
                                const void* prm, const Geo& g, double dt, double* acc, unsigned long long* work,
                                unsigned long long base, cudaStream_t s) {
    if (kernel == kAdjointStrip) {
        if (dtype == 0)
            return launch_adjoint_strip<double>((const double*)x, (const double*)lam_in, (double*)lam_out, prm, g, dt,
                                                acc, work, base, s);
        return launch_adjoint_strip<float>((const float*)x, (const float*)lam_in, (float*)lam_out, prm, g, dt, acc,
                                           work, base, s);
    }
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
    const unsigned grid = (unsigned)std::min<int64_t>(items, (int64_t)lg::device_sm_count() * 32);
    if (dtype == 0)
        loss_seed_kernel<double><<<grid, 256, 0, s>>>((const double*)x, target, (double*)lam, g, loss);
    else
        loss_seed_kernel<float><<<grid, 256, 0, s>>>((const float*)x, target, (float*)lam, g, loss);
    return cudaGetLastError();
}

int64_t loss_items(const Geo& g) { return (int64_t)g.ninst * ((g.N0 + TW - 1) / TW) * ((g.N1 + 7) / 8); }

int64_t adjoint_items(int dtype, int kernel, const Geo& g) {
    if (kernel == kAdjointStrip) {
        const int rows = adjoint_strip_rows(g);
        return g.ninst * adjoint_strips(g) * ((g.N1 + rows - 1) / rows);
    }
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
