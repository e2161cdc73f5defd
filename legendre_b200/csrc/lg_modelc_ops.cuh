// Model C device arithmetic shared by the step kernels, written in the
// reference's operand order.  Include only from translation units compiled
// with -fmad=false (see lg_kernels.cu).
#pragma once

#include "lg_common.cuh"
#include "lg_kernels.h"

namespace lg {

template <class T>
struct MC {
    T lambda, d_thermal, a_bar, eps_prime, tol, f_a_bar, f_eps_prime, f_a12, f_tol, inv_h2_flux, ih0, ih1;
    T c_far, inv_c_far;  // a_bar * a_bar, the far-field mobility divisor, and RN(1 / c_far)
};

template <class T>
inline MC<T> to_mc(const ModelCDev& m) {
    MC<T> r;
    r.lambda = (T)m.lambda;
    r.d_thermal = (T)m.d_thermal;
    r.a_bar = (T)m.a_bar;
    r.eps_prime = (T)m.eps_prime;
    r.tol = (T)m.tol;
    r.f_a_bar = (T)m.f_a_bar;
    r.f_eps_prime = (T)m.f_eps_prime;
    r.f_a12 = (T)m.f_a12;
    r.f_tol = (T)m.f_tol;
    r.inv_h2_flux = (T)m.inv_h2_flux;
    r.ih0 = (T)m.inv_h2[0];
    r.ih1 = (T)m.inv_h2[1];
    r.c_far = r.a_bar * r.a_bar;
    r.inv_c_far = T(1) / r.c_far;
    return r;
}

// KarmaRappelFlux::face (finite_volume.rs:129-142)
template <class T>
__device__ __forceinline__ void kr_face(const MC<T>& m, T dx, T dy, T& a, T& da) {
    T dx2 = dx * dx;
    T dy2 = dy * dy;
    T sum = dx2 + dy2;
    T mag2 = sum * sum;
    if (mag2 <= m.f_tol) {
        a = m.f_a_bar;
        da = T(0);
    } else {
        a = m.f_a_bar * (T(1) + m.f_eps_prime * (dx2 * dx2 + dy2 * dy2) / mag2);
        da = -(m.f_a12) * dx * dy * (dx2 - dy2) / mag2;
    }
}

// ModelC::center_anisotropy (phasefield.rs:159-175) from the half
// differences dx = 0.5 (p(i+1) - p(i-1)), dy likewise.
template <class T>
__device__ __forceinline__ T center_anisotropy(const MC<T>& m, T dx, T dy) {
    T dx2 = dx * dx;
    T dy2 = dy * dy;
    T sum = dx2 + dy2;
    T mag2 = sum * sum;
    if (mag2 <= m.tol) return m.a_bar;
    return m.a_bar * (T(1) + m.eps_prime * (dx2 * dx2 + dy2 * dy2) / mag2);
}

__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }

__device__ __forceinline__ double normal_t(uint64_t key, double) { return standard_normal(key); }

// x / c_far, the IEEE quotient, for the far-field cells (a = a_bar).  For
// double operands whose quotient neither underflows nor overflows, the
// quotient q = RN(x y) by the correctly rounded reciprocal y = RN(1/c)
// followed by one correction with the exact residual r = x - c q (an fma),
// RN(q + r y), is the correctly rounded x / c (Markstein's theorem; the
// same bits as the division, checked against it on 3.8e9 operands over
// 600 divisors, half of them next to rounding midpoints).  Zeros are x y
// (their sign kept); tiny and huge x take the division.
__device__ __forceinline__ double div_far(double x, double c, double y) {
    const double ax = fabs(x);
    const double q = x * y;
    const double qc = fma(fma(-q, c, x), y, q);
    if (ax >= 0x1p-960 && ax <= 0x1p+960) return qc;
    return x == 0.0 ? q : x / c;  // +-0 / c = +-0 = +-0 y (y > 0)
}
__device__ __forceinline__ float div_far(float x, float c, float) { return x / c; }
__device__ __forceinline__ float normal_t(uint64_t key, float) { return standard_normal_f32(key); }

// The exact FP64 arithmetic policy of the step kernels: face fluxes from
// the normal difference dn and the transverse quarter sum 0.25 ((d1 + c) - e)
// (finite_volume.rs:258-283), the cell update (phasefield.rs:395-421) and
// the Euler-Maruyama axpy (driver.rs:210-236), in the reference's operand
// order.
template <class T>
struct OpsExact {
    using Params = MC<T>;
    static constexpr bool kFarPass = true;  // the paired rows test for the far field first (quarter, *_far)

    // x face: KarmaRappelFlux::face(derx, dery) and j = a (a derx - da dery)
    static __device__ __forceinline__ T xface(const MC<T>& m, T dn, T d1, T c, T e) {
        const T dt = T(0.25) * (d1 + c - e);
        T a, da;
        kr_face(m, dn, dt, a, da);
        return a * (a * dn - da * dt);
    }
    // y face: face(derx, dery) with derx transverse, j = a (a dery + da derx)
    static __device__ __forceinline__ T yface(const MC<T>& m, T dn, T d1, T c, T e) {
        const T dt = T(0.25) * (d1 + c - e);
        T a, da;
        kr_face(m, dt, dn, a, da);
        return a * (a * dn + da * dt);
    }
    // The far-field forms: the face fluxes and the cell update with the
    // anisotropy branches decided (kr_face and center_anisotropy both flat),
    // the same expressions as the branches they stand for, so their bits.
    // `quarter` is the transverse quarter sum of xface / yface and the
    // *_mag2 the |grad|^4 those branches test.
    static __device__ __forceinline__ T quarter(T d1, T c, T e) { return T(0.25) * (d1 + c - e); }
    static __device__ __forceinline__ T face_mag2(T dx, T dy) {
        const T dx2 = dx * dx;
        const T dy2 = dy * dy;
        const T sum = dx2 + dy2;
        return sum * sum;
    }
    static __device__ __forceinline__ T center_mag2(T cdx, T cdy) { return face_mag2(T(0.5) * cdx, T(0.5) * cdy); }
    static __device__ __forceinline__ bool face_flat(const MC<T>& m, T dx, T dy) { return face_mag2(dx, dy) <= m.f_tol; }
    static __device__ __forceinline__ bool center_flat(const MC<T>& m, T cdx, T cdy) {
        return center_mag2(cdx, cdy) <= m.tol;
    }
    static __device__ __forceinline__ T xface_far(const MC<T>& m, T dn, T dt) {
        const T a = m.f_a_bar, da = T(0);
        return a * (a * dn - da * dt);
    }
    static __device__ __forceinline__ T yface_far(const MC<T>& m, T dn, T dt) {
        const T a = m.f_a_bar, da = T(0);
        return a * (a * dn + da * dt);
    }
    static __device__ __forceinline__ void cell_far(const MC<T>& m, T jr, T jl, T jt, T jb, T p, T uc, T ul, T ur,
                                                    T up, T um, T& kphi, T& ku) {
        const T flux = (jr - jl + jt - jb) * m.inv_h2_flux;
        const T g_prime = fma_t(p * p, p, -p);
        const T one_m_p2 = fma_t(p, -p, T(1));
        const T p_prime = one_m_p2 * one_m_p2;
        kphi = div_far(fma_t(m.lambda * uc, -p_prime, flux - g_prime), m.c_far, m.inv_c_far);
        T acc = T(0);
        acc += ((ur - (uc + uc)) + ul) * m.ih0;
        acc += ((up - (uc + uc)) + um) * m.ih1;
        ku = fma_t(acc, m.d_thermal, T(0.5) * kphi);
    }
    static __device__ __forceinline__ void cell(const MC<T>& m, T jr, T jl, T jt, T jb, T p, T cdx, T cdy, T uc,
                                                T ul, T ur, T up, T um, T& kphi, T& ku) {
        const T flux = (jr - jl + jt - jb) * m.inv_h2_flux;
        const T g_prime = fma_t(p * p, p, -p);
        const T one_m_p2 = fma_t(p, -p, T(1));
        const T p_prime = one_m_p2 * one_m_p2;
        const T a = center_anisotropy(m, T(0.5) * cdx, T(0.5) * cdy);
        const T num = fma_t(m.lambda * uc, -p_prime, flux - g_prime);
        // a == a_bar: the divisor a a is c_far (whichever branch of the
        // anisotropy gave it)
        kphi = a == m.a_bar ? div_far(num, m.c_far, m.inv_c_far) : num / (a * a);
        T acc = T(0);
        acc += ((ur - (uc + uc)) + ul) * m.ih0;
        acc += ((up - (uc + uc)) + um) * m.ih1;
        ku = fma_t(acc, m.d_thermal, T(0.5) * kphi);
    }
    // Multi-grain faces and cell (finite_volume.rs:196-234, phasefield.rs:
    // 378-392): a face's anisotropy in the crystal frame (c0, s0) = (cos, sin)
    // theta0 of the cell being updated, the flux in the lab frame; the centre
    // anisotropy rotated likewise with the flux's constants
    // (center_anisotropy_rotated).  derx/dery are the face's lab-frame
    // differences in the reference's operand order.
    static __device__ __forceinline__ T oxface(const MC<T>& m, T c0, T s0, T derx, T dery) {
        T a, da;
        kr_face(m, c0 * derx + s0 * dery, c0 * dery - s0 * derx, a, da);
        return a * (a * derx - da * dery);
    }
    static __device__ __forceinline__ T oyface(const MC<T>& m, T c0, T s0, T derx, T dery) {
        T a, da;
        kr_face(m, c0 * derx + s0 * dery, c0 * dery - s0 * derx, a, da);
        return a * (a * dery + da * derx);
    }
    static __device__ __forceinline__ void ocell(const MC<T>& m, T jr, T jl, T jt, T jb, T p, T cdx, T cdy, T c0, T s0,
                                                 T uc, T ul, T ur, T up, T um, T& kphi, T& ku) {
        const T flux = (jr - jl + jt - jb) * m.inv_h2_flux;
        const T g_prime = fma_t(p * p, p, -p);
        const T one_m_p2 = fma_t(p, -p, T(1));
        const T p_prime = one_m_p2 * one_m_p2;
        const T dx = T(0.5) * cdx, dy = T(0.5) * cdy;
        T a, da;
        kr_face(m, c0 * dx + s0 * dy, c0 * dy - s0 * dx, a, da);
        kphi = fma_t(m.lambda * uc, -p_prime, flux - g_prime) / (a * a);
        T acc = T(0);
        acc += ((ur - (uc + uc)) + ul) * m.ih0;
        acc += ((up - (uc + uc)) + um) * m.ih1;
        ku = fma_t(acc, m.d_thermal, T(0.5) * kphi);
    }
    static __device__ __forceinline__ T axpy(T dt, T k, T x) { return x + dt * k; }
    static __device__ __forceinline__ T noise(uint64_t key) { return normal_t(key, T(0)); }
    static __device__ __forceinline__ T add_noise(T x, T scale_amp, T n) { return x + scale_amp * n; }
};

__device__ __forceinline__ int64_t slab_base(const SlabLayout& L, int b, int field) {
    return ((int64_t)b * L.nfields + field) * L.slab_stride;
}

// The eight neighbours of one block of a 2-D Cartesian grid, for ghost
// pushes: face neighbours from the topology table, diagonals by chaining
// (x step, then y step).  -1 where the step leaves the domain through a
// physical boundary; such steps are never taken (mirror images stay in the
// block itself).
struct Nbr2 {
    int b, l, r, d, u, dl, dr, ul, ur;

    __device__ __forceinline__ void load(const CartTopo& topo, int blk) {
        b = blk;
        l = topo.nbr[(blk * 3 + 0) * 2 + 0];
        r = topo.nbr[(blk * 3 + 0) * 2 + 1];
        d = topo.nbr[(blk * 3 + 1) * 2 + 0];
        u = topo.nbr[(blk * 3 + 1) * 2 + 1];
        dl = l >= 0 ? topo.nbr[(l * 3 + 1) * 2 + 0] : -1;
        ul = l >= 0 ? topo.nbr[(l * 3 + 1) * 2 + 1] : -1;
        dr = r >= 0 ? topo.nbr[(r * 3 + 1) * 2 + 0] : -1;
        ur = r >= 0 ? topo.nbr[(r * 3 + 1) * 2 + 1] : -1;
    }
    __device__ __forceinline__ int at(int sx, int sy) const {
        if (sy == 0) return sx == 0 ? b : (sx < 0 ? l : r);
        if (sx == 0) return sy < 0 ? d : u;
        if (sy < 0) return sx < 0 ? dl : dr;
        return sx < 0 ? ul : ur;
    }
};

// Ghost push of 2-D, ghost-width-1 fields: the value of interior cell (i, j)
// goes to every ghost entry whose source it is (the separable map of the
// reference's dimension sweep, cartesian.rs:439-526).  Scalars only, no
// local arrays.
template <class T>
__device__ __forceinline__ void push_ghosts_2d_g1(T* __restrict__ out, const SlabLayout& L, int field,
                                                  const Nbr2& nb, int n0, int n1, int i, int j, T v) {
    const bool lo_x = i == 0, hi_x = i == n0 - 1, lo_y = j == 0, hi_y = j == n1 - 1;
    if (!(lo_x | hi_x | lo_y | hi_y)) return;
    const int sy = L.gdim[0];
    const int sA = nb.l >= 0 ? -1 : 0, iA = nb.l >= 0 ? n0 : -1;
    const int sB = nb.r >= 0 ? 1 : 0, iB = nb.r >= 0 ? -1 : n0;
    const int sC = nb.d >= 0 ? -1 : 0, jC = nb.d >= 0 ? n1 : -1;
    const int sD = nb.u >= 0 ? 1 : 0, jD = nb.u >= 0 ? -1 : n1;
    auto put = [&](int sx, int syy, int ii, int jj) {
        out[slab_base(L, nb.at(sx, syy), field) + (ii + 1) + (int64_t)(jj + 1) * sy] = v;
    };
    if (lo_x) put(sA, 0, iA, j);
    if (hi_x) put(sB, 0, iB, j);
    if (lo_y) put(0, sC, i, jC);
    if (hi_y) put(0, sD, i, jD);
    if (lo_x && lo_y) put(sA, sC, iA, jC);
    if (lo_x && hi_y) put(sA, sD, iA, jD);
    if (hi_x && lo_y) put(sB, sC, iB, jC);
    if (hi_x && hi_y) put(sB, sD, iB, jD);
}

}  // namespace lg
