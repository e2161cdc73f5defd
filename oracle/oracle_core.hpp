// legendre oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// Shared pieces of the CPU restatement of the reference's SerialScheduler
// path (rng, per-block stencils, Model C right-hand side, driver kernels),
// written against a plain block extent so the Cartesian and AMR oracles use
// the same code.  Rules: compiled with -ffp-contract=off, std::fma exactly
// at the reference's mul_add sites, reference operand order, glibc libm.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "legendre_oracle.h"

namespace orc {

// ---------------------------------------------------------------- rng ------
// src/util/rng.rs:13-18
inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// src/util/rng.rs:23-29
inline uint64_t mix_key(uint64_t seed, const uint64_t* parts, size_t n) {
    uint64_t s = splitmix64(seed);
    for (size_t i = 0; i < n; ++i) s = splitmix64(s ^ parts[i]);
    return s;
}
// src/util/rng.rs:35-37
inline double unit_open(uint64_t bits) { return (double)((bits >> 11) + 1) * (1.0 / 9007199254740992.0); }
// std::f64::consts::TAU
constexpr double kTau = 6.283185307179586476925286766559;
// src/util/rng.rs:43-49
inline double standard_normal(uint64_t key) {
    uint64_t a = splitmix64(key);
    uint64_t b = splitmix64(a ^ 0xD1B54A32D192ED03ull);
    double u = unit_open(a);
    double v = unit_open(b);
    return std::sqrt(-2.0 * std::log(u)) * std::cos(kTau * v);
}

// ------------------------------------------------------------- extents ----
// A uniform box of cells (a Cartesian block or an AMR patch) with a ghost
// ring: dense, dimension 0 fastest (src/geometry/cartesian.rs:8-11, 189-204).
struct Ext {
    int D = 2;
    int64_t n[3] = {1, 1, 1};
    int64_t len(int g) const {
        int64_t r = 1;
        for (int d = 0; d < D; ++d) r *= n[d] + 2 * g;
        return r;
    }
    int64_t lin(const int64_t* idx, int g) const {
        int64_t off = 0, stride = 1;
        for (int d = 0; d < D; ++d) {
            off += (idx[d] + g) * stride;
            stride *= n[d] + 2 * g;
        }
        return off;
    }
    // Grid::cell_key for a box (cartesian.rs:599-619, amr/grid.rs:397-417)
    bool cell_key(int g, int64_t offset, uint64_t* key) const {
        int64_t rem = offset, k = 0, stride = 1;
        for (int d = 0; d < D; ++d) {
            int64_t gh = n[d] + 2 * g;
            int64_t c = rem % gh;
            rem /= gh;
            if (c < g || c >= n[d] + g) return false;
            k += (c - g) * stride;
            stride *= n[d];
        }
        *key = (uint64_t)k;
        return true;
    }
};

// Visit every index of the half-open box lo..hi, dimension 0 fastest
// (cartesian.rs:338-358).
template <class F>
void for_each_box(int D, const int64_t* lo, const int64_t* hi, F f) {
    for (int d = 0; d < D; ++d)
        if (lo[d] >= hi[d]) return;
    int64_t idx[3] = {lo[0], D > 1 ? lo[1] : 0, D > 2 ? lo[2] : 0};
    for (;;) {
        f(idx);
        int d = 0;
        for (;;) {
            idx[d] += 1;
            if (idx[d] < hi[d]) break;
            idx[d] = lo[d];
            if (++d == D) return;
        }
    }
}

template <class F>
void for_each_interior(const Ext& e, F f) {
    int64_t lo[3] = {0, 0, 0};
    for_each_box(e.D, lo, e.n, f);
}

template <class F>
void parallel_blocks(int64_t nblocks, int nthreads, F f) {
#ifdef _OPENMP
    if (nthreads > 1) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
        for (int64_t b = 0; b < nblocks; ++b) f(b);
        return;
    }
#endif
    (void)nthreads;
    for (int64_t b = 0; b < nblocks; ++b) f(b);
}

// src/discretization/finite_difference.rs:49-67 ; output interior only
inline void central_laplacian(const Ext& e, const double* h, const double* in, double* out, int g) {
    double inv_h2[3];
    for (int d = 0; d < e.D; ++d) inv_h2[d] = 1.0 / (h[d] * h[d]);
    for_each_interior(e, [&](const int64_t* idx) {
        double center = in[e.lin(idx, g)];
        double acc = 0.0;
        for (int d = 0; d < e.D; ++d) {
            int64_t p[3] = {idx[0], idx[1], idx[2]}, m[3] = {idx[0], idx[1], idx[2]};
            p[d] += 1;
            m[d] -= 1;
            acc += ((in[e.lin(p, g)] - (center + center)) + in[e.lin(m, g)]) * inv_h2[d];
        }
        out[e.lin(idx, g)] = acc;
    });
}

// Heat<D>::vector_field_block (tests/heat3d.rs:58-74): Laplacian then *= kappa
inline void heat_drift_block(const Ext& e, const double* h, double kappa, const double* u, double* k) {
    central_laplacian(e, h, u, k, 1);
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, 1);
        k[o] = k[o] * kappa;
    });
}

// ---------------------------------------------------------- Model C -------
struct ModelC {
    double eps4, lambda, d_thermal, noise_amplitude, tol;
    double a_bar, eps_prime;                    // model (phasefield.rs:100-116)
    double f_a_bar, f_eps_prime, f_a12, f_tol;  // flux (finite_volume.rs:113-122)
};

inline ModelC make_model(const orc_modelc_params* p) {
    ModelC m;
    m.eps4 = p->eps4;
    m.lambda = p->lambda;
    m.d_thermal = p->d_thermal;
    m.noise_amplitude = p->noise_amplitude;
    m.tol = p->anisotropy_tol;
    m.a_bar = std::fma(3.0, -m.eps4, 1.0);
    m.eps_prime = 3.0 * m.eps4 / m.a_bar;
    m.f_a_bar = std::fma(3.0, -m.eps4, 1.0);
    m.f_eps_prime = 3.0 * m.eps4 / m.f_a_bar;
    m.f_a12 = 4.0 * m.f_a_bar * m.f_eps_prime;
    m.f_tol = p->flux_tol;
    return m;
}

// finite_volume.rs:129-142
inline void kr_face(const ModelC& m, double dx, double dy, double* a, double* da) {
    double dx2 = dx * dx;
    double dy2 = dy * dy;
    double sum = dx2 + dy2;
    double mag2 = sum * sum;
    if (mag2 <= m.f_tol) {
        *a = m.f_a_bar;
        *da = 0.0;
    } else {
        *a = m.f_a_bar * (1.0 + m.f_eps_prime * (dx2 * dx2 + dy2 * dy2) / mag2);
        *da = -(m.f_a12) * dx * dy * (dx2 - dy2) / mag2;
    }
}

// phasefield.rs:159-175
inline double center_anisotropy(const ModelC& m, const double* p, int64_t sx, int64_t sy, int64_t o) {
    double dx = 0.5 * (p[o + sx] - p[o - sx]);
    double dy = 0.5 * (p[o + sy] - p[o - sy]);
    double dx2 = dx * dx;
    double dy2 = dy * dy;
    double sum = dx2 + dy2;
    double mag2 = sum * sum;
    if (mag2 <= m.tol) return m.a_bar;
    return m.a_bar * (1.0 + m.eps_prime * (dx2 * dx2 + dy2 * dy2) / mag2);
}

// ModelC::vector_field_block(Driver::Time) on a 2-D box (phasefield.rs:367-421):
// KarmaRappelFlux::kernel (finite_volume.rs:248-285) into dphi, the local
// terms (phasefield.rs:393-404), the u Laplacian and coupling
// (phasefield.rs:412-421).  Interior entries of kphi/ku only.
inline void modelc_drift_block(const Ext& e, const double* h, const ModelC& m, const double* p, const double* u,
                               double* kphi, double* ku) {
    const int g = 1;
    const int64_t sx = 1, sy = e.n[0] + 2 * g;
    double inv_h2 = 1.0 / (h[0] * h[1]);
    double quarter = 0.25;
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, g);
        auto P = [&](int di, int dj) { return p[o + di * sx + dj * sy]; };
        double derx_r = P(1, 0) - P(0, 0);
        double derx_l = P(0, 0) - P(-1, 0);
        double derx_t = quarter * (P(1, 1) - P(-1, 1) + P(1, 0) - P(-1, 0));
        double derx_b = quarter * (P(1, 0) - P(-1, 0) + P(1, -1) - P(-1, -1));
        double dery_t = P(0, 1) - P(0, 0);
        double dery_b = P(0, 0) - P(0, -1);
        double dery_r = quarter * (P(1, 1) - P(1, -1) + P(0, 1) - P(0, -1));
        double dery_l = quarter * (P(0, 1) - P(0, -1) + P(-1, 1) - P(-1, -1));
        double a_r, da_r, a_l, da_l, a_t, da_t, a_b, da_b;
        kr_face(m, derx_r, dery_r, &a_r, &da_r);
        kr_face(m, derx_l, dery_l, &a_l, &da_l);
        kr_face(m, derx_t, dery_t, &a_t, &da_t);
        kr_face(m, derx_b, dery_b, &a_b, &da_b);
        double j_r = a_r * (a_r * derx_r - da_r * dery_r);
        double j_l = a_l * (a_l * derx_l - da_l * dery_l);
        double j_t = a_t * (a_t * dery_t + da_t * derx_t);
        double j_b = a_b * (a_b * dery_b + da_b * derx_b);
        kphi[o] = (j_r - j_l + j_t - j_b) * inv_h2;
    });
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, g);
        double pv = p[o];
        double g_prime = std::fma(pv * pv, pv, -pv);
        double one_m_p2 = std::fma(pv, -pv, 1.0);
        double p_prime = one_m_p2 * one_m_p2;
        double a = center_anisotropy(m, p, sx, sy, o);
        kphi[o] = std::fma(m.lambda * u[o], -p_prime, kphi[o] - g_prime) / (a * a);
    });
    central_laplacian(e, h, u, ku, g);
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, g);
        ku[o] = std::fma(ku[o], m.d_thermal, 0.5 * kphi[o]);
    });
}

// The multi-grain form: KarmaRappelFlux::apply_oriented (finite_volume.rs:
// 178-235) with every face's anisotropy taken in the crystal frame of the
// cell's own orientation theta0 (read at the cell centre, ghost width 0),
// rotate() at finite_volume.rs:238-242, and the local terms with
// center_anisotropy_rotated (finite_volume.rs:159-172, phasefield.rs:378-392).
// (s0, c0) = theta0.sin_cos(): glibc sin and cos, as Rust's f64::sin_cos.
inline void modelc_drift_block_oriented(const Ext& e, const double* h, const ModelC& m, const double* p,
                                        const double* u, const double* theta, double* kphi, double* ku) {
    const int g = 1;
    const int64_t sx = 1, sy = e.n[0] + 2 * g;
    double inv_h2 = 1.0 / (h[0] * h[1]);
    double quarter = 0.25;
    auto rotate = [](double c0, double s0, double dx, double dy, double* rx, double* ry) {
        *rx = c0 * dx + s0 * dy;
        *ry = c0 * dy - s0 * dx;
    };
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, g);
        double th = theta[e.lin(idx, 0)];
        double s0 = std::sin(th), c0 = std::cos(th);
        auto P = [&](int di, int dj) { return p[o + di * sx + dj * sy]; };
        double derx_r = P(1, 0) - P(0, 0);
        double derx_l = P(0, 0) - P(-1, 0);
        double derx_t = quarter * (P(1, 1) - P(-1, 1) + P(1, 0) - P(-1, 0));
        double derx_b = quarter * (P(1, 0) - P(-1, 0) + P(1, -1) - P(-1, -1));
        double dery_t = P(0, 1) - P(0, 0);
        double dery_b = P(0, 0) - P(0, -1);
        double dery_r = quarter * (P(1, 1) - P(1, -1) + P(0, 1) - P(0, -1));
        double dery_l = quarter * (P(0, 1) - P(0, -1) + P(-1, 1) - P(-1, -1));
        double rx, ry, a_r, da_r, a_l, da_l, a_t, da_t, a_b, da_b;
        rotate(c0, s0, derx_r, dery_r, &rx, &ry);
        kr_face(m, rx, ry, &a_r, &da_r);
        rotate(c0, s0, derx_l, dery_l, &rx, &ry);
        kr_face(m, rx, ry, &a_l, &da_l);
        rotate(c0, s0, derx_t, dery_t, &rx, &ry);
        kr_face(m, rx, ry, &a_t, &da_t);
        rotate(c0, s0, derx_b, dery_b, &rx, &ry);
        kr_face(m, rx, ry, &a_b, &da_b);
        double j_r = a_r * (a_r * derx_r - da_r * dery_r);
        double j_l = a_l * (a_l * derx_l - da_l * dery_l);
        double j_t = a_t * (a_t * dery_t + da_t * derx_t);
        double j_b = a_b * (a_b * dery_b + da_b * derx_b);
        kphi[o] = (j_r - j_l + j_t - j_b) * inv_h2;
    });
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, g);
        double th = theta[e.lin(idx, 0)];
        double s0 = std::sin(th), c0 = std::cos(th);
        double pv = p[o];
        double g_prime = std::fma(pv * pv, pv, -pv);
        double one_m_p2 = std::fma(pv, -pv, 1.0);
        double p_prime = one_m_p2 * one_m_p2;
        double dx = 0.5 * (p[o + sx] - p[o - sx]);
        double dy = 0.5 * (p[o + sy] - p[o - sy]);
        double rx, ry, a, da;
        rotate(c0, s0, dx, dy, &rx, &ry);
        kr_face(m, rx, ry, &a, &da);  // the flux's face(): flux constants
        kphi[o] = std::fma(m.lambda * u[o], -p_prime, kphi[o] - g_prime) / (a * a);
    });
    central_laplacian(e, h, u, ku, g);
    for_each_interior(e, [&](const int64_t* idx) {
        int64_t o = e.lin(idx, g);
        ku[o] = std::fma(ku[o], m.d_thermal, 0.5 * kphi[o]);
    });
}

// ------------------------------------------------------------ drivers -----
// Driver::Time (driver.rs:210-217): x += dt * v over every slab entry
inline void apply_time(std::vector<double>& x, const std::vector<double>& v, double dt) {
    for (size_t i = 0; i < x.size(); ++i) x[i] += dt * v[i];
}

// Driver::Wiener(0) (driver.rs:218-237) on one field of one block
inline void apply_wiener(const Ext& e, int g, std::vector<double>& x, const std::vector<double>& amp, double dt,
                         uint64_t seed, uint64_t salt, uint64_t block) {
    double scale = std::sqrt(dt);
    uint64_t parts[3] = {salt, (1ull << 32) | 0ull, block};
    uint64_t block_key = mix_key(seed, parts, 3);
    for (size_t i = 0; i < x.size(); ++i) {
        if (amp[i] == 0.0) continue;
        uint64_t cell;
        if (!e.cell_key(g, (int64_t)i, &cell)) continue;
        uint64_t key = splitmix64(block_key ^ cell);
        x[i] += scale * amp[i] * standard_normal(key);
    }
}

inline uint64_t bits_of(double t) {
    uint64_t s;
    std::memcpy(&s, &t, sizeof s);
    return s;
}

}  // namespace orc
