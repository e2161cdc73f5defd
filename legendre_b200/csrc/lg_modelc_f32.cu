// Model C column-tile step in FP32 storage and arithmetic.
//
// Same tile schedule as the FP64 kernel, but the arithmetic is restructured
// for single precision (this unit is compiled with contraction allowed):
//   * one approximate reciprocal per face serves both of its ratios, using
//     (dx^4 + dy^4)/(dx^2 + dy^2)^2 = 1 - 2 dx^2 dy^2/(dx^2 + dy^2)^2, so
//     A = a(1 + e') - 2 a e' dx^2 dy^2 / |grad|^4;
//   * the 1/A^2 mobility is a reciprocal times the numerator;
//   * the Gaussian is drawn from the same counter-based key as the FP64
//     path, with the Box-Muller transform in single precision.
// Its error against the FP64 oracle is measured by the tests.
#include <cmath>

#include "lg_modelc_tile.cuh"

namespace lg {
namespace {

struct Fast32 {
    float lambda, d_thermal, inv_h2_flux, ih0, ih1;
    float f_a_bar, f_a1pe, f_2ae, f_a12, f_tol;  // flux: a, a(1+e'), 2 a e', a12, tol
    float c_a_bar, c_a1pe, c_2ae, c_tol;         // cell-centred anisotropy
};

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct OpsFast32 {
    using Params = Fast32;
    static constexpr bool kFarPass = true;  // the paired rows test for the far field first (quarter, *_far)

    static __device__ __forceinline__ void aniso(float dx, float dy, float a_bar, float a1pe, float two_ae,
                                                 float tol, float& a, float& inv) {
        const float dx2 = dx * dx, dy2 = dy * dy;
        const float s = dx2 + dy2;
        const float mag2 = s * s;
        inv = rcp_approx(mag2);
        const bool flat = mag2 <= tol;
        a = flat ? a_bar : a1pe - two_ae * (dx2 * dy2) * inv;
        inv = flat ? 0.0f : inv;
    }
    static __device__ __forceinline__ float xface(const Fast32& m, float dn, float d1, float c, float e) {
        const float dt = 0.25f * ((d1 + c) - e);
        float a, inv;
        aniso(dn, dt, m.f_a_bar, m.f_a1pe, m.f_2ae, m.f_tol, a, inv);
        const float da = -m.f_a12 * dn * dt * (dn * dn - dt * dt) * inv;
        return a * (a * dn - da * dt);
    }
    static __device__ __forceinline__ float yface(const Fast32& m, float dn, float d1, float c, float e) {
        const float dt = 0.25f * ((d1 + c) - e);
        float a, inv;
        aniso(dt, dn, m.f_a_bar, m.f_a1pe, m.f_2ae, m.f_tol, a, inv);
        const float da = -m.f_a12 * dt * dn * (dt * dt - dn * dn) * inv;
        return a * (a * dn + da * dt);
    }
    static __device__ __forceinline__ void cell(const Fast32& m, float jr, float jl, float jt, float jb, float p,
                                                float cdx, float cdy, float uc, float ul, float ur, float up,
                                                float um, float& kphi, float& ku) {
        const float flux = ((jr - jl) + (jt - jb)) * m.inv_h2_flux;
        const float g_prime = p * p * p - p;
        const float one_m_p2 = 1.0f - p * p;
        const float p_prime = one_m_p2 * one_m_p2;
        float a, inv;
        aniso(0.5f * cdx, 0.5f * cdy, m.c_a_bar, m.c_a1pe, m.c_2ae, m.c_tol, a, inv);
        kphi = ((flux - g_prime) - m.lambda * uc * p_prime) * rcp_approx(a * a);
        const float lap = ((ur + ul) - 2.0f * uc) * m.ih0 + ((up + um) - 2.0f * uc) * m.ih1;
        ku = lap * m.d_thermal + 0.5f * kphi;
    }
    // multi-grain faces and cell (see OpsExact::oxface for the reference form):
    // one reciprocal per face
    static __device__ __forceinline__ float oaniso(const Fast32& m, float rx, float ry, float& da) {
        float a, inv;
        aniso(rx, ry, m.f_a_bar, m.f_a1pe, m.f_2ae, m.f_tol, a, inv);
        da = -m.f_a12 * rx * ry * (rx * rx - ry * ry) * inv;
        return a;
    }
    static __device__ __forceinline__ float oxface(const Fast32& m, float c0, float s0, float derx, float dery) {
        float da;
        const float a = oaniso(m, c0 * derx + s0 * dery, c0 * dery - s0 * derx, da);
        return a * (a * derx - da * dery);
    }
    static __device__ __forceinline__ float oyface(const Fast32& m, float c0, float s0, float derx, float dery) {
        float da;
        const float a = oaniso(m, c0 * derx + s0 * dery, c0 * dery - s0 * derx, da);
        return a * (a * dery + da * derx);
    }
    static __device__ __forceinline__ void ocell(const Fast32& m, float jr, float jl, float jt, float jb, float p,
                                                 float cdx, float cdy, float c0, float s0, float uc, float ul, float ur,
                                                 float up, float um, float& kphi, float& ku) {
        const float flux = ((jr - jl) + (jt - jb)) * m.inv_h2_flux;
        const float g_prime = p * p * p - p;
        const float one_m_p2 = 1.0f - p * p;
        const float p_prime = one_m_p2 * one_m_p2;
        const float dx = 0.5f * cdx, dy = 0.5f * cdy;
        float dac;
        const float a = oaniso(m, c0 * dx + s0 * dy, c0 * dy - s0 * dx, dac);
        kphi = ((flux - g_prime) - m.lambda * uc * p_prime) * rcp_approx(a * a);
        const float lap = ((ur + ul) - 2.0f * uc) * m.ih0 + ((up + um) - 2.0f * uc) * m.ih1;
        ku = lap * m.d_thermal + 0.5f * kphi;
    }
    // The far-field forms (every anisotropy of a pass flat): a = a_bar and no
    // reciprocal per face; the cell's 1/a_bar^2 by the same approximate
    // reciprocal the general form takes.  Same values as the general forms
    // with the flat selects taken.
    static __device__ __forceinline__ float quarter(float d1, float c, float e) { return 0.25f * ((d1 + c) - e); }
    static __device__ __forceinline__ float face_mag2(float dx, float dy) {
        const float s = dx * dx + dy * dy;
        return s * s;
    }
    static __device__ __forceinline__ bool face_flat(const Fast32& m, float dx, float dy) {
        return face_mag2(dx, dy) <= m.f_tol;
    }
    static __device__ __forceinline__ bool center_flat(const Fast32& m, float cdx, float cdy) {
        return face_mag2(0.5f * cdx, 0.5f * cdy) <= m.c_tol;
    }
    static __device__ __forceinline__ float xface_far(const Fast32& m, float dn, float) {
        return m.f_a_bar * (m.f_a_bar * dn);
    }
    static __device__ __forceinline__ float yface_far(const Fast32& m, float dn, float) {
        return m.f_a_bar * (m.f_a_bar * dn);
    }
    static __device__ __forceinline__ void cell_far(const Fast32& m, float jr, float jl, float jt, float jb, float p,
                                                    float uc, float ul, float ur, float up, float um, float& kphi,
                                                    float& ku) {
        const float flux = ((jr - jl) + (jt - jb)) * m.inv_h2_flux;
        const float g_prime = p * p * p - p;
        const float one_m_p2 = 1.0f - p * p;
        const float p_prime = one_m_p2 * one_m_p2;
        kphi = ((flux - g_prime) - m.lambda * uc * p_prime) * rcp_approx(m.c_a_bar * m.c_a_bar);
        const float lap = ((ur + ul) - 2.0f * uc) * m.ih0 + ((up + um) - 2.0f * uc) * m.ih1;
        ku = lap * m.d_thermal + 0.5f * kphi;
    }
    static __device__ __forceinline__ float axpy(float dt, float k, float x) { return x + dt * k; }
    static __device__ __forceinline__ float noise(uint64_t key) { return normal_fast32(key); }
    static __device__ __forceinline__ float add_noise(float x, float scale_amp, float n) { return x + scale_amp * n; }
    // Box-Muller from the reference's two uniforms (rng.rs:43-49), single
    // precision: u keeps its full 53-bit tail (rounded to 24 bits), and
    // cos(2 pi v) = -cos(2 pi (v - 1/2)) keeps the argument in [-pi, pi].
    static __device__ __forceinline__ float normal_fast32(uint64_t key) {
        const uint64_t a = splitmix64(key);
        const uint64_t b = splitmix64(a ^ 0xD1B54A32D192ED03ull);
        const float u = __ull2float_rn((a >> 11) + 1) * 0x1p-53f;
        const float v = __ull2float_rn((b >> 11) + 1) * 0x1p-53f;
        // the hardware's approximate square root (sqrt.approx; +0 and -0 map to
        // themselves): the IEEE sqrtf cost 5 % of the step
        float r;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(-2.0f * __logf(u)));
        return -r * __cosf(6.28318530717958647692f * (v - 0.5f));
    }
};

}  // namespace

namespace {
Fast32 fast32_of(const ModelCDev& m) {
    Fast32 f{};
    f.lambda = (float)m.lambda;
    f.d_thermal = (float)m.d_thermal;
    f.inv_h2_flux = (float)m.inv_h2_flux;
    f.ih0 = (float)m.inv_h2[0];
    f.ih1 = (float)m.inv_h2[1];
    f.f_a_bar = (float)m.f_a_bar;
    f.f_a1pe = (float)(m.f_a_bar * (1.0 + m.f_eps_prime));
    f.f_2ae = (float)(2.0 * m.f_a_bar * m.f_eps_prime);
    f.f_a12 = (float)m.f_a12;
    f.f_tol = (float)m.f_tol;
    f.c_a_bar = (float)m.a_bar;
    f.c_a1pe = (float)(m.a_bar * (1.0 + m.eps_prime));
    f.c_2ae = (float)(2.0 * m.a_bar * m.eps_prime);
    f.c_tol = (float)m.tol;
    return f;
}
}  // namespace

cudaError_t launch_modelc_tile_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, int minb, unsigned* work, cudaStream_t s) {
    TileArgs g{topo, L, dt, nz.seed, tdev, slot, rows, 0, 0, 0, work};
    const Fast32 f = fast32_of(m);
    const float scale_amp = (float)(std::sqrt(dt) * nz.amp);
    if (nz.on) return launch_strip_ops<float, OpsFast32, true, 1>(in, out, g, f, (float)dt, scale_amp, minb, s);
    return launch_strip_ops<float, OpsFast32, false, 1>(in, out, g, f, (float)dt, scale_amp, minb, s);
}

cudaError_t launch_modelc_oriented_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                       const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                       const float* trig, int64_t ncells, int rows, cudaStream_t s) {
    TileArgs g{topo, L, dt, nz.seed, tdev, slot, rows, 0, 0, 0};
    const Fast32 f = fast32_of(m);
    const float scale_amp = (float)(std::sqrt(dt) * nz.amp);
    const OrientArgs oa{trig, ncells};
    if (nz.on) return launch_strip_oriented<float, OpsFast32, true, 2, true>(in, out, g, f, (float)dt, scale_amp, oa, s);
    return launch_strip_oriented<float, OpsFast32, false, 2, true>(in, out, g, f, (float)dt, scale_amp, oa, s);
}

cudaError_t launch_modelc_rk_stage_f32(int mode, const float* in, float* out, const CartTopo& topo,
                                       const SlabLayout& L, const ModelCDev& m, const float* y, float* k,
                                       const float* k1, const float* k2, const float* k3, double c, double s6,
                                       double s3, const float* trig, int64_t ncells, double* tdev, int slot,
                                       double dt, cudaStream_t s) {
    TileArgs g{topo, L, dt, 0, tdev, slot, 0, 0, 0, 0};
    const Fast32 f = fast32_of(m);
    const OrientArgs oa{trig, ncells};
    const RkArgs<float> rk{y, k, k1, k2, k3, (float)c, (float)s6, (float)s3};
    if (mode == 1)
        return trig ? launch_strip_rk<float, OpsFast32, 1, true>(in, out, g, f, (float)dt, oa, rk, s)
                    : launch_strip_rk<float, OpsFast32, 1, false>(in, out, g, f, (float)dt, oa, rk, s);
    return trig ? launch_strip_rk<float, OpsFast32, 2, true>(in, out, g, f, (float)dt, oa, rk, s)
                : launch_strip_rk<float, OpsFast32, 2, false>(in, out, g, f, (float)dt, oa, rk, s);
}

size_t modelc_record_size_f32() { return sizeof(Fast32); }
void modelc_record_f32(const ModelCDev& m, void* out) { *static_cast<Fast32*>(out) = fast32_of(m); }

cudaError_t launch_modelc_batch_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                    const void* params, const uint64_t* seeds, int bpi, double dt, double amp,
                                    double* tdev, int slot, int rows, cudaStream_t s) {
    TileArgs g{topo, L, dt, 0, tdev, slot, rows, 0, 0, 0};
    const BatchArgs bt{params, seeds, bpi};
    const float scale_amp = (float)(std::sqrt(dt) * amp);
    if (amp != 0.0) return launch_strip_batch<float, OpsFast32, true, 2, true>(in, out, g, bt, (float)dt, scale_amp, s);
    return launch_strip_batch<float, OpsFast32, false, 2, true>(in, out, g, bt, (float)dt, scale_amp, s);
}

}  // namespace lg
