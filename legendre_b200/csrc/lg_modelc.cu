// Model C column-tile step, FP64, bit-identical to the reference.
//
// Compiled with -fmad=false: every operation below rounds separately and
// fma appears exactly where the reference calls f64::mul_add, in the
// reference's operand order (finite_volume.rs:129-142, 258-283;
// phasefield.rs:159-175, 395-421; driver.rs:210-236).
#include <cmath>

#include "lg_modelc_tile.cuh"

namespace lg {
namespace {

template <class T>
struct OpsExact {
    using Params = MC<T>;

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
    static __device__ __forceinline__ void cell(const MC<T>& m, T jr, T jl, T jt, T jb, T p, T cdx, T cdy, T uc,
                                                T ul, T ur, T up, T um, T& kphi, T& ku) {
        const T flux = (jr - jl + jt - jb) * m.inv_h2_flux;
        const T g_prime = fma_t(p * p, p, -p);
        const T one_m_p2 = fma_t(p, -p, T(1));
        const T p_prime = one_m_p2 * one_m_p2;
        const T a = center_anisotropy(m, T(0.5) * cdx, T(0.5) * cdy);
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

}  // namespace

bool modelc_tile_supported(const CartTopo& topo) { return topo.D == 2 && topo.n[0] >= 1; }

cudaError_t launch_modelc_tile_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, int minb, cudaStream_t s) {
    TileArgs g{topo, L, dt, nz.seed, tdev, slot, rows, 0, 0, 0};
    const MC<double> mc = to_mc<double>(m);
    const double scale_amp = std::sqrt(dt) * nz.amp;
    if (nz.on) return launch_strip_ops<double, OpsExact<double>, true, 1>(in, out, g, mc, dt, scale_amp, minb, s);
    return launch_strip_ops<double, OpsExact<double>, false, 1>(in, out, g, mc, dt, scale_amp, minb, s);
}

}  // namespace lg
