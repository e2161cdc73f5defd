// Model C column-tile step, FP64, bit-identical to the reference.
//
// Compiled with -fmad=false: every operation below rounds separately and
// fma appears exactly where the reference calls f64::mul_add, in the
// reference's operand order (finite_volume.rs:129-142, 258-283;
// phasefield.rs:159-175, 395-421; driver.rs:210-236).
#include <cmath>

#include "lg_modelc_tile.cuh"

namespace lg {

bool modelc_tile_supported(const CartTopo& topo) { return topo.D == 2 && topo.n[0] >= 1; }

cudaError_t launch_modelc_tile_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, int minb, unsigned* work, cudaStream_t s) {
    TileArgs g{topo, L, dt, nz.seed, tdev, slot, rows, 0, 0, 0, work};
    const MC<double> mc = to_mc<double>(m);
    const double scale_amp = std::sqrt(dt) * nz.amp;
    if (nz.on) return launch_strip_ops<double, OpsExact<double>, true, 1>(in, out, g, mc, dt, scale_amp, minb, s);
    return launch_strip_ops<double, OpsExact<double>, false, 1>(in, out, g, mc, dt, scale_amp, minb, s);
}

cudaError_t launch_modelc_oriented_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                       const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                       const double* trig, int64_t ncells, int rows, cudaStream_t s) {
    TileArgs g{topo, L, dt, nz.seed, tdev, slot, rows, 0, 0, 0};
    const MC<double> mc = to_mc<double>(m);
    const double scale_amp = std::sqrt(dt) * nz.amp;
    const OrientArgs oa{trig, ncells};
    if (nz.on) return launch_strip_oriented<double, OpsExact<double>, true, 2, true>(in, out, g, mc, dt, scale_amp, oa, s);
    return launch_strip_oriented<double, OpsExact<double>, false, 2, true>(in, out, g, mc, dt, scale_amp, oa, s);
}

cudaError_t launch_modelc_rk_stage_f64(int mode, const double* in, double* out, const CartTopo& topo,
                                       const SlabLayout& L, const ModelCDev& m, const double* y, double* k,
                                       const double* k1, const double* k2, const double* k3, double c, double s6,
                                       double s3, const double* trig, int64_t ncells, double* tdev, int slot,
                                       double dt, cudaStream_t s) {
    TileArgs g{topo, L, dt, 0, tdev, slot, 0, 0, 0, 0};
    const MC<double> mc = to_mc<double>(m);
    const OrientArgs oa{trig, ncells};
    const RkArgs<double> rk{y, k, k1, k2, k3, c, s6, s3};
    if (mode == 1)
        return trig ? launch_strip_rk<double, OpsExact<double>, 1, true>(in, out, g, mc, dt, oa, rk, s)
                    : launch_strip_rk<double, OpsExact<double>, 1, false>(in, out, g, mc, dt, oa, rk, s);
    return trig ? launch_strip_rk<double, OpsExact<double>, 2, true>(in, out, g, mc, dt, oa, rk, s)
                : launch_strip_rk<double, OpsExact<double>, 2, false>(in, out, g, mc, dt, oa, rk, s);
}

size_t modelc_record_size_f64() { return sizeof(MC<double>); }
void modelc_record_f64(const ModelCDev& m, void* out) { *static_cast<MC<double>*>(out) = to_mc<double>(m); }

cudaError_t launch_modelc_batch_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                    const void* params, const uint64_t* seeds, int bpi, double dt, double amp,
                                    double* tdev, int slot, int rows, cudaStream_t s) {
    TileArgs g{topo, L, dt, 0, tdev, slot, rows, 0, 0, 0};
    const BatchArgs bt{params, seeds, bpi};
    const double scale_amp = std::sqrt(dt) * amp;
    if (amp != 0.0) return launch_strip_batch<double, OpsExact<double>, true, 2, true>(in, out, g, bt, dt, scale_amp, s);
    return launch_strip_batch<double, OpsExact<double>, false, 2, true>(in, out, g, bt, dt, scale_amp, s);
}

}  // namespace lg
