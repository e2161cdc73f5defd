// Launchers of the legendre B200 kernels (host side, C++ linkage).  Each
// returns the cudaError_t of its launch; the C-ABI layer turns that into a
// status code and an error string.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lg_common.cuh"

namespace lg {

// Model C parameters as the kernels consume them (derived constants are
// computed on the host exactly as the reference derives them).
struct ModelCDev {
    double lambda, d_thermal;
    double a_bar, eps_prime, tol;                 // ModelC (phasefield.rs:100-116)
    double f_a_bar, f_eps_prime, f_a12, f_tol;    // KarmaRappelFlux (finite_volume.rs:113-122)
    double inv_h2_flux;                           // 1/(hx*hy)   (finite_volume.rs:254)
    double inv_h2[2];                             // 1/(h_d*h_d) (finite_difference.rs:54)
};

struct NoiseDev {
    int on;               // Wiener<1> with a non-zero amplitude
    uint64_t seed;
    double amp;           // noise amplitude b (the Wiener amplitude field)
};

// (b) ghost fill of one field (pull form): every ghost entry of every block
// copies its source interior entry (exchange, periodic wrap or mirror).
cudaError_t launch_halo_fill(void* arena, int elem_size, const CartTopo& topo, const SlabLayout& L, int field,
                             cudaStream_t s);

// (d) forward-Euler heat step: out = in + dt * (kappa * lap(in)) on the
// interiors, plus the ghost ring of `out` filled from the new interiors.
cudaError_t launch_heat_step(const double* in, double* out, const CartTopo& topo, const SlabLayout& L, int field,
                             double kappa, double dt, const double inv_h2[3], cudaStream_t s);

// (d) the same heat step for 3-D grids of ghost width 1, with every halo
// value read from the neighbour blocks' interiors: `out` gets interiors only
// (its ghost entries are left as they were).  Bit-identical to
// launch_heat_step.  Needs n0 * n1 <= 1024.
bool heat3d_pull_supported(const CartTopo& topo, const SlabLayout& L);
cudaError_t launch_heat3d_pull(const double* in, double* out, const CartTopo& topo, const SlabLayout& L, int field,
                               double kappa, double dt, const double inv_h2[3], cudaStream_t s);

// The same step with each CTA's tile and its six halo faces staged by
// tensor copies (TMA) onto one mbarrier; needs an even block width too.  A
// wait for the copies that gives up sets *err (the context's device word).
bool heat3d_tma_supported(const CartTopo& topo, const SlabLayout& L);
cudaError_t launch_heat3d_tma(const double* in, double* out, const CartTopo& topo, const SlabLayout& L, int field,
                              double kappa, double dt, const double inv_h2[3], int* err, cudaStream_t s);

// (a) fused Model C Euler-Maruyama step, FP64, bit-exact to the reference.
// Reads phi (field 0) and u (field 1) from `in`, writes both to `out` with
// ghosts filled.  `tdev[slot]` holds the step's time (its bits are the noise
// salt); block 0 writes tdev[slot ^ 1] = t + dt.
cudaError_t launch_modelc_step_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int variant, cudaStream_t s);

// FP32 storage and arithmetic variant of the same step.
cudaError_t launch_modelc_step_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int variant, cudaStream_t s);

// One RungeKutta4 stage of the heat model (rk4.rs:40-79): mode 1 writes
// k = kappa lap(in) to kout and y + c k to out; mode 2 writes
// (((y + s6 k1) + s3 k2) + s3 k3) + s6 k to out.  Ghost images of out are
// pushed.  FP64, any dimension, bit-identical to the reference's stages.
cudaError_t launch_heat_rk_stage(int mode, const double* in, double* out, const double* y, double* kout,
                                 const double* k1, const double* k2, const double* k3, const CartTopo& topo,
                                 const SlabLayout& L, int field, double kappa, const double* inv_h2, double c,
                                 double s6, double s3, cudaStream_t s);

// Warp-strip variants of the same steps (lg_modelc.cu, lg_modelc_f32.cu):
// each face flux is evaluated once and shared by its two cells; `rows` rows
// of one block per warp (0 = chosen from the grid); `minb` = the form: 2, 3
// or 4 CTAs per SM the register allocation must allow, 5, 6, 7 the same
// with two rows per pass of the row loop.  With `work` (two counters, the
// step's at `slot`) the launch is one wave of CTAs whose warps take further
// units from the counter; null gives the static grid-stride schedule.  The
// FP64 results are bit-identical to the reference-order kernel above.
bool modelc_tile_supported(const CartTopo& topo);
cudaError_t launch_modelc_tile_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, int minb, unsigned* work, cudaStream_t s);
cudaError_t launch_modelc_tile_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                   const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                   int rows, int minb, unsigned* work, cudaStream_t s);
// The multi-grain step (lg_modelc.cu, lg_modelc_f32.cu): the strip schedule
// with every cell's four faces in its own crystal frame; `trig` holds cos
// theta0 of the ncells interior cells (blocks in order, dimension 0 fastest)
// then sin theta0, in the state's element type.  FP64 is bit-identical to
// the reference's apply_oriented path.
cudaError_t launch_modelc_oriented_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                       const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                       const double* trig, int64_t ncells, int rows, cudaStream_t s);
cudaError_t launch_modelc_oriented_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                       const ModelCDev& m, double dt, const NoiseDev& nz, double* tdev, int slot,
                                       const float* trig, int64_t ncells, int rows, cudaStream_t s);

// One RungeKutta4 stage of Model C without noise (rk4.rs:40-79) on the
// strip schedule: mode 1 writes the drift of `in` to k and y + c k to out;
// mode 2 writes (((y + s6 k1) + s3 k2) + s3 k3) + s6 k4 to out.  trig
// (cos then sin theta0, or null) selects the multi-grain form.  FP64 is
// bit-identical to the reference's stages.
cudaError_t launch_modelc_rk_stage_f64(int mode, const double* in, double* out, const CartTopo& topo,
                                       const SlabLayout& L, const ModelCDev& m, const double* y, double* k,
                                       const double* k1, const double* k2, const double* k3, double c, double s6,
                                       double s3, const double* trig, int64_t ncells, double* tdev, int slot,
                                       double dt, cudaStream_t s);
cudaError_t launch_modelc_rk_stage_f32(int mode, const float* in, float* out, const CartTopo& topo,
                                       const SlabLayout& L, const ModelCDev& m, const float* y, float* k,
                                       const float* k1, const float* k2, const float* k3, double c, double s6,
                                       double s3, const float* trig, int64_t ncells, double* tdev, int slot,
                                       double dt, cudaStream_t s);

// Batched instances (an ensemble of independent grids of one geometry):
// block b of the topology belongs to instance b / bpi, with the parameter
// record params[instance] (built by modelc_record_*) and Wiener seed
// seeds[instance]; noise keys use the instance-local block index.
size_t modelc_record_size_f64();
void modelc_record_f64(const ModelCDev& m, void* out);
size_t modelc_record_size_f32();
void modelc_record_f32(const ModelCDev& m, void* out);
cudaError_t launch_modelc_batch_f64(const double* in, double* out, const CartTopo& topo, const SlabLayout& L,
                                    const void* params, const uint64_t* seeds, int bpi, double dt, double amp,
                                    double* tdev, int slot, int rows, cudaStream_t s);
cudaError_t launch_modelc_batch_f32(const float* in, float* out, const CartTopo& topo, const SlabLayout& L,
                                    const void* params, const uint64_t* seeds, int bpi, double dt, double amp,
                                    double* tdev, int slot, int rows, cudaStream_t s);

// Standard normals of a key array (tests of the generator).
cudaError_t launch_standard_normal(const uint64_t* keys, double* out, int64_t n, cudaStream_t s);

}  // namespace lg
