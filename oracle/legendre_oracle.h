/* legendre oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * C interface of the CPU restatement of the reference's SerialScheduler path
 * (see legendre_oracle.cpp for the file:line each function follows).  Loaded
 * by the tests, by __graft_entry__.smoke() and by bench.py's CPU baseline leg
 * only; the product library never links or calls it.
 */
#ifndef LEGENDRE_ORACLE_H
#define LEGENDRE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ModelC public fields (src/physics/phasefield.rs:55-66) plus the flux
 * policy's regularisation threshold (FiniteVolume::tol,
 * src/discretization/finite_volume.rs:41-50). */
typedef struct orc_modelc_params {
    double eps4;
    double lambda;
    double d_thermal;
    double noise_amplitude;
    double anisotropy_tol;
    double flux_tol;
} orc_modelc_params;

uint64_t orc_splitmix64(uint64_t z);
uint64_t orc_mix_key(uint64_t seed, const uint64_t* parts, int64_t n);
double orc_unit_open(uint64_t bits);
double orc_standard_normal(uint64_t key);
void orc_standard_normal_batch(const uint64_t* keys, int64_t n, double* out);

void* orc_grid_create(int D, const int64_t* cells, const int64_t* block, const double* origin,
                      const double* spacing, const int* periodic);
void orc_grid_destroy(void* g);
int64_t orc_grid_num_blocks(const void* g);
int64_t orc_grid_block_len(const void* g, int ghost);
int64_t orc_grid_face_neighbor(const void* g, int64_t b, int dim, int dir);
void orc_grid_cell_center(const void* g, int64_t b, const int64_t* idx, double* out);
int orc_grid_cell_key(const void* g, int ghost, int64_t offset, uint64_t* key);

void* orc_state_create(const void* grid, int nfields, const int* ghosts);
void orc_state_destroy(void* s);
void orc_state_set_field(void* s, int f, const double* data);
void orc_state_get_field(const void* s, int f, double* data);

void orc_fill_ghosts_mirror(const void* grid, void* s, int f);
double orc_heat_run(const void* grid, void* s, int f, double kappa, double t0, double dt, int64_t steps,
                    int nthreads);
double orc_modelc_run(const void* grid, void* s, const orc_modelc_params* p, double t0, double dt, uint64_t seed,
                      int64_t steps, int wiener, int nthreads);
void orc_modelc_drift(const void* grid, void* s, const orc_modelc_params* p, double* kphi_out, double* ku_out);
void orc_modelc_initialize_grains(const void* grid, void* s, const double* grains, int64_t n, double u0);
/* the multi-grain form: theta0 in field `theta_field` (ghost width 0) */
double orc_modelc_run_oriented(const void* grid, void* s, const orc_modelc_params* p, int theta_field, double t0,
                               double dt, uint64_t seed, int64_t steps, int wiener, int nthreads);
void orc_modelc_initialize_orientations(const void* grid, void* s, int theta_field, const double* grains,
                                        int64_t n);
/* RungeKutta4 (rk4.rs:40-79): heat on field f, Model C without noise */
double orc_heat_run_rk4(const void* grid, void* s, int f, double kappa, double t0, double dt, int64_t steps,
                        int nthreads);
double orc_modelc_run_rk4(const void* grid, void* s, const orc_modelc_params* p, int theta_field, double t0,
                          double dt, int64_t steps, int nthreads);
int orc_num_threads_available(void);

#ifdef __cplusplus
}
#endif
#endif
