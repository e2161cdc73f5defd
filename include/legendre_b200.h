/* legendre_b200 -- C ABI of the B200 block-stepping library.
 *
 * The reference (trbritt/legendre 0.1.4, Rust) has no FFI of its own: its
 * device seam is two traits, `Scheduler` (src/core/scheduler.rs:25-38) and
 * `Allocator`/`StorageBackend` (src/core/storage.rs:126-154).  A
 * `CudaScheduler` cannot carry device work through `for_each_block_mut`
 * (its closure is opaque host code), so the device path enters at
 * integrator-step granularity and at the storage seam.  The entry points
 * below are exactly what a Rust `CudaScheduler` / `CudaAllocator` /
 * device-integrator wrapper binds; each comment names the reference
 * interface it replaces.
 *
 * Conventions
 *  - Every function returns an int status: LG_OK (0) or a negative LG_ERR_*;
 *    lg_last_error(ctx) gives the text of the last failure on that context.
 *  - All device work of a context runs in order on its one stream; calls on
 *    one context are not re-entrant (one host thread per context).
 *  - Host arrays are plain pointers + element counts; nothing here takes
 *    PyTorch or CUDA-runtime C++ types.
 *  - Field data crosses the boundary in the reference's layout: for each
 *    block in BlockId order, the field's ghost-inclusive slab, dimension 0
 *    fastest (src/geometry/cartesian.rs:8-11).
 */
#ifndef LEGENDRE_B200_H
#define LEGENDRE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LG_ABI_VERSION 1

enum lg_status {
    LG_OK = 0,
    LG_ERR_INVALID = -1,   /* bad argument (the reference panics or returns GridError) */
    LG_ERR_CUDA = -2,      /* a CUDA runtime call failed */
    LG_ERR_NOMEM = -3,     /* device allocation failed */
    LG_ERR_TIMEOUT = -4,   /* lg_sync gave up waiting */
    LG_ERR_STATE = -5,     /* call out of order (e.g. wrong dtype or field) */
    LG_ERR_DEVICE = -6     /* a kernel reported a device-side error flag */
};

enum lg_dtype { LG_F64 = 0, LG_F32 = 1 };

/* Run flags. */
#define LG_RUN_GRAPH 1u      /* capture the step sequence once in a CUDA graph and replay it */
#define LG_RUN_PERSISTENT 2u /* AMR: every phase of a coarse step in one cooperative launch */

typedef struct lg_ctx lg_ctx;
typedef struct lg_grid lg_grid;
typedef struct lg_state lg_state;

/* ---------------------------------------------------------------- context
 * The `CudaScheduler` itself: device, stream, error text.  Replaces
 * `SerialScheduler`/`RayonScheduler` (src/core/scheduler.rs:39-84) as the
 * type-level selector of the device path.  `stream` may be NULL (the
 * context creates its own) or an existing cudaStream_t to run on. */
int lg_abi_version(void);
int lg_ctx_create(int device, void* stream, lg_ctx** out);
int lg_ctx_destroy(lg_ctx* ctx);
const char* lg_last_error(const lg_ctx* ctx);
/* Wait for all work of the context; LG_ERR_TIMEOUT after timeout_ms (< 0: no limit). */
int lg_sync(lg_ctx* ctx, int64_t timeout_ms);
/* Number of kernels this context has launched (its own kernels only). */
int64_t lg_ctx_kernel_launches(const lg_ctx* ctx);

/* ------------------------------------------------------------------- grid
 * Device block-topology table of a `CartesianGrid<D>`
 * (src/geometry/cartesian.rs:48-97): D <= 3, cells[d] % block[d] == 0,
 * spacing > 0 (CartesianGrid::new errors -> LG_ERR_INVALID); periodic[d]
 * is `with_periodic`.  Face neighbours follow `face_neighbor`
 * (cartesian.rs:162-181). */
int lg_grid_create_cartesian(lg_ctx* ctx, int D, const int64_t* cells, const int64_t* block_cells,
                             const double* origin, const double* spacing, const int* periodic, lg_grid** out);
int lg_grid_destroy(lg_grid* grid);
int64_t lg_grid_num_blocks(const lg_grid* grid);
/* Neighbour of `block` across face (dim, dir = -1/+1); *out = -1 at a physical boundary. */
int lg_grid_face_neighbor(const lg_grid* grid, int64_t block, int dim, int dir, int64_t* out);

/* ------------------------------------------------------------------ state
 * The `CudaAllocator`: one device arena per state, block-major slabs, zero
 * initialised (replaces StateBuilder::build / BlockStorage::allocate,
 * src/core/state.rs:207-264, and SystemAllocator, storage.rs:177-189).
 * Field f has ghost width ghosts[f] <= every block extent
 * (cartesian.rs:456-462).  The arena is double-buffered: steps read one
 * copy and write the other, which stands in for the reference's stage
 * buffers (simulation.rs:187-202). */
int lg_state_create(lg_ctx* ctx, const lg_grid* grid, int dtype, int nfields, const int* ghosts, lg_state** out);
int lg_state_destroy(lg_state* st);
/* Host <-> device copies of one field, every block, ghost-inclusive slabs in
 * BlockId order (`State::slab`/`slab_mut`, state.rs:413-424).  `nelem` must
 * equal num_blocks * block_len(ghost).  Uploading marks ghosts stale; the
 * next step refills them first. */
int lg_state_upload_field(lg_state* st, int field, const void* host, int64_t nelem);
int lg_state_download_field(lg_state* st, int field, void* host, int64_t nelem);
/* Device address and length of one slab of the current buffer
 * (`StorageBackend::as_slice`, storage.rs:126-138, on device memory). */
int lg_state_slab(lg_state* st, int64_t block, int field, void** dev, int64_t* len);
/* `Simulation::time` / its step counter (simulation.rs:225-233). */
int lg_state_get_time(const lg_state* st, double* t, int64_t* step_index);
int lg_state_set_time(lg_state* st, double t, int64_t step_index);

/* -------------------------------------------------------------- kernels */

/* (b) Ghost fill of one field: halo exchange, periodic wrap and mirror
 * (no-flux) boundaries -- `fill_ghosts_mirror` (cartesian.rs:392-401,
 * 439-526; FaceBc::Mirror, boundary.rs:63-66).  Result identical to the
 * reference's dimension sweep, corners included. */
int lg_fill_ghosts(lg_state* st, int field);

/* (d) `nsteps` forward-Euler steps of the heat model `Heat<D>`
 * (examples/heat3d.rs:41-85, tests/heat3d.rs:33-80): u += dt * (kappa *
 * CentralLaplacian(u)) (finite_difference.rs:49-67, euler.rs:28-54).  The
 * field must have ghost width 1.  Advances the state's time by dt per step. */
int lg_heat_fe_run(lg_state* st, int field, double kappa, double dt, int64_t nsteps, uint32_t flags);

/* Model C parameters: the public fields of `ModelC`
 * (src/physics/phasefield.rs:55-66) and `FiniteVolume::tol`
 * (finite_volume.rs:41-50).  noise_amplitude != 0 selects
 * `ModelC<Wiener<1>>`, 0 selects `ModelC<NoNoise>`. */
typedef struct lg_modelc_params {
    double eps4;
    double lambda;
    double d_thermal;
    double noise_amplitude;
    double anisotropy_tol;
    double flux_tol;
} lg_modelc_params;

/* (a) `nsteps` Euler-Maruyama steps of Model C on a 2-D Cartesian state with
 * fields phi (0) and u (1), ghost 1 -- EulerMaruyama::step
 * (src/integrators/euler_maruyama.rs:34-75) with
 * ModelC::vector_field_block (phasefield.rs:353-422), fill_ghosts
 * (phasefield.rs:431-439) and State::apply_step_with (state.rs:656-699) in
 * one fused kernel per step.  The noise salt of each step is the bit
 * pattern of the state's time before the step; `seed` is
 * `EulerMaruyama::seed`.  FP64 states are bit-identical to the reference
 * without noise; with noise the integer key stream is exact and the
 * Gaussian is within 1e-12 relative.  `variant` selects a kernel shape
 * (0 = library default). */
int lg_modelc_em_run(lg_state* st, const lg_modelc_params* p, double dt, uint64_t seed, int64_t nsteps,
                     int variant, uint32_t flags);
/* Autotuner of the fused Model C step: times every strip-kernel variant
 * (2, 3 or 4 CTAs per SM by register budget x strip heights chosen by the
 * library, 8, 16 or 32 rows) for `trial_steps` steps from a copy of the
 * state, restores the state, its time and step index, and remembers the
 * fastest for this context, block shape, block count, element type and noise
 * setting: lg_modelc_em_run with variant 0 then uses it.  Returns it in
 * *best_variant and its time per step in *best_ms (if non-null).  No
 * counterpart in the reference, whose block size is the user's only knob. */
int lg_modelc_autotune(lg_state* st, const lg_modelc_params* p, double dt, uint64_t seed, int trial_steps,
                       int* best_variant, double* best_ms);

/* Initial conditions, computed on the host exactly as the reference does and
 * uploaded.  `ModelC::initialize_grains` without orientations
 * (phasefield.rs:227-314): grains = n x (cx, cy, radius, orientation). */
int lg_modelc_initialize_grains(lg_state* st, const double* grains, int64_t n, double u0);
/* Multi-grain Model C (ModelC::with_orientations, phasefield.rs:118-125):
 * theta0 is a static field of ghost width 0 beyond phi and u.
 * lg_modelc_set_orientations takes theta0 from field `theta_field` of the
 * state (copying it into both step buffers) and computes cos and sin theta0
 * of every cell on the host, as the reference's sin_cos; from then on
 * lg_modelc_em_run steps the oriented form, each cell's four faces with
 * their anisotropy in its crystal frame (finite_volume.rs:178-235).  A
 * negative theta_field returns to the axis-aligned step.
 * lg_modelc_initialize_orientations writes theta0 by the nearest-seed
 * Voronoi rule of initialize_grains (phasefield.rs:286-311; grains as x, y,
 * radius, orientation) and sets it. */
int lg_modelc_set_orientations(lg_state* st, int theta_field);
int lg_modelc_initialize_orientations(lg_state* st, int theta_field, const double* grains, int64_t n);
/* RungeKutta4 (src/integrators/rk4.rs:22-79): classic fourth-order steps of
 * the heat model on `field` (any dimension, FP64) and of Model C (2-D,
 * axis-aligned or multi-grain, FP64 or FP32), deterministic models only (the
 * reference pairs RK4 with NoNoise): a non-zero noise amplitude is refused.
 * Each step is four stage launches, k_i of the stage input written beside
 * y + c_i k_i, the last one applying y += dt/6 k1, dt/3 k2, dt/3 k3, dt/6 k4
 * in the reference's order; FP64 is bit-identical to the reference.  The
 * first run allocates five more arenas of the state's size. */
int lg_heat_rk4_run(lg_state* st, int field, double kappa, double dt, int64_t nsteps, uint32_t flags);
int lg_modelc_rk4_run(lg_state* st, const lg_modelc_params* p, double dt, int64_t nsteps, uint32_t flags);
/* Heat initial condition of the 96^3 benchmark: sin(2 pi x) sin(2 pi y)
 * sin(2 pi z) + amp * (2 * unit_open(mix_key(seed, [gx, gy, gz])) - 1) at
 * cell centres (gx.. = global cell index); the reference has no such
 * helper, it is a `fill_from_fn` closure (cartesian.rs:546-559). */
int lg_heat_initialize_sine_noise(lg_state* st, int field, uint64_t seed, double amp);

/* ------------------------------------------------------------------ AMR
 * A 2-D Berger-Oliger simulation on a patch hierarchy: `AmrGrid<2>`
 * (src/geometry/amr/grid.rs:55-279) with its state, the `Subcycling`
 * integrator (src/integrators/subcycling.rs:48-268) or a global-dt
 * Euler-Maruyama, and optionally the `BergerOliger` adaptivity policy
 * (src/geometry/amr/adapt.rs:131-237), as `Simulation::adaptive` owns them
 * (src/core/simulation.rs:137-183).  Ghost fill, restriction, tagging and
 * the per-level steps run on the device; clustering (cluster.rs:144-290)
 * and migration (adapt.rs:323-402) run on the host at regrid cadence.
 * Fields have ghost width 1 (the models of the path).  FP64. */
typedef struct lg_amr_sim lg_amr_sim;

enum lg_model { LG_MODEL_HEAT = 0, LG_MODEL_C = 1 };
enum lg_amr_integrator { LG_AMR_SUBCYCLING = 0, LG_AMR_GLOBAL_DT = 1 };

/* RegridPolicy + ClusterParams + GradientTagger (adapt.rs:48-129,
 * cluster.rs:115-135); `field` is the tagged field's index. */
typedef struct lg_amr_policy {
    int64_t every;
    int64_t buffer;
    int64_t min_width;
    double efficiency;
    double threshold;
    int field;
} lg_amr_policy;

/* Base grid (cells, block, origin, spacing; 2 entries each), refinement
 * ratios, and initial patches as npatches x (level, lo_x, lo_y, hi_x, hi_y)
 * in their level's cell coordinates (AmrGrid::from_patches,
 * amr/grid.rs:90-196: invalid hierarchies -> LG_ERR_INVALID).
 * model LG_MODEL_C uses *mp; LG_MODEL_HEAT uses kappa (the heat model of
 * tests/amr.rs:297-345).  policy NULL = the Static policy. */
int lg_amr_sim_create(lg_ctx* ctx, const int64_t* cells, const int64_t* block, const double* origin,
                      const double* spacing, const uint32_t* ratios, int nratios, const int64_t* patches,
                      int64_t npatches, int model, const lg_modelc_params* mp, double kappa, int integrator,
                      uint64_t seed, const lg_amr_policy* policy, lg_amr_sim** out);
int lg_amr_sim_destroy(lg_amr_sim* sim);
/* Blocks (patches), populated levels, grid epoch (simulation.rs:210-213). */
int lg_amr_sim_info(const lg_amr_sim* sim, int64_t* num_blocks, int* num_levels, int64_t* epoch);
/* Patch of a block: (level, lo_x, lo_y, hi_x, hi_y) (AmrGrid::patch). */
int lg_amr_sim_patch(const lg_amr_sim* sim, int64_t block, int64_t* out5);
/* Field data: every block's ghost-inclusive slab in BlockId order. */
int lg_amr_sim_field_len(const lg_amr_sim* sim, int64_t* nelem);
int lg_amr_sim_get_field(lg_amr_sim* sim, int field, double* host, int64_t nelem);
int lg_amr_sim_set_field(lg_amr_sim* sim, int field, const double* host, int64_t nelem);
int lg_amr_sim_time(const lg_amr_sim* sim, double* t, int64_t* step_index);
/* Integrator::suggested_dt (integrators/mod.rs:218-223, subcycling.rs:54-61). */
int lg_amr_sim_suggested_dt(const lg_amr_sim* sim, double* dt);
/* `nsteps` of Simulation::step(dt) (simulation.rs:255-290): regrid at the
 * policy's cadence, then one coarse step.  LG_RUN_GRAPH replays pairs of
 * coarse steps between regrids from a captured CUDA graph.
 * LG_RUN_PERSISTENT runs every phase of a pair of coarse steps (each
 * level's fused ghost fill + step, each restriction) in one cooperative
 * launch whose CTAs meet at grid barriers; a barrier wait is bounded, and
 * if one gives up the call returns LG_ERR_TIMEOUT and the state is invalid.
 * It takes precedence over LG_RUN_GRAPH. */
int lg_amr_sim_step(lg_amr_sim* sim, double dt, int64_t nsteps, uint32_t flags);
/* Polls (each of at least 128 ns) a grid barrier of the LG_RUN_PERSISTENT
 * launch waits for the other CTAs before it gives up and the step returns
 * LG_ERR_TIMEOUT (default 4,000,000: over a second).  No counterpart in the
 * reference, whose Rayon scheduler has no device waits; a watchdog knob,
 * and the way to make a barrier give up at once (0) to exercise the
 * timeout path without any fault. */
int lg_amr_sim_set_barrier_spin_limit(lg_amr_sim* sim, int64_t polls);
/* (c) transfers on the current state: `restrict` (intergrid.rs:97-105) of
 * one field, finest level first; `fill_ghosts_mirror` of every level
 * (intergrid.rs:155-168); `GradientTagger::tag_level` (adapt.rs:78-103),
 * flagged cells sorted, *count = total (cells_out holds min(total, cap)). */
int lg_amr_restrict(lg_amr_sim* sim, int field);
int lg_amr_fill_ghosts(lg_amr_sim* sim);
int lg_amr_tag_level(lg_amr_sim* sim, int field, int level, double threshold, int64_t* cells_out, int64_t cap,
                     int64_t* count);
/* lg_amr_tag_level without any allocation.  No counterpart in the reference:
 * it serves callers that cannot allocate device memory (a step loop whose
 * memory a caching allocator holds, or a latency-bound loop that a
 * synchronising cudaMalloc/cudaFree would stall).  The flags are compacted in
 * a static device scratch of 2^18 cells (4 MiB) and sorted in place in
 * cells_out.  Fails with LG_ERR_INVALID when the level has more than 2^18
 * cells, or when cap < *count (nothing copied, *count set).  Calls that
 * overlap on the GPU race on the scratch.  Every call synchronises the
 * context's stream (the flag count is read back), so it must not be called
 * while that stream is being captured.  The first call on a device resolves
 * the scratch's address and caches it: not valid across a cudaDeviceReset.
 * Only the error paths allocate (a host message string). */
int lg_amr_tag_level_static(lg_amr_sim* sim, int field, int level, double threshold, int64_t* cells_out,
                            int64_t cap, int64_t* count);
/* Berger-Rigoutsos clustering of flagged cells, `cluster` (amr/cluster.rs:
 * 144-290): flags are nflags (x, y) pairs of one level, in any order (the
 * boxes do not depend on it; flags must not repeat); *nboxes receives the number of boxes,
 * boxes the first min(cap, *nboxes) as (lo_x, lo_y, hi_x, hi_y), half-open.
 * efficiency in (0, 1], min_width >= 1 (LG_ERR_INVALID otherwise).  Host
 * only: it needs no device and no context; the regrid uses the same code. */
int lg_amr_cluster(const int64_t* flags, int64_t nflags, double efficiency, int64_t min_width, int64_t* boxes,
                   int64_t cap, int64_t* nboxes);
/* `AmrGrid::from_patches` validation (amr/grid.rs:90-196) of a 2-D
 * hierarchy: base cells and block as for lg_amr_sim_create, patches as
 * (level, lo_x, lo_y, hi_x, hi_y) rows.  LG_OK, or LG_ERR_INVALID with the
 * reason (the GridError) in err (NUL-terminated, at most errlen bytes).
 * The same check lg_amr_sim_create and every regrid run; host only. */
int lg_amr_check_hierarchy(const int64_t* cells, const int64_t* block, const uint32_t* ratios, int nratios,
                           const int64_t* patches, int64_t npatches, char* err, int64_t errlen);

/* ----------------------------------------------------------- ensembles --
 * Batched Model C: `ninst` independent instances of one 2-D grid geometry
 * (cells[2] in blocks of block[2], spacing[2], zero-flux boundaries), each
 * with its own eps4 and Wiener seed, sharing lambda, D, the noise amplitude
 * and the tolerances of `p`.  No counterpart in the reference, which runs
 * one Simulation per realisation; each instance's trajectory is the one its
 * own Simulation (lg_modelc_em_run on the same grid) produces -- bit for bit
 * in FP64.  Host arrays are instance-major, then row-major (x fastest):
 * n = ninst * cells[0] * cells[1]. */
typedef struct lg_ensemble lg_ensemble;
int lg_ensemble_create(lg_ctx* ctx, const int64_t* cells, const int64_t* block, const double* spacing, int64_t ninst,
                       const lg_modelc_params* p, const double* eps4, const uint64_t* seeds, int dtype,
                       lg_ensemble** out);
int lg_ensemble_destroy(lg_ensemble* e);
int lg_ensemble_upload(lg_ensemble* e, int field, const double* host, int64_t n);
int lg_ensemble_download(lg_ensemble* e, int field, double* host, int64_t n);
int lg_ensemble_set_time(lg_ensemble* e, double t, int64_t step_index);
int lg_ensemble_get_time(const lg_ensemble* e, double* t, int64_t* step_index);
/* `nsteps` Euler-Maruyama steps of every instance (LG_RUN_GRAPH: pairs of
 * steps replayed from a CUDA graph). */
int lg_ensemble_run(lg_ensemble* e, double dt, int64_t nsteps, uint32_t flags);
/* Differentiation.  From the current state x_0, runs `nsteps` steps storing
 * the state every `ckpt_every` steps, evaluates
 * L_i = sum over the cells of (phi_T - target)^2 per instance, and runs the
 * hand-written adjoint of the fused step back to x_0, recomputing each
 * segment from its checkpoint (the noise replays from its keys).  Returns
 * loss[i], grad_params[4 i + k] = dL_i/d(lambda, D, eps4, Delta) -- Delta
 * taken as the undercooling of an initial u = -Delta on every cell -- and,
 * when non-null, dL_i/dphi_0 and dL_i/du_0 per cell.  The state is left at
 * x_T.  Parameter gradients accumulate in FP64 (FP32 ensembles included). */
int lg_ensemble_value_and_grad(lg_ensemble* e, double dt, int64_t nsteps, int64_t ckpt_every, const double* target,
                               double* loss, double* grad_params, double* grad_phi0, double* grad_u0);
/* The backward API of one Simulation (north of `Simulation::step`,
 * simulation.rs:255-290; the reference has no adjoint): the same
 * differentiation for a 2-D zero-flux Model C state of phi and u (ghost 1)
 * stepped by Euler-Maruyama with `p` and Wiener `seed` from the state's
 * current time.  target, grad_phi0 and grad_u0 are row-major over the whole
 * grid (x fastest, cells[0] * cells[1] values); loss[0] and grad_params[0..3]
 * = dL/d(lambda, D, eps4, Delta), Delta shifting the initial u by -Delta on
 * every cell.  The state is left at x_T with its time advanced, as after
 * lg_modelc_em_run of nsteps.  LG_ERR_STATE for other states. */
int lg_modelc_value_and_grad(lg_state* state, const lg_modelc_params* p, double dt, uint64_t seed, int64_t nsteps,
                             int64_t ckpt_every, const double* target, double* loss, double* grad_params,
                             double* grad_phi0, double* grad_u0);
/* The form of the step adjoint value_and_grad runs: LG_ADJOINT_STRIP (warp
 * strips walking up the rows; the default) or LG_ADJOINT_TILE (shared-memory
 * tiles with a two-cell halo).  Both give the same gradients up to rounding. */
#define LG_ADJOINT_STRIP 0
#define LG_ADJOINT_TILE 1
int lg_ensemble_set_adjoint_kernel(lg_ensemble* e, int kernel);
/* Device bytes value_and_grad may spend on a resident tail: the last
 * segments whose every state fits are kept from the forward pass instead of
 * being recomputed from their checkpoints (the gradients are the same bits).
 * 0, the default, is pure checkpointing; 0 also frees the kept states.  The
 * budget is taken as given: it must fit in the free device memory beside the
 * checkpoints and recomputed states, or value_and_grad returns LG_ERR_NOMEM
 * (a caller sizes it from cudaMemGetInfo less a margin). */
int lg_ensemble_set_resident_budget(lg_ensemble* e, uint64_t bytes);

/* ---- Observation: snapshots off the stepping stream --------------------
 * The device side of AsyncObserver (src/core/observer.rs:65-165): a ring of
 * `nslots` snapshot slots of a state, each a device buffer and a pinned host
 * buffer holding the interior cells of the chosen fields (1 to 8) in the row
 * order of the reference's Parquet snapshots (src/io/parquet.rs:150-215):
 * blocks in order, each block's interior cells dimension-0-fastest, one
 * column of `rows` FP64 values per field (FP32 states are widened).
 *
 * lg_snapshot_ring_capture gathers the state as it stands after the work
 * already enqueued on the state's stream into a free slot (one kernel on
 * that stream) and copies the slot to the host on a stream of the ring's own
 * after an event, so the stepping stream never waits for the host.  The
 * calling thread first waits until the device has gathered the previous
 * capture, so it runs at most one snapshot interval ahead of the device while
 * the device keeps the work already enqueued.  With no free slot (the
 * consumer has not finished with the earlier snapshots) it drops the
 * snapshot and sets *slot = -1, as the reference's observer drops rather
 * than blocks (observer.rs:17-25, 149-156).
 * lg_snapshot_ring_poll hands out the oldest captured snapshot whose copy
 * has finished, waiting up to timeout_ms (0: just look; LG_ERR_TIMEOUT if
 * none); the caller reads `columns` (nfields x rows doubles) and gives the
 * slot back with lg_snapshot_ring_release.  capture runs on the thread that
 * steps the state; poll and release may run on another thread.  The state
 * must outlive the ring. */
typedef struct lg_snapshot_ring lg_snapshot_ring;
int lg_snapshot_ring_create(lg_state* st, const int* fields, int nfields, int nslots, lg_snapshot_ring** out);
int lg_snapshot_ring_destroy(lg_snapshot_ring* r);
int lg_snapshot_ring_capture(lg_snapshot_ring* r, int64_t step, double t, int64_t epoch, int* slot);
int lg_snapshot_ring_poll(lg_snapshot_ring* r, int timeout_ms, int* slot, int64_t* step, double* t, int64_t* epoch,
                          const double** columns);
int lg_snapshot_ring_release(lg_snapshot_ring* r, int slot);
int lg_snapshot_ring_stats(lg_snapshot_ring* r, int64_t* captured, int64_t* dropped, int64_t* rows);
/* Cell centres of a Cartesian grid in the same row order, one column of
 * cells[0] x ... x cells[D-1] values per dimension: (block origin cell +
 * index + 0.5) * spacing + origin as one fused multiply-add, the reference's
 * cell_center (src/geometry/cartesian.rs:589-597).  Host only: it needs no
 * device and no context. */
int lg_cell_centers(int D, const int64_t* cells, const int64_t* block_cells, const double* origin,
                    const double* spacing, double* out);
/* FP64 sum of one field over every block's interior cells of the current
 * state (values widened from the state's precision), in a fixed order: per
 * block, 256 strided partial sums joined by a fixed shuffle tree and the
 * warps in order; then the blocks in index order.  The same state gives the
 * same bits.  Model C's enthalpy is h^D (sum u - sum phi / 2); with no noise
 * and periodic or zero-flux boundaries a step changes it only by rounding
 * (du/dt = D lap u + dphi/dt / 2, phasefield.rs:353-422).  The reference has
 * no such reduction.  Waits for the context's stream. */
int lg_state_field_sum(lg_state* st, int field, double* sum);

/* Standard normals of n keys on the device (`rng::standard_normal`,
 * src/util/rng.rs:43-49); host arrays in and out. */
int lg_standard_normal(lg_ctx* ctx, const uint64_t* keys, int64_t n, double* out);

/* Compute-side roofline denominators, measured on the context's device (no
 * counterpart in the reference, which publishes no device figures):
 * retired operations per second, over all SMs, of independent chains of
 * FP64 FMAs, FP32 FMAs, 32-bit integer multiply-adds and plain 32-bit ALU
 * operations (xor, add) at full occupancy; best of three ~ms-long launches
 * timed with CUDA events.  Waits for the context's stream. */
typedef struct lg_compute_peaks {
    double dfma_per_s;
    double ffma_per_s;
    double imad_per_s;
    double alu_per_s;
    int32_t sms;
    double clock_mhz;  /* the device's reported maximum SM clock */
} lg_compute_peaks;
int lg_measure_compute_peaks(lg_ctx* ctx, lg_compute_peaks* out);

#ifdef __cplusplus
}
#endif
#endif
