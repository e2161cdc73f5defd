// legendre oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A serial CPU restatement of the reference's `SerialScheduler` path for the
// block-stepping hot path (trbritt/legendre 0.1.4, Rust).  It exists only to
// check the CUDA library: the tests, `__graft_entry__.smoke()` and the CPU
// baseline leg of `bench.py` may call it; nothing in the product links it.
//
// Bit-exactness rules (the reference is Rust, which never contracts a*b+c):
//   * compiled with -ffp-contract=off,
//   * std::fma exactly where the reference calls `f64::mul_add`,
//   * the reference's operand order, left-to-right evaluation of a-b+c-d,
//   * glibc log/cos/sqrt/tanh/hypot (what Rust's f64 methods call on
//     linux-gnu).
// Each function names the reference file:line it restates.
//
// OpenMP (optional `nthreads`) parallelises only the per-block dispatches,
// mirroring `RayonScheduler` (src/core/scheduler.rs:65-84): blocks are
// disjoint, so results are identical for every thread count.

#include <limits>

#include "oracle_core.hpp"

namespace {

using namespace orc;

// --------------------------------------------------------- Cartesian ------
// src/geometry/cartesian.rs:28-187
struct Grid {
    int D;
    int64_t cells[3], block[3], nb[3];
    double origin[3], spacing[3];
    bool periodic[3];

    int64_t num_blocks() const {
        int64_t n = 1;
        for (int d = 0; d < D; ++d) n *= nb[d];
        return n;
    }
    int64_t ghosted(int d, int g) const { return block[d] + 2 * g; }
    int64_t block_len(int g) const {
        int64_t n = 1;
        for (int d = 0; d < D; ++d) n *= ghosted(d, g);
        return n;
    }
    // cartesian.rs:145-154
    void block_coords(int64_t b, int64_t* out) const {
        int64_t rem = b;
        for (int d = 0; d < D; ++d) { out[d] = rem % nb[d]; rem /= nb[d]; }
    }
    // cartesian.rs:162-181 ; -1 for a non-periodic domain boundary
    int64_t face_neighbor(int64_t b, int dim, int dir) const {
        int64_t c[3];
        block_coords(b, c);
        int64_t stepped = c[dim] + (dir < 0 ? -1 : 1);
        int64_t next;
        if (stepped >= 0 && stepped < nb[dim]) next = stepped;
        else if (periodic[dim]) next = ((stepped % nb[dim]) + nb[dim]) % nb[dim];
        else return -1;
        int64_t id = 0, stride = 1;
        for (int d = 0; d < D; ++d) {
            id += (d == dim ? next : c[d]) * stride;
            stride *= nb[d];
        }
        return id;
    }
    // cartesian.rs:189-204
    int64_t linearize(const int64_t* idx, int g) const {
        int64_t off = 0, stride = 1;
        for (int d = 0; d < D; ++d) {
            off += (idx[d] + g) * stride;
            stride *= block[d] + 2 * g;
        }
        return off;
    }
    // cartesian.rs:588-597
    void cell_center(int64_t b, const int64_t* idx, double* out) const {
        int64_t c[3];
        block_coords(b, c);
        for (int d = 0; d < D; ++d) {
            int64_t global = c[d] * block[d];
            out[d] = std::fma(((double)global + (double)idx[d]) + 0.5, spacing[d], origin[d]);
        }
    }
    // cartesian.rs:599-619 ; returns false for a ghost entry
    bool cell_key(int g, int64_t offset, uint64_t* key) const {
        int64_t rem = offset, k = 0, stride = 1;
        for (int d = 0; d < D; ++d) {
            int64_t gh = block[d] + 2 * g;
            int64_t c = rem % gh;
            rem /= gh;
            if (c < g || c >= block[d] + g) return false;
            k += (c - g) * stride;
            stride *= block[d];
        }
        *key = (uint64_t)k;
        return true;
    }
};

template <class F>
void for_each_interior(const Grid& g, F f) {
    int64_t lo[3] = {0, 0, 0};
    for_each_box(g.D, lo, g.block, f);
}

Ext ext_of(const Grid& g) {
    Ext e;
    e.D = g.D;
    for (int d = 0; d < 3; ++d) e.n[d] = g.block[d];
    return e;
}

// Block-major state: blocks x fields, each slab ghost-inclusive
// (src/core/state.rs:219-296).  A zero-length slab marks a field the buffer
// does not carry (state.rs:237-264).
struct State {
    std::vector<int> ghost;
    std::vector<std::vector<std::vector<double>>> slab;  // [block][field]
};

State make_state(const Grid& g, const std::vector<int>& ghosts, const std::vector<bool>& keep) {
    State s;
    s.ghost = ghosts;
    s.slab.resize(g.num_blocks());
    for (auto& b : s.slab) {
        b.resize(ghosts.size());
        for (size_t f = 0; f < ghosts.size(); ++f)
            if (keep[f]) b[f].assign(g.block_len(ghosts[f]), 0.0);
    }
    return s;
}

// cartesian.rs:439-526 with FaceBc::Mirror (boundary.rs:63-66)
void fill_ghosts_mirror(const Grid& grid, State& st, int f) {
    int g = st.ghost[f];
    if (g == 0) return;
    const int D = grid.D;
    for (int d = 0; d < D; ++d) {
        int64_t n = grid.block[d];
        int64_t lo[3], hi[3];
        for (int e = 0; e < D; ++e) { lo[e] = -g; hi[e] = grid.block[e] + g; }
        for (int64_t b = 0; b < grid.num_blocks(); ++b) {
            for (int dir : {-1, 1}) {
                if (dir < 0) { lo[d] = -g; hi[d] = 0; }
                else { lo[d] = n; hi[d] = n + g; }
                int64_t nbk = grid.face_neighbor(b, d, dir);
                std::vector<double>& dst = st.slab[b][f];
                if (nbk == b) {
                    for_each_box(D, lo, hi, [&](const int64_t* idx) {
                        int64_t s[3] = {idx[0], idx[1], idx[2]};
                        s[d] = dir < 0 ? n + idx[d] : idx[d] - n;
                        dst[grid.linearize(idx, g)] = dst[grid.linearize(s, g)];
                    });
                } else if (nbk >= 0) {
                    const std::vector<double>& src = st.slab[nbk][f];
                    for_each_box(D, lo, hi, [&](const int64_t* idx) {
                        int64_t s[3] = {idx[0], idx[1], idx[2]};
                        s[d] = dir < 0 ? n + idx[d] : idx[d] - n;
                        dst[grid.linearize(idx, g)] = src[grid.linearize(s, g)];
                    });
                } else {
                    for_each_box(D, lo, hi, [&](const int64_t* idx) {
                        int64_t layer = dir < 0 ? -1 - idx[d] : idx[d] - n;
                        int64_t s[3] = {idx[0], idx[1], idx[2]};
                        s[d] = dir < 0 ? layer : n - 1 - layer;  // Mirror: interior(k)
                        dst[grid.linearize(idx, g)] = dst[grid.linearize(s, g)];
                    });
                }
            }
        }
    }
}

// ------------------------------------------------------------- heat -------
// examples/heat3d.rs:41-85 (Heat3 / tests/heat3d.rs Heat<D>): u registered
// with ghost 1; drift = CentralLaplacian(u) then *= kappa (heat3d.rs:76-78).
// ForwardEuler::step (src/integrators/euler.rs:51-53): eval_drift, then
// state.axpy_with(dt, k) over every slab entry (state.rs:485-498).
double heat_run(const Grid& grid, State& st, int f, double kappa, double t, double dt, int64_t steps,
                int nthreads) {
    int g = st.ghost[f];
    std::vector<std::vector<double>> k(grid.num_blocks(), std::vector<double>(grid.block_len(g), 0.0));
    const Ext e = ext_of(grid);
    for (int64_t s = 0; s < steps; ++s) {
        fill_ghosts_mirror(grid, st, f);
        parallel_blocks(grid.num_blocks(), nthreads, [&](int64_t b) {
            heat_drift_block(e, grid.spacing, kappa, st.slab[b][f].data(), k[b].data());
        });
        parallel_blocks(grid.num_blocks(), nthreads, [&](int64_t b) { apply_time(st.slab[b][f], k[b], dt); });
        t += dt;  // src/core/simulation.rs:285
    }
    return t;
}

// EulerMaruyama::step (src/integrators/euler_maruyama.rs:34-75) with
// ModelC<Wiener<1>> (noise != 0) or ModelC<NoNoise>, fields phi=0, u=1.
double modelc_run(const Grid& grid, State& st, const ModelC& m, double t, double dt, uint64_t seed,
                  int64_t steps, bool wiener, int nthreads, int theta_field = -1) {
    const int64_t nb = grid.num_blocks();
    const int64_t len = grid.block_len(1);
    // Stage buffers (simulation.rs:187-202): Tendency(Time) carries phi and
    // u; Tendency(Wiener(0)) carries phi only (phasefield.rs:340-341).
    std::vector<std::vector<double>> kphi(nb, std::vector<double>(len, 0.0));
    std::vector<std::vector<double>> ku(nb, std::vector<double>(len, 0.0));
    std::vector<std::vector<double>> amp(wiener ? nb : 0, std::vector<double>(len, 0.0));
    for (int64_t s = 0; s < steps; ++s) {
        // StepCtx::eval_drift (integrators/mod.rs:190-198)
        fill_ghosts_mirror(grid, st, 0);
        fill_ghosts_mirror(grid, st, 1);
        const Ext e = ext_of(grid);
        parallel_blocks(nb, nthreads, [&](int64_t b) {
            if (theta_field >= 0)
                modelc_drift_block_oriented(e, grid.spacing, m, st.slab[b][0].data(), st.slab[b][1].data(),
                                            st.slab[b][theta_field].data(), kphi[b].data(), ku[b].data());
            else
                modelc_drift_block(e, grid.spacing, m, st.slab[b][0].data(), st.slab[b][1].data(), kphi[b].data(),
                                   ku[b].data());
        });
        if (wiener) {
            // eval_tendency_impl: fill_zero then amp_phi = b on the interior
            // (integrators/mod.rs:251-277, phasefield.rs:361-366)
            parallel_blocks(nb, nthreads, [&](int64_t b) {
                std::fill(amp[b].begin(), amp[b].end(), 0.0);
                for_each_interior(grid, [&](const int64_t* idx) { amp[b][grid.linearize(idx, 1)] = m.noise_amplitude; });
            });
        }
        // State::apply_step_with (state.rs:656-699), salt = t.to_bits()
        const uint64_t salt = bits_of(t);
        parallel_blocks(nb, nthreads, [&](int64_t b) {
            apply_time(st.slab[b][0], kphi[b], dt);  // Driver::Time over phi then u
            apply_time(st.slab[b][1], ku[b], dt);
            if (wiener) apply_wiener(e, 1, st.slab[b][0], amp[b], dt, seed, salt, (uint64_t)b);
        });
        t += dt;
    }
    return t;
}

// phasefield.rs:227-286 (initialize_grains, orientations disabled)
void modelc_initialize_grains(const Grid& grid, State& st, const double* grains, int64_t n, double u0) {
    const double CUTOFF = 27.0;
    const int64_t nx = grid.block[0], ny = grid.block[1];
    for (int64_t b = 0; b < grid.num_blocks(); ++b) {
        double hx = grid.spacing[0], hy = grid.spacing[1];
        int64_t i0[3] = {0, 0, 0}, i1[3] = {nx - 1, ny - 1, 0};
        double c0[3], c1[3];
        grid.cell_center(b, i0, c0);
        grid.cell_center(b, i1, c1);
        double lo[2] = {std::fma(0.5, -hx, c0[0]), std::fma(0.5, -hy, c0[1])};
        double hi[2] = {std::fma(0.5, hx, c1[0]), std::fma(0.5, hy, c1[1])};
        auto dist_box = [&](double cx, double cy) {
            double dx = std::max(std::max(lo[0] - cx, cx - hi[0]), 0.0);
            double dy = std::max(std::max(lo[1] - cy, cy - hi[1]), 0.0);
            return std::hypot(dx, dy);
        };
        std::vector<int64_t> near;
        for (int64_t k = 0; k < n; ++k)
            if (dist_box(grains[4 * k], grains[4 * k + 1]) <= grains[4 * k + 2] + CUTOFF) near.push_back(k);
        std::vector<double>& phi = st.slab[b][0];
        std::vector<double>& u = st.slab[b][1];
        for_each_interior(grid, [&](const int64_t* idx) {
            double v = -1.0;
            if (!near.empty()) {
                double xy[3];
                grid.cell_center(b, idx, xy);
                for (int64_t k : near) {
                    double r = std::hypot(xy[0] - grains[4 * k], xy[1] - grains[4 * k + 1]);
                    double pk = -std::tanh((r - grains[4 * k + 2]) / std::sqrt(2.0));
                    v = std::fmax(v, pk);
                }
            }
            phi[grid.linearize(idx, 1)] = v;
        });
        for_each_interior(grid, [&](const int64_t* idx) { u[grid.linearize(idx, 1)] = -u0; });
    }
}

// RungeKutta4::step (src/integrators/rk4.rs:40-79) over the fields `fields`
// of a state: k1 = f(y); y_tmp = y; y_tmp += (0.5 dt) k1; k2 = f(y_tmp);
// y_tmp = y; y_tmp += (0.5 dt) k2; k3 = f(y_tmp); y_tmp = y; y_tmp += dt k3;
// k4 = f(y_tmp); y += (dt/6) k1; y += (dt/3) k2; y += (dt/3) k3;
// y += (dt/6) k4.  Copies and axpys run over every slab entry (state.rs:
// 559-568); a drift writes interior entries only (tendency ghosts stay 0)
// and fills the ghosts of its input first (StepCtx::eval_drift).  Static
// fields (theta0) are copied into y_tmp and never stepped.
template <class Drift>
double rk4_run(const Grid& grid, State& st, const std::vector<int>& fields, double t, double dt, int64_t steps,
               int nthreads, Drift drift) {
    const int64_t nb = grid.num_blocks();
    const size_t nf = fields.size();
    auto zeros = [&]() {
        std::vector<std::vector<std::vector<double>>> k(nf);
        for (size_t i = 0; i < nf; ++i)
            k[i].assign(nb, std::vector<double>(grid.block_len(st.ghost[fields[i]]), 0.0));
        return k;
    };
    auto k1 = zeros(), k2 = zeros(), k3 = zeros(), k4 = zeros();
    State tmp = st;
    const double half_dt = 0.5 * dt, sixth = dt / 6.0, third = dt / 3.0;
    auto axpy = [&](State& x, double a, std::vector<std::vector<std::vector<double>>>& k) {
        parallel_blocks(nb, nthreads, [&](int64_t b) {
            for (size_t i = 0; i < nf; ++i) {
                std::vector<double>& xs = x.slab[b][fields[i]];
                for (size_t e = 0; e < xs.size(); ++e) xs[e] += a * k[i][b][e];
            }
        });
    };
    auto copy = [&]() {
        for (int64_t b = 0; b < nb; ++b) tmp.slab[b] = st.slab[b];
    };
    for (int64_t s = 0; s < steps; ++s) {
        drift(st, k1);
        copy();
        axpy(tmp, half_dt, k1);
        drift(tmp, k2);
        copy();
        axpy(tmp, half_dt, k2);
        drift(tmp, k3);
        copy();
        axpy(tmp, dt, k3);
        drift(tmp, k4);
        axpy(st, sixth, k1);
        axpy(st, third, k2);
        axpy(st, third, k3);
        axpy(st, sixth, k4);
        t += dt;
    }
    return t;
}

// phasefield.rs:286-311: theta0 by nearest-seed Voronoi.  Per block, the
// candidates are the grains whose box distance is at most the smallest
// farthest-corner distance of any grain; each cell takes the orientation of
// the candidate minimising fma(dy, dy, dx * dx) (the first one on ties, as
// min_by), or 0 without candidates.  Written into field f (ghost width 0).
void modelc_initialize_orientations(const Grid& grid, State& st, int f, const double* grains, int64_t n) {
    const int64_t nx = grid.block[0], ny = grid.block[1];
    for (int64_t b = 0; b < grid.num_blocks(); ++b) {
        double hx = grid.spacing[0], hy = grid.spacing[1];
        int64_t i0[3] = {0, 0, 0}, i1[3] = {nx - 1, ny - 1, 0};
        double c0[3], c1[3];
        grid.cell_center(b, i0, c0);
        grid.cell_center(b, i1, c1);
        double lo[2] = {std::fma(0.5, -hx, c0[0]), std::fma(0.5, -hy, c0[1])};
        double hi[2] = {std::fma(0.5, hx, c1[0]), std::fma(0.5, hy, c1[1])};
        auto dist_box = [&](double cx, double cy) {
            double dx = std::max(std::max(lo[0] - cx, cx - hi[0]), 0.0);
            double dy = std::max(std::max(lo[1] - cy, cy - hi[1]), 0.0);
            return std::hypot(dx, dy);
        };
        auto dist_far = [&](double cx, double cy) {
            double dx = std::max(std::fabs(cx - lo[0]), std::fabs(cx - hi[0]));
            double dy = std::max(std::fabs(cy - lo[1]), std::fabs(cy - hi[1]));
            return std::hypot(dx, dy);
        };
        double threshold = std::numeric_limits<double>::max();
        for (int64_t k = 0; k < n; ++k) threshold = std::min(threshold, dist_far(grains[4 * k], grains[4 * k + 1]));
        std::vector<int64_t> cand;
        for (int64_t k = 0; k < n; ++k)
            if (dist_box(grains[4 * k], grains[4 * k + 1]) <= threshold) cand.push_back(k);
        std::vector<double>& th = st.slab[b][f];
        for_each_interior(grid, [&](const int64_t* idx) {
            double xy[3];
            grid.cell_center(b, idx, xy);
            double best = 0.0, bd = 0.0;
            bool any = false;
            for (int64_t k : cand) {
                double dx = xy[0] - grains[4 * k], dy = xy[1] - grains[4 * k + 1];
                double d = std::fma(dy, dy, dx * dx);
                if (!any || d < bd) {  // strict: the first minimum stays (total_cmp on finite values)
                    any = true;
                    bd = d;
                    best = grains[4 * k + 3];
                }
            }
            th[grid.linearize(idx, 0)] = any ? best : 0.0;
        });
    }
}

}  // namespace

// ============================================================ C ABI =======
extern "C" {

uint64_t orc_splitmix64(uint64_t z) { return splitmix64(z); }
uint64_t orc_mix_key(uint64_t seed, const uint64_t* parts, int64_t n) { return mix_key(seed, parts, (size_t)n); }
double orc_unit_open(uint64_t bits) { return unit_open(bits); }
double orc_standard_normal(uint64_t key) { return standard_normal(key); }
void orc_standard_normal_batch(const uint64_t* keys, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = standard_normal(keys[i]);
}

void* orc_grid_create(int D, const int64_t* cells, const int64_t* block, const double* origin,
                      const double* spacing, const int* periodic) {
    if (D < 1 || D > 3) return nullptr;
    Grid* g = new Grid();
    g->D = D;
    for (int d = 0; d < 3; ++d) {
        bool on = d < D;
        g->cells[d] = on ? cells[d] : 1;
        g->block[d] = on ? block[d] : 1;
        g->origin[d] = on ? origin[d] : 0.0;
        g->spacing[d] = on ? spacing[d] : 1.0;
        g->periodic[d] = on ? periodic[d] != 0 : false;
        if (on && (g->cells[d] <= 0 || g->block[d] <= 0 || g->cells[d] % g->block[d] != 0 ||
                   !(g->spacing[d] > 0.0) || !std::isfinite(g->spacing[d]))) {
            delete g;
            return nullptr;
        }
        g->nb[d] = g->cells[d] / g->block[d];
    }
    return g;
}
void orc_grid_destroy(void* g) { delete static_cast<Grid*>(g); }
int64_t orc_grid_num_blocks(const void* g) { return static_cast<const Grid*>(g)->num_blocks(); }
int64_t orc_grid_block_len(const void* g, int ghost) { return static_cast<const Grid*>(g)->block_len(ghost); }
int64_t orc_grid_face_neighbor(const void* g, int64_t b, int dim, int dir) {
    return static_cast<const Grid*>(g)->face_neighbor(b, dim, dir);
}
void orc_grid_cell_center(const void* g, int64_t b, const int64_t* idx, double* out) {
    static_cast<const Grid*>(g)->cell_center(b, idx, out);
}
int orc_grid_cell_key(const void* g, int ghost, int64_t offset, uint64_t* key) {
    return static_cast<const Grid*>(g)->cell_key(ghost, offset, key) ? 1 : 0;
}

void* orc_state_create(const void* grid, int nfields, const int* ghosts) {
    const Grid& g = *static_cast<const Grid*>(grid);
    std::vector<int> gh(ghosts, ghosts + nfields);
    for (int f = 0; f < nfields; ++f)
        for (int d = 0; d < g.D; ++d)
            if (gh[f] < 0 || gh[f] > g.block[d]) return nullptr;  // cartesian.rs:456-462
    std::vector<bool> keep(nfields, true);
    return new State(make_state(g, gh, keep));
}
void orc_state_destroy(void* s) { delete static_cast<State*>(s); }

// Copy field f of every block, block order, each slab ghost-inclusive.
void orc_state_set_field(void* s, int f, const double* data) {
    State& st = *static_cast<State*>(s);
    size_t off = 0;
    for (auto& b : st.slab) {
        std::memcpy(b[f].data(), data + off, b[f].size() * sizeof(double));
        off += b[f].size();
    }
}
void orc_state_get_field(const void* s, int f, double* data) {
    const State& st = *static_cast<const State*>(s);
    size_t off = 0;
    for (auto& b : st.slab) {
        std::memcpy(data + off, b[f].data(), b[f].size() * sizeof(double));
        off += b[f].size();
    }
}

void orc_fill_ghosts_mirror(const void* grid, void* s, int f) {
    fill_ghosts_mirror(*static_cast<const Grid*>(grid), *static_cast<State*>(s), f);
}

double orc_heat_run(const void* grid, void* s, int f, double kappa, double t0, double dt, int64_t steps,
                    int nthreads) {
    return heat_run(*static_cast<const Grid*>(grid), *static_cast<State*>(s), f, kappa, t0, dt, steps, nthreads);
}

double orc_heat_run_rk4(const void* grid, void* s, int f, double kappa, double t0, double dt, int64_t steps,
                        int nthreads) {
    const Grid& g = *static_cast<const Grid*>(grid);
    State& st = *static_cast<State*>(s);
    const Ext e = ext_of(g);
    return rk4_run(g, st, {f}, t0, dt, steps, nthreads, [&](State& y, std::vector<std::vector<std::vector<double>>>& k) {
        fill_ghosts_mirror(g, y, f);
        parallel_blocks(g.num_blocks(), nthreads,
                        [&](int64_t b) { heat_drift_block(e, g.spacing, kappa, y.slab[b][f].data(), k[0][b].data()); });
    });
}

// Model C (no noise: RK4 pairs with NoNoise, rk4.rs:15-19) with
// RungeKutta4; theta_field >= 0 for the multi-grain form.
double orc_modelc_run_rk4(const void* grid, void* s, const orc_modelc_params* p, int theta_field, double t0,
                          double dt, int64_t steps, int nthreads) {
    const Grid& g = *static_cast<const Grid*>(grid);
    State& st = *static_cast<State*>(s);
    const ModelC m = make_model(p);
    const Ext e = ext_of(g);
    return rk4_run(g, st, {0, 1}, t0, dt, steps, nthreads,
                   [&](State& y, std::vector<std::vector<std::vector<double>>>& k) {
                       fill_ghosts_mirror(g, y, 0);
                       fill_ghosts_mirror(g, y, 1);
                       parallel_blocks(g.num_blocks(), nthreads, [&](int64_t b) {
                           if (theta_field >= 0)
                               modelc_drift_block_oriented(e, g.spacing, m, y.slab[b][0].data(), y.slab[b][1].data(),
                                                           y.slab[b][theta_field].data(), k[0][b].data(),
                                                           k[1][b].data());
                           else
                               modelc_drift_block(e, g.spacing, m, y.slab[b][0].data(), y.slab[b][1].data(),
                                                  k[0][b].data(), k[1][b].data());
                       });
                   });
}

double orc_modelc_run(const void* grid, void* s, const orc_modelc_params* p, double t0, double dt, uint64_t seed,
                      int64_t steps, int wiener, int nthreads) {
    ModelC m = make_model(p);
    return modelc_run(*static_cast<const Grid*>(grid), *static_cast<State*>(s), m, t0, dt, seed, steps,
                      wiener != 0, nthreads);
}

// One drift evaluation (k interior) without an update, for kernel-level tests.
void orc_modelc_drift(const void* grid, void* s, const orc_modelc_params* p, double* kphi_out, double* ku_out) {
    const Grid& g = *static_cast<const Grid*>(grid);
    State& st = *static_cast<State*>(s);
    ModelC m = make_model(p);
    int64_t len = g.block_len(1);
    const Ext e = ext_of(g);
    for (int64_t b = 0; b < g.num_blocks(); ++b) {
        std::vector<double> kp(len, 0.0), ku(len, 0.0);
        modelc_drift_block(e, g.spacing, m, st.slab[b][0].data(), st.slab[b][1].data(), kp.data(), ku.data());
        std::memcpy(kphi_out + b * len, kp.data(), len * sizeof(double));
        std::memcpy(ku_out + b * len, ku.data(), len * sizeof(double));
    }
}

double orc_modelc_run_oriented(const void* grid, void* s, const orc_modelc_params* p, int theta_field, double t0,
                               double dt, uint64_t seed, int64_t steps, int wiener, int nthreads) {
    ModelC m = make_model(p);
    return modelc_run(*static_cast<const Grid*>(grid), *static_cast<State*>(s), m, t0, dt, seed, steps,
                      wiener != 0, nthreads, theta_field);
}

void orc_modelc_initialize_orientations(const void* grid, void* s, int theta_field, const double* grains,
                                        int64_t n) {
    modelc_initialize_orientations(*static_cast<const Grid*>(grid), *static_cast<State*>(s), theta_field, grains, n);
}

void orc_modelc_initialize_grains(const void* grid, void* s, const double* grains, int64_t n, double u0) {
    modelc_initialize_grains(*static_cast<const Grid*>(grid), *static_cast<State*>(s), grains, n, u0);
}

int orc_num_threads_available(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
