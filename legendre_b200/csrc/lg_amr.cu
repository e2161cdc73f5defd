// 2-D AMR on the device: Berger-Oliger subcycling of Model C or the heat
// model on a patch hierarchy, with plan-driven ghost fill (exchange, mirror,
// time-interpolated bilinear prolongation), restriction, gradient tagging
// and per-level work-list step kernels.  The hierarchy and its plans are
// built on the host (lg_amr_host.cu); regrids (tag on the device, cluster
// and migrate on the host) happen at the policy's cadence.
//
// Compiled with -fmad=false: every kernel keeps the reference's operand
// order, so FP64 results are bit-identical to the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/legendre_b200.h"
#include "lg_amr_host.h"
#include "lg_kernels.h"
#include "lg_modelc_ops.cuh"

namespace lg {
// lg_abi.cu
int abi_fail(lg_ctx* ctx, int code, const std::string& msg);
cudaStream_t abi_stream(lg_ctx* ctx);
int abi_device(lg_ctx* ctx);
void abi_count_launch(lg_ctx* ctx, int64_t n);
int64_t abi_launches(lg_ctx* ctx);
void abi_set_launches(lg_ctx* ctx, int64_t n);
}  // namespace lg

namespace {

using lg::amr::BlockDesc;
using lg::amr::Corner;
using lg::amr::FillOp;
using lg::amr::RestrictOp;
using lg::amr::Unit;

constexpr int kMaxDepth = 8;

// Substep time of one level: t_l = fma(s_l, dt_l, t_{l-1}) down the
// recursion from the level-0 time in the device slot (subcycling.rs:256).
struct TimeChain {
    int depth;
    int s[kMaxDepth];
    double dt[kMaxDepth];
};

__device__ __forceinline__ double chain_time(double t0, const TimeChain& c) {
    double t = t0;
    for (int k = 0; k < c.depth; ++k) t = fma((double)c.s[k], c.dt[k], t);
    return t;
}

// ------------------------------------------------------------ kernels ----
// Ghost entries of one level (intergrid.rs:183-223 / 358-408): a copy of a
// same-level interior entry, or the bilinear fold acc + v w over coarse
// interior corners, blended in time as old (1 - alpha) + new alpha.
// A (this level) and Ac (the coarser level) may be the same arena: the
// kernel writes ghost entries only and reads interior entries only.
__global__ void amr_fill_kernel(const BlockDesc* __restrict__ blocks, double* A, const double* Ac, const double* Sc,
                                const FillOp* __restrict__ ops, int64_t nops, const Corner* __restrict__ corners,
                                int nfields, double alpha, int interp) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += (int64_t)gridDim.x * blockDim.x) {
        const FillOp op = ops[i];
        const BlockDesc tb = blocks[op.tblock];
        for (int f = 0; f < nfields; ++f) {
            double v;
            if (op.b >= 0) {
                const BlockDesc sb = blocks[op.a];
                v = A[sb.off + f * sb.stride + op.b];
            } else {
                double acc = 0.0, old = 0.0;
                for (int k = op.a; k < op.a - op.b; ++k) {
                    const Corner c = corners[k];
                    const BlockDesc cb = blocks[c.block];
                    const int64_t o = cb.off + f * cb.stride + c.off;
                    acc = acc + Ac[o] * c.w;
                    if (interp) old = old + Sc[o] * c.w;
                }
                v = interp ? old * (1.0 - alpha) + acc * alpha : acc;
            }
            A[tb.off + f * tb.stride + op.toff] = v;
        }
    }
}

// Covered coarse cells <- sum of r x r fine children (dimension 0 fastest,
// from zero) times 1/r^2 (intergrid.rs:110-150).
// C (coarse level) and F (fine level) may be the same arena (disjoint slabs).
__global__ void amr_restrict_kernel(const BlockDesc* __restrict__ blocks, double* C, const double* F,
                                    const RestrictOp* __restrict__ ops, int64_t nops,
                                    int r, double inv, int f0, int f1) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += (int64_t)gridDim.x * blockDim.x) {
        const RestrictOp op = ops[i];
        const BlockDesc fb = blocks[op.fblock], cb = blocks[op.cblock];
        const int sy = fb.nx + 2;
        for (int f = f0; f < f1; ++f) {
            const double* src = F + fb.off + f * fb.stride + op.foff;
            double sum = 0.0;
            for (int ky = 0; ky < r; ++ky)
                for (int kx = 0; kx < r; ++kx) sum += src[kx + ky * sy];
            C[cb.off + f * cb.stride + op.coff] = sum * inv;
        }
    }
}

// GradientTagger::tag_level (adapt.rs:78-103): flag where
// max_d |(u(+e_d) - u(-e_d)) 0.5| > threshold; cells in level coordinates.
__global__ void amr_tag_kernel(const BlockDesc* __restrict__ blocks, const int64_t* __restrict__ lo,
                               const Unit* __restrict__ units, int64_t nunits, const double* __restrict__ A,
                               int field, double threshold, int64_t* __restrict__ out, int64_t cap,
                               unsigned long long* __restrict__ count) {
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const BlockDesc b = blocks[un.block];
        const double* v = A + b.off + field * b.stride;
        const int sy = b.nx + 2;
        for (int c = un.start + threadIdx.x; c < un.start + un.count; c += blockDim.x) {
            const int i = c % b.nx, j = c / b.nx;
            const int o = (i + 1) + (j + 1) * sy;
            double gmax = 0.0;
            gmax = fmax(gmax, fabs((v[o + 1] - v[o - 1]) * 0.5));
            gmax = fmax(gmax, fabs((v[o + sy] - v[o - sy]) * 0.5));
            if (gmax > threshold) {
                const unsigned long long k = atomicAdd(count, 1ull);
                if ((int64_t)k < cap) {
                    out[2 * k] = lo[2 * un.block] + i;
                    out[2 * k + 1] = lo[2 * un.block + 1] + j;
                }
            }
        }
    }
}

struct StepArgs {
    const BlockDesc* blocks;
    const Unit* units;
    int64_t nunits;
    const double* in;
    double* out;
    double dt;
    double* tdev;
    int slot;
    int write_t;   // this launch advances the level-0 time slot
    double dt0;    // level-0 step (for that advance)
    TimeChain chain;
    int noise;
    uint64_t seed;
    double scale_amp;
};

// Model C Euler-Maruyama on the cells of one level's work list (the
// reference-order cell update of phasefield.rs:353-422 with the Time and
// Wiener drivers, state.rs:706-753).  Ghosts are not pushed: under AMR
// they come from the fill plan.
__global__ void __launch_bounds__(256) amr_modelc_kernel(StepArgs a, lg::MC<double> m) {
    const double t0 = a.tdev[a.slot];
    if (a.write_t && blockIdx.x == 0 && threadIdx.x == 0) a.tdev[a.slot ^ 1] = t0 + a.dt0;
    const double t = chain_time(t0, a.chain);
    for (int64_t u = blockIdx.x; u < a.nunits; u += gridDim.x) {
        const Unit un = a.units[u];
        const BlockDesc b = a.blocks[un.block];
        const double* ph = a.in + b.off;
        const double* uu = a.in + b.off + b.stride;
        double* po = a.out + b.off;
        double* uo = a.out + b.off + b.stride;
        const int sy = b.nx + 2;
        uint64_t block_key = 0;
        if (a.noise)
            block_key = lg::wiener_block_key(a.seed, (uint64_t)__double_as_longlong(t), lg::kWienerStream0,
                                             (uint64_t)un.block);
        for (int c = un.start + threadIdx.x; c < un.start + un.count; c += blockDim.x) {
            const int i = c % b.nx, j = c / b.nx;
            const int o = (i + 1) + (j + 1) * sy;
            auto P = [&](int di, int dj) { return ph[o + di + dj * sy]; };
            double derx_r = P(1, 0) - P(0, 0);
            double derx_l = P(0, 0) - P(-1, 0);
            double derx_t = 0.25 * (P(1, 1) - P(-1, 1) + P(1, 0) - P(-1, 0));
            double derx_b = 0.25 * (P(1, 0) - P(-1, 0) + P(1, -1) - P(-1, -1));
            double dery_t = P(0, 1) - P(0, 0);
            double dery_b = P(0, 0) - P(0, -1);
            double dery_r = 0.25 * (P(1, 1) - P(1, -1) + P(0, 1) - P(0, -1));
            double dery_l = 0.25 * (P(0, 1) - P(0, -1) + P(-1, 1) - P(-1, -1));
            double a_r, da_r, a_l, da_l, a_t, da_t, a_b, da_b;
            lg::kr_face(m, derx_r, dery_r, a_r, da_r);
            lg::kr_face(m, derx_l, dery_l, a_l, da_l);
            lg::kr_face(m, derx_t, dery_t, a_t, da_t);
            lg::kr_face(m, derx_b, dery_b, a_b, da_b);
            double j_r = a_r * (a_r * derx_r - da_r * dery_r);
            double j_l = a_l * (a_l * derx_l - da_l * dery_l);
            double j_t = a_t * (a_t * dery_t + da_t * derx_t);
            double j_b = a_b * (a_b * dery_b + da_b * derx_b);
            double flux = (j_r - j_l + j_t - j_b) * m.inv_h2_flux;
            double p = P(0, 0);
            double g_prime = fma(p * p, p, -p);
            double one_m_p2 = fma(p, -p, 1.0);
            double p_prime = one_m_p2 * one_m_p2;
            double ac = lg::center_anisotropy(m, 0.5 * (P(1, 0) - P(-1, 0)), 0.5 * (P(0, 1) - P(0, -1)));
            double uc = uu[o];
            double kphi = fma(m.lambda * uc, -p_prime, flux - g_prime) / (ac * ac);
            double acc = 0.0;
            acc += ((uu[o + 1] - (uc + uc)) + uu[o - 1]) * m.ih0;
            acc += ((uu[o + sy] - (uc + uc)) + uu[o - sy]) * m.ih1;
            double ku = fma(acc, m.d_thermal, 0.5 * kphi);
            double phin = p + a.dt * kphi;
            if (a.noise) phin += a.scale_amp * lg::standard_normal(lg::splitmix64(block_key ^ (uint64_t)c));
            po[o] = phin;
            uo[o] = uc + a.dt * ku;
        }
    }
}

// Heat on the cells of one level's work list: k = lap(u) kappa, u + dt k
// (tests/amr.rs:324-339, euler.rs:51-53).
__global__ void __launch_bounds__(256) amr_heat_kernel(StepArgs a, double kappa, double ih0, double ih1) {
    const double t0 = a.tdev[a.slot];
    if (a.write_t && blockIdx.x == 0 && threadIdx.x == 0) a.tdev[a.slot ^ 1] = t0 + a.dt0;
    for (int64_t u = blockIdx.x; u < a.nunits; u += gridDim.x) {
        const Unit un = a.units[u];
        const BlockDesc b = a.blocks[un.block];
        const double* s = a.in + b.off;
        double* o_ = a.out + b.off;
        const int sy = b.nx + 2;
        for (int c = un.start + threadIdx.x; c < un.start + un.count; c += blockDim.x) {
            const int i = c % b.nx, j = c / b.nx;
            const int o = (i + 1) + (j + 1) * sy;
            const double center = s[o];
            double acc = 0.0;
            acc += ((s[o + 1] - (center + center)) + s[o - 1]) * ih0;
            acc += ((s[o + sy] - (center + center)) + s[o - sy]) * ih1;
            const double k = acc * kappa;
            o_[o] = center + a.dt * k;
        }
    }
}

unsigned grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

template <class T>
T* dev_upload(const std::vector<T>& v, cudaError_t* err) {
    T* p = nullptr;
    if (v.empty()) return nullptr;
    *err = cudaMalloc(&p, v.size() * sizeof(T));
    if (*err != cudaSuccess) return nullptr;
    *err = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
}

}  // namespace

struct lg_amr_sim {
    lg_ctx* ctx = nullptr;
    lg::amr::Layout layout;
    lg::amr::Plans plans;
    int model = LG_MODEL_C;
    lg_modelc_params mp{};
    double kappa = 0.0;
    int integrator = LG_AMR_SUBCYCLING;
    uint64_t seed = 0;
    bool has_policy = false;
    lg::amr::Policy policy;
    int nfields = 2;
    // device
    double* arena[2] = {nullptr, nullptr};
    double* snap = nullptr;
    BlockDesc* d_blocks = nullptr;
    int64_t* d_lo = nullptr;
    FillOp* d_fill = nullptr;
    Corner* d_corners = nullptr;
    RestrictOp* d_restrict = nullptr;
    Unit* d_units = nullptr;
    int64_t* d_tags = nullptr;
    int64_t tag_cap = 0;
    unsigned long long* d_count = nullptr;
    double* d_t = nullptr;
    std::vector<int> cur;  // current buffer per level
    int tslot = 0;
    double t = 0.0;
    int64_t step_index = 0, epoch = 0;
    std::map<std::string, std::pair<cudaGraphExec_t, int64_t>> graphs;  // exec, launches
};

namespace {

int fail(lg_amr_sim* s, int code, const std::string& m) { return lg::abi_fail(s ? s->ctx : nullptr, code, m); }

#define AMR_CUDA(s, call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail((s), LG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_device(lg_amr_sim* s) {
    for (double*& a : s->arena) {
        cudaFree(a);
        a = nullptr;
    }
    cudaFree(s->snap);
    cudaFree(s->d_blocks);
    cudaFree(s->d_lo);
    cudaFree(s->d_fill);
    cudaFree(s->d_corners);
    cudaFree(s->d_restrict);
    cudaFree(s->d_units);
    s->snap = nullptr;
    s->d_blocks = nullptr;
    s->d_lo = nullptr;
    s->d_fill = nullptr;
    s->d_corners = nullptr;
    s->d_restrict = nullptr;
    s->d_units = nullptr;
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second.first);
    s->graphs.clear();
}

// (re)build plans and device tables for s->layout; fresh zeroed arenas
int setup_device(lg_amr_sim* s) {
    free_device(s);
    s->plans = lg::amr::build_plans(s->layout, s->nfields, 1024);
    if (!s->plans.error.empty()) return fail(s, LG_ERR_STATE, s->plans.error);
    cudaError_t e = cudaSuccess;
    std::vector<int64_t> lo;
    for (const auto& p : s->layout.patches) {
        lo.push_back(p.bx.lo[0]);
        lo.push_back(p.bx.lo[1]);
    }
    s->d_blocks = dev_upload(s->plans.blocks, &e);
    if (e == cudaSuccess) s->d_lo = dev_upload(lo, &e);
    if (e == cudaSuccess) s->d_fill = dev_upload(s->plans.fill, &e);
    if (e == cudaSuccess) s->d_corners = dev_upload(s->plans.corners, &e);
    if (e == cudaSuccess) s->d_restrict = dev_upload(s->plans.restrict_ops, &e);
    if (e == cudaSuccess) s->d_units = dev_upload(s->plans.units, &e);
    const size_t bytes = (size_t)s->plans.arena_elems * sizeof(double);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMalloc(&s->arena[k], bytes);
        if (e == cudaSuccess) e = cudaMemset(s->arena[k], 0, bytes);
    }
    if (e == cudaSuccess) e = cudaMalloc(&s->snap, bytes);
    if (e == cudaSuccess) e = cudaMemset(s->snap, 0, bytes);
    if (e != cudaSuccess) return fail(s, LG_ERR_NOMEM, std::string("AMR device setup: ") + cudaGetErrorString(e));
    s->cur.assign(s->layout.num_levels(), 0);
    return LG_OK;
}

// level l's slabs are contiguous in the arena: [off of its first block, end of its last)
std::pair<int64_t, int64_t> level_range(const lg_amr_sim* s, int level) {
    const uint32_t b0 = s->layout.level_start[level], b1 = s->layout.level_start[level + 1];
    if (b0 == b1) return {0, 0};
    const BlockDesc& last = s->plans.blocks[b1 - 1];
    return {s->plans.blocks[b0].off, last.off + last.stride * s->nfields};
}

int launch_fill(lg_amr_sim* s, int level, bool interp, double alpha) {
    const int64_t a = s->plans.fill_start[level], b = s->plans.fill_start[level + 1];
    if (b == a) return LG_OK;
    const double* coarse = level > 0 ? s->arena[s->cur[level - 1]] : nullptr;
    amr_fill_kernel<<<grid_for(b - a, 256), 256, 0, lg::abi_stream(s->ctx)>>>(
        s->d_blocks, s->arena[s->cur[level]], coarse, s->snap, s->d_fill + a, b - a, s->d_corners, s->nfields, alpha,
        interp ? 1 : 0);
    lg::abi_count_launch(s->ctx, 1);
    AMR_CUDA(s, cudaGetLastError());
    return LG_OK;
}

int launch_restrict(lg_amr_sim* s, int fine, int f0, int f1) {
    const int64_t a = s->plans.restrict_start[fine], b = s->plans.restrict_start[fine + 1];
    if (b == a) return LG_OK;
    const int r = (int)s->layout.ratios[fine - 1];
    const double inv = 1.0 / ((double)r * (double)r);
    amr_restrict_kernel<<<grid_for(b - a, 256), 256, 0, lg::abi_stream(s->ctx)>>>(
        s->d_blocks, s->arena[s->cur[fine - 1]], s->arena[s->cur[fine]], s->d_restrict + a, b - a, r, inv, f0, f1);
    lg::abi_count_launch(s->ctx, 1);
    AMR_CUDA(s, cudaGetLastError());
    return LG_OK;
}

lg::MC<double> level_mc(const lg_amr_sim* s, int level) {
    lg::ModelCDev m{};
    const lg_modelc_params* p = &s->mp;
    m.lambda = p->lambda;
    m.d_thermal = p->d_thermal;
    m.a_bar = std::fma(3.0, -p->eps4, 1.0);
    m.eps_prime = 3.0 * p->eps4 / m.a_bar;
    m.tol = p->anisotropy_tol;
    m.f_a_bar = std::fma(3.0, -p->eps4, 1.0);
    m.f_eps_prime = 3.0 * p->eps4 / m.f_a_bar;
    m.f_a12 = 4.0 * m.f_a_bar * m.f_eps_prime;
    m.f_tol = p->flux_tol;
    const auto& h = s->layout.level_spacing[level];
    m.inv_h2_flux = 1.0 / (h[0] * h[1]);
    m.inv_h2[0] = 1.0 / (h[0] * h[0]);
    m.inv_h2[1] = 1.0 / (h[1] * h[1]);
    return lg::to_mc<double>(m);
}

// one Euler-Maruyama update of the units [u0, u1) (level l, or every level
// for the global-dt path), reading buffer `in_buf` and writing the other
int launch_step(lg_amr_sim* s, int level_for_consts, int64_t u0, int64_t u1, int in_buf, double dt,
                const TimeChain& chain, bool write_t, double dt0) {
    if (u1 == u0) return LG_OK;
    StepArgs a{};
    a.blocks = s->d_blocks;
    a.units = s->d_units + u0;
    a.nunits = u1 - u0;
    a.in = s->arena[in_buf];
    a.out = s->arena[in_buf ^ 1];
    a.dt = dt;
    a.tdev = s->d_t;
    a.slot = s->tslot;
    a.write_t = write_t ? 1 : 0;
    a.dt0 = dt0;
    a.chain = chain;
    a.noise = (s->model == LG_MODEL_C && s->mp.noise_amplitude != 0.0) ? 1 : 0;
    a.seed = s->seed;
    a.scale_amp = std::sqrt(dt) * s->mp.noise_amplitude;
    const unsigned g = (unsigned)std::min<int64_t>(u1 - u0, 65535);
    if (s->model == LG_MODEL_C) {
        amr_modelc_kernel<<<g, 256, 0, lg::abi_stream(s->ctx)>>>(a, level_mc(s, level_for_consts));
    } else {
        const auto& h = s->layout.level_spacing[level_for_consts];
        amr_heat_kernel<<<g, 256, 0, lg::abi_stream(s->ctx)>>>(a, s->kappa, 1.0 / (h[0] * h[0]), 1.0 / (h[1] * h[1]));
    }
    lg::abi_count_launch(s->ctx, 1);
    AMR_CUDA(s, cudaGetLastError());
    return LG_OK;
}

double stable_dt_at(const lg_amr_sim* s, int level) {
    const auto& h = s->layout.level_spacing[level];
    const double hm = std::min(h[0], h[1]);
    if (s->model == LG_MODEL_C) return 0.2 * (hm * hm) / s->mp.d_thermal;  // phasefield.rs:446-449
    return 0.25 * (hm * hm) / s->kappa;                                     // tests/amr.rs:341-343
}

// Subcycle::advance (subcycling.rs:195-267)
int advance(lg_amr_sim* s, int level, TimeChain chain, double dt, double alpha, bool first) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    // 1. snapshot this level (only level-l slabs are ever read from it)
    auto rng = level_range(s, level);
    if (rng.second > rng.first)
        AMR_CUDA(s, cudaMemcpyAsync(s->snap + rng.first, s->arena[s->cur[level]] + rng.first,
                                    (rng.second - rng.first) * sizeof(double), cudaMemcpyDeviceToDevice, st));
    // 2. ghosts of this level, coarse source interpolated in time
    int rc = launch_fill(s, level, level > 0, alpha);
    if (rc != LG_OK) return rc;
    // 3. Euler-Maruyama on this level's blocks
    rc = launch_step(s, level, s->plans.unit_start[level], s->plans.unit_start[level + 1], s->cur[level], dt, chain,
                     first, dt);
    if (rc != LG_OK) return rc;
    s->cur[level] ^= 1;
    // 4. subcycle the next level, then restrict it
    const int child = level + 1;
    if (child < s->layout.num_levels()) {
        const double n_f = std::round(stable_dt_at(s, level) / stable_dt_at(s, child));
        const uint64_t n = (uint64_t)std::max(n_f, 1.0);
        const double dt_child = dt / (double)n;
        if (chain.depth >= kMaxDepth) return fail(s, LG_ERR_INVALID, "too many refinement levels");
        for (uint64_t k = 0; k < n; ++k) {
            TimeChain c = chain;
            c.s[c.depth] = (int)k;
            c.dt[c.depth] = dt_child;
            c.depth += 1;
            rc = advance(s, child, c, dt_child, (double)k / (double)n, false);
            if (rc != LG_OK) return rc;
        }
        rc = launch_restrict(s, child, 0, s->nfields);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

// the model's AMR fill_ghosts (phasefield.rs:454-467): restrict then fill,
// for fields [f0, f1)
int sync_fields(lg_amr_sim* s, int f0, int f1) {
    for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
        int rc = launch_restrict(s, fine, f0, f1);
        if (rc != LG_OK) return rc;
    }
    // per-field fill: the plan fills all fields; fill only [f0, f1) by
    // temporarily narrowing nfields is not possible, so fill all fields --
    // their values are consistent with the reference only when every field
    // is being synchronised, which is the case for the model's fill.
    for (int level = 0; level < s->layout.num_levels(); ++level) {
        int rc = launch_fill(s, level, false, 0.0);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

int one_coarse_step(lg_amr_sim* s, double dt) {
    TimeChain c{};
    if (s->integrator == LG_AMR_SUBCYCLING) {
        int rc = advance(s, 0, c, dt, 0.0, true);
        if (rc != LG_OK) return rc;
    } else {
        int rc = sync_fields(s, 0, s->nfields);
        if (rc != LG_OK) return rc;
        // every level steps together; buffers of all levels agree here
        for (int l = 1; l < s->layout.num_levels(); ++l)
            if (s->cur[l] != s->cur[0]) return fail(s, LG_ERR_STATE, "level buffers out of step");
        for (int l = 0; l < s->layout.num_levels(); ++l) {
            rc = launch_step(s, l, s->plans.unit_start[l], s->plans.unit_start[l + 1], s->cur[l], dt, c, l == 0, dt);
            if (rc != LG_OK) return rc;
        }
        for (int l = 0; l < s->layout.num_levels(); ++l) s->cur[l] ^= 1;
    }
    s->tslot ^= 1;
    return LG_OK;
}

// host copies of field f of every block (current buffer of its level)
int download_blocks(lg_amr_sim* s, int f, std::vector<std::vector<double>>& out) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    out.assign(s->layout.num_blocks(), {});
    for (int b = 0; b < s->layout.num_blocks(); ++b) {
        const BlockDesc& d = s->plans.blocks[b];
        out[b].resize((size_t)(d.nx + 2) * (d.ny + 2));
        AMR_CUDA(s, cudaMemcpyAsync(out[b].data(), s->arena[s->cur[d.level]] + d.off + f * d.stride,
                                    out[b].size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    AMR_CUDA(s, cudaStreamSynchronize(st));
    return LG_OK;
}

int upload_blocks(lg_amr_sim* s, int f, const std::vector<std::vector<double>>& in) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    for (int b = 0; b < s->layout.num_blocks(); ++b) {
        const BlockDesc& d = s->plans.blocks[b];
        AMR_CUDA(s, cudaMemcpyAsync(s->arena[s->cur[d.level]] + d.off + f * d.stride, in[b].data(),
                                    in[b].size() * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    AMR_CUDA(s, cudaStreamSynchronize(st));
    return LG_OK;
}

int tag_level(lg_amr_sim* s, int field, int level, double threshold, std::vector<std::array<int64_t, 2>>& cells) {
    cudaStream_t st = lg::abi_stream(s->ctx);
    int64_t need = 0;
    for (uint32_t b = s->layout.level_start[level]; b < s->layout.level_start[level + 1]; ++b)
        need += (int64_t)s->plans.blocks[b].nx * s->plans.blocks[b].ny;
    if (need > s->tag_cap) {
        cudaFree(s->d_tags);
        s->d_tags = nullptr;
        AMR_CUDA(s, cudaMalloc(&s->d_tags, 2 * need * sizeof(int64_t)));
        s->tag_cap = need;
    }
    if (!s->d_count) AMR_CUDA(s, cudaMalloc(&s->d_count, sizeof(unsigned long long)));
    AMR_CUDA(s, cudaMemsetAsync(s->d_count, 0, sizeof(unsigned long long), st));
    const int64_t u0 = s->plans.unit_start[level], u1 = s->plans.unit_start[level + 1];
    if (u1 > u0) {
        amr_tag_kernel<<<(unsigned)std::min<int64_t>(u1 - u0, 65535), 256, 0, st>>>(
            s->d_blocks, s->d_lo, s->d_units + u0, u1 - u0, s->arena[s->cur[level]], field, threshold, s->d_tags,
            s->tag_cap, s->d_count);
        lg::abi_count_launch(s->ctx, 1);
        AMR_CUDA(s, cudaGetLastError());
    }
    unsigned long long n = 0;
    AMR_CUDA(s, cudaMemcpyAsync(&n, s->d_count, sizeof n, cudaMemcpyDeviceToHost, st));
    AMR_CUDA(s, cudaStreamSynchronize(st));
    std::vector<int64_t> host(2 * n);
    if (n) AMR_CUDA(s, cudaMemcpy(host.data(), s->d_tags, 2 * n * sizeof(int64_t), cudaMemcpyDeviceToHost));
    cells.resize(n);
    for (unsigned long long k = 0; k < n; ++k) cells[k] = {host[2 * k], host[2 * k + 1]};
    return LG_OK;
}

// BergerOliger::regrid (adapt.rs:152-237): prepare (restrict + fill of the
// tagged field), tag every level on the device, build boxes on the host,
// keep the hierarchy if acceptable, else rebuild and migrate.
int maybe_regrid(lg_amr_sim* s) {
    if (!s->has_policy || s->step_index % s->policy.every != 0) return LG_OK;
    const int f = s->policy.field;
    for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
        int rc = launch_restrict(s, fine, f, f + 1);
        if (rc != LG_OK) return rc;
    }
    // the global fill of the tagged field only: fill writes every field's
    // ghosts, and ghosts are rewritten before any other read, so the extra
    // fields' ghost values are unobservable
    for (int level = 0; level < s->layout.num_levels(); ++level) {
        int rc = launch_fill(s, level, false, 0.0);
        if (rc != LG_OK) return rc;
    }
    std::vector<std::vector<std::array<int64_t, 2>>> flags(s->layout.num_levels());
    for (int level = 0; level < s->layout.num_levels() && level < s->layout.max_levels() - 1; ++level) {
        int rc = tag_level(s, f, level, s->policy.threshold, flags[level]);
        if (rc != LG_OK) return rc;
    }
    auto proposed = lg::amr::propose(s->layout, flags, s->policy);
    if (lg::amr::acceptable(s->layout, proposed)) return LG_OK;
    lg::amr::Layout ng;
    std::string err = lg::amr::build_layout(s->layout.base, s->layout.ratios, proposed, &ng);
    if (!err.empty()) return fail(s, LG_ERR_STATE, "regrid produced an invalid hierarchy: " + err);
    std::vector<std::vector<std::vector<double>>> migrated(s->nfields);
    for (int k = 0; k < s->nfields; ++k) {
        std::vector<std::vector<double>> old;
        int rc = download_blocks(s, k, old);
        if (rc != LG_OK) return rc;
        lg::amr::migrate_field(s->layout, old, ng, migrated[k]);
    }
    s->layout = std::move(ng);
    int rc = setup_device(s);
    if (rc != LG_OK) return rc;
    for (int k = 0; k < s->nfields; ++k) {
        rc = upload_blocks(s, k, migrated[k]);
        if (rc != LG_OK) return rc;
    }
    s->epoch += 1;
    return LG_OK;
}

}  // namespace

extern "C" {

int lg_amr_sim_create(lg_ctx* ctx, const int64_t* cells, const int64_t* block, const double* origin,
                      const double* spacing, const uint32_t* ratios, int nratios, const int64_t* patches,
                      int64_t npatches, int model, const lg_modelc_params* mp, double kappa, int integrator,
                      uint64_t seed, const lg_amr_policy* policy, lg_amr_sim** out) {
    if (!ctx || !out || !cells || !block || !origin || !spacing || (nratios > 0 && !ratios) ||
        (npatches > 0 && !patches))
        return lg::abi_fail(ctx, LG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (model != LG_MODEL_C && model != LG_MODEL_HEAT) return lg::abi_fail(ctx, LG_ERR_INVALID, "unknown model");
    if (model == LG_MODEL_C && !mp) return lg::abi_fail(ctx, LG_ERR_INVALID, "Model C needs parameters");
    if (integrator != LG_AMR_SUBCYCLING && integrator != LG_AMR_GLOBAL_DT)
        return lg::abi_fail(ctx, LG_ERR_INVALID, "unknown integrator");
    if (nratios + 1 > kMaxDepth) return lg::abi_fail(ctx, LG_ERR_INVALID, "too many refinement levels");
    lg::amr::Base base{};
    for (int d = 0; d < 2; ++d) {
        base.cells[d] = cells[d];
        base.block[d] = block[d];
        base.origin[d] = origin[d];
        base.spacing[d] = spacing[d];
        if (!(spacing[d] > 0.0) || !std::isfinite(spacing[d]))
            return lg::abi_fail(ctx, LG_ERR_INVALID, "invalid spacing");
    }
    std::vector<uint32_t> r(ratios, ratios + nratios);
    std::vector<std::vector<lg::amr::Box>> levels;
    for (int64_t i = 0; i < npatches; ++i) {
        const int64_t lv = patches[5 * i];
        if (lv < 1 || lv > nratios) return lg::abi_fail(ctx, LG_ERR_INVALID, "patch level out of range");
        if ((int64_t)levels.size() < lv) levels.resize(lv);
        lg::amr::Box b;
        b.lo[0] = patches[5 * i + 1];
        b.lo[1] = patches[5 * i + 2];
        b.hi[0] = patches[5 * i + 3];
        b.hi[1] = patches[5 * i + 4];
        levels[lv - 1].push_back(b);
    }
    lg_amr_sim* s = new lg_amr_sim();
    s->ctx = ctx;
    std::string err = lg::amr::build_layout(base, r, levels, &s->layout);
    if (!err.empty()) {
        delete s;
        return lg::abi_fail(ctx, LG_ERR_INVALID, "AmrGrid: " + err);
    }
    s->model = model;
    if (mp) s->mp = *mp;
    s->kappa = kappa;
    s->integrator = integrator;
    s->seed = seed;
    s->nfields = model == LG_MODEL_C ? 2 : 1;
    if (policy) {
        s->has_policy = true;
        s->policy.every = std::max<int64_t>(1, policy->every);
        s->policy.buffer = policy->buffer;
        s->policy.min_width = policy->min_width;
        s->policy.efficiency = policy->efficiency;
        s->policy.threshold = policy->threshold;
        s->policy.field = policy->field;
        if (policy->field < 0 || policy->field >= s->nfields) {
            delete s;
            return lg::abi_fail(ctx, LG_ERR_INVALID, "tagged field out of range");
        }
    }
    cudaSetDevice(lg::abi_device(ctx));
    int rc = setup_device(s);
    if (rc == LG_OK && cudaMalloc(&s->d_t, 2 * sizeof(double)) != cudaSuccess) rc = LG_ERR_NOMEM;
    if (rc == LG_OK && cudaMemset(s->d_t, 0, 2 * sizeof(double)) != cudaSuccess) rc = LG_ERR_CUDA;
    if (rc != LG_OK) {
        free_device(s);
        cudaFree(s->d_t);
        delete s;
        return lg::abi_fail(ctx, rc, "AMR state allocation failed");
    }
    *out = s;
    return LG_OK;
}

int lg_amr_sim_destroy(lg_amr_sim* s) {
    if (!s) return LG_ERR_INVALID;
    cudaSetDevice(lg::abi_device(s->ctx));
    cudaStreamSynchronize(lg::abi_stream(s->ctx));
    free_device(s);
    cudaFree(s->d_t);
    cudaFree(s->d_tags);
    cudaFree(s->d_count);
    delete s;
    return LG_OK;
}

int lg_amr_sim_info(const lg_amr_sim* s, int64_t* num_blocks, int* num_levels, int64_t* epoch) {
    if (!s || !num_blocks || !num_levels || !epoch) return LG_ERR_INVALID;
    *num_blocks = s->layout.num_blocks();
    *num_levels = s->layout.num_levels();
    *epoch = s->epoch;
    return LG_OK;
}

int lg_amr_sim_patch(const lg_amr_sim* s, int64_t block, int64_t* out5) {
    if (!s || !out5 || block < 0 || block >= s->layout.num_blocks()) return LG_ERR_INVALID;
    const auto& p = s->layout.patches[block];
    out5[0] = p.level;
    out5[1] = p.bx.lo[0];
    out5[2] = p.bx.lo[1];
    out5[3] = p.bx.hi[0];
    out5[4] = p.bx.hi[1];
    return LG_OK;
}

int lg_amr_sim_field_len(const lg_amr_sim* s, int64_t* n) {
    if (!s || !n) return LG_ERR_INVALID;
    int64_t k = 0;
    for (const auto& b : s->plans.blocks) k += (int64_t)(b.nx + 2) * (b.ny + 2);
    *n = k;
    return LG_OK;
}

int lg_amr_sim_get_field(lg_amr_sim* s, int field, double* host, int64_t nelem) {
    if (!s || !host || field < 0 || field >= s->nfields) return fail(s, LG_ERR_INVALID, "bad field");
    int64_t n = 0;
    lg_amr_sim_field_len(s, &n);
    if (nelem != n) return fail(s, LG_ERR_INVALID, "element count must equal lg_amr_sim_field_len");
    cudaSetDevice(lg::abi_device(s->ctx));
    std::vector<std::vector<double>> blocks;
    int rc = download_blocks(s, field, blocks);
    if (rc != LG_OK) return rc;
    for (const auto& b : blocks) {
        std::memcpy(host, b.data(), b.size() * sizeof(double));
        host += b.size();
    }
    return LG_OK;
}

int lg_amr_sim_set_field(lg_amr_sim* s, int field, const double* host, int64_t nelem) {
    if (!s || !host || field < 0 || field >= s->nfields) return fail(s, LG_ERR_INVALID, "bad field");
    int64_t n = 0;
    lg_amr_sim_field_len(s, &n);
    if (nelem != n) return fail(s, LG_ERR_INVALID, "element count must equal lg_amr_sim_field_len");
    cudaSetDevice(lg::abi_device(s->ctx));
    std::vector<std::vector<double>> blocks(s->layout.num_blocks());
    for (int b = 0; b < s->layout.num_blocks(); ++b) {
        const auto& d = s->plans.blocks[b];
        blocks[b].assign(host, host + (size_t)(d.nx + 2) * (d.ny + 2));
        host += blocks[b].size();
    }
    return upload_blocks(s, field, blocks);
}

int lg_amr_sim_time(const lg_amr_sim* s, double* t, int64_t* step_index) {
    if (!s || !t || !step_index) return LG_ERR_INVALID;
    *t = s->t;
    *step_index = s->step_index;
    return LG_OK;
}

int lg_amr_sim_suggested_dt(const lg_amr_sim* s, double* dt) {
    if (!s || !dt) return LG_ERR_INVALID;
    // Subcycling::suggested_dt: level 0; a global-dt scheme: the finest
    // level the ratios allow (integrators/mod.rs:218-223, subcycling.rs:54-61)
    *dt = stable_dt_at(s, s->integrator == LG_AMR_SUBCYCLING ? 0 : (int)s->layout.level_spacing.size() - 1);
    return LG_OK;
}

int lg_amr_sim_step(lg_amr_sim* s, double dt, int64_t nsteps, uint32_t flags) {
    if (!s) return LG_ERR_INVALID;
    if (nsteps < 0) return fail(s, LG_ERR_INVALID, "negative step count");
    cudaSetDevice(lg::abi_device(s->ctx));
    cudaStream_t st = lg::abi_stream(s->ctx);
    AMR_CUDA(s, cudaMemcpyAsync(s->d_t + s->tslot, &s->t, sizeof(double), cudaMemcpyHostToDevice, st));
    int64_t done = 0;
    while (done < nsteps) {
        int rc = maybe_regrid(s);
        if (rc != LG_OK) return rc;
        // steps until the next regrid point, in pairs through a CUDA graph
        int64_t run = nsteps - done;
        if (s->has_policy) {
            const int64_t next = (s->step_index / s->policy.every + 1) * s->policy.every;
            run = std::min(run, next - s->step_index);
        }
        int64_t k = 0;
        if ((flags & LG_RUN_GRAPH) && run >= 2) {
            char key[160];
            snprintf(key, sizeof key, "%lld|%a|%d", (long long)s->epoch, dt, s->tslot);
            std::string gk = key;
            for (int c : s->cur) gk += c ? '1' : '0';
            auto it = s->graphs.find(gk);
            if (it == s->graphs.end()) {
                const std::vector<int> cur0 = s->cur;
                const int slot0 = s->tslot;
                const int64_t before = lg::abi_launches(s->ctx);
                cudaGraph_t graph = nullptr;
                AMR_CUDA(s, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                int rc2 = one_coarse_step(s, dt);
                if (rc2 == LG_OK) rc2 = one_coarse_step(s, dt);
                cudaError_t ec = cudaStreamEndCapture(st, &graph);
                const int64_t captured = lg::abi_launches(s->ctx) - before;
                lg::abi_set_launches(s->ctx, before);
                if (rc2 != LG_OK) {
                    if (graph) cudaGraphDestroy(graph);
                    return rc2;
                }
                AMR_CUDA(s, ec);
                if (s->cur != cur0 || s->tslot != slot0) {
                    cudaGraphDestroy(graph);
                    return fail(s, LG_ERR_STATE, "a captured pair of coarse steps must restore the buffer parity");
                }
                cudaGraphExec_t exec = nullptr;
                cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                AMR_CUDA(s, ei);
                it = s->graphs.emplace(gk, std::make_pair(exec, captured)).first;
            }
            for (; k + 2 <= run; k += 2) {
                AMR_CUDA(s, cudaGraphLaunch(it->second.first, st));
                lg::abi_count_launch(s->ctx, it->second.second);
                for (int r2 = 0; r2 < 2; ++r2) {
                    s->t += dt;
                    s->step_index += 1;
                }
            }
        }
        for (; k < run; ++k) {
            int rc2 = one_coarse_step(s, dt);
            if (rc2 != LG_OK) return rc2;
            s->t += dt;  // simulation.rs:285-286
            s->step_index += 1;
        }
        done += run;
    }
    return LG_OK;
}

int lg_amr_restrict(lg_amr_sim* s, int field) {
    if (!s || field < 0 || field >= s->nfields) return fail(s, LG_ERR_INVALID, "bad field");
    cudaSetDevice(lg::abi_device(s->ctx));
    for (int fine = s->layout.num_levels() - 1; fine >= 1; --fine) {
        int rc = launch_restrict(s, fine, field, field + 1);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

int lg_amr_fill_ghosts(lg_amr_sim* s) {
    if (!s) return LG_ERR_INVALID;
    cudaSetDevice(lg::abi_device(s->ctx));
    for (int level = 0; level < s->layout.num_levels(); ++level) {
        int rc = launch_fill(s, level, false, 0.0);
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

int lg_amr_tag_level(lg_amr_sim* s, int field, int level, double threshold, int64_t* cells_out, int64_t cap,
                     int64_t* count) {
    if (!s || !count || field < 0 || field >= s->nfields || level < 0 || level >= s->layout.num_levels())
        return fail(s, LG_ERR_INVALID, "bad tag arguments");
    cudaSetDevice(lg::abi_device(s->ctx));
    std::vector<std::array<int64_t, 2>> cells;
    int rc = tag_level(s, field, level, threshold, cells);
    if (rc != LG_OK) return rc;
    std::sort(cells.begin(), cells.end());
    *count = (int64_t)cells.size();
    for (int64_t k = 0; k < (int64_t)cells.size() && k < cap; ++k) {
        cells_out[2 * k] = cells[k][0];
        cells_out[2 * k + 1] = cells[k][1];
    }
    return LG_OK;
}

}  // extern "C"
