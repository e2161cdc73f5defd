// Batched Model C ensembles: many independent instances of one 2-D grid
// geometry (zero-flux boundaries) stepped together by the warp-strip kernel,
// each with its own eps4 and Wiener seed; and the gradient of a terminal
// loss by the hand-written adjoint (lg_adjoint.cu) with checkpointing.
//
// Device layout: every instance is a CartesianGrid's block-major state
// (phi and u slabs, ghost 1); the instances follow each other, so block b of
// the batch is block b % bpi of instance b / bpi.  The topology table wires
// the blocks of each instance and leaves -1 (mirror) at instance edges.
//
// value_and_grad: the forward pass stores the state every K steps; the
// backward sweep walks the segments from the last, recomputes a segment's
// states from its checkpoint (the noise replays from its counter-based keys
// and the stored segment-start time), and runs the adjoint steps back
// through it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/legendre_b200.h"
#include "lg_adjoint.h"
#include "lg_kernels.h"
#include "lg_state_view.h"

struct lg_ensemble {
    lg_ctx* ctx = nullptr;
    int dtype = LG_F64;
    int esize = 8;
    int64_t ninst = 0;
    int N0 = 0, N1 = 0, n0 = 0, n1 = 0, nb0 = 0, nb1 = 0, bpi = 0;
    double h[2] = {1.0, 1.0};
    lg_modelc_params p{};
    std::vector<double> eps4;
    std::vector<uint64_t> seeds;
    int64_t slab_stride = 0;
    int64_t state_elems = 0;  // per buffer: ninst * bpi * 2 * slab_stride
    // device
    int* d_nbr = nullptr;
    void* state[2] = {nullptr, nullptr};
    int cur = 0;
    double* d_t = nullptr;
    int tslot = 0;
    double t = 0.0;
    int64_t step_index = 0;
    void* d_fwd_params = nullptr;
    uint64_t* d_seeds = nullptr;
    void* d_adj_params = nullptr;
    std::map<std::string, std::pair<cudaGraphExec_t, int64_t>> graphs;  // exec, launches per replay
    // backward workspace
    std::vector<void*> ckpt, seg;
    std::vector<void*> res;   // every state of the resident tail segments
    uint64_t res_budget = 0;  // device bytes value_and_grad may keep states in
    void* adj[2] = {nullptr, nullptr};
    double* d_acc = nullptr;
    int64_t acc_cap = 0;  // doubles held by d_acc
    double* d_loss = nullptr;
    double* d_target = nullptr;
    double* d_usum = nullptr;  // per instance: the sum of the u cotangents (the Delta gradient's)
    int adj_kernel = lg::adj::kAdjointStrip;
    cudaStream_t aux = nullptr;          // the target's upload, beside the forward pass
    cudaEvent_t target_ready = nullptr;  // ... and its completion, awaited by the loss kernel
};

namespace {

int efail(lg_ensemble* e, int code, const std::string& m) { return lg::abi_fail(e ? e->ctx : nullptr, code, m); }

#define ENS_CUDA(e, call)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return efail((e), LG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

lg::CartTopo topo_of(const lg_ensemble* e) {
    lg::CartTopo t{};
    t.D = 2;
    t.n[0] = e->n0;
    t.n[1] = e->n1;
    t.n[2] = 1;
    t.nb[0] = e->nb0;
    t.nb[1] = e->nb1 * (int)e->ninst;
    t.nb[2] = 1;
    t.nblocks = (int)(e->ninst * e->bpi);
    t.nbr = e->d_nbr;
    return t;
}

lg::SlabLayout layout_of(const lg_ensemble* e) {
    lg::SlabLayout L{};
    L.nfields = 2;
    L.ghost = 1;
    L.slab_stride = e->slab_stride;
    L.len = (int64_t)(e->n0 + 2) * (e->n1 + 2);
    L.gdim[0] = e->n0 + 2;
    L.gdim[1] = e->n1 + 2;
    L.gdim[2] = 1;
    return L;
}

lg::adj::Geo geo_of(const lg_ensemble* e) {
    lg::adj::Geo g{};
    g.ninst = e->ninst;
    g.N0 = e->N0;
    g.N1 = e->N1;
    g.n0 = e->n0;
    g.n1 = e->n1;
    g.nb0 = e->nb0;
    g.bpi = e->bpi;
    g.slab_stride = e->slab_stride;
    return g;
}

// ModelC::new and KarmaRappelFlux::new for one instance's eps4
// (phasefield.rs:100-116, finite_volume.rs:113-122)
lg::ModelCDev model_of(const lg_ensemble* e, double eps4) {
    lg::ModelCDev m{};
    m.lambda = e->p.lambda;
    m.d_thermal = e->p.d_thermal;
    m.a_bar = std::fma(3.0, -eps4, 1.0);
    m.eps_prime = 3.0 * eps4 / m.a_bar;
    m.tol = e->p.anisotropy_tol;
    m.f_a_bar = std::fma(3.0, -eps4, 1.0);
    m.f_eps_prime = 3.0 * eps4 / m.f_a_bar;
    m.f_a12 = 4.0 * m.f_a_bar * m.f_eps_prime;
    m.f_tol = e->p.flux_tol;
    m.inv_h2_flux = 1.0 / (e->h[0] * e->h[1]);
    m.inv_h2[0] = 1.0 / (e->h[0] * e->h[0]);
    m.inv_h2[1] = 1.0 / (e->h[1] * e->h[1]);
    return m;
}

size_t state_bytes(const lg_ensemble* e) { return (size_t)e->state_elems * e->esize; }

int64_t slab_index(const lg_ensemble* e, int64_t inst, int X, int Y, int f) {
    const int bx = X / e->n0, by = Y / e->n1;
    const int64_t b = inst * e->bpi + bx + by * e->nb0;
    return (b * 2 + f) * e->slab_stride + (X - bx * e->n0 + 1) + (int64_t)(Y - by * e->n1 + 1) * (e->n0 + 2);
}

int fill_ghosts(lg_ensemble* e, void* buf) {
    const lg::CartTopo topo = topo_of(e);
    const lg::SlabLayout L = layout_of(e);
    for (int f = 0; f < 2; ++f) {
        ENS_CUDA(e, lg::launch_halo_fill(buf, e->esize, topo, L, f, lg::abi_stream(e->ctx)));
        lg::abi_count_launch(e->ctx, 1);
    }
    return LG_OK;
}

// one step x(in) -> x(out), reading time slot `slot`
int step_once(lg_ensemble* e, const void* in, void* out, double dt, int slot) {
    const lg::CartTopo topo = topo_of(e);
    const lg::SlabLayout L = layout_of(e);
    cudaError_t err;
    if (e->dtype == LG_F64)
        err = lg::launch_modelc_batch_f64((const double*)in, (double*)out, topo, L, e->d_fwd_params, e->d_seeds,
                                          e->bpi, dt, e->p.noise_amplitude, e->d_t, slot, 0, lg::abi_stream(e->ctx));
    else
        err = lg::launch_modelc_batch_f32((const float*)in, (float*)out, topo, L, e->d_fwd_params, e->d_seeds, e->bpi,
                                          dt, e->p.noise_amplitude, e->d_t, slot, 0, lg::abi_stream(e->ctx));
    lg::abi_count_launch(e->ctx, 1);
    if (err != cudaSuccess) return efail(e, LG_ERR_CUDA, std::string("ensemble step: ") + cudaGetErrorString(err));
    return LG_OK;
}

void free_workspace(lg_ensemble* e) {
    for (void* p : e->ckpt) cudaFree(p);
    for (void* p : e->seg) cudaFree(p);
    for (void* p : e->res) cudaFree(p);
    e->ckpt.clear();
    e->seg.clear();
    e->res.clear();
    for (void*& p : e->adj) {
        cudaFree(p);
        p = nullptr;
    }
    cudaFree(e->d_acc);
    cudaFree(e->d_loss);
    cudaFree(e->d_target);
    cudaFree(e->d_usum);
    e->d_acc = e->d_loss = e->d_target = e->d_usum = nullptr;
}

void free_all(lg_ensemble* e) {
    if (e->target_ready) cudaEventDestroy(e->target_ready);
    if (e->aux) cudaStreamDestroy(e->aux);
    e->target_ready = nullptr;
    e->aux = nullptr;
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second.first);
    e->graphs.clear();
    free_workspace(e);
    cudaFree(e->d_nbr);
    for (void* p : e->state) cudaFree(p);
    cudaFree(e->d_t);
    cudaFree(e->d_fwd_params);
    cudaFree(e->d_seeds);
    cudaFree(e->d_adj_params);
}

int alloc_states(lg_ensemble* e, std::vector<void*>& v, size_t n) {
    while (v.size() > n) {
        cudaFree(v.back());
        v.pop_back();
    }
    while (v.size() < n) {
        void* p = nullptr;
        if (cudaMalloc(&p, state_bytes(e)) != cudaSuccess) {
            cudaGetLastError();
            return efail(e, LG_ERR_NOMEM, "ensemble checkpoint storage: out of device memory");
        }
        v.push_back(p);
    }
    return LG_OK;
}

// The sum of field f's interior cells of every instance, in a fixed order
// (the same bits on every call): CTA i takes instance i, thread t the cells
// t, t + 256, ... in (block, row, column) order, then a fixed shuffle tree
// and the warps in order.
template <class T>
__global__ void __launch_bounds__(256) instance_field_sum_kernel(const T* __restrict__ arena, int64_t slab_stride,
                                                                 int bpi, int n0, int n1, int f, double* out) {
    const int64_t per_block = (int64_t)n0 * n1, cells = per_block * bpi;
    const T* base = arena + (int64_t)blockIdx.x * bpi * 2 * slab_stride;
    double s = 0.0;
    for (int64_t c = threadIdx.x; c < cells; c += blockDim.x) {
        const int b = (int)(c / per_block);
        const int rem = (int)(c - (int64_t)b * per_block);
        const int y = rem / n0, x = rem - y * n0;
        s += (double)base[((int64_t)b * 2 + f) * slab_stride + (x + 1) + (int64_t)(y + 1) * (n0 + 2)];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ double w[8];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += w[k];
        out[blockIdx.x] = t;
    }
}

// interior rows of one field of every instance, from a host image of the
// arena into the instance-major, row-major host layout
template <class T>
void gather_rows(const lg_ensemble* e, const std::vector<char>& img, int f, double* host) {
    const T* a = reinterpret_cast<const T*>(img.data());
    for (int64_t i = 0; i < e->ninst; ++i)
        for (int by = 0; by < e->nb1; ++by)
            for (int bx = 0; bx < e->nb0; ++bx) {
                const int64_t b = i * e->bpi + bx + (int64_t)by * e->nb0;
                const T* slab = a + (b * 2 + f) * e->slab_stride;
                for (int y = 0; y < e->n1; ++y) {
                    const T* src = slab + 1 + (int64_t)(y + 1) * (e->n0 + 2);
                    double* dst = host + (i * e->N1 + (int64_t)by * e->n1 + y) * e->N0 + (int64_t)bx * e->n0;
                    for (int x = 0; x < e->n0; ++x) dst[x] = (double)src[x];
                }
            }
}

}  // namespace

extern "C" {

int lg_ensemble_create(lg_ctx* ctx, const int64_t* cells, const int64_t* block, const double* spacing, int64_t ninst,
                       const lg_modelc_params* p, const double* eps4, const uint64_t* seeds, int dtype,
                       lg_ensemble** out) {
    if (!ctx || !cells || !block || !spacing || !p || !eps4 || !seeds || !out || ninst < 1)
        return lg::abi_fail(ctx, LG_ERR_INVALID, "bad ensemble arguments");
    *out = nullptr;
    if (dtype != LG_F64 && dtype != LG_F32) return lg::abi_fail(ctx, LG_ERR_INVALID, "dtype must be LG_F64 or LG_F32");
    for (int d = 0; d < 2; ++d) {
        if (block[d] < 2 || cells[d] < block[d] || cells[d] % block[d] != 0 || cells[d] > (int64_t(1) << 20))
            return lg::abi_fail(ctx, LG_ERR_INVALID, "cells must be positive multiples of a block of at least 2");
        if (!(spacing[d] > 0.0) || !std::isfinite(spacing[d])) return lg::abi_fail(ctx, LG_ERR_INVALID, "bad spacing");
    }
    const int64_t bpi = (cells[0] / block[0]) * (cells[1] / block[1]);
    if (bpi * ninst > (int64_t(1) << 30)) return lg::abi_fail(ctx, LG_ERR_INVALID, "too many blocks");
    lg_ensemble* e = new lg_ensemble();
    e->ctx = ctx;
    e->dtype = dtype;
    e->esize = dtype == LG_F64 ? 8 : 4;
    e->ninst = ninst;
    e->N0 = (int)cells[0];
    e->N1 = (int)cells[1];
    e->n0 = (int)block[0];
    e->n1 = (int)block[1];
    e->nb0 = e->N0 / e->n0;
    e->nb1 = e->N1 / e->n1;
    e->bpi = (int)bpi;
    e->h[0] = spacing[0];
    e->h[1] = spacing[1];
    e->p = *p;
    e->eps4.assign(eps4, eps4 + ninst);
    e->seeds.assign(seeds, seeds + ninst);
    const int64_t align = 256 / e->esize;
    e->slab_stride = ((int64_t)(e->n0 + 2) * (e->n1 + 2) + align - 1) / align * align;
    e->state_elems = ninst * e->bpi * 2 * e->slab_stride;
    cudaSetDevice(lg::abi_device(ctx));
    // topology: each instance's blocks, mirror (-1) at instance edges
    std::vector<int> nbr((size_t)(ninst * e->bpi) * 6, -1);
    for (int64_t i = 0; i < ninst; ++i)
        for (int by = 0; by < e->nb1; ++by)
            for (int bx = 0; bx < e->nb0; ++bx) {
                const int64_t b = i * e->bpi + bx + by * e->nb0;
                int* q = &nbr[(size_t)b * 6];
                q[0] = bx > 0 ? (int)(b - 1) : -1;
                q[1] = bx < e->nb0 - 1 ? (int)(b + 1) : -1;
                q[2] = by > 0 ? (int)(b - e->nb0) : -1;
                q[3] = by < e->nb1 - 1 ? (int)(b + e->nb0) : -1;
            }
    const int kind = dtype == LG_F64 ? 0 : 1;
    const size_t fsz = dtype == LG_F64 ? lg::modelc_record_size_f64() : lg::modelc_record_size_f32();
    const size_t asz = lg::adj::adj_params_size(kind);
    std::vector<char> fwd((size_t)ninst * fsz), adjp((size_t)ninst * asz);
    for (int64_t i = 0; i < ninst; ++i) {
        const lg::ModelCDev m = model_of(e, eps4[i]);
        if (dtype == LG_F64)
            lg::modelc_record_f64(m, fwd.data() + i * fsz);
        else
            lg::modelc_record_f32(m, fwd.data() + i * fsz);
        lg::adj::adj_params(kind, m, adjp.data() + i * asz);
    }
    cudaError_t err = cudaMalloc(&e->d_nbr, nbr.size() * sizeof(int));
    if (err == cudaSuccess) err = cudaMemcpy(e->d_nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice);
    for (int k = 0; k < 2 && err == cudaSuccess; ++k) {
        err = cudaMalloc(&e->state[k], state_bytes(e));
        if (err == cudaSuccess) err = cudaMemset(e->state[k], 0, state_bytes(e));
    }
    if (err == cudaSuccess) err = cudaMalloc(&e->d_t, 2 * sizeof(double));
    if (err == cudaSuccess) err = cudaMemset(e->d_t, 0, 2 * sizeof(double));
    if (err == cudaSuccess) err = cudaMalloc(&e->d_fwd_params, fwd.size());
    if (err == cudaSuccess) err = cudaMemcpy(e->d_fwd_params, fwd.data(), fwd.size(), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMalloc(&e->d_adj_params, adjp.size());
    if (err == cudaSuccess) err = cudaMemcpy(e->d_adj_params, adjp.data(), adjp.size(), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMalloc(&e->d_seeds, ninst * sizeof(uint64_t));
    if (err == cudaSuccess) err = cudaMemcpy(e->d_seeds, seeds, ninst * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        cudaGetLastError();
        free_all(e);
        delete e;
        return lg::abi_fail(ctx, LG_ERR_NOMEM, std::string("ensemble allocation: ") + cudaGetErrorString(err));
    }
    *out = e;
    return LG_OK;
}

int lg_ensemble_destroy(lg_ensemble* e) {
    if (!e) return LG_ERR_INVALID;
    cudaSetDevice(lg::abi_device(e->ctx));
    cudaStreamSynchronize(lg::abi_stream(e->ctx));
    free_all(e);
    delete e;
    return LG_OK;
}

int lg_ensemble_upload(lg_ensemble* e, int field, const double* host, int64_t n) {
    if (!e || !host || field < 0 || field > 1) return efail(e, LG_ERR_INVALID, "bad field");
    if (n != e->ninst * e->N0 * e->N1) return efail(e, LG_ERR_INVALID, "element count must be instances * cells");
    cudaSetDevice(lg::abi_device(e->ctx));
    cudaStream_t st = lg::abi_stream(e->ctx);
    std::vector<char> img(state_bytes(e));
    ENS_CUDA(e, cudaMemcpyAsync(img.data(), e->state[e->cur], img.size(), cudaMemcpyDeviceToHost, st));
    ENS_CUDA(e, cudaStreamSynchronize(st));
    for (int64_t i = 0; i < e->ninst; ++i)
        for (int Y = 0; Y < e->N1; ++Y)
            for (int X = 0; X < e->N0; ++X) {
                const double v = host[(i * e->N1 + Y) * e->N0 + X];
                const int64_t o = slab_index(e, i, X, Y, field);
                if (e->dtype == LG_F64)
                    reinterpret_cast<double*>(img.data())[o] = v;
                else
                    reinterpret_cast<float*>(img.data())[o] = (float)v;
            }
    ENS_CUDA(e, cudaMemcpyAsync(e->state[e->cur], img.data(), img.size(), cudaMemcpyHostToDevice, st));
    int rc = fill_ghosts(e, e->state[e->cur]);
    if (rc != LG_OK) return rc;
    ENS_CUDA(e, cudaStreamSynchronize(st));
    return LG_OK;
}

int lg_ensemble_download(lg_ensemble* e, int field, double* host, int64_t n) {
    if (!e || !host || field < 0 || field > 1) return efail(e, LG_ERR_INVALID, "bad field");
    if (n != e->ninst * e->N0 * e->N1) return efail(e, LG_ERR_INVALID, "element count must be instances * cells");
    cudaSetDevice(lg::abi_device(e->ctx));
    cudaStream_t st = lg::abi_stream(e->ctx);
    std::vector<char> img(state_bytes(e));
    ENS_CUDA(e, cudaMemcpyAsync(img.data(), e->state[e->cur], img.size(), cudaMemcpyDeviceToHost, st));
    ENS_CUDA(e, cudaStreamSynchronize(st));
    if (e->dtype == LG_F64)
        gather_rows<double>(e, img, field, host);
    else
        gather_rows<float>(e, img, field, host);
    return LG_OK;
}

int lg_ensemble_set_time(lg_ensemble* e, double t, int64_t step_index) {
    if (!e) return LG_ERR_INVALID;
    e->t = t;
    e->step_index = step_index;
    return LG_OK;
}

int lg_ensemble_get_time(const lg_ensemble* e, double* t, int64_t* step_index) {
    if (!e || !t || !step_index) return LG_ERR_INVALID;
    *t = e->t;
    *step_index = e->step_index;
    return LG_OK;
}

int lg_ensemble_run(lg_ensemble* e, double dt, int64_t nsteps, uint32_t flags) {
    if (!e || nsteps < 0) return efail(e, LG_ERR_INVALID, "bad run arguments");
    cudaSetDevice(lg::abi_device(e->ctx));
    cudaStream_t st = lg::abi_stream(e->ctx);
    ENS_CUDA(e, cudaMemcpyAsync(e->d_t + e->tslot, &e->t, sizeof(double), cudaMemcpyHostToDevice, st));
    ENS_CUDA(e, cudaStreamSynchronize(st));
    int64_t k = 0;
    if ((flags & LG_RUN_GRAPH) && nsteps >= 2) {  // pairs of steps restore the buffer and the time slot
        char key[96];
        snprintf(key, sizeof key, "%a|%d|%d", dt, e->cur, e->tslot);
        auto it = e->graphs.find(key);
        if (it == e->graphs.end()) {
            cudaGraph_t g = nullptr;
            ENS_CUDA(e, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int rc = step_once(e, e->state[e->cur], e->state[e->cur ^ 1], dt, e->tslot);
            if (rc == LG_OK) rc = step_once(e, e->state[e->cur ^ 1], e->state[e->cur], dt, e->tslot ^ 1);
            const cudaError_t ec = cudaStreamEndCapture(st, &g);
            lg::abi_count_launch(e->ctx, -2);  // captured, not launched: counted on each replay
            if (rc != LG_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            ENS_CUDA(e, ec);
            cudaGraphExec_t ex = nullptr;
            const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            ENS_CUDA(e, ei);
            it = e->graphs.emplace(key, std::make_pair(ex, int64_t(2))).first;
        }
        for (; k + 2 <= nsteps; k += 2) {
            ENS_CUDA(e, cudaGraphLaunch(it->second.first, st));
            lg::abi_count_launch(e->ctx, it->second.second);
            for (int r = 0; r < 2; ++r) {
                e->t += dt;
                e->step_index += 1;
            }
        }
    }
    for (; k < nsteps; ++k) {
        int rc = step_once(e, e->state[e->cur], e->state[e->cur ^ 1], dt, e->tslot);
        if (rc != LG_OK) return rc;
        e->cur ^= 1;
        e->tslot ^= 1;
        e->t += dt;  // simulation.rs:285-286
        e->step_index += 1;
    }
    return LG_OK;
}

int lg_ensemble_value_and_grad(lg_ensemble* e, double dt, int64_t nsteps, int64_t ckpt_every, const double* target,
                               double* loss, double* grad_params, double* grad_phi0, double* grad_u0) {
    if (!e || !target || !loss || !grad_params || nsteps < 1 || ckpt_every < 1)
        return efail(e, LG_ERR_INVALID, "bad value_and_grad arguments");
    cudaSetDevice(lg::abi_device(e->ctx));
    cudaStream_t st = lg::abi_stream(e->ctx);
    const int kind = e->dtype == LG_F64 ? 0 : 1;
    const int64_t K = std::min(ckpt_every, nsteps);
    const int64_t nseg = (nsteps + K - 1) / K;
    const lg::adj::Geo geo = geo_of(e);
    const int64_t cells = e->ninst * e->N0 * e->N1;
    // resident tail: the last segments whose every state fits in the budget
    // keep them from the forward pass and skip their recomputation
    int64_t nres = 0, used = 0;
    for (int64_t s = nseg - 1; s >= 0; --s) {
        const int64_t len = std::min(K, nsteps - s * K);
        if ((uint64_t)(used + len) * (uint64_t)state_bytes(e) > e->res_budget) break;
        used += len;
        ++nres;
    }
    const int64_t first_res = nseg - nres, n_res0 = first_res * K;
    // workspace: a checkpoint per recomputed segment, K - 1 recomputed
    // states, the resident states, two cotangent buffers
    int rc = alloc_states(e, e->ckpt, (size_t)first_res);
    if (rc == LG_OK) rc = alloc_states(e, e->seg, (size_t)(first_res > 0 ? std::max<int64_t>(K - 1, 0) : 0));
    if (rc == LG_OK) rc = alloc_states(e, e->res, (size_t)used);
    if (rc != LG_OK) return rc;
    const int64_t acc_n = 3 * lg::adj::adjoint_items(kind, e->adj_kernel, geo), loss_n = lg::adj::loss_items(geo);
    if (!e->adj[0]) {
        for (void*& q : e->adj) ENS_CUDA(e, cudaMalloc(&q, state_bytes(e)));
        ENS_CUDA(e, cudaMalloc(&e->d_loss, loss_n * sizeof(double)));
        ENS_CUDA(e, cudaMalloc(&e->d_target, cells * sizeof(double)));
        ENS_CUDA(e, cudaMalloc(&e->d_usum, e->ninst * sizeof(double)));
    }
    // the accumulator slots, then the strip form's work-list counter
    if (e->acc_cap < acc_n + 1) {
        cudaFree(e->d_acc);
        e->d_acc = nullptr;
        e->acc_cap = 0;
        ENS_CUDA(e, cudaMalloc(&e->d_acc, (acc_n + 1) * sizeof(double)));
        e->acc_cap = acc_n + 1;
    }
    const bool listed = e->adj_kernel == lg::adj::kAdjointStrip;
    unsigned long long* work = listed ? reinterpret_cast<unsigned long long*>(e->d_acc + acc_n) : nullptr;
    // each strip launch advances the counter by its number of units, so the
    // base of a launch is the units of the launches before it in this call
    const unsigned long long per_launch = (unsigned long long)(acc_n / 3);
    unsigned long long ticket = 0;
    ENS_CUDA(e, cudaMemsetAsync(e->d_acc, 0, (acc_n + 1) * sizeof(double), st));
    for (void* q : e->adj) ENS_CUDA(e, cudaMemsetAsync(q, 0, state_bytes(e), st));

    // forward pass: checkpoints of the recomputed segments; the resident
    // segments' states are written in place (x_n in res[n - n_res0])
    std::vector<double> tseg((size_t)nseg);
    ENS_CUDA(e, cudaMemcpyAsync(e->d_t + e->tslot, &e->t, sizeof(double), cudaMemcpyHostToDevice, st));
    ENS_CUDA(e, cudaStreamSynchronize(st));
    for (int64_t n = 0; n < nsteps; ++n) {
        if (n % K == 0) tseg[(size_t)(n / K)] = e->t;
        if (n < n_res0) {
            if (n % K == 0)
                ENS_CUDA(e, cudaMemcpyAsync(e->ckpt[(size_t)(n / K)], e->state[e->cur], state_bytes(e),
                                            cudaMemcpyDeviceToDevice, st));
            rc = step_once(e, e->state[e->cur], e->state[e->cur ^ 1], dt, e->tslot);
            if (rc != LG_OK) return rc;
            e->cur ^= 1;
        } else {
            const int64_t i = n - n_res0;
            if (i == 0)
                ENS_CUDA(e, cudaMemcpyAsync(e->res[0], e->state[e->cur], state_bytes(e), cudaMemcpyDeviceToDevice,
                                            st));
            const bool last = i + 1 == used;
            rc = step_once(e, e->res[(size_t)i], last ? e->state[e->cur ^ 1] : e->res[(size_t)(i + 1)], dt, e->tslot);
            if (rc != LG_OK) return rc;
            if (last) e->cur ^= 1;
        }
        e->tslot ^= 1;
        e->t += dt;
        e->step_index += 1;
    }
    // the target crosses from the host while the queued forward steps run:
    // its copy goes on a second stream (from pageable memory it holds this
    // thread until the bytes are staged), and the loss kernel, its first
    // reader, waits for it.  The previous call's reads of d_target ended at
    // that call's closing synchronisation.
    if (!e->aux) {
        ENS_CUDA(e, cudaStreamCreateWithFlags(&e->aux, cudaStreamNonBlocking));
        ENS_CUDA(e, cudaEventCreateWithFlags(&e->target_ready, cudaEventDisableTiming));
    }
    ENS_CUDA(e, cudaMemcpyAsync(e->d_target, target, cells * sizeof(double), cudaMemcpyHostToDevice, e->aux));
    ENS_CUDA(e, cudaEventRecord(e->target_ready, e->aux));
    ENS_CUDA(e, cudaStreamWaitEvent(st, e->target_ready, 0));
    // terminal loss and the seed of the backward sweep
    int a = 0;
    ENS_CUDA(e, lg::adj::launch_loss_seed(kind, e->state[e->cur], e->d_target, e->adj[a], geo, e->d_loss, st));
    lg::abi_count_launch(e->ctx, 1);
    // backward sweep
    double t_start = 0.0;
    for (int64_t s = nseg - 1; s >= 0; --s) {
        const int64_t len = std::min(K, nsteps - s * K);
        if (s >= first_res) {  // resident: x_{sK+i} is res[sK + i - n_res0]
            for (int64_t i = len - 1; i >= 0; --i) {
                const void* x = e->res[(size_t)(s * K + i - n_res0)];
                ENS_CUDA(e, lg::adj::launch_adjoint_step(kind, e->adj_kernel, x, e->adj[a], e->adj[a ^ 1],
                                                         e->d_adj_params, geo, dt, e->d_acc, work, ticket, st));
                lg::abi_count_launch(e->ctx, 1);
                ticket += per_launch;
                a ^= 1;
            }
            continue;
        }
        t_start = tseg[(size_t)s];
        ENS_CUDA(e, cudaMemcpyAsync(e->d_t, &t_start, sizeof(double), cudaMemcpyHostToDevice, st));
        ENS_CUDA(e, cudaStreamSynchronize(st));  // the host scalar is rewritten for the next segment
        int slot = 0;
        for (int64_t i = 1; i < len; ++i) {  // x_{sK+i} into seg[i-1]
            const void* in = i == 1 ? e->ckpt[(size_t)s] : e->seg[(size_t)(i - 2)];
            rc = step_once(e, in, e->seg[(size_t)(i - 1)], dt, slot);
            if (rc != LG_OK) return rc;
            slot ^= 1;
        }
        for (int64_t i = len - 1; i >= 0; --i) {
            const void* x = i == 0 ? e->ckpt[(size_t)s] : e->seg[(size_t)(i - 1)];
            ENS_CUDA(e, lg::adj::launch_adjoint_step(kind, e->adj_kernel, x, e->adj[a], e->adj[a ^ 1],
                                                     e->d_adj_params, geo, dt, e->d_acc, work, ticket, st));
            lg::abi_count_launch(e->ctx, 1);
            ticket += per_launch;
            a ^= 1;
        }
    }
    // the device time slot of the state holds the state's time again
    ENS_CUDA(e, cudaMemcpyAsync(e->d_t + e->tslot, &e->t, sizeof(double), cudaMemcpyHostToDevice, st));
    // results: the parameter partials, the loss, the Delta gradient as the
    // device's fixed-order sum of the u cotangents (u_0 = -Delta on every
    // cell); the cell cotangents cross to the host only when asked for
    if (e->dtype == LG_F64)
        instance_field_sum_kernel<double><<<(unsigned)e->ninst, 256, 0, st>>>(
            static_cast<const double*>(e->adj[a]), e->slab_stride, e->bpi, e->n0, e->n1, 1, e->d_usum);
    else
        instance_field_sum_kernel<float><<<(unsigned)e->ninst, 256, 0, st>>>(
            static_cast<const float*>(e->adj[a]), e->slab_stride, e->bpi, e->n0, e->n1, 1, e->d_usum);
    lg::abi_count_launch(e->ctx, 1);
    ENS_CUDA(e, cudaGetLastError());
    std::vector<double> acc((size_t)acc_n), lossv((size_t)loss_n), usum((size_t)e->ninst);
    ENS_CUDA(e, cudaMemcpyAsync(acc.data(), e->d_acc, acc_n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ENS_CUDA(e, cudaMemcpyAsync(lossv.data(), e->d_loss, loss_n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ENS_CUDA(e, cudaMemcpyAsync(usum.data(), e->d_usum, e->ninst * sizeof(double), cudaMemcpyDeviceToHost, st));
    std::vector<char> img;
    if (grad_phi0 || grad_u0) {
        img.resize(state_bytes(e));
        ENS_CUDA(e, cudaMemcpyAsync(img.data(), e->adj[a], img.size(), cudaMemcpyDeviceToHost, st));
    }
    ENS_CUDA(e, cudaStreamSynchronize(st));
    for (int f = 0; f < 2; ++f) {
        double* dst = f == 0 ? grad_phi0 : grad_u0;
        if (!dst) continue;
        if (e->dtype == LG_F64)
            gather_rows<double>(e, img, f, dst);
        else
            gather_rows<float>(e, img, f, dst);
    }
    const int64_t acc_tiles = acc_n / 3 / e->ninst, loss_tiles = loss_n / e->ninst;
    for (int64_t i = 0; i < e->ninst; ++i) {  // fixed summation order: reproducible
        double l = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
        for (int64_t k = 0; k < loss_tiles; ++k) l += lossv[(size_t)(i * loss_tiles + k)];
        for (int64_t k = 0; k < acc_tiles; ++k) {
            const double* q = &acc[(size_t)(3 * (i * acc_tiles + k))];
            g0 += q[0];
            g1 += q[1];
            g2 += q[2];
        }
        const double gd = -usum[(size_t)i];
        loss[i] = l;
        grad_params[4 * i + 0] = g0;
        grad_params[4 * i + 1] = g1;
        grad_params[4 * i + 2] = g2;
        grad_params[4 * i + 3] = gd;
    }
    return LG_OK;
}

int lg_ensemble_set_resident_budget(lg_ensemble* e, uint64_t bytes) {
    if (!e) return LG_ERR_INVALID;
    e->res_budget = bytes;
    if (bytes == 0) {  // give the resident states back
        for (void* p : e->res) cudaFree(p);
        e->res.clear();
    }
    return LG_OK;
}

int lg_ensemble_set_adjoint_kernel(lg_ensemble* e, int kernel) {
    if (!e) return LG_ERR_INVALID;
    if (kernel != LG_ADJOINT_STRIP && kernel != LG_ADJOINT_TILE)
        return efail(e, LG_ERR_INVALID, "unknown adjoint kernel");
    e->adj_kernel = kernel == LG_ADJOINT_STRIP ? lg::adj::kAdjointStrip : lg::adj::kAdjointTile;
    return LG_OK;
}

// The backward API of one Simulation: its state (a 2-D zero-flux Model C
// state of phi and u, ghost 1) is exactly the block-major arena of a
// one-instance ensemble -- same slabs, same order, same stride -- so the
// state moves into such an ensemble by one device copy, goes through
// value_and_grad, and x_T moves back the same way.  The instance's noise
// keys are the Simulation's (its seed, its time, the block ids), so the
// forward pass inside is the trajectory lg_modelc_em_run produces.
int lg_modelc_value_and_grad(lg_state* state, const lg_modelc_params* p, double dt, uint64_t seed, int64_t nsteps,
                             int64_t ckpt_every, const double* target, double* loss, double* grad_params,
                             double* grad_phi0, double* grad_u0) {
    lg::StateView v{};
    if (!state || !p || lg::abi_state_view(state, &v) != LG_OK) return LG_ERR_INVALID;
    if (v.D != 2 || v.nfields != 2 || v.ghosts[0] != 1 || v.ghosts[1] != 1)
        return lg::abi_fail(v.ctx, LG_ERR_STATE, "value_and_grad needs a 2-D Model C state of phi and u (ghost 1)");
    if (v.periodic[0] || v.periodic[1])
        return lg::abi_fail(v.ctx, LG_ERR_STATE, "value_and_grad supports zero-flux (mirror) boundaries only");
    double t = 0.0;
    int64_t step = 0;
    lg_state_get_time(state, &t, &step);
    const int64_t cells[2] = {v.block[0] * v.nb[0], v.block[1] * v.nb[1]};
    const int64_t block[2] = {v.block[0], v.block[1]};
    const double spacing[2] = {v.spacing[0], v.spacing[1]};
    const double eps4 = p->eps4;
    lg_ensemble* e = nullptr;
    int rc = lg_ensemble_create(v.ctx, cells, block, spacing, 1, p, &eps4, &seed, v.dtype, &e);
    if (rc != LG_OK) return rc;
    cudaStream_t st = lg::abi_stream(v.ctx);
    const size_t bytes = (size_t)state_bytes(e);
    if (e->slab_stride != v.slab_stride || bytes != (size_t)v.nblocks * 2 * v.slab_stride * v.esize) {
        lg_ensemble_destroy(e);
        return lg::abi_fail(v.ctx, LG_ERR_STATE, "state layout differs from the ensemble's");
    }
    cudaError_t ce = cudaMemcpyAsync(e->state[e->cur], v.arena, bytes, cudaMemcpyDeviceToDevice, st);
    if (ce == cudaSuccess) rc = fill_ghosts(e, e->state[e->cur]);
    else rc = lg::abi_fail(v.ctx, LG_ERR_CUDA, std::string("state copy: ") + cudaGetErrorString(ce));
    if (rc == LG_OK) {
        e->t = t;
        e->step_index = step;
        rc = lg_ensemble_value_and_grad(e, dt, nsteps, ckpt_every, target, loss, grad_params, grad_phi0, grad_u0);
    }
    if (rc == LG_OK) {
        ce = cudaMemcpyAsync(v.arena_rw, e->state[e->cur], bytes, cudaMemcpyDeviceToDevice, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) rc = lg::abi_fail(v.ctx, LG_ERR_CUDA, std::string("state copy: ") + cudaGetErrorString(ce));
        else lg_state_set_time(state, e->t, e->step_index);
    }
    lg_ensemble_destroy(e);
    return rc;
}

}  // extern "C"
