// C ABI of the legendre B200 library: contexts (the CudaScheduler), device
// block-topology tables, state arenas (the CudaAllocator), run loops and
// CUDA-graph capture of step sequences.  Declarations and contracts live in
// include/legendre_b200.h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/legendre_b200.h"
#include "lg_state_view.h"
#include "lg_kernels.h"

struct lg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int64_t launches = 0;
    std::map<std::string, int> tuned;  // Model C variant chosen by lg_modelc_autotune, per shape
    int* d_flag = nullptr;  // set by a kernel whose bounded device wait gave up (allocated on first use)
};

struct lg_grid {
    lg_ctx* ctx = nullptr;
    int D = 0;
    int64_t cells[3] = {1, 1, 1}, block[3] = {1, 1, 1}, nb[3] = {1, 1, 1};
    double origin[3] = {0, 0, 0}, spacing[3] = {1, 1, 1};
    int periodic[3] = {0, 0, 0};
    int64_t nblocks = 0;
    std::vector<int> h_nbr;  // nblocks * 3 * 2
    int* d_nbr = nullptr;
};

struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t steps = 0;
    int64_t launches = 0;
};

struct lg_state {
    lg_ctx* ctx = nullptr;
    const lg_grid* grid = nullptr;
    int dtype = LG_F64;
    int esize = 8;
    int nfields = 0;
    std::vector<int> ghosts;
    int64_t slab_stride = 0;  // elements
    void* arena[2] = {nullptr, nullptr};
    int cur = 0;
    double* d_t = nullptr;    // two time slots
    int tslot = 0;
    double t = 0.0;
    int64_t step_index = 0;
    bool ghosts_valid = false;
    std::map<std::string, GraphEntry> graphs;
    // multi-grain Model C: the theta0 field and cos/sin theta0 of every
    // interior cell on the device (cos block-major, then sin), state dtype
    int theta_field = -1;
    void* orient = nullptr;
    // RungeKutta4 workspace (allocated at the first RK4 run): k1, k2, k3 and
    // two stage states, each an arena of the state's layout
    void* rk[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

namespace {

int fail(lg_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(lg_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, LG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define LG_CUDA(ctx, call)                                        \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
    } while (0)

int64_t block_len(const lg_grid* g, int ghost) {
    int64_t n = 1;
    for (int d = 0; d < g->D; ++d) n *= g->block[d] + 2 * ghost;
    return n;
}

lg::CartTopo topo_of(const lg_grid* g) {
    lg::CartTopo t{};
    t.D = g->D;
    for (int d = 0; d < 3; ++d) {
        t.n[d] = (int)g->block[d];
        t.nb[d] = (int)g->nb[d];
    }
    t.nblocks = (int)g->nblocks;
    t.nbr = g->d_nbr;
    return t;
}

lg::SlabLayout layout_of(const lg_state* st, int field) {
    lg::SlabLayout L{};
    L.nfields = st->nfields;
    L.ghost = st->ghosts[field];
    L.slab_stride = st->slab_stride;
    L.len = block_len(st->grid, L.ghost);
    for (int d = 0; d < 3; ++d) L.gdim[d] = d < st->grid->D ? (int)st->grid->block[d] + 2 * L.ghost : 1;
    return L;
}

// face_neighbor (cartesian.rs:162-181)
int64_t face_neighbor(const lg_grid* g, int64_t b, int dim, int dir) {
    int64_t c[3] = {0, 0, 0}, rem = b;
    for (int d = 0; d < g->D; ++d) {
        c[d] = rem % g->nb[d];
        rem /= g->nb[d];
    }
    int64_t stepped = c[dim] + (dir < 0 ? -1 : 1), next;
    if (stepped >= 0 && stepped < g->nb[dim]) next = stepped;
    else if (g->periodic[dim]) next = ((stepped % g->nb[dim]) + g->nb[dim]) % g->nb[dim];
    else return -1;
    int64_t id = 0, stride = 1;
    for (int d = 0; d < g->D; ++d) {
        id += (d == dim ? next : c[d]) * stride;
        stride *= g->nb[d];
    }
    return id;
}

int fill_all_ghosts(lg_state* st) {
    lg_ctx* ctx = st->ctx;
    for (int f = 0; f < st->nfields; ++f) {
        if (st->ghosts[f] == 0) continue;
        cudaError_t e = lg::launch_halo_fill(st->arena[st->cur], st->esize, topo_of(st->grid), layout_of(st, f), f,
                                             ctx->stream);
        ctx->launches++;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "halo fill launch");
    }
    st->ghosts_valid = true;
    return LG_OK;
}

// Run `nsteps` of a step functor, optionally through a cached CUDA graph of
// an even number of steps (so the ping-pong buffer and time slot return to
// their starting parity after every replay).
template <class StepFn>
int run_steps(lg_state* st, const std::string& key, int64_t nsteps, uint32_t flags, StepFn step) {
    lg_ctx* ctx = st->ctx;
    int64_t done = 0;
    if ((flags & LG_RUN_GRAPH) && nsteps >= 2) {
        const int64_t chunk = std::min<int64_t>(nsteps - (nsteps & 1), 64);
        std::string gk = key + "|chunk=" + std::to_string(chunk) + "|cur=" + std::to_string(st->cur) +
                         "|slot=" + std::to_string(st->tslot);
        auto it = st->graphs.find(gk);
        if (it == st->graphs.end()) {
            GraphEntry ge;
            ge.steps = chunk;
            int64_t before = ctx->launches;
            LG_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            int cur0 = st->cur, slot0 = st->tslot;
            int rc = LG_OK;
            for (int64_t s = 0; s < chunk && rc == LG_OK; ++s) rc = step();
            cudaError_t ec = cudaStreamEndCapture(ctx->stream, &ge.graph);
            st->cur = cur0;
            st->tslot = slot0;
            ge.launches = ctx->launches - before;
            ctx->launches = before;
            if (rc != LG_OK) {
                if (ge.graph) cudaGraphDestroy(ge.graph);
                return rc;
            }
            if (ec != cudaSuccess) return cuda_fail(ctx, ec, "cudaStreamEndCapture");
            LG_CUDA(ctx, cudaGraphInstantiate(&ge.exec, ge.graph, 0));
            it = st->graphs.emplace(gk, ge).first;
        }
        const GraphEntry& ge = it->second;
        while (nsteps - done >= ge.steps) {
            LG_CUDA(ctx, cudaGraphLaunch(ge.exec, ctx->stream));
            ctx->launches += ge.launches;
            done += ge.steps;
        }
    }
    for (; done < nsteps; ++done) {
        int rc = step();
        if (rc != LG_OK) return rc;
    }
    return LG_OK;
}

// the autotuner's cache key: the grid's block shape and count, the element
// type and whether the noise term is on
std::string tune_key(const lg_state* st, bool noise) {
    const lg_grid* g = st->grid;
    return std::to_string(g->D) + "|" + std::to_string(g->block[0]) + "x" + std::to_string(g->block[1]) + "|" +
           std::to_string(g->nblocks) + "|" + std::to_string(st->dtype) + "|" + (noise ? "n" : "q");
}

// Host-side time bookkeeping of `steps` steps: t += dt each
// (simulation.rs:285-286), the same IEEE additions the kernels perform.
void advance_time(lg_state* st, double dt, int64_t steps) {
    for (int64_t s = 0; s < steps; ++s) st->t += dt;
    st->step_index += steps;
}

}  // namespace

namespace lg {
// context services for the other translation units of the library
int abi_fail(lg_ctx* ctx, int code, const std::string& msg) { return fail(ctx, code, msg); }
int abi_state_view(const lg_state* st, StateView* v) {
    if (!st || !v) return LG_ERR_INVALID;
    const lg_grid* g = st->grid;
    v->ctx = st->ctx;
    v->arena = st->arena[st->cur];
    v->dtype = st->dtype;
    v->esize = st->esize;
    v->D = g->D;
    v->nfields = st->nfields;
    v->ghosts = st->ghosts.data();
    v->slab_stride = st->slab_stride;
    v->nblocks = g->nblocks;
    for (int d = 0; d < 3; ++d) {
        v->block[d] = g->block[d];
        v->nb[d] = g->nb[d];
        v->spacing[d] = g->spacing[d];
        v->periodic[d] = g->periodic[d];
    }
    v->arena_rw = st->arena[st->cur];
    return LG_OK;
}
int* abi_device_flag(lg_ctx* ctx) {
    if (!ctx->d_flag) {
        if (cudaMalloc(&ctx->d_flag, sizeof(int)) != cudaSuccess) {
            ctx->d_flag = nullptr;
            return nullptr;
        }
        if (cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream) != cudaSuccess) return nullptr;
    }
    return ctx->d_flag;
}
cudaStream_t abi_stream(lg_ctx* ctx) { return ctx->stream; }
int abi_device(lg_ctx* ctx) { return ctx->device; }
void abi_count_launch(lg_ctx* ctx, int64_t n) { ctx->launches += n; }
int64_t abi_launches(lg_ctx* ctx) { return ctx->launches; }
void abi_set_launches(lg_ctx* ctx, int64_t n) { ctx->launches = n; }
}  // namespace lg

extern "C" {

int lg_abi_version(void) { return LG_ABI_VERSION; }

int lg_ctx_create(int device, void* stream, lg_ctx** out) {
    if (!out) return LG_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return LG_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return LG_ERR_CUDA;
    lg_ctx* ctx = new lg_ctx();
    ctx->device = device;
    if (stream) {
        ctx->stream = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return LG_ERR_CUDA;
        }
        ctx->own_stream = true;
    }
    *out = ctx;
    return LG_OK;
}

int lg_ctx_destroy(lg_ctx* ctx) {
    if (!ctx) return LG_ERR_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->d_flag) cudaFree(ctx->d_flag);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return LG_OK;
}

const char* lg_last_error(const lg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t lg_ctx_kernel_launches(const lg_ctx* ctx) { return ctx ? ctx->launches : -1; }

// after the stream has drained: did a kernel's bounded device wait give up?
static int check_device_flag(lg_ctx* ctx) {
    if (!ctx->d_flag) return LG_OK;
    int v = 0;
    LG_CUDA(ctx, cudaMemcpy(&v, ctx->d_flag, sizeof v, cudaMemcpyDeviceToHost));
    if (v == 0) return LG_OK;
    LG_CUDA(ctx, cudaMemset(ctx->d_flag, 0, sizeof(int)));
    return fail(ctx, LG_ERR_DEVICE, "a kernel's bounded wait for its tile copies gave up; results are invalid");
}

int lg_sync(lg_ctx* ctx, int64_t timeout_ms) {
    if (!ctx) return LG_ERR_INVALID;
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(ctx->stream);
        if (e == cudaSuccess) return check_device_flag(ctx);
        if (e != cudaErrorNotReady) return cuda_fail(ctx, e, "stream");
        if (timeout_ms >= 0) {
            auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0);
            if (ms.count() > timeout_ms) return fail(ctx, LG_ERR_TIMEOUT, "lg_sync timed out");
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

int lg_grid_create_cartesian(lg_ctx* ctx, int D, const int64_t* cells, const int64_t* block_cells,
                             const double* origin, const double* spacing, const int* periodic, lg_grid** out) {
    if (!ctx || !out || !cells || !block_cells || !origin || !spacing || !periodic)
        return fail(ctx, LG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (D < 1 || D > 3) return fail(ctx, LG_ERR_INVALID, "dimension must be 1, 2 or 3");
    lg_grid* g = new lg_grid();
    g->ctx = ctx;
    g->D = D;
    g->nblocks = 1;
    for (int d = 0; d < D; ++d) {
        // CartesianGrid::new (cartesian.rs:48-82)
        if (!(cells[d] > 0 && block_cells[d] > 0)) {
            delete g;
            return fail(ctx, LG_ERR_INVALID, "empty dimension " + std::to_string(d));
        }
        if (cells[d] % block_cells[d] != 0) {
            delete g;
            return fail(ctx, LG_ERR_INVALID, "cells not divisible by block cells in dimension " + std::to_string(d));
        }
        if (!(spacing[d] > 0.0) || !std::isfinite(spacing[d])) {
            delete g;
            return fail(ctx, LG_ERR_INVALID, "invalid spacing in dimension " + std::to_string(d));
        }
        g->cells[d] = cells[d];
        g->block[d] = block_cells[d];
        g->nb[d] = cells[d] / block_cells[d];
        g->origin[d] = origin[d];
        g->spacing[d] = spacing[d];
        g->periodic[d] = periodic[d] ? 1 : 0;
        g->nblocks *= g->nb[d];
    }
    if (g->nblocks > (int64_t)1 << 30) {
        delete g;
        return fail(ctx, LG_ERR_INVALID, "too many blocks");
    }
    g->h_nbr.assign(g->nblocks * 6, -1);
    for (int64_t b = 0; b < g->nblocks; ++b)
        for (int d = 0; d < D; ++d)
            for (int s = 0; s < 2; ++s) g->h_nbr[(b * 3 + d) * 2 + s] = (int)face_neighbor(g, b, d, s ? 1 : -1);
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaMalloc(&g->d_nbr, g->h_nbr.size() * sizeof(int));
    if (e != cudaSuccess) {
        delete g;
        return fail(ctx, LG_ERR_NOMEM, "topology table allocation failed");
    }
    e = cudaMemcpy(g->d_nbr, g->h_nbr.data(), g->h_nbr.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(g->d_nbr);
        delete g;
        return cuda_fail(ctx, e, "topology upload");
    }
    *out = g;
    return LG_OK;
}

int lg_grid_destroy(lg_grid* g) {
    if (!g) return LG_ERR_INVALID;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    cudaFree(g->d_nbr);
    delete g;
    return LG_OK;
}

int64_t lg_grid_num_blocks(const lg_grid* g) { return g ? g->nblocks : -1; }

int lg_grid_face_neighbor(const lg_grid* g, int64_t block, int dim, int dir, int64_t* out) {
    if (!g || !out || block < 0 || block >= g->nblocks || dim < 0 || dim >= g->D || (dir != 1 && dir != -1))
        return LG_ERR_INVALID;
    *out = face_neighbor(g, block, dim, dir);
    return LG_OK;
}

int lg_state_create(lg_ctx* ctx, const lg_grid* grid, int dtype, int nfields, const int* ghosts, lg_state** out) {
    if (!ctx || !grid || !out || nfields < 1 || !ghosts) return fail(ctx, LG_ERR_INVALID, "bad state arguments");
    *out = nullptr;
    if (dtype != LG_F64 && dtype != LG_F32) return fail(ctx, LG_ERR_INVALID, "dtype must be LG_F64 or LG_F32");
    int64_t maxlen = 0;
    for (int f = 0; f < nfields; ++f) {
        for (int d = 0; d < grid->D; ++d)
            if (ghosts[f] < 0 || ghosts[f] > grid->block[d])
                return fail(ctx, LG_ERR_INVALID,
                            "ghost width " + std::to_string(ghosts[f]) + " exceeds block extent in dimension " +
                                std::to_string(d));
        maxlen = std::max(maxlen, block_len(grid, ghosts[f]));
    }
    lg_state* st = new lg_state();
    st->ctx = ctx;
    st->grid = grid;
    st->dtype = dtype;
    st->esize = dtype == LG_F64 ? 8 : 4;
    st->nfields = nfields;
    st->ghosts.assign(ghosts, ghosts + nfields);
    const int64_t align = 256 / st->esize;
    st->slab_stride = (maxlen + align - 1) / align * align;
    const size_t bytes = (size_t)grid->nblocks * nfields * st->slab_stride * st->esize;
    cudaSetDevice(ctx->device);
    for (int k = 0; k < 2; ++k) {
        if (cudaMalloc(&st->arena[k], bytes) != cudaSuccess) {
            cudaGetLastError();
            for (int j = 0; j < k; ++j) cudaFree(st->arena[j]);
            delete st;
            return fail(ctx, LG_ERR_NOMEM, "state arena allocation of " + std::to_string(bytes) + " bytes failed");
        }
        cudaMemsetAsync(st->arena[k], 0, bytes, ctx->stream);
    }
    // two time slots, then the two work-list counters of the strip kernel
    if (cudaMalloc(&st->d_t, 4 * sizeof(double)) != cudaSuccess) {
        cudaFree(st->arena[0]);
        cudaFree(st->arena[1]);
        delete st;
        return fail(ctx, LG_ERR_NOMEM, "time slot allocation failed");
    }
    cudaMemsetAsync(st->d_t, 0, 4 * sizeof(double), ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        lg_state_destroy(st);
        return cuda_fail(ctx, e, "state initialisation");
    }
    *out = st;
    return LG_OK;
}

int lg_state_destroy(lg_state* st) {
    if (!st) return LG_ERR_INVALID;
    cudaSetDevice(st->ctx->device);
    cudaStreamSynchronize(st->ctx->stream);
    for (auto& kv : st->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    cudaFree(st->arena[0]);
    cudaFree(st->arena[1]);
    cudaFree(st->d_t);
    cudaFree(st->orient);
    for (void* q : st->rk) cudaFree(q);
    delete st;
    return LG_OK;
}

static int field_copy(lg_state* st, int field, void* host, int64_t nelem, bool upload) {
    lg_ctx* ctx = st->ctx;
    if (field < 0 || field >= st->nfields) return fail(ctx, LG_ERR_INVALID, "field index out of range");
    const int64_t len = block_len(st->grid, st->ghosts[field]);
    if (!host || nelem != len * st->grid->nblocks)
        return fail(ctx, LG_ERR_INVALID, "element count must be num_blocks * block_len(ghost)");
    char* dev = static_cast<char*>(st->arena[st->cur]) + (size_t)field * st->slab_stride * st->esize;
    const size_t dpitch = (size_t)st->nfields * st->slab_stride * st->esize;
    const size_t width = (size_t)len * st->esize;
    cudaSetDevice(ctx->device);
    if (upload) {
        LG_CUDA(ctx, cudaMemcpy2DAsync(dev, dpitch, host, width, width, st->grid->nblocks, cudaMemcpyHostToDevice,
                                       ctx->stream));
        st->ghosts_valid = false;
    } else {
        LG_CUDA(ctx, cudaMemcpy2DAsync(host, width, dev, dpitch, width, st->grid->nblocks, cudaMemcpyDeviceToHost,
                                       ctx->stream));
    }
    LG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return upload ? LG_OK : check_device_flag(ctx);
}

int lg_state_upload_field(lg_state* st, int field, const void* host, int64_t nelem) {
    if (!st) return LG_ERR_INVALID;
    return field_copy(st, field, const_cast<void*>(host), nelem, true);
}

int lg_state_download_field(lg_state* st, int field, void* host, int64_t nelem) {
    if (!st) return LG_ERR_INVALID;
    return field_copy(st, field, host, nelem, false);
}

int lg_state_slab(lg_state* st, int64_t block, int field, void** dev, int64_t* len) {
    if (!st || !dev || !len) return LG_ERR_INVALID;
    if (block < 0 || block >= st->grid->nblocks || field < 0 || field >= st->nfields)
        return fail(st->ctx, LG_ERR_INVALID, "block or field out of range");
    *dev = static_cast<char*>(st->arena[st->cur]) + ((size_t)block * st->nfields + field) * st->slab_stride * st->esize;
    *len = block_len(st->grid, st->ghosts[field]);
    return LG_OK;
}

int lg_state_get_time(const lg_state* st, double* t, int64_t* step_index) {
    if (!st || !t || !step_index) return LG_ERR_INVALID;
    *t = st->t;
    *step_index = st->step_index;
    return LG_OK;
}

int lg_state_set_time(lg_state* st, double t, int64_t step_index) {
    if (!st) return LG_ERR_INVALID;
    st->t = t;
    st->step_index = step_index;
    return LG_OK;
}

int lg_fill_ghosts(lg_state* st, int field) {
    if (!st) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    if (field < 0 || field >= st->nfields) return fail(ctx, LG_ERR_INVALID, "field index out of range");
    cudaSetDevice(ctx->device);
    cudaError_t e = lg::launch_halo_fill(st->arena[st->cur], st->esize, topo_of(st->grid), layout_of(st, field),
                                         field, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "halo fill launch");
    return LG_OK;
}

int lg_heat_fe_run(lg_state* st, int field, double kappa, double dt, int64_t nsteps, uint32_t flags) {
    if (!st) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    if (st->dtype != LG_F64) return fail(ctx, LG_ERR_STATE, "the heat path is FP64");
    if (field < 0 || field >= st->nfields || st->ghosts[field] != 1)
        return fail(ctx, LG_ERR_STATE, "heat field must exist and have ghost width 1");
    if (nsteps < 0) return fail(ctx, LG_ERR_INVALID, "negative step count");
    cudaSetDevice(ctx->device);
    if (!st->ghosts_valid) {
        int rc = fill_all_ghosts(st);
        if (rc != LG_OK) return rc;
    }
    double inv_h2[3] = {0, 0, 0};
    for (int d = 0; d < st->grid->D; ++d) inv_h2[d] = 1.0 / (st->grid->spacing[d] * st->grid->spacing[d]);
    const lg::CartTopo topo = topo_of(st->grid);
    const lg::SlabLayout L = layout_of(st, field);
    char key[256];
    snprintf(key, sizeof key, "heat|f=%d|k=%a|dt=%a", field, kappa, dt);
    // 3-D: halos pulled from the neighbour blocks, ghosts filled once at the
    // end; otherwise the push kernel, which keeps the ghosts valid each step
    // (even block widths: the tiles staged by tensor copies; odd: by cp.async)
    const bool pull = lg::heat3d_pull_supported(topo, L);
    int* dflag = nullptr;
    const bool tma = pull && lg::heat3d_tma_supported(topo, L) && (dflag = lg::abi_device_flag(ctx)) != nullptr;
    auto step = [&]() -> int {
        const double* in = static_cast<const double*>(st->arena[st->cur]);
        double* out = static_cast<double*>(st->arena[st->cur ^ 1]);
        cudaError_t e = tma    ? lg::launch_heat3d_tma(in, out, topo, L, field, kappa, dt, inv_h2, dflag, ctx->stream)
                        : pull ? lg::launch_heat3d_pull(in, out, topo, L, field, kappa, dt, inv_h2, ctx->stream)
                               : lg::launch_heat_step(in, out, topo, L, field, kappa, dt, inv_h2, ctx->stream);
        ctx->launches++;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "heat step launch");
        st->cur ^= 1;
        st->tslot ^= 1;
        return LG_OK;
    };
    int rc = run_steps(st, key, nsteps, flags, step);
    if (rc != LG_OK) return rc;
    if (pull && nsteps > 0) {
        rc = fill_all_ghosts(st);
        if (rc != LG_OK) return rc;
    }
    if (nsteps & 1) {
        // graph replays keep parity; the remainder steps already flipped it
    }
    advance_time(st, dt, nsteps);
    return LG_OK;
}

int lg_modelc_em_run(lg_state* st, const lg_modelc_params* p, double dt, uint64_t seed, int64_t nsteps,
                     int variant, uint32_t flags) {
    if (!st || !p) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    if (st->grid->D != 2 || st->nfields < 2 || st->ghosts[0] != 1 || st->ghosts[1] != 1)
        return fail(ctx, LG_ERR_STATE, "Model C needs a 2-D state with phi and u of ghost width 1");
    if (nsteps < 0) return fail(ctx, LG_ERR_INVALID, "negative step count");
    if (variant < 0 || variant % 1000 % 10 > 7 || variant % 1000 > 17 || (variant % 1000 >= 10 && variant % 10 < 2))
        return fail(ctx, LG_ERR_INVALID, "unknown kernel variant");
    cudaSetDevice(ctx->device);
    if (!st->ghosts_valid) {
        int rc = fill_all_ghosts(st);
        if (rc != LG_OK) return rc;
    }
    lg::ModelCDev m{};
    m.lambda = p->lambda;
    m.d_thermal = p->d_thermal;
    m.a_bar = std::fma(3.0, -p->eps4, 1.0);            // phasefield.rs:101
    m.eps_prime = 3.0 * p->eps4 / m.a_bar;             // phasefield.rs:109
    m.tol = p->anisotropy_tol;
    m.f_a_bar = std::fma(3.0, -p->eps4, 1.0);          // finite_volume.rs:114
    m.f_eps_prime = 3.0 * p->eps4 / m.f_a_bar;         // finite_volume.rs:115
    m.f_a12 = 4.0 * m.f_a_bar * m.f_eps_prime;         // finite_volume.rs:119
    m.f_tol = p->flux_tol;
    m.inv_h2_flux = 1.0 / (st->grid->spacing[0] * st->grid->spacing[1]);
    m.inv_h2[0] = 1.0 / (st->grid->spacing[0] * st->grid->spacing[0]);
    m.inv_h2[1] = 1.0 / (st->grid->spacing[1] * st->grid->spacing[1]);
    lg::NoiseDev nz{};
    nz.on = p->noise_amplitude != 0.0 ? 1 : 0;
    nz.seed = seed;
    nz.amp = p->noise_amplitude;
    // the device time slot starts from the host's time
    LG_CUDA(ctx, cudaMemcpyAsync(st->d_t + st->tslot, &st->t, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    const lg::CartTopo topo = topo_of(st->grid);
    const lg::SlabLayout L = layout_of(st, 0);
    if (variant == 0) {  // the autotuned choice for this shape, if any
        auto it = ctx->tuned.find(tune_key(st, nz.on != 0));
        if (it != ctx->tuned.end()) variant = it->second;
    }
    char key[512];
    snprintf(key, sizeof key, "modelc|%a|%a|%a|%a|%a|%a|dt=%a|seed=%llu|v=%d|orient=%p", p->eps4, p->lambda,
             p->d_thermal, p->noise_amplitude, p->anisotropy_tol, p->flux_tol, dt, (unsigned long long)seed, variant,
             st->orient);
    const int64_t ncells = st->grid->nblocks * st->grid->block[0] * st->grid->block[1];
    // variant = kind + 1000 * rows: kind 0 library default, 1 one thread per
    // cell in reference order, 2/3/4 warp strips with 2/3/4 CTAs per SM, 5/6/7
    // the same with two rows per pass of the row loop, 12..17 those forms as
    // a persistent work list; rows fixes the strip height
    const int kind = variant % 1000 % 10, rows = variant / 1000;
    const bool listed = variant % 1000 >= 10;
    const bool tile = kind != 1 && lg::modelc_tile_supported(topo);
    const int minb = kind >= 2 ? kind : (st->dtype == LG_F32 ? 3 : 2);
    unsigned* work = listed ? reinterpret_cast<unsigned*>(st->d_t + 2) : nullptr;
    // the run's first step takes its units from a cleared list (each step
    // clears the other slot's list for the step after it)
    if (work) LG_CUDA(ctx, cudaMemsetAsync(work + st->tslot, 0, sizeof(unsigned), ctx->stream));
    if (kind == 2 && !tile) return fail(ctx, LG_ERR_INVALID, "the strip kernel needs a 2-D grid");
    auto step = [&]() -> int {
        cudaError_t e;
        const void* in = st->arena[st->cur];
        void* out = st->arena[st->cur ^ 1];
        if (st->orient)  // multi-grain: the oriented strip step, whatever the variant's kind
            e = st->dtype == LG_F64
                    ? lg::launch_modelc_oriented_f64(static_cast<const double*>(in), static_cast<double*>(out), topo,
                                                     L, m, dt, nz, st->d_t, st->tslot,
                                                     static_cast<const double*>(st->orient), ncells, rows, ctx->stream)
                    : lg::launch_modelc_oriented_f32(static_cast<const float*>(in), static_cast<float*>(out), topo, L,
                                                     m, dt, nz, st->d_t, st->tslot,
                                                     static_cast<const float*>(st->orient), ncells, rows, ctx->stream);
        else if (st->dtype == LG_F64)
            e = tile ? lg::launch_modelc_tile_f64(static_cast<const double*>(in), static_cast<double*>(out), topo, L,
                                                  m, dt, nz, st->d_t, st->tslot, rows, minb, work, ctx->stream)
                     : lg::launch_modelc_step_f64(static_cast<const double*>(in), static_cast<double*>(out), topo, L,
                                                  m, dt, nz, st->d_t, st->tslot, variant, ctx->stream);
        else
            e = tile ? lg::launch_modelc_tile_f32(static_cast<const float*>(in), static_cast<float*>(out), topo, L,
                                                  m, dt, nz, st->d_t, st->tslot, rows, minb, work, ctx->stream)
                     : lg::launch_modelc_step_f32(static_cast<const float*>(in), static_cast<float*>(out), topo, L, m,
                                                  dt, nz, st->d_t, st->tslot, variant, ctx->stream);
        ctx->launches++;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "Model C step launch");
        st->cur ^= 1;
        st->tslot ^= 1;
        return LG_OK;
    };
    int rc = run_steps(st, key, nsteps, flags, step);
    if (rc != LG_OK) return rc;
    advance_time(st, dt, nsteps);
    return LG_OK;
}

int lg_modelc_autotune(lg_state* st, const lg_modelc_params* p, double dt, uint64_t seed, int trial_steps,
                       int* best_variant, double* best_ms) {
    if (!st || !p || !best_variant || trial_steps < 1) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    if (st->grid->D != 2) return fail(ctx, LG_ERR_STATE, "the Model C autotuner needs a 2-D state");
    cudaSetDevice(ctx->device);
    if (!st->ghosts_valid) {
        int rc = fill_all_ghosts(st);
        if (rc != LG_OK) return rc;
    }
    // every candidate starts from a copy of the current state; the state,
    // its time and its step index are restored afterwards
    const size_t bytes = (size_t)st->grid->nblocks * st->nfields * st->slab_stride * st->esize;
    void* saved = nullptr;
    LG_CUDA(ctx, cudaMalloc(&saved, bytes));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int cur0 = st->cur, slot0 = st->tslot;
    const double t0 = st->t;
    const int64_t k0 = st->step_index;
    int rc = LG_OK;
    cudaError_t ce = cudaMemcpyAsync(saved, st->arena[cur0], bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    if (ce != cudaSuccess) rc = cuda_fail(ctx, ce, "autotune state copy");
    const std::string key = tune_key(st, p->noise_amplitude != 0.0);
    ctx->tuned.erase(key);
    // time one candidate over `steps` steps from the saved state (after two
    // warm-up steps); ms per step, or a negative value on failure
    auto trial = [&](int v, int steps) -> float {
        ce = cudaMemcpyAsync(st->arena[cur0], saved, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
        if (ce != cudaSuccess) {
            rc = cuda_fail(ctx, ce, "autotune state copy");
            return -1.0f;
        }
        st->cur = cur0;
        st->tslot = slot0;
        st->t = t0;
        rc = lg_modelc_em_run(st, p, dt, seed, 2, v, 0);  // warm-up
        if (rc != LG_OK) return -1.0f;
        cudaEventRecord(e0, ctx->stream);
        rc = lg_modelc_em_run(st, p, dt, seed, steps, v, 0);
        cudaEventRecord(e1, ctx->stream);
        if (rc != LG_OK) return -1.0f;
        ce = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce != cudaSuccess) {
            rc = cuda_fail(ctx, ce, "autotune timing");
            return -1.0f;
        }
        return ms / steps;
    };
    // every candidate once, then the three fastest again in three interleaved
    // rounds of twice as many steps, each scored by its fastest round: short
    // windows alone mis-rank variants within a few percent, and a clock that
    // drifts (the power cap of a long FP64 run) slows every candidate of a
    // round alike instead of whichever was timed last
    std::vector<std::pair<float, int>> first;
    for (int kind : {2, 3, 4, 5, 6, 7, 12, 13, 14, 15, 16, 17}) {
        for (int rows : {0, 8, 16, 32}) {
            if (rc != LG_OK) break;
            const int v = kind + 1000 * rows;
            const float ms = trial(v, trial_steps);
            if (rc == LG_OK) first.emplace_back(ms, v);
        }
    }
    std::sort(first.begin(), first.end());
    const size_t finalists = std::min<size_t>(first.size(), 3);
    std::vector<float> fastest(finalists, 0.0f);
    for (int round = 0; round < 3 && rc == LG_OK; ++round)
        for (size_t i = 0; i < finalists && rc == LG_OK; ++i) {
            const float ms = trial(first[i].second, 2 * trial_steps);
            if (rc == LG_OK && (round == 0 || ms < fastest[i])) fastest[i] = ms;
        }
    int best = 0;
    float best_t = 0.0f;
    for (size_t i = 0; i < finalists && rc == LG_OK; ++i)
        if (best == 0 || fastest[i] < best_t) {
            best = first[i].second;
            best_t = fastest[i];
        }
    if (rc == LG_OK) {
        ce = cudaMemcpyAsync(st->arena[cur0], saved, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
        if (ce != cudaSuccess) rc = cuda_fail(ctx, ce, "autotune state restore");
    }
    cudaFree(saved);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st->cur = cur0;
    st->tslot = slot0;
    st->t = t0;
    st->step_index = k0;
    if (rc != LG_OK) return rc;
    ctx->tuned[key] = best;
    *best_variant = best;
    if (best_ms) *best_ms = best_t;
    return LG_OK;
}

int lg_modelc_initialize_grains(lg_state* st, const double* grains, int64_t n, double u0) {
    if (!st || (n > 0 && !grains)) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    const lg_grid* g = st->grid;
    if (g->D != 2 || st->nfields < 2 || st->ghosts[0] != 1 || st->ghosts[1] != 1)
        return fail(ctx, LG_ERR_STATE, "Model C needs a 2-D state with phi and u of ghost width 1");
    const int64_t nx = g->block[0], ny = g->block[1];
    const int64_t len = block_len(g, 1), sy = nx + 2;
    std::vector<double> phi(len * g->nblocks, 0.0), u(len * g->nblocks, 0.0);
    auto center = [&](int64_t b, int64_t i, int64_t j, double* out) {
        // CartesianGrid::cell_center (cartesian.rs:588-597)
        int64_t c0 = b % g->nb[0], c1 = b / g->nb[0];
        out[0] = std::fma(((double)(c0 * nx) + (double)i) + 0.5, g->spacing[0], g->origin[0]);
        out[1] = std::fma(((double)(c1 * ny) + (double)j) + 0.5, g->spacing[1], g->origin[1]);
    };
    const double CUTOFF = 27.0;
    auto work = [&](int64_t b0, int64_t b1) {
        for (int64_t b = b0; b < b1; ++b) {
            // ModelC::initialize_grains (phasefield.rs:238-286)
            double hx = g->spacing[0], hy = g->spacing[1], c0[2], c1[2];
            center(b, 0, 0, c0);
            center(b, nx - 1, ny - 1, c1);
            double lo[2] = {std::fma(0.5, -hx, c0[0]), std::fma(0.5, -hy, c0[1])};
            double hi[2] = {std::fma(0.5, hx, c1[0]), std::fma(0.5, hy, c1[1])};
            std::vector<int64_t> near;
            for (int64_t k = 0; k < n; ++k) {
                double cx = grains[4 * k], cy = grains[4 * k + 1];
                double dx = std::max(std::max(lo[0] - cx, cx - hi[0]), 0.0);
                double dy = std::max(std::max(lo[1] - cy, cy - hi[1]), 0.0);
                if (std::hypot(dx, dy) <= grains[4 * k + 2] + CUTOFF) near.push_back(k);
            }
            double* ph = phi.data() + b * len;
            double* uu = u.data() + b * len;
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    double v = -1.0;
                    if (!near.empty()) {
                        double xy[2];
                        center(b, i, j, xy);
                        for (int64_t k : near) {
                            double r = std::hypot(xy[0] - grains[4 * k], xy[1] - grains[4 * k + 1]);
                            v = std::fmax(v, -std::tanh((r - grains[4 * k + 2]) / std::sqrt(2.0)));
                        }
                    }
                    ph[(i + 1) + (j + 1) * sy] = v;
                    uu[(i + 1) + (j + 1) * sy] = -u0;
                }
        }
    };
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (g->nblocks < 4) nt = 1;
    std::vector<std::thread> pool;
    int64_t per = (g->nblocks + nt - 1) / nt;
    for (unsigned k = 0; k < nt; ++k) {
        int64_t b0 = k * per, b1 = std::min<int64_t>(g->nblocks, b0 + per);
        if (b0 < b1) pool.emplace_back(work, b0, b1);
    }
    for (auto& th : pool) th.join();
    int rc = lg_state_upload_field(st, 0, phi.data(), (int64_t)phi.size());
    if (rc != LG_OK) return rc;
    return lg_state_upload_field(st, 1, u.data(), (int64_t)u.size());
}

// the RungeKutta4 workspace: five arenas of the state's layout, zeroed
static int rk_workspace(lg_state* st) {
    if (st->rk[0]) return LG_OK;
    const size_t bytes = (size_t)st->grid->nblocks * st->nfields * st->slab_stride * st->esize;
    for (void*& q : st->rk) {
        cudaError_t e = cudaMalloc(&q, bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(q, 0, bytes, st->ctx->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            for (void*& r : st->rk) {
                cudaFree(r);
                r = nullptr;
            }
            return fail(st->ctx, LG_ERR_NOMEM, "RungeKutta4 workspace: out of device memory");
        }
    }
    return LG_OK;
}

int lg_heat_rk4_run(lg_state* st, int field, double kappa, double dt, int64_t nsteps, uint32_t flags) {
    if (!st) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    if (st->dtype != LG_F64) return fail(ctx, LG_ERR_STATE, "the heat path is FP64");
    if (field < 0 || field >= st->nfields || st->ghosts[field] != 1)
        return fail(ctx, LG_ERR_STATE, "heat field must exist and have ghost width 1");
    if (nsteps < 0) return fail(ctx, LG_ERR_INVALID, "negative step count");
    cudaSetDevice(ctx->device);
    int rc = rk_workspace(st);
    if (rc != LG_OK) return rc;
    if (!st->ghosts_valid) {
        rc = fill_all_ghosts(st);
        if (rc != LG_OK) return rc;
    }
    double inv_h2[3] = {0, 0, 0};
    for (int d = 0; d < st->grid->D; ++d) inv_h2[d] = 1.0 / (st->grid->spacing[d] * st->grid->spacing[d]);
    const lg::CartTopo topo = topo_of(st->grid);
    const lg::SlabLayout L = layout_of(st, field);
    const double half_dt = 0.5 * dt, sixth = dt / 6.0, third = dt / 3.0;  // rk4.rs:57, 74-75
    char key[256];
    snprintf(key, sizeof key, "heat-rk4|f=%d|k=%a|dt=%a", field, kappa, dt);
    double* k1 = static_cast<double*>(st->rk[0]);
    double* k2 = static_cast<double*>(st->rk[1]);
    double* k3 = static_cast<double*>(st->rk[2]);
    double* t0 = static_cast<double*>(st->rk[3]);
    double* t1 = static_cast<double*>(st->rk[4]);
    auto step = [&]() -> int {
        const double* y = static_cast<const double*>(st->arena[st->cur]);
        double* out = static_cast<double*>(st->arena[st->cur ^ 1]);
        cudaError_t e = lg::launch_heat_rk_stage(1, y, t0, y, k1, nullptr, nullptr, nullptr, topo, L, field, kappa,
                                                 inv_h2, half_dt, 0.0, 0.0, ctx->stream);
        if (e == cudaSuccess)
            e = lg::launch_heat_rk_stage(1, t0, t1, y, k2, nullptr, nullptr, nullptr, topo, L, field, kappa, inv_h2,
                                         half_dt, 0.0, 0.0, ctx->stream);
        if (e == cudaSuccess)
            e = lg::launch_heat_rk_stage(1, t1, t0, y, k3, nullptr, nullptr, nullptr, topo, L, field, kappa, inv_h2,
                                         dt, 0.0, 0.0, ctx->stream);
        if (e == cudaSuccess)
            e = lg::launch_heat_rk_stage(2, t0, out, y, nullptr, k1, k2, k3, topo, L, field, kappa, inv_h2, 0.0,
                                         sixth, third, ctx->stream);
        ctx->launches += 4;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "heat RK4 stage launch");
        st->cur ^= 1;
        st->tslot ^= 1;
        return LG_OK;
    };
    rc = run_steps(st, key, nsteps, flags, step);
    if (rc != LG_OK) return rc;
    advance_time(st, dt, nsteps);
    return LG_OK;
}

int lg_modelc_rk4_run(lg_state* st, const lg_modelc_params* p, double dt, int64_t nsteps, uint32_t flags) {
    if (!st || !p) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    if (st->grid->D != 2 || st->nfields < 2 || st->ghosts[0] != 1 || st->ghosts[1] != 1)
        return fail(ctx, LG_ERR_STATE, "Model C needs a 2-D state with phi and u of ghost width 1");
    if (p->noise_amplitude != 0.0)
        return fail(ctx, LG_ERR_INVALID, "RungeKutta4 steps deterministic models only (rk4.rs:15-19): noise must be 0");
    if (nsteps < 0) return fail(ctx, LG_ERR_INVALID, "negative step count");
    cudaSetDevice(ctx->device);
    int rc = rk_workspace(st);
    if (rc != LG_OK) return rc;
    if (!st->ghosts_valid) {
        rc = fill_all_ghosts(st);
        if (rc != LG_OK) return rc;
    }
    lg::ModelCDev m{};
    m.lambda = p->lambda;
    m.d_thermal = p->d_thermal;
    m.a_bar = std::fma(3.0, -p->eps4, 1.0);    // phasefield.rs:101
    m.eps_prime = 3.0 * p->eps4 / m.a_bar;     // phasefield.rs:109
    m.tol = p->anisotropy_tol;
    m.f_a_bar = std::fma(3.0, -p->eps4, 1.0);  // finite_volume.rs:114
    m.f_eps_prime = 3.0 * p->eps4 / m.f_a_bar;
    m.f_a12 = 4.0 * m.f_a_bar * m.f_eps_prime;
    m.f_tol = p->flux_tol;
    m.inv_h2_flux = 1.0 / (st->grid->spacing[0] * st->grid->spacing[1]);
    m.inv_h2[0] = 1.0 / (st->grid->spacing[0] * st->grid->spacing[0]);
    m.inv_h2[1] = 1.0 / (st->grid->spacing[1] * st->grid->spacing[1]);
    LG_CUDA(ctx, cudaMemcpyAsync(st->d_t + st->tslot, &st->t, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    const lg::CartTopo topo = topo_of(st->grid);
    const lg::SlabLayout L = layout_of(st, 0);
    const int64_t ncells = st->grid->nblocks * st->grid->block[0] * st->grid->block[1];
    const double half_dt = 0.5 * dt, sixth = dt / 6.0, third = dt / 3.0;  // rk4.rs:57, 74-75
    char key[512];
    snprintf(key, sizeof key, "modelc-rk4|%a|%a|%a|%a|%a|dt=%a|orient=%p", p->eps4, p->lambda, p->d_thermal,
             p->anisotropy_tol, p->flux_tol, dt, st->orient);
    auto step = [&]() -> int {
        const void* y = st->arena[st->cur];
        void* out = st->arena[st->cur ^ 1];
        void *k1 = st->rk[0], *k2 = st->rk[1], *k3 = st->rk[2], *t0 = st->rk[3], *t1 = st->rk[4];
        const void* stage_in[4] = {y, t0, t1, t0};
        void* stage_out[4] = {t0, t1, t0, out};
        void* stage_k[3] = {k1, k2, k3};
        const double stage_c[3] = {half_dt, half_dt, dt};
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
            const int mode = i < 3 ? 1 : 2;
            if (st->dtype == LG_F64)
                e = lg::launch_modelc_rk_stage_f64(
                    mode, static_cast<const double*>(stage_in[i]), static_cast<double*>(stage_out[i]), topo, L, m,
                    static_cast<const double*>(y), i < 3 ? static_cast<double*>(stage_k[i]) : nullptr,
                    static_cast<const double*>(k1), static_cast<const double*>(k2), static_cast<const double*>(k3),
                    i < 3 ? stage_c[i] : 0.0, sixth, third, static_cast<const double*>(st->orient), ncells, st->d_t,
                    st->tslot, dt, ctx->stream);
            else
                e = lg::launch_modelc_rk_stage_f32(
                    mode, static_cast<const float*>(stage_in[i]), static_cast<float*>(stage_out[i]), topo, L, m,
                    static_cast<const float*>(y), i < 3 ? static_cast<float*>(stage_k[i]) : nullptr,
                    static_cast<const float*>(k1), static_cast<const float*>(k2), static_cast<const float*>(k3),
                    i < 3 ? stage_c[i] : 0.0, sixth, third, static_cast<const float*>(st->orient), ncells, st->d_t,
                    st->tslot, dt, ctx->stream);
        }
        ctx->launches += 4;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "Model C RK4 stage launch");
        st->cur ^= 1;
        st->tslot ^= 1;
        return LG_OK;
    };
    rc = run_steps(st, key, nsteps, flags, step);
    if (rc != LG_OK) return rc;
    advance_time(st, dt, nsteps);
    return LG_OK;
}

int lg_modelc_set_orientations(lg_state* st, int theta_field) {
    if (!st) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    cudaSetDevice(ctx->device);
    if (theta_field < 0) {  // back to the axis-aligned step
        LG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(st->orient);
        st->orient = nullptr;
        st->theta_field = -1;
        return LG_OK;
    }
    const lg_grid* g = st->grid;
    if (g->D != 2 || st->nfields < 3 || st->ghosts[0] != 1 || st->ghosts[1] != 1)
        return fail(ctx, LG_ERR_STATE, "multi-grain Model C needs a 2-D state with phi, u and theta0");
    if (theta_field < 2 || theta_field >= st->nfields || st->ghosts[theta_field] != 0)
        return fail(ctx, LG_ERR_INVALID, "theta0 must be a field beyond phi and u with ghost width 0");
    const int64_t bc = g->block[0] * g->block[1], ncells = g->nblocks * bc;
    // theta0 of the current arena to the host, and into the other arena (the
    // step writes phi and u only, so both buffers keep the static field)
    const size_t pitch = (size_t)st->nfields * st->slab_stride * st->esize, width = (size_t)bc * st->esize;
    const size_t off = (size_t)theta_field * st->slab_stride * st->esize;
    std::vector<char> raw((size_t)ncells * st->esize);
    const char* cur = static_cast<const char*>(st->arena[st->cur]) + off;
    char* other = static_cast<char*>(st->arena[st->cur ^ 1]) + off;
    LG_CUDA(ctx, cudaMemcpy2DAsync(raw.data(), width, cur, pitch, width, g->nblocks, cudaMemcpyDeviceToHost,
                                   ctx->stream));
    LG_CUDA(ctx, cudaMemcpy2DAsync(other, pitch, cur, pitch, width, g->nblocks, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
    LG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // (s0, c0) = theta0.sin_cos() on the host, as the reference evaluates it
    // (phasefield.rs:383, finite_volume.rs:202)
    const size_t tbytes = 2 * (size_t)ncells * st->esize;
    std::vector<char> trig(tbytes);
    for (int64_t k = 0; k < ncells; ++k) {
        const double th = st->dtype == LG_F64 ? reinterpret_cast<const double*>(raw.data())[k]
                                              : (double)reinterpret_cast<const float*>(raw.data())[k];
        const double c0 = std::cos(th), s0 = std::sin(th);
        if (st->dtype == LG_F64) {
            reinterpret_cast<double*>(trig.data())[k] = c0;
            reinterpret_cast<double*>(trig.data())[ncells + k] = s0;
        } else {
            reinterpret_cast<float*>(trig.data())[k] = (float)c0;
            reinterpret_cast<float*>(trig.data())[ncells + k] = (float)s0;
        }
    }
    cudaFree(st->orient);
    st->orient = nullptr;
    st->theta_field = -1;
    LG_CUDA(ctx, cudaMalloc(&st->orient, tbytes));
    LG_CUDA(ctx, cudaMemcpy(st->orient, trig.data(), tbytes, cudaMemcpyHostToDevice));
    st->theta_field = theta_field;
    return LG_OK;
}

int lg_modelc_initialize_orientations(lg_state* st, int theta_field, const double* grains, int64_t n) {
    if (!st || (n > 0 && !grains)) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    const lg_grid* g = st->grid;
    if (g->D != 2 || theta_field < 2 || theta_field >= st->nfields || st->ghosts[theta_field] != 0)
        return fail(ctx, LG_ERR_INVALID, "theta0 must be a field beyond phi and u with ghost width 0");
    const int64_t nx = g->block[0], ny = g->block[1], bc = nx * ny;
    std::vector<double> theta((size_t)(bc * g->nblocks), 0.0);
    auto center = [&](int64_t b, int64_t i, int64_t j, double* out) {
        int64_t c0 = b % g->nb[0], c1 = b / g->nb[0];
        out[0] = std::fma(((double)(c0 * nx) + (double)i) + 0.5, g->spacing[0], g->origin[0]);
        out[1] = std::fma(((double)(c1 * ny) + (double)j) + 0.5, g->spacing[1], g->origin[1]);
    };
    // ModelC::initialize_grains, theta0 by nearest-seed Voronoi
    // (phasefield.rs:286-311): per block the candidates are the grains whose
    // box distance is at most the smallest farthest-corner distance; a cell
    // takes the first candidate minimising fma(dy, dy, dx * dx)
    auto work = [&](int64_t b0, int64_t b1) {
        for (int64_t b = b0; b < b1; ++b) {
            double hx = g->spacing[0], hy = g->spacing[1], c0[2], c1[2];
            center(b, 0, 0, c0);
            center(b, nx - 1, ny - 1, c1);
            double lo[2] = {std::fma(0.5, -hx, c0[0]), std::fma(0.5, -hy, c0[1])};
            double hi[2] = {std::fma(0.5, hx, c1[0]), std::fma(0.5, hy, c1[1])};
            double threshold = std::numeric_limits<double>::max();
            for (int64_t k = 0; k < n; ++k) {
                double cx = grains[4 * k], cy = grains[4 * k + 1];
                double dx = std::max(std::fabs(cx - lo[0]), std::fabs(cx - hi[0]));
                double dy = std::max(std::fabs(cy - lo[1]), std::fabs(cy - hi[1]));
                threshold = std::min(threshold, std::hypot(dx, dy));
            }
            std::vector<int64_t> cand;
            for (int64_t k = 0; k < n; ++k) {
                double cx = grains[4 * k], cy = grains[4 * k + 1];
                double dx = std::max(std::max(lo[0] - cx, cx - hi[0]), 0.0);
                double dy = std::max(std::max(lo[1] - cy, cy - hi[1]), 0.0);
                if (std::hypot(dx, dy) <= threshold) cand.push_back(k);
            }
            double* th = theta.data() + b * bc;
            for (int64_t j = 0; j < ny; ++j)
                for (int64_t i = 0; i < nx; ++i) {
                    double xy[2];
                    center(b, i, j, xy);
                    double best = 0.0, bd = 0.0;
                    bool any = false;
                    for (int64_t k : cand) {
                        double dx = xy[0] - grains[4 * k], dy = xy[1] - grains[4 * k + 1];
                        double d = std::fma(dy, dy, dx * dx);
                        if (!any || d < bd) {
                            any = true;
                            bd = d;
                            best = grains[4 * k + 3];
                        }
                    }
                    th[i + j * nx] = any ? best : 0.0;
                }
        }
    };
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (g->nblocks < 4) nt = 1;
    std::vector<std::thread> pool;
    int64_t per = (g->nblocks + nt - 1) / nt;
    for (unsigned k = 0; k < nt; ++k) {
        int64_t b0 = k * per, b1 = std::min<int64_t>(g->nblocks, b0 + per);
        if (b0 < b1) pool.emplace_back(work, b0, b1);
    }
    for (auto& t : pool) t.join();
    int rc;
    if (st->dtype == LG_F64) {
        rc = lg_state_upload_field(st, theta_field, theta.data(), (int64_t)theta.size());
    } else {
        std::vector<float> tf(theta.begin(), theta.end());
        rc = lg_state_upload_field(st, theta_field, tf.data(), (int64_t)tf.size());
    }
    if (rc != LG_OK) return rc;
    return lg_modelc_set_orientations(st, theta_field);
}

int lg_heat_initialize_sine_noise(lg_state* st, int field, uint64_t seed, double amp) {
    if (!st) return LG_ERR_INVALID;
    lg_ctx* ctx = st->ctx;
    const lg_grid* g = st->grid;
    if (st->dtype != LG_F64 || field < 0 || field >= st->nfields)
        return fail(ctx, LG_ERR_STATE, "heat initial condition needs an FP64 field");
    const int gh = st->ghosts[field];
    const int64_t len = block_len(g, gh);
    std::vector<double> host(len * g->nblocks, 0.0);
    const double two_pi = 2.0 * 3.14159265358979323846;
    for (int64_t b = 0; b < g->nblocks; ++b) {
        int64_t c[3] = {0, 0, 0}, rem = b;
        for (int d = 0; d < g->D; ++d) {
            c[d] = rem % g->nb[d];
            rem /= g->nb[d];
        }
        int64_t n[3] = {g->block[0], g->D > 1 ? g->block[1] : 1, g->D > 2 ? g->block[2] : 1};
        for (int64_t k = 0; k < n[2]; ++k)
            for (int64_t j = 0; j < n[1]; ++j)
                for (int64_t i = 0; i < n[0]; ++i) {
                    int64_t idx[3] = {i, j, k};
                    uint64_t parts_key = lg::splitmix64(seed);
                    double s = 1.0;
                    int64_t off = 0, stride = 1;
                    for (int d = 0; d < g->D; ++d) {
                        int64_t global = c[d] * g->block[d] + idx[d];
                        double x = std::fma(((double)(c[d] * g->block[d]) + (double)idx[d]) + 0.5, g->spacing[d],
                                            g->origin[d]);
                        s = s * std::sin(two_pi * x);
                        parts_key = lg::splitmix64(parts_key ^ (uint64_t)global);
                        off += (idx[d] + gh) * stride;
                        stride *= g->block[d] + 2 * gh;
                    }
                    host[b * len + off] = s + amp * (2.0 * lg::unit_open(parts_key) - 1.0);
                }
    }
    return lg_state_upload_field(st, field, host.data(), (int64_t)host.size());
}

int lg_standard_normal(lg_ctx* ctx, const uint64_t* keys, int64_t n, double* out) {
    if (!ctx || n < 0 || (n > 0 && (!keys || !out))) return fail(ctx, LG_ERR_INVALID, "bad arguments");
    if (n == 0) return LG_OK;
    cudaSetDevice(ctx->device);
    uint64_t* dk = nullptr;
    double* dout = nullptr;
    LG_CUDA(ctx, cudaMalloc(&dk, n * sizeof(uint64_t)));
    cudaError_t e = cudaMalloc(&dout, n * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(dk);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    e = cudaMemcpyAsync(dk, keys, n * sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        e = lg::launch_standard_normal(dk, dout, n, ctx->stream);
        ctx->launches++;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dk);
    cudaFree(dout);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "standard normal");
    return LG_OK;
}

}  // extern "C"
