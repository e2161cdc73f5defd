// Observation: the device side of the reference's AsyncObserver
// (src/core/observer.rs:65-165), the coordinate columns of its Parquet
// snapshots (src/io/parquet.rs:150-215), and an FP64 sum of a field over the
// interior cells (the conserved totals of a run: Model C's enthalpy).
//
// A snapshot ring holds `nslots` slots, each a device buffer and a pinned
// host buffer of the chosen fields' interior cells in the Parquet row order
// (block-major, interior cells dimension-0-fastest; one FP64 column per
// field).  capture() gathers the current state into a free slot's device
// buffer with one kernel on the state's stream, then copies it to the host
// buffer on the ring's own stream after an event, so the stepping stream
// never waits for the host (the host waits, at each capture, until the
// device has reached the previous one).  A slot goes FREE -> IN_FLIGHT (capture) ->
// HELD (poll, once its copy has finished) -> FREE (release).  With no free
// slot the snapshot is dropped and counted, as the reference drops a
// snapshot rather than block the solver (observer.rs:17-25, 149-156).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/legendre_b200.h"
#include "lg_common.cuh"
#include "lg_state_view.h"

namespace {

constexpr int kMaxPackFields = 8;

struct PackArgs {
    int nf;
    int field[kMaxPackFields], ghost[kMaxPackFields];
    int D, n0, n1;
    int64_t nfields, slab_stride, nblocks, bcells, ncells;
};

// out[k * ncells + b * bcells + i] = field k of block b at interior cell i
// (i dimension-0-fastest), widened to FP64.
template <class T>
__global__ void __launch_bounds__(256) snapshot_pack_kernel(const T* __restrict__ arena, double* __restrict__ out,
                                                            PackArgs a) {
    const int k = blockIdx.z;
    const int g = a.ghost[k];
    const int64_t gx = a.n0 + 2 * g;
    const int64_t gy = a.D > 1 ? a.n1 + 2 * g : 1;
    const int g1 = a.D > 1 ? g : 0, g2 = a.D > 2 ? g : 0;
    for (int64_t b = blockIdx.y; b < a.nblocks; b += gridDim.y) {
        const T* slab = arena + (b * a.nfields + a.field[k]) * a.slab_stride;
        double* dst = out + k * a.ncells + b * a.bcells;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.bcells;
             i += (int64_t)gridDim.x * blockDim.x) {
            const int64_t x = i % a.n0, r = i / a.n0;
            const int64_t y = r % a.n1, z = r / a.n1;
            dst[i] = (double)slab[(x + g) + (y + g1) * gx + (z + g2) * gx * gy];
        }
    }
}

struct SumArgs {
    int field, ghost, D, n0, n1;
    int64_t nfields, slab_stride, nblocks, bcells;
};

// partial[b] = the FP64 sum of field `field`'s interior cells of block b.
// The order is fixed: thread t adds cells t, t + 256, ... in turn, the
// warps' sums meet by a fixed shuffle tree and the eight warp sums in warp
// order, so a state gives the same bits on every call.
constexpr int kSumThreads = 256;

template <class T>
__global__ void __launch_bounds__(kSumThreads) field_sum_kernel(const T* __restrict__ arena,
                                                                double* __restrict__ partial, SumArgs a) {
    __shared__ double warp_sum[kSumThreads / 32];
    const int g = a.ghost;
    const int64_t gx = a.n0 + 2 * g;
    const int64_t gy = a.D > 1 ? a.n1 + 2 * g : 1;
    const int g1 = a.D > 1 ? g : 0, g2 = a.D > 2 ? g : 0;
    for (int64_t b = blockIdx.x; b < a.nblocks; b += gridDim.x) {
        const T* slab = arena + (b * a.nfields + a.field) * a.slab_stride;
        double s = 0.0;
        for (int64_t i = threadIdx.x; i < a.bcells; i += kSumThreads) {
            const int64_t x = i % a.n0, r = i / a.n0;
            const int64_t y = r % a.n1, z = r / a.n1;
            s += (double)slab[(x + g) + (y + g1) * gx + (z + g2) * gx * gy];
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < kSumThreads / 32; ++w) t += warp_sum[w];
            partial[b] = t;
        }
        __syncthreads();  // warp_sum is rewritten for the next block
    }
}

enum SlotStatus { kFree = 0, kInFlight = 1, kHeld = 2 };

}  // namespace

struct lg_snapshot_ring {
    lg_state* st = nullptr;
    lg_ctx* ctx = nullptr;
    int device = 0;
    int nslots = 0;
    std::vector<int> fields;
    int64_t bcells = 0, ncells = 0;
    cudaStream_t copy = nullptr;
    std::vector<double*> dslot, hslot;
    std::vector<cudaEvent_t> packed, copied;
    std::vector<int> status;
    std::vector<uint64_t> seq;
    std::vector<int64_t> step, epoch;
    std::vector<double> t;
    uint64_t next_seq = 0;
    int last = -1;  // slot of the latest capture
    int64_t captured = 0, dropped = 0;
    std::mutex mu;
};

namespace {

int rfail(lg_snapshot_ring* r, int code, const std::string& m) { return lg::abi_fail(r ? r->ctx : nullptr, code, m); }

void free_ring(lg_snapshot_ring* r) {
    cudaSetDevice(r->device);
    if (r->copy) cudaStreamSynchronize(r->copy);
    for (double* p : r->dslot)
        if (p) cudaFree(p);
    for (double* p : r->hslot)
        if (p) cudaFreeHost(p);
    for (cudaEvent_t e : r->packed)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : r->copied)
        if (e) cudaEventDestroy(e);
    if (r->copy) cudaStreamDestroy(r->copy);
    delete r;
}

}  // namespace

extern "C" {

int lg_snapshot_ring_create(lg_state* st, const int* fields, int nfields, int nslots, lg_snapshot_ring** out) {
    if (!st || !fields || !out) return LG_ERR_INVALID;
    *out = nullptr;
    lg::StateView v;
    int rc = lg::abi_state_view(st, &v);
    if (rc != LG_OK) return rc;
    if (nfields < 1 || nfields > kMaxPackFields)
        return lg::abi_fail(v.ctx, LG_ERR_INVALID, "a snapshot holds 1 to 8 fields");
    if (nslots < 1) return lg::abi_fail(v.ctx, LG_ERR_INVALID, "a snapshot ring needs at least one slot");
    for (int k = 0; k < nfields; ++k)
        if (fields[k] < 0 || fields[k] >= v.nfields)
            return lg::abi_fail(v.ctx, LG_ERR_INVALID, "snapshot field index out of range");
    lg_snapshot_ring* r = new lg_snapshot_ring();
    r->st = st;
    r->ctx = v.ctx;
    r->device = lg::abi_device(v.ctx);
    r->nslots = nslots;
    r->fields.assign(fields, fields + nfields);
    r->bcells = v.block[0] * v.block[1] * v.block[2];
    r->ncells = r->bcells * v.nblocks;
    cudaSetDevice(r->device);
    const size_t bytes = (size_t)nfields * (size_t)r->ncells * sizeof(double);
    r->dslot.assign(nslots, nullptr);
    r->hslot.assign(nslots, nullptr);
    r->packed.assign(nslots, nullptr);
    r->copied.assign(nslots, nullptr);
    r->status.assign(nslots, kFree);
    r->seq.assign(nslots, 0);
    r->step.assign(nslots, 0);
    r->epoch.assign(nslots, 0);
    r->t.assign(nslots, 0.0);
    cudaError_t e = cudaStreamCreateWithFlags(&r->copy, cudaStreamNonBlocking);
    for (int i = 0; i < nslots && e == cudaSuccess; ++i) {
        e = cudaMalloc(&r->dslot[i], bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&r->hslot[i], bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->packed[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->copied[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        lg_ctx* ctx = r->ctx;
        free_ring(r);
        return lg::abi_fail(ctx, e == cudaErrorMemoryAllocation ? LG_ERR_NOMEM : LG_ERR_CUDA,
                            std::string("snapshot ring: ") + cudaGetErrorString(e));
    }
    *out = r;
    return LG_OK;
}

int lg_snapshot_ring_destroy(lg_snapshot_ring* r) {
    if (!r) return LG_ERR_INVALID;
    free_ring(r);
    return LG_OK;
}

int lg_snapshot_ring_capture(lg_snapshot_ring* r, int64_t step, double t, int64_t epoch, int* slot) {
    if (!r || !slot) return LG_ERR_INVALID;
    *slot = -1;
    // pace the host: wait until the device has gathered the previous
    // snapshot, so the caller runs at most one snapshot interval ahead of
    // the device and a full ring means the consumer is behind (the device
    // keeps the steps already enqueued)
    cudaEvent_t prev = nullptr;
    {
        std::lock_guard<std::mutex> lock(r->mu);
        if (r->last >= 0) prev = r->packed[r->last];
    }
    if (prev) {
        cudaSetDevice(r->device);
        const cudaError_t w = cudaEventSynchronize(prev);
        if (w != cudaSuccess) return rfail(r, LG_ERR_CUDA, std::string("snapshot pacing: ") + cudaGetErrorString(w));
    }
    std::lock_guard<std::mutex> lock(r->mu);
    int i = 0;
    while (i < r->nslots && r->status[i] != kFree) ++i;
    if (i == r->nslots) {  // every slot in flight or held by the consumer
        ++r->dropped;
        return LG_OK;
    }
    lg::StateView v;
    int rc = lg::abi_state_view(r->st, &v);
    if (rc != LG_OK) return rc;
    cudaSetDevice(r->device);
    cudaStream_t st = lg::abi_stream(r->ctx);
    PackArgs a{};
    a.nf = (int)r->fields.size();
    for (int k = 0; k < a.nf; ++k) {
        a.field[k] = r->fields[k];
        a.ghost[k] = v.ghosts[r->fields[k]];
    }
    a.D = v.D;
    a.n0 = (int)v.block[0];
    a.n1 = (int)v.block[1];
    a.nfields = v.nfields;
    a.slab_stride = v.slab_stride;
    a.nblocks = v.nblocks;
    a.bcells = r->bcells;
    a.ncells = r->ncells;
    const dim3 grid((unsigned)std::min<int64_t>((r->bcells + 255) / 256, 1024),
                    (unsigned)std::min<int64_t>(v.nblocks, 65535), (unsigned)a.nf);
    if (v.dtype == LG_F64)
        snapshot_pack_kernel<double><<<grid, 256, 0, st>>>(static_cast<const double*>(v.arena), r->dslot[i], a);
    else
        snapshot_pack_kernel<float><<<grid, 256, 0, st>>>(static_cast<const float*>(v.arena), r->dslot[i], a);
    cudaError_t e = cudaGetLastError();
    lg::abi_count_launch(r->ctx, 1);
    const size_t bytes = r->fields.size() * (size_t)r->ncells * sizeof(double);
    if (e == cudaSuccess) e = cudaEventRecord(r->packed[i], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(r->copy, r->packed[i], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->hslot[i], r->dslot[i], bytes, cudaMemcpyDeviceToHost, r->copy);
    if (e == cudaSuccess) e = cudaEventRecord(r->copied[i], r->copy);
    if (e != cudaSuccess) return rfail(r, LG_ERR_CUDA, std::string("snapshot capture: ") + cudaGetErrorString(e));
    r->status[i] = kInFlight;
    r->last = i;
    r->seq[i] = r->next_seq++;
    r->step[i] = step;
    r->t[i] = t;
    r->epoch[i] = epoch;
    ++r->captured;
    *slot = i;
    return LG_OK;
}

int lg_snapshot_ring_poll(lg_snapshot_ring* r, int timeout_ms, int* slot, int64_t* step, double* t, int64_t* epoch,
                          const double** columns) {
    if (!r || !slot || !step || !t || !epoch || !columns) return LG_ERR_INVALID;
    *slot = -1;
    cudaSetDevice(r->device);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(std::max(timeout_ms, 0));
    for (;;) {
        {
            std::lock_guard<std::mutex> lock(r->mu);
            int oldest = -1;
            for (int i = 0; i < r->nslots; ++i)
                if (r->status[i] == kInFlight && (oldest < 0 || r->seq[i] < r->seq[oldest])) oldest = i;
            if (oldest >= 0) {
                const cudaError_t q = cudaEventQuery(r->copied[oldest]);
                if (q == cudaSuccess) {
                    r->status[oldest] = kHeld;
                    *slot = oldest;
                    *step = r->step[oldest];
                    *t = r->t[oldest];
                    *epoch = r->epoch[oldest];
                    *columns = r->hslot[oldest];
                    return LG_OK;
                }
                if (q != cudaErrorNotReady)
                    return rfail(r, LG_ERR_CUDA, std::string("snapshot copy: ") + cudaGetErrorString(q));
            }
        }
        if (std::chrono::steady_clock::now() >= deadline) return LG_ERR_TIMEOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

int lg_snapshot_ring_release(lg_snapshot_ring* r, int slot) {
    if (!r) return LG_ERR_INVALID;
    std::lock_guard<std::mutex> lock(r->mu);
    if (slot < 0 || slot >= r->nslots || r->status[slot] != kHeld)
        return rfail(r, LG_ERR_INVALID, "release of a snapshot slot the consumer does not hold");
    r->status[slot] = kFree;
    return LG_OK;
}

int lg_snapshot_ring_stats(lg_snapshot_ring* r, int64_t* captured, int64_t* dropped, int64_t* rows) {
    if (!r || !captured || !dropped || !rows) return LG_ERR_INVALID;
    std::lock_guard<std::mutex> lock(r->mu);
    *captured = r->captured;
    *dropped = r->dropped;
    *rows = r->ncells;
    return LG_OK;
}

int lg_cell_centers(int D, const int64_t* cells, const int64_t* block_cells, const double* origin,
                    const double* spacing, double* out) {
    if (!cells || !block_cells || !origin || !spacing || !out || D < 1 || D > 3) return LG_ERR_INVALID;
    int64_t n[3] = {1, 1, 1}, nb[3] = {1, 1, 1};
    for (int d = 0; d < D; ++d) {
        if (cells[d] <= 0 || block_cells[d] <= 0 || cells[d] % block_cells[d] != 0) return LG_ERR_INVALID;
        n[d] = block_cells[d];
        nb[d] = cells[d] / block_cells[d];
    }
    const int64_t bcells = n[0] * n[1] * n[2], nblocks = nb[0] * nb[1] * nb[2], ncells = bcells * nblocks;
    int64_t row = 0;
    for (int64_t b = 0; b < nblocks; ++b) {
        const int64_t bc[3] = {b % nb[0], (b / nb[0]) % nb[1], b / (nb[0] * nb[1])};  // block_coords
        for (int64_t z = 0; z < n[2]; ++z)
            for (int64_t y = 0; y < n[1]; ++y)
                for (int64_t x = 0; x < n[0]; ++x, ++row) {
                    const int64_t idx[3] = {x, y, z};
                    for (int d = 0; d < D; ++d) {
                        // (global as f64 + idx as f64 + 0.5).mul_add(spacing, origin)
                        const double a = ((double)(bc[d] * n[d]) + (double)idx[d]) + 0.5;
                        out[d * ncells + row] = std::fma(a, spacing[d], origin[d]);
                    }
                }
    }
    return LG_OK;
}

int lg_state_field_sum(lg_state* st, int field, double* sum) {
    if (!st || !sum) return LG_ERR_INVALID;
    lg::StateView v;
    int rc = lg::abi_state_view(st, &v);
    if (rc != LG_OK) return rc;
    if (field < 0 || field >= v.nfields) return lg::abi_fail(v.ctx, LG_ERR_INVALID, "field index out of range");
    cudaSetDevice(lg::abi_device(v.ctx));
    cudaStream_t s = lg::abi_stream(v.ctx);
    SumArgs a{};
    a.field = field;
    a.ghost = v.ghosts[field];
    a.D = v.D;
    a.n0 = (int)v.block[0];
    a.n1 = (int)v.block[1];
    a.nfields = v.nfields;
    a.slab_stride = v.slab_stride;
    a.nblocks = v.nblocks;
    a.bcells = v.block[0] * v.block[1] * v.block[2];
    double* d = nullptr;
    cudaError_t e = cudaMallocAsync(&d, (size_t)v.nblocks * sizeof(double), s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return lg::abi_fail(v.ctx, e == cudaErrorMemoryAllocation ? LG_ERR_NOMEM : LG_ERR_CUDA,
                            std::string("field sum: ") + cudaGetErrorString(e));
    }
    const unsigned grid = (unsigned)std::min<int64_t>(v.nblocks, (int64_t)lg::device_sm_count() * 8);
    if (v.dtype == LG_F64)
        field_sum_kernel<double><<<grid, kSumThreads, 0, s>>>(static_cast<const double*>(v.arena), d, a);
    else
        field_sum_kernel<float><<<grid, kSumThreads, 0, s>>>(static_cast<const float*>(v.arena), d, a);
    e = cudaGetLastError();
    lg::abi_count_launch(v.ctx, 1);
    std::vector<double> part((size_t)v.nblocks);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(part.data(), d, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
    const cudaError_t f = cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return lg::abi_fail(v.ctx, LG_ERR_CUDA, std::string("field sum: ") + cudaGetErrorString(e));
    double total = 0.0;
    for (double p : part) total += p;  // blocks in index order
    *sum = total;
    return LG_OK;
}

}  // extern "C"
