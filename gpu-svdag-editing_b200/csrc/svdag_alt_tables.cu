// svdag_alt_tables.cu - kernels and C ABI of the alternative table layouts (svdag_alt_tables.cuh).
//
// Two launch forms per operation, as the reference's table benchmark has them
// (extras/hashmap_bench/src/main.cu:125-200):
//  * thread per key (lanes = 1): the layout functions of svdag_alt_tables.cuh as they are;
//  * warp-hybrid (lanes = 32; addAsWarpHybrid / findAsWarpHybrid): every lane holds a key, and the
//    warp serves the lanes' keys one at a time, each lane inspecting one slot of the slab, so a slab
//    is read with one coalesced load of its slot words (128 to 256 bytes) instead of 31 dependent ones.
// The warp-hybrid functions live in svdag_alt_tables.cuh beside the thread-per-key ones, written
// against a warp type (here the intrinsics) so that the host can run them too. Layouts are template
// arguments: a kernel's copy of the table descriptor gets its layout field set to the constant, so
// the layout branches of the shared functions fold at compile time.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>

#include "svdag_alt_tables.cuh"
#include "svdag_host.hpp"

using namespace svdag;
using namespace svdag::alt;

struct svdag_alt_table {
    svdag_ctx* ctx = nullptr;
    AltTable t {};
    void* mem = nullptr;
    unsigned long long* countDev = nullptr; // stats scratch
};

namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xFFFFFFFFu;

// The warp collectives of the warp-hybrid forms (svdag_alt_tables.cuh), every lane taking part.
// The call-site argument only serves the host's emulated warp.
struct DeviceWarp {
    __device__ __forceinline__ uint32_t lane() const { return threadIdx.x & 31u; }
    __device__ __forceinline__ uint32_t ballot(bool p, uint32_t) const { return __ballot_sync(kFull, p); }
    __device__ __forceinline__ uint32_t shfl(uint32_t v, uint32_t src, uint32_t) const { return __shfl_sync(kFull, v, (int)src); }
    __device__ __forceinline__ uint64_t shfl64(uint64_t v, uint32_t src, uint32_t) const
    {
        return __shfl_sync(kFull, (unsigned long long)v, (int)src);
    }
};

template <uint32_t L>
__device__ __forceinline__ AltTable with_layout(const AltTable& t)
{
    AltTable c = t;
    c.layout = L;
    return c;
}

template <uint32_t L>
__global__ void k_alt_add(AltTable t0, const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ handles)
{
    const AltTable t = with_layout<L>(t0);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        handles[i] = add(t, keys + (uint64_t)i * t.k);
}

template <uint32_t L>
__global__ void k_alt_find(AltTable t0, const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ handles)
{
    const AltTable t = with_layout<L>(t0);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        handles[i] = find(t, keys + (uint64_t)i * t.k);
}

// Warp-hybrid forms: the loop bound is warp-uniform (every lane of a warp shares `base`).
template <uint32_t L, bool ADD>
__global__ void k_alt_warp(AltTable t0, const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ handles)
{
    const AltTable t = with_layout<L>(t0);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint64_t i = base + lane;
        const bool valid = i < n;
        const uint32_t* key = keys + (valid ? i : 0) * t.k;
        const DeviceWarp w;
        const uint32_t h = ADD ? warp_add<L>(w, t, key, valid) : warp_find<L>(w, t, key, valid);
        if (valid)
            handles[i] = h;
    }
}

__global__ void k_alt_read(AltTable t, const uint32_t* __restrict__ handles, uint32_t n, uint32_t* __restrict__ out)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        read(t, handles[i], out + (uint64_t)i * t.k);
}

__global__ void k_alt_mark(AltTable t, const uint32_t* __restrict__ handles, uint32_t n)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        mark_active(t, handles[i]);
}

// freeInactiveItems: thread per slab (slab layouts) or per bucket list (IndividualChaining), the
// freed count summed per warp into *count.
__global__ void k_alt_free(AltTable t, uint32_t units, unsigned long long* count)
{
    unsigned long long n = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < units; i += stride)
        n += t.layout == kIndividualChaining ? free_inactive_chain(t, i) : free_inactive_slab(t, i);
    for (int o = 16; o; o >>= 1)
        n += __shfl_xor_sync(kFull, n, o);
    if ((threadIdx.x & 31u) == 0 && n)
        atomicAdd(count, n);
}

// Nodes reachable from the IndividualChaining heads (thread per bucket, walks bounded by the arena).
__global__ void k_chain_count(AltTable t, unsigned long long* count)
{
    unsigned long long n = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.numBuckets; b += stride)
        for (uint32_t cur = t.heads[b], steps = 0; cur != 0 && cur <= t.slabCount && steps < t.slabCount; ++steps) {
            ++n;
            cur = slab_at(t, cur - 1u)[t.k];
        }
    for (int o = 16; o; o >>= 1)
        n += __shfl_xor_sync(kFull, n, o);
    if ((threadIdx.x & 31u) == 0 && n)
        atomicAdd(count, n);
}

__global__ void k_alt_count(AltTable t, uint32_t slabs, unsigned long long* count)
{
    unsigned long long n = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slabs; i += stride)
        n += slab_items(t.layout, slab_at(t, i));
    for (int o = 16; o; o >>= 1)
        n += __shfl_xor_sync(kFull, n, o);
    if ((threadIdx.x & 31u) == 0 && n)
        atomicAdd(count, n);
}

int grid_of(const svdag_alt_table* at, unsigned long long threads)
{
    static int smCount = 0;
    if (!smCount) {
        cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, at->ctx->device);
        if (smCount <= 0)
            smCount = 148;
    }
    const unsigned long long need = (threads + kThreads - 1) / kThreads;
    return (int)std::max<unsigned long long>(1, std::min<unsigned long long>(need, (unsigned long long)smCount * 8));
}

template <bool ADD>
svdag_status launch_op(svdag_alt_table* at, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t lanes, void* stream)
{
    if (!at || (n && (!keys || !handles)) || (lanes != 0 && lanes != 1 && lanes != 32))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    cudaSetDevice(at->ctx->device);
    const cudaStream_t s = (cudaStream_t)stream;
    const AltTable& t = at->t;
    const int grid = grid_of(at, n);
    if (lanes != 1 && t.layout != kIndividualChaining) { // a chain walk is one key's: no warp form
        switch (t.layout) {
        case kTicketBoard: k_alt_warp<kTicketBoard, ADD><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        case kAtomic64: k_alt_warp<kAtomic64, ADD><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        default: k_alt_warp<kAcceleration, ADD><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        }
    } else if (ADD) {
        switch (t.layout) {
        case kTicketBoard: k_alt_add<kTicketBoard><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        case kAtomic64: k_alt_add<kAtomic64><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        case kIndividualChaining: k_alt_add<kIndividualChaining><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        default: k_alt_add<kAcceleration><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        }
    } else {
        switch (t.layout) {
        case kTicketBoard: k_alt_find<kTicketBoard><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        case kAtomic64: k_alt_find<kAtomic64><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        case kIndividualChaining: k_alt_find<kIndividualChaining><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        default: k_alt_find<kAcceleration><<<grid, kThreads, 0, s>>>(t, keys, n, handles); break;
        }
    }
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

} // namespace

extern "C" {

svdag_status svdag_alt_table_create(svdag_ctx* ctx, uint32_t layout, uint32_t itemWords, uint32_t numBuckets,
    uint64_t reservedItems, svdag_alt_table** out)
{
    if (!ctx || !out || !layout_ok(layout, itemWords) || numBuckets == 0)
        return SVDAG_ERR_INVALID;
    *out = nullptr;
    const unsigned long long bytes = table_layout(layout, itemWords, numBuckets, reservedItems, nullptr, nullptr);
    if (!bytes)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(ctx->device);
    auto* at = new (std::nothrow) svdag_alt_table();
    if (!at)
        return SVDAG_ERR_OOM;
    at->ctx = ctx;
    if (cudaMalloc(&at->mem, bytes) != cudaSuccess || cudaMalloc(&at->countDev, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(at->mem);
        delete at;
        return SVDAG_ERR_OOM;
    }
    AltTable& t = at->t;
    table_layout(layout, itemWords, numBuckets, reservedItems, at->mem, &t);
    const uint32_t ctlInit[kCtlWords] = { initial_counter(layout, numBuckets) };
    svdag_status st = SVDAG_OK;
    // Both run on the legacy default stream and may still be in flight when they return; the wait
    // orders them before work on any stream, non-blocking streams included.
    if (cudaMemset(at->mem, 0, bytes) != cudaSuccess
        || cudaMemcpy(t.ctl, ctlInit, sizeof(ctlInit), cudaMemcpyHostToDevice) != cudaSuccess
        || cudaStreamSynchronize(0) != cudaSuccess)
        st = SVDAG_ERR_CUDA;
    if (st) {
        cudaGetLastError();
        cudaFree(at->countDev);
        cudaFree(at->mem);
        delete at;
        return st;
    }
    *out = at;
    return SVDAG_OK;
}

svdag_status svdag_alt_table_destroy(svdag_alt_table* at)
{
    if (!at)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(at->ctx->device);
    cudaFree(at->countDev);
    cudaFree(at->mem);
    delete at;
    return SVDAG_OK;
}

svdag_status svdag_alt_table_add(svdag_alt_table* at, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t lanes, void* stream)
{
    return launch_op<true>(at, keys, n, handles, lanes, stream);
}

svdag_status svdag_alt_table_find(svdag_alt_table* at, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t lanes, void* stream)
{
    return launch_op<false>(at, keys, n, handles, lanes, stream);
}

svdag_status svdag_alt_table_read(svdag_alt_table* at, const uint32_t* handles, uint32_t n, uint32_t* outWords, void* stream)
{
    if (!at || (n && (!handles || !outWords)))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    cudaSetDevice(at->ctx->device);
    k_alt_read<<<grid_of(at, n), kThreads, 0, (cudaStream_t)stream>>>(at->t, handles, n, outWords);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

svdag_status svdag_alt_table_sync(svdag_alt_table* at, void* stream)
{
    if (!at)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(at->ctx->device);
    const cudaStream_t s = (cudaStream_t)stream;
    uint32_t st = 0;
    SVDAG_CUDA(cudaMemcpyAsync(&st, &at->t.ctl[kCtlStatus], sizeof(st), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    if (st) {
        SVDAG_CUDA(cudaMemsetAsync(&at->t.ctl[kCtlStatus], 0, sizeof(uint32_t), s));
        SVDAG_CUDA(cudaStreamSynchronize(s));
    }
    return (svdag_status)st;
}

svdag_status svdag_alt_table_get_stats(svdag_alt_table* at, svdag_table_stats* out, void* stream)
{
    if (!at || !out)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(at->ctx->device);
    const cudaStream_t s = (cudaStream_t)stream;
    uint32_t next = 0;
    SVDAG_CUDA(cudaMemcpyAsync(&next, &at->t.ctl[kCtlNextSlab], sizeof(next), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    const uint32_t used = std::min(next, at->t.slabCount);
    const bool chain = at->t.layout == kIndividualChaining;
    SVDAG_CUDA(cudaMemsetAsync(at->countDev, 0, sizeof(unsigned long long), s));
    if (chain)
        k_chain_count<<<grid_of(at, at->t.numBuckets), kThreads, 0, s>>>(at->t, at->countDev);
    else
        k_alt_count<<<grid_of(at, used), kThreads, 0, s>>>(at->t, used, at->countDev);
    SVDAG_CUDA(cudaGetLastError());
    unsigned long long items = 0;
    SVDAG_CUDA(cudaMemcpyAsync(&items, at->countDev, sizeof(items), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    out->items = items;
    out->buckets = at->t.numBuckets;
    out->overflow_slabs = chain ? 0 : used - at->t.numBuckets;
    out->bytes = (chain ? ((unsigned long long)at->t.numBuckets * 4ull + 255ull) / 256ull * 256ull : 0ull)
        + (unsigned long long)used * at->t.slabWords * 4ull;
    return svdag_alt_table_sync(at, stream);
}

svdag_status svdag_alt_table_clear_active(svdag_alt_table* at, void* stream)
{
    if (!at)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(at->ctx->device);
    SVDAG_CUDA(cudaMemsetAsync(at->t.active, 0, (size_t)active_words(at->t) * 4u, (cudaStream_t)stream));
    return SVDAG_OK;
}

svdag_status svdag_alt_table_mark_active(svdag_alt_table* at, const uint32_t* handles, uint32_t n, void* stream)
{
    if (!at || (n && !handles))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    cudaSetDevice(at->ctx->device);
    k_alt_mark<<<grid_of(at, n), kThreads, 0, (cudaStream_t)stream>>>(at->t, handles, n);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

svdag_status svdag_alt_table_free_inactive(svdag_alt_table* at, uint64_t* freed, void* stream)
{
    if (!at)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(at->ctx->device);
    const cudaStream_t s = (cudaStream_t)stream;
    const bool chain = at->t.layout == kIndividualChaining;
    uint32_t next = 0;
    if (!chain) {
        SVDAG_CUDA(cudaMemcpyAsync(&next, &at->t.ctl[kCtlNextSlab], sizeof(next), cudaMemcpyDeviceToHost, s));
        SVDAG_CUDA(cudaStreamSynchronize(s));
    }
    const uint32_t units = chain ? at->t.numBuckets : std::min(next, at->t.slabCount);
    SVDAG_CUDA(cudaMemsetAsync(at->countDev, 0, sizeof(unsigned long long), s));
    k_alt_free<<<grid_of(at, units), kThreads, 0, s>>>(at->t, units, at->countDev);
    SVDAG_CUDA(cudaGetLastError());
    unsigned long long n = 0;
    SVDAG_CUDA(cudaMemcpyAsync(&n, at->countDev, sizeof(n), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    if (freed)
        *freed = n;
    return svdag_alt_table_sync(at, stream);
}

svdag_status svdag_alt_table_tune(svdag_ctx* ctx, const uint32_t* keys, uint32_t n, uint32_t itemWords, uint32_t itemsPerBucket,
    svdag_alt_tuning* best, svdag_alt_tuning* all, void* stream)
{
    if (!ctx || !keys || !n || !best || itemWords < 1 || itemWords > alt::kMaxItemWords)
        return SVDAG_ERR_INVALID;
    const uint32_t ipb = itemsPerBucket ? itemsPerBucket : 64u;
    const uint32_t buckets = n / ipb + 1;
    const cudaStream_t s = (cudaStream_t)stream;
    cudaSetDevice(ctx->device);
    uint32_t* handles = nullptr;
    cudaEvent_t ev[3] = {};
    if (cudaMalloc(&handles, (size_t)n * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return SVDAG_ERR_OOM;
    }
    svdag_status st = SVDAG_OK;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess)
            st = SVDAG_ERR_CUDA;
    svdag_alt_tuning cand[SVDAG_ALT_TUNING_CANDIDATES] = {};
    int bestIdx = -1;
    // (layout, lanes): each slab layout thread per key and warp-hybrid, IndividualChaining thread per key
    const uint32_t layouts[SVDAG_ALT_TUNING_CANDIDATES] = { kTicketBoard, kTicketBoard, kAtomic64, kAtomic64, kAcceleration,
        kAcceleration, kIndividualChaining };
    const uint32_t laneCounts[SVDAG_ALT_TUNING_CANDIDATES] = { 1, 32, 1, 32, 1, 32, 1 };
    for (uint32_t c = 0; c < SVDAG_ALT_TUNING_CANDIDATES && st == SVDAG_OK; ++c) {
        svdag_alt_tuning& r = cand[c];
        r.layout = layouts[c];
        r.lanes = laneCounts[c];
        r.add_ms = r.find_ms = -1.0f;
        if (!layout_ok(r.layout, itemWords))
            continue;
        { // untimed warm-up on a small table: a kernel's first launch also loads it (lazy module loading)
            svdag_alt_table* w = nullptr;
            const uint32_t wn = std::min(n, 1024u);
            if (svdag_alt_table_create(ctx, r.layout, itemWords, 64, 2ull * wn, &w) == SVDAG_OK) {
                svdag_alt_table_add(w, keys, wn, handles, r.lanes, stream);
                svdag_alt_table_find(w, keys, wn, handles, r.lanes, stream);
                svdag_alt_table_sync(w, stream); // a latched error here shows again in the timed run
                svdag_alt_table_destroy(w);
            }
        }
        svdag_alt_table* t = nullptr;
        const svdag_status cs = svdag_alt_table_create(ctx, r.layout, itemWords, buckets, 2ull * n, &t);
        if (cs == SVDAG_ERR_OOM)
            continue;
        if (cs != SVDAG_OK) {
            st = cs;
            break;
        }
        svdag_status ts = SVDAG_OK;
        if (cudaEventRecord(ev[0], s) != cudaSuccess || (ts = svdag_alt_table_add(t, keys, n, handles, r.lanes, stream)) != SVDAG_OK
            || cudaEventRecord(ev[1], s) != cudaSuccess || (ts = svdag_alt_table_find(t, keys, n, handles, r.lanes, stream)) != SVDAG_OK
            || cudaEventRecord(ev[2], s) != cudaSuccess)
            ts = ts ? ts : SVDAG_ERR_CUDA;
        const svdag_status ds = ts ? ts : svdag_alt_table_sync(t, stream); // a latched error: the sample does not fit this layout
        if (ds == SVDAG_OK) {
            float a = 0, f = 0;
            cudaEventElapsedTime(&a, ev[0], ev[1]);
            cudaEventElapsedTime(&f, ev[1], ev[2]);
            r.add_ms = a;
            r.find_ms = f;
            if (bestIdx < 0 || a + f < cand[bestIdx].add_ms + cand[bestIdx].find_ms)
                bestIdx = (int)c;
        } else if (ds == SVDAG_ERR_CUDA) {
            st = ds;
        }
        svdag_alt_table_destroy(t);
    }
    for (auto& e : ev)
        if (e)
            cudaEventDestroy(e);
    cudaFree(handles);
    if (st != SVDAG_OK)
        return st;
    if (bestIdx < 0)
        return SVDAG_ERR_OOM;
    *best = cand[bestIdx];
    if (all)
        for (uint32_t c = 0; c < SVDAG_ALT_TUNING_CANDIDATES; ++c)
            all[c] = cand[c];
    return SVDAG_OK;
}

} // extern "C"
