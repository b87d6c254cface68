// svdag_ctx.cu - context lifetime (one preallocated HBM pool), status, statistics, garbage collection.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>

#include "svdag_edit.cuh"
#include "svdag_host.hpp"

using namespace svdag;

namespace {

constexpr unsigned long long kCtlBytes = 64 * 1024;
constexpr unsigned long long kBatchBytes = 2 * 1024 * 1024;

// ---------------------------------------------------------------- garbage collection
// MyGPUHashDAG::garbageCollect(activeRootNodes) (my_gpu_hash_dag.cu:373-463) marks level by level
// from the active roots and the canonical fully-filled nodes; freeInactiveItems
// (gpu_hash_table_base.cu:265-374) then clears every unmarked slot and hands every overflow slab it
// leaves empty back to the slab allocator. Here marking is a bitmap with one bit per handle (an
// 16-byte handle unit of the item region) and the frontier is deduplicated by the test-and-set on it; the
// sweep unlinks empty overflow slabs and pushes them on the free list of their size class.
// MyGPUHashDAGUndoRedo::garbageCollect (my_gpu_base_dag.h:66-77) passes the current root alone and
// clears the history (svdag_gc); svdag_gc_keep_history passes the current root and every undo and
// redo root, and keeps the history.

__device__ __forceinline__ bool mark_once(uint32_t* bits, uint32_t handle)
{
    const uint32_t m = 1u << (handle & 31u);
    if (__ldcg(&bits[handle >> 5]) & m) // most children of a shared DAG are marked already
        return false;
    return !(atomicOr(&bits[handle >> 5], m) & m);
}

__device__ __forceinline__ void push_root(const DevDag& d, uint32_t* bits, uint32_t h, uint32_t* frontier, uint32_t& n)
{
    if (h == kNone)
        return;
    if (!handle_ok(d, h)) {
        set_status(d.ctl, SVDAG_ERR_CORRUPT);
        return;
    }
    if (mark_once(bits, h))
        frontier[n++] = h;
}

// Level-0 frontier: the root, the canonical fully-filled nodes of level 0 and, with `history`,
// every root of the undo ring and the redo stack (at most 1 + 16 + 64 + 64 entries).
__global__ void k_gc_roots(DevDag d, uint32_t* bits, uint32_t* frontier, uint32_t* count, uint32_t history)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    const Control* c = d.ctl;
    uint32_t n = 0;
    push_root(d, bits, c->root, frontier, n);
    for (uint32_t m = 0; m < SVDAG_NUM_MATERIALS; ++m)
        push_root(d, bits, c->fullyFilled[0][m], frontier, n);
    if (history) {
        const uint32_t nu = c->undoCount < 64u ? c->undoCount : 64u;
        for (uint32_t i = 0; i < nu; ++i)
            push_root(d, bits, c->undo[(c->undoHead + 63u - i) & 63u], frontier, n);
        const uint32_t nr = c->redoCount < 64u ? c->redoCount : 64u;
        for (uint32_t i = 0; i < nr; ++i)
            push_root(d, bits, c->redo[i], frontier, n);
    }
    count[0] = n;
}

// Marks the children of the level's frontier and gathers the newly marked ones (plus the canonical
// fully-filled items of the level below) as the next frontier. A frontier longer than `cap` latches
// SVDAG_ERR_OOM; the next level then reads only the first `cap` entries and the host leaves the
// tables untouched (no sweep runs after an incomplete mark).
__global__ void k_gc_mark(DevDag d, uint32_t* bits, uint32_t level, const uint32_t* in, const uint32_t* inCount, uint32_t* out,
    uint32_t* outCount, uint32_t cap)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (uint32_t m = 0; m < SVDAG_NUM_MATERIALS; ++m) {
            const uint32_t h = d.ctl->fullyFilled[level + 1][m];
            if (h == kNone || !handle_ok(d, h) || !mark_once(bits, h))
                continue;
            const uint32_t at = atomicAdd(outCount, 1u);
            if (at < cap)
                out[at] = h;
            else
                set_status(d.ctl, SVDAG_ERR_OOM);
        }
    }
    const uint32_t n = min(*inCount, cap);
    // Whole warps iterate together (the bound is rounded up to a warp multiple) so that the
    // children a warp marks in one step take a single atomic on the frontier counter.
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += stride) {
        const uint32_t i = base + lane;
        const uint32_t* node = i < n ? item_ptr(d, in[i]) : nullptr;
        const uint32_t mask = node ? node[0] & 0xFFu : 0u;
        uint32_t children[8];
        uint32_t mine = 0; // children this lane marked first
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) {
            if (j < (uint32_t)__popc(mask)) {
                const uint32_t c = node[1 + j];
                if (!handle_ok(d, c))
                    set_status(d.ctl, SVDAG_ERR_CORRUPT);
                else if (mark_once(bits, c))
                    children[mine++] = c;
            }
        }
        // warp-wide exclusive scan of `mine`
        uint32_t prefix = mine;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, prefix, o);
            if (lane >= o)
                prefix += v;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, prefix, 31);
        uint32_t first = 0;
        if (lane == 31 && total)
            first = atomicAdd(outCount, total);
        first = __shfl_sync(0xFFFFFFFFu, first, 31) + prefix - mine;
        for (uint32_t j = 0; j < mine; ++j) {
            if (first + j < cap)
                out[first + j] = children[j];
            else
                set_status(d.ctl, SVDAG_ERR_OOM);
        }
    }
}

// One thread per bucket: clears the unmarked occupied slots (tag and item words) of its chain and
// unlinks every overflow slab left without an occupied slot (the bucket's own slab stays); the
// unlinked slabs of a thread are pushed on their class's free list as one chain.
__global__ void k_gc_sweep(DevDag d, DevTable t, const uint32_t* bits, unsigned long long* freed)
{
    unsigned long long nfreed = 0, nslabs = 0;
    for (uint32_t c = 0; c < kNumClasses; ++c) {
        const uint32_t k = c + 2;
        uint32_t first = kEnd, last = kEnd, count = 0; // unlinked slabs, linked through word 7
        for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.numBuckets[c]; b += gridDim.x * blockDim.x) {
            uint32_t slab = t.bucketBase[c] + b;
            uint32_t* prevLink = nullptr; // the link word that leads to `slab` (none for the bucket's slab)
            for (uint32_t steps = 0; steps < kMaxChain; ++steps) {
                uint32_t* h = slab_ptr(d, slab);
                const uint32_t body = h[6];
                uint32_t live = 0;
                for (uint32_t s = 0; s < kSlots; ++s) {
                    const uint32_t tag = header_tag(h, s);
                    if (tag == 0)
                        continue;
                    const uint32_t item = slot_handle(body, s, k);
                    if (tag == kTagBusy || ((bits[item >> 5] >> (item & 31u)) & 1u)) {
                        ++live;
                        continue;
                    }
                    if (!handle_ok(d, item)) {
                        set_status(d.ctl, SVDAG_ERR_CORRUPT);
                        ++live;
                        continue;
                    }
                    uint32_t* ip = handle_ptr(d, item);
                    for (uint32_t j = 0; j < k; ++j)
                        ip[j] = 0;
                    h[s >> 2] &= ~(0xFFu << (8u * (s & 3u)));
                    ++nfreed;
                }
                const uint32_t next = h[7];
                if (next != kEnd && !slab_ok(d, next)) {
                    set_status(d.ctl, SVDAG_ERR_CORRUPT);
                    break;
                }
                if (live == 0 && prevLink) { // an empty overflow slab: out of the chain, onto the free list
                    *prevLink = next;
                    h[7] = first;
                    first = slab;
                    if (last == kEnd)
                        last = slab;
                    ++count;
                } else {
                    prevLink = h + 7;
                }
                if (next == kEnd)
                    break;
                slab = next;
            }
        }
        if (count) {
            push_free_chain(d, c, first, last, count);
            nslabs += count;
        }
    }
    if (nfreed)
        atomicAdd(&freed[0], nfreed);
    if (nslabs)
        atomicAdd(&freed[1], nslabs);
}

__global__ void k_gc_finish(Control* c, const unsigned long long* freed, const uint32_t* counts, uint32_t levels, uint32_t clearHistory)
{
    unsigned long long live = 0;
    for (uint32_t l = 0; l < levels; ++l) // counts[l]: the frontier of level l, every item marked once
        live += counts[l];
    c->gcLiveItems = live;
    c->gcFreedItems = freed[0];
    c->gcFreedSlabs = freed[1];
    if (clearHistory) {
        c->undoCount = 0;
        c->redoCount = 0;
    }
}

svdag_status collect(svdag_ctx* ctx, bool keepHistory, cudaStream_t s)
{
    SVDAG_TRY(ensure_level_tables(ctx, s));
    // A collection reports its own errors: an error latched by earlier work (which its own call or
    // record reported) is cleared first.
    (void)read_status(ctx, s);
    unsigned long long top = 0;
    SVDAG_CUDA(cudaMemcpyAsync(&top, &ctx->ctl->itemTop, sizeof(top), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    top = std::min<unsigned long long>(top, ctx->itemWords);
    const unsigned long long bitmapBytes = align256(((top / kUnitWords) + 64) / 8 + 8); // one bit per handle unit
    const unsigned long long rest = ctx->scratchBytes > bitmapBytes + 4096 ? ctx->scratchBytes - bitmapBytes - 4096 : 0;
    uint32_t frontierCap = (uint32_t)std::min<unsigned long long>(rest / 8, 0xFFFFFFFFull); // two frontiers of u32
    // SVDAG_GC_MAX_FRONTIER lowers the frontier capacity (tests reach the overflow path with it
    // without a DAG larger than the scratch arena).
    if (const char* cap = std::getenv("SVDAG_GC_MAX_FRONTIER"))
        frontierCap = (uint32_t)std::min<unsigned long long>(frontierCap, std::strtoull(cap, nullptr, 10));
    if (frontierCap < 1024)
        return SVDAG_ERR_OOM;
    auto* bits = reinterpret_cast<uint32_t*>(ctx->scratch);
    auto* counts = reinterpret_cast<uint32_t*>(ctx->scratch + bitmapBytes);
    auto* fa = reinterpret_cast<uint32_t*>(ctx->scratch + bitmapBytes + 4096);
    auto* fb = fa + frontierCap;
    ctx->scratchHighWater = std::max(ctx->scratchHighWater, bitmapBytes + 4096);
    SVDAG_CUDA(cudaMemsetAsync(ctx->scratch, 0, bitmapBytes + 4096, s));
    const DevDag d = ctx->dag();
    k_gc_roots<<<1, 32, 0, s>>>(d, bits, fa, counts + 0, keepHistory ? 1u : 0u);
    const uint32_t LL = d.leafLevel;
    for (uint32_t level = 0; level < LL; ++level) {
        uint32_t* in = (level & 1) ? fb : fa;
        uint32_t* out = (level & 1) ? fa : fb;
        k_gc_mark<<<grid_for(ctx, 1ull << 24, 256), 256, 0, s>>>(d, bits, level, in, counts + level, out, counts + level + 1, frontierCap);
    }
    SVDAG_CUDA(cudaGetLastError());
    // An incomplete mark (frontier overflow, a corrupt handle) must not free anything.
    SVDAG_TRY(read_status(ctx, s));
    auto* freed = reinterpret_cast<unsigned long long*>(counts + 64);
    for (uint32_t level = 0; level <= LL; ++level) {
        const DevTable t = ctx->levelTables[level].dev;
        unsigned long long nb = 0;
        for (uint32_t c = 0; c < kNumClasses; ++c)
            nb = std::max<unsigned long long>(nb, t.numBuckets[c]);
        k_gc_sweep<<<grid_for(ctx, nb, 256), 256, 0, s>>>(d, t, bits, freed);
    }
    k_gc_finish<<<1, 1, 0, s>>>(ctx->ctl, freed, counts, LL + 1, keepHistory ? 0u : 1u);
    SVDAG_CUDA(cudaGetLastError());
    return read_status(ctx, s);
}

} // namespace

extern "C" {

uint32_t svdag_abi_version(void) { return SVDAG_ABI_VERSION; }

const char* svdag_status_string(svdag_status s)
{
    switch (s) {
    case SVDAG_OK:
        return "ok";
    case SVDAG_ERR_INVALID:
        return "invalid argument";
    case SVDAG_ERR_OOM:
        return "out of memory (pool, item region or scratch arena)";
    case SVDAG_ERR_TIMEOUT:
        return "bounded device wait or retry loop gave up";
    case SVDAG_ERR_CORRUPT:
        return "structural invariant violated";
    case SVDAG_ERR_CUDA:
        return "CUDA runtime error";
    case SVDAG_ERR_NO_DEVICE:
        return "no usable sm_100 device";
    case SVDAG_ERR_UNSUPPORTED:
        return "unsupported";
    case SVDAG_ERR_BUSY:
        return "busy";
    }
    return "unknown status";
}

svdag_status svdag_create(const svdag_config* cfg, svdag_ctx** out)
{
    if (!cfg || !out || cfg->levels < SVDAG_MIN_LEVELS || cfg->levels > SVDAG_MAX_LEVELS || (cfg->flags & ~(SVDAG_FLAG_PHASE_KERNELS | SVDAG_FLAG_PERSISTENT)) != 0)
        return SVDAG_ERR_INVALID;
    if (cfg->probe_lanes && cfg->probe_lanes != 1 && cfg->probe_lanes != 2 && cfg->probe_lanes != 4 && cfg->probe_lanes != 8
        && cfg->probe_lanes != 16 && cfg->probe_lanes != 32)
        return SVDAG_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || cfg->device < 0 || cfg->device >= ndev) {
        cudaGetLastError();
        return SVDAG_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop {};
    SVDAG_CUDA(cudaGetDeviceProperties(&prop, cfg->device));
    if (prop.major != 10)
        return SVDAG_ERR_NO_DEVICE; // built for sm_100a only
    SVDAG_CUDA(cudaSetDevice(cfg->device));
    const unsigned long long pool = cfg->pool_bytes ? cfg->pool_bytes : (1ull << 30);
    const unsigned long long scratch = (cfg->scratch_bytes ? cfg->scratch_bytes : pool / 4) & ~255ull;
    if (scratch + kCtlBytes + kBatchBytes + (1ull << 20) > pool)
        return SVDAG_ERR_INVALID;
    auto* ctx = new (std::nothrow) svdag_ctx();
    if (!ctx)
        return SVDAG_ERR_OOM;
    ctx->cfg = *cfg;
    ctx->device = cfg->device;
    ctx->probeLanes = cfg->probe_lanes ? cfg->probe_lanes : 1; // thread per key: measured fastest on B200
    ctx->loadFactor = cfg->target_load_factor ? cfg->target_load_factor : 16;
    ctx->persistentLeaves = (cfg->flags & SVDAG_FLAG_PERSISTENT) ? 16384.0 : 0.0;
    ctx->cfg.undo_depth = cfg->undo_depth ? std::min<uint32_t>(cfg->undo_depth, 64) : 32;
    if (cudaMalloc(&ctx->pool, pool) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return SVDAG_ERR_OOM;
    }
    ctx->poolBytes = pool;
    ctx->ctl = reinterpret_cast<Control*>(ctx->pool);
    ctx->batch = ctx->pool + kCtlBytes;
    ctx->batchBytes = kBatchBytes - 4096; // the last 4 KiB hold the editor queue of the phase launches
    ctx->queue = reinterpret_cast<EditQueue*>(ctx->batch + ctx->batchBytes);
    static_assert(sizeof(EditQueue) <= 4096, "editor queue too large");
    ctx->scratch = ctx->pool + kCtlBytes + kBatchBytes;
    ctx->scratchBytes = scratch;
    // The rest: slab headers (a thirteenth: 32 bytes per slab, whose body of 24 items takes at least
    // 24 * 16 = 384 bytes) then items.
    const unsigned long long rest = pool - kCtlBytes - kBatchBytes - scratch;
    const unsigned long long headerBytes = align256(rest / 13);
    ctx->headers = reinterpret_cast<uint32_t*>(ctx->pool + kCtlBytes + kBatchBytes + scratch);
    ctx->headerCount = std::min<unsigned long long>(headerBytes / 32, 0xFFFFFFF0ull);
    ctx->items = reinterpret_cast<uint32_t*>(ctx->pool + kCtlBytes + kBatchBytes + scratch + headerBytes);
    ctx->itemWords = std::min<unsigned long long>((rest - headerBytes) / 4 - 64, kMaxItemWords) & ~31ull;
    static_assert(sizeof(Control) <= kCtlBytes, "control block too large");
    cudaError_t e = cudaMemset(ctx->pool, 0, pool);
    if (e == cudaSuccess) {
        Control init {};
        init.headerTop = 1;
        init.root = kNone;
        init.undoDepth = ctx->cfg.undo_depth;
        init.savedRoot = kNone;
        for (auto& lv : init.fullyFilled)
            for (auto& m : lv)
                m = kNone;
        e = cudaMemcpy(ctx->ctl, &init, sizeof(init), cudaMemcpyHostToDevice);
    }
    // The memset and the copy run on the legacy default stream and may still be in flight when they
    // return; waiting here orders them before the caller's work on any stream (non-blocking included).
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        cudaFree(ctx->pool);
        delete ctx;
        return cuda_status(e);
    }
    *out = ctx;
    return SVDAG_OK;
}

svdag_status svdag_destroy(svdag_ctx* ctx)
{
    if (!ctx)
        return SVDAG_ERR_INVALID;
    cudaSetDevice(ctx->device);
    for (auto* t : ctx->standalone)
        delete t;
    for (auto& g : ctx->graphs)
        if (g)
            cudaGraphExecDestroy(g);
    cudaDeviceSynchronize();
    cudaFree(ctx->pool);
    delete ctx;
    return SVDAG_OK;
}

svdag_status svdag_sync(svdag_ctx* ctx, void* stream)
{
    if (!ctx)
        return SVDAG_ERR_INVALID;
    return read_status(ctx, as_stream(stream));
}

svdag_status svdag_get_root(svdag_ctx* ctx, uint32_t* root, void* stream)
{
    if (!ctx || !root)
        return SVDAG_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    SVDAG_CUDA(cudaMemcpyAsync(root, &ctx->ctl->root, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    return SVDAG_OK;
}

svdag_status svdag_gc(svdag_ctx* ctx, void* stream)
{
    if (!ctx)
        return SVDAG_ERR_INVALID;
    return collect(ctx, false, as_stream(stream));
}

svdag_status svdag_gc_keep_history(svdag_ctx* ctx, void* stream)
{
    if (!ctx)
        return SVDAG_ERR_INVALID;
    return collect(ctx, true, as_stream(stream));
}

svdag_status svdag_get_stats(svdag_ctx* ctx, svdag_stats* out, void* stream)
{
    if (!ctx || !out)
        return SVDAG_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    std::memset(out, 0, sizeof(*out));
    Control c;
    SVDAG_CUDA(cudaMemcpyAsync(&c, ctx->ctl, sizeof(c), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    out->levels = ctx->cfg.levels;
    out->root = c.root;
    out->pool_bytes = ctx->poolBytes;
    out->item_region_bytes = ctx->itemWords * 4 + ctx->headerCount * 32;
    out->item_region_used_bytes = used_region_bytes(ctx, c.itemTop, c.headerTop, c.freeBytes);
    out->free_list_bytes = c.freeBytes;
    for (uint32_t k = 0; k < kNumClasses; ++k)
        out->free_list_slabs += c.freeSlabs[k];
    out->gc_freed_items = c.gcFreedItems;
    out->gc_freed_slabs = c.gcFreedSlabs;
    out->gc_live_items = c.gcLiveItems;
    out->scratch_bytes = ctx->scratchBytes;
    out->scratch_high_water_bytes = ctx->scratchHighWater;
    out->undo_count = c.undoCount;
    out->redo_count = c.redoCount;
    for (uint32_t l = 0; l + 1 < ctx->cfg.levels; ++l) {
        svdag_table& t = ctx->levelTables[l];
        if (!t.ready)
            continue;
        svdag_table_stats ts {};
        SVDAG_TRY(svdag_table_get_stats(&t, &ts, stream));
        out->level_items[l] = ts.items;
        out->level_buckets[l] = ts.buckets;
    }
    return SVDAG_OK;
}

} // extern "C"
