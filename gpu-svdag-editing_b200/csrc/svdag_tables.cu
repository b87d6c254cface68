// svdag_tables.cu - level/standalone slab hash tables: allocation, batched add/find, export.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "svdag_host.hpp"

using namespace svdag;

namespace svdag {

int grid_for(const svdag_ctx* ctx, unsigned long long work, int threadsPerBlock, int blocksPerSm)
{
    static int smCount = 0;
    if (!smCount) {
        cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, ctx->device);
        if (smCount <= 0)
            smCount = 148;
    }
    const unsigned long long maxBlocks = (unsigned long long)smCount * blocksPerSm;
    const unsigned long long need = (work + threadsPerBlock - 1) / threadsPerBlock;
    return (int)std::max<unsigned long long>(1, std::min(maxBlocks, need));
}

svdag_status read_status(svdag_ctx* ctx, cudaStream_t s)
{
    uint32_t st = 0;
    SVDAG_CUDA(cudaMemcpyAsync(&st, &ctx->ctl->status, sizeof(st), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    if (st) {
        const uint32_t zero = 0;
        SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->status, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
        SVDAG_CUDA(cudaStreamSynchronize(s));
    }
    return (svdag_status)st;
}

// Writes the body handle of every bucket header of a table (the rest of each header is cleared).
__global__ void k_init_bucket_headers(DevDag d, DevTable t)
{
    for (uint32_t c = 0; c < kNumClasses; ++c) {
        const uint32_t units = body_words(c + 2) / kUnitWords;
        for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.numBuckets[c]; b += gridDim.x * blockDim.x) {
            uint4* h = reinterpret_cast<uint4*>(slab_ptr(d, t.bucketBase[c] + b));
            h[0] = make_uint4(0, 0, 0, 0);
            h[1] = make_uint4(0, 0, t.bodyBase[c] + b * units, kEnd);
        }
    }
}

// Reserves a table's bucket headers at the top of the header region and its first slab bodies at the
// top of the item region, clears them and links each header to its body.
svdag_status alloc_table(svdag_ctx* ctx, svdag_table* t, uint32_t kind, const uint32_t* bucketsPerClass, cudaStream_t s, bool recycle)
{
    unsigned long long tops[2] = { 0, 0 }; // itemTop (words), headerTop (headers)
    SVDAG_CUDA(cudaMemcpyAsync(tops, &ctx->ctl->itemTop, sizeof(tops), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    DevTable dev {};
    dev.kind = kind;
    dev.recycle = recycle ? 1u : 0u;
    unsigned long long words = 0, headers = 0, buckets = 0;
    for (uint32_t c = 0; c < kNumClasses; ++c) {
        dev.numBuckets[c] = bucketsPerClass[c];
        dev.bucketBase[c] = (uint32_t)(tops[1] + headers);
        dev.bodyBase[c] = (uint32_t)((tops[0] + words) / kUnitWords); // tops[0] and body sizes are multiples of 32 words
        words += (unsigned long long)bucketsPerClass[c] * body_words(c + 2);
        headers += bucketsPerClass[c];
        buckets = std::max<unsigned long long>(buckets, bucketsPerClass[c]);
    }
    if (tops[0] + words > ctx->itemWords || tops[1] + headers > ctx->headerCount)
        return SVDAG_ERR_OOM;
    SVDAG_CUDA(cudaMemsetAsync(ctx->items + tops[0], 0, words * 4, s));
    k_init_bucket_headers<<<grid_for(ctx, buckets, 256), 256, 0, s>>>(ctx->dag(), dev);
    SVDAG_CUDA(cudaGetLastError());
    const unsigned long long newTops[2] = { tops[0] + words, tops[1] + headers };
    SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->itemTop, newTops, sizeof(newTops), cudaMemcpyHostToDevice, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    t->ctx = ctx;
    t->dev = dev;
    t->ready = true;
    t->words = words + headers * kHeaderWords;
    return SVDAG_OK;
}

__global__ void k_insert_canonical(DevDag d, DevTable t, uint32_t level)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    Grp<1> g;
    Spare spare;
    for (uint32_t m = 0; m < SVDAG_NUM_MATERIALS; ++m) {
        Key<1> key;
        if (level == d.leafLevel) { // fully filled leaf of material m (my_gpu_hash_dag.cu:40-49)
            key.w[0] = key.w[1] = 0xFFFFFFFFu;
            for (uint32_t i = 2; i < 10; ++i)
                key.w[i] = m * 0x11111111u;
            key.n = 10;
        } else { // node with 8 fully-filled children (my_gpu_hash_dag.cu:50-63)
            key.w[0] = 0xFFu | (1u << 8) | (m << 9);
            for (uint32_t i = 1; i < 9; ++i)
                key.w[i] = d.ctl->fullyFilled[level + 1][m];
            key.w[9] = 0;
            key.n = 9;
        }
        hash_words(key.w, key.n, key.ha, key.hb);
        bool inserted;
        d.ctl->fullyFilled[level][m] = table_find_or_insert<1>(g, d, t, key, spare, inserted);
    }
    release_spare<1>(g, d, t, spare);
}

svdag_status insert_canonical(svdag_ctx* ctx, uint32_t level, cudaStream_t s)
{
    k_insert_canonical<<<1, 32, 0, s>>>(ctx->dag(), ctx->levelTables[level].dev, level);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

void reset_level_tables(svdag_ctx* ctx)
{
    for (auto& t : ctx->levelTables)
        t = svdag_table {};
}

// Default bucket counts for a level that was not sized by a scene build: the surface of a scene
// grows as 4^level, capped; chains absorb the rest.
svdag_status ensure_level_tables(svdag_ctx* ctx, cudaStream_t s)
{
    const uint32_t leaf = ctx->cfg.levels - 2;
    bool created = false;
    for (int level = (int)leaf; level >= 0; --level) {
        svdag_table& t = ctx->levelTables[level];
        if (t.ready)
            continue;
        const unsigned long long expect = std::min<unsigned long long>(1ull << (2 * (level + 1)), 1ull << 20);
        uint32_t buckets[kNumClasses];
        for (uint32_t c = 0; c < kNumClasses; ++c)
            buckets[c] = (uint32_t)std::max<unsigned long long>(1, expect / (4ull * ctx->loadFactor));
        SVDAG_TRY(alloc_table(ctx, &t, level == (int)leaf ? SVDAG_KIND_LEAF : SVDAG_KIND_NODE, buckets, s, true));
        t.level = level;
        SVDAG_TRY(insert_canonical(ctx, (uint32_t)level, s));
        created = true;
    }
    return created ? upload_tables(ctx, s) : SVDAG_OK;
}

svdag_status upload_tables(svdag_ctx* ctx, cudaStream_t s)
{
    DevTable t[kMaxLevels];
    for (uint32_t l = 0; l < kMaxLevels; ++l)
        t[l] = ctx->levelTables[l].dev;
    SVDAG_CUDA(cudaMemcpyAsync(ctx->ctl->tables, t, sizeof(t), cudaMemcpyHostToDevice, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    return SVDAG_OK;
}

} // namespace svdag

// ---------------------------------------------------------------- batched table kernels

namespace {

enum { OP_FIND = 0, OP_ADD = 1, OP_FIND_OR_INSERT = 2 };

template <int G, int OP>
__global__ void __launch_bounds__(256) k_table_op(DevDag d, DevTable t, const uint32_t* __restrict__ keys,
    const uint32_t* __restrict__ offsets, uint32_t n, unsigned long long totalWords, const uint32_t* __restrict__ reps,
    uint32_t* __restrict__ out)
{
    Grp<G> g;
    const uint32_t groupsPerBlock = blockDim.x / G;
    const unsigned long long stride = (unsigned long long)gridDim.x * groupsPerBlock;
    Spare spare;
    for (unsigned long long i = blockIdx.x * groupsPerBlock + threadIdx.x / G; i < n; i += stride) {
        if (reps && reps[i] != i)
            continue;
        const uint32_t off = offsets[i];
        if (off >= totalWords) {
            if (g.lane == 0)
                out[i] = kNone;
            set_status(d.ctl, SVDAG_ERR_INVALID);
            continue;
        }
        Key<G> key;
        load_key<G>(g, keys + off, totalWords - off, t.kind, key);
        uint32_t h;
        if constexpr (OP == OP_FIND) {
            h = table_find<G>(g, d, t, key);
        } else if constexpr (OP == OP_ADD) {
            h = table_add<G>(g, d, t, key, spare);
        } else {
            bool ins;
            h = table_find_or_insert<G>(g, d, t, key, spare, ins);
        }
        if (g.lane == 0)
            out[i] = h;
    }
    release_spare<G>(g, d, t, spare);
}

// Batch dedup into an open-addressing scratch table of 64-bit entries (tag hash << 32 | index+1).
__global__ void __launch_bounds__(256) k_batch_dedup(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ offsets,
    uint32_t n, unsigned long long totalWords, uint32_t kind, unsigned long long* table, uint32_t capMask, uint32_t* reps,
    Control* ctl)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t off = offsets[i];
        if (off >= totalWords) {
            reps[i] = i;
            set_status(ctl, SVDAG_ERR_INVALID);
            continue;
        }
        const uint32_t* p = keys + off;
        const unsigned long long lim = totalWords - off;
        uint32_t w[kItemStride] = {};
        w[0] = lim > 0 ? p[0] : 0u;
        w[1] = lim > 1 ? p[1] : 0u;
        const uint32_t nw = kind == SVDAG_KIND_NODE ? dev_node_words(w[0]) : dev_leaf_words(w[0], w[1]);
        for (uint32_t j = 2; j < nw && j < lim; ++j)
            w[j] = p[j];
        uint32_t ha, hb;
        hash_words(w, nw, ha, hb);
        const unsigned long long entry = ((unsigned long long)hb << 32) | (unsigned long long)(i + 1u);
        uint32_t slot = ha & capMask;
        uint32_t rep = i;
        for (uint32_t probe = 0;; ++probe) {
            if (probe > capMask) {
                set_status(ctl, SVDAG_ERR_OOM);
                break;
            }
            unsigned long long e = table[slot];
            if (e == 0) {
                e = atomicCAS(&table[slot], 0ull, entry);
                if (e == 0)
                    break;
            }
            if ((uint32_t)(e >> 32) == hb) {
                const uint32_t j = (uint32_t)e - 1u;
                const uint32_t* q = keys + offsets[j];
                const unsigned long long qlim = totalWords - offsets[j];
                bool same = true;
                for (uint32_t k = 0; k < nw && same; ++k)
                    same = k < qlim && q[k] == w[k];
                if (same) {
                    rep = j;
                    break;
                }
            }
            slot = (slot + 1u) & capMask;
        }
        reps[i] = rep;
    }
}

__global__ void k_gather(const uint32_t* reps, uint32_t n, uint32_t* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (reps[i] != i)
            out[i] = out[reps[i]];
}

__global__ void k_table_read(DevDag d, uint32_t kind, const uint32_t* handles, uint32_t n, uint32_t* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t h = handles[i];
        uint32_t* o = out + (size_t)i * kItemStride;
        if (h == kNone || !handle_ok(d, h)) {
            for (uint32_t j = 0; j < kItemStride; ++j)
                o[j] = 0;
            continue;
        }
        const uint32_t* p = handle_ptr(d, h);
        const uint32_t nw = kind == SVDAG_KIND_NODE ? dev_node_words(p[0]) : dev_leaf_words(p[0], p[1]);
        for (uint32_t j = 0; j < kItemStride; ++j)
            o[j] = j < nw ? p[j] : 0u;
    }
}

// One thread per bucket walks the chain: counts items and overflow slabs, optionally dumps items.
__global__ void k_table_walk(DevDag d, DevTable t, unsigned long long* counters, uint32_t* outHandles, uint32_t* outWords,
    unsigned long long capacity)
{
    for (uint32_t c = 0; c < kNumClasses; ++c) {
        const uint32_t k = c + 2;
        const uint32_t nb = t.numBuckets[c];
        for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
            uint32_t slab = t.bucketBase[c] + b;
            unsigned long long items = 0, slabs = 0;
            for (uint32_t steps = 0; steps < kMaxChain; ++steps) {
                const uint32_t* h = slab_ptr(d, slab);
                for (uint32_t s = 0; s < kSlots; ++s) {
                    const uint32_t tag = header_tag(h, s);
                    if (tag == 0 || tag == kTagBusy)
                        continue;
                    ++items;
                    if (outHandles) {
                        const unsigned long long pos = atomicAdd(&counters[2], 1ull);
                        if (pos < capacity) {
                            const uint32_t item = slot_handle(h[6], s, k);
                            outHandles[pos] = item;
                            const uint32_t* ip = handle_ptr(d, item);
                            for (uint32_t j = 0; j < kItemStride; ++j)
                                outWords[pos * kItemStride + j] = j < k ? ip[j] : 0u;
                        }
                    }
                }
                const uint32_t next = h[7];
                if (next == kEnd)
                    break;
                if (!slab_ok(d, next)) {
                    set_status(d.ctl, SVDAG_ERR_CORRUPT);
                    break;
                }
                ++slabs;
                slab = next;
            }
            atomicAdd(&counters[0], items);
            atomicAdd(&counters[1], slabs);
        }
    }
}

template <int OP>
svdag_status launch_table_op(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    unsigned long long totalWords, const uint32_t* reps, uint32_t* out, uint32_t lanes, cudaStream_t s)
{
    svdag_ctx* ctx = t->ctx;
    if (!lanes)
        lanes = ctx->probeLanes;
    const int threads = 256;
    const unsigned long long workThreads = (unsigned long long)n * lanes;
    const int grid = grid_for(ctx, workThreads, threads, 8);
    const DevDag d = ctx->dag();
    switch (lanes) {
    case 1:
        k_table_op<1, OP><<<grid, threads, 0, s>>>(d, t->dev, keys, offsets, n, totalWords, reps, out);
        break;
    case 2:
        k_table_op<2, OP><<<grid, threads, 0, s>>>(d, t->dev, keys, offsets, n, totalWords, reps, out);
        break;
    case 4:
        k_table_op<4, OP><<<grid, threads, 0, s>>>(d, t->dev, keys, offsets, n, totalWords, reps, out);
        break;
    case 8:
        k_table_op<8, OP><<<grid, threads, 0, s>>>(d, t->dev, keys, offsets, n, totalWords, reps, out);
        break;
    case 16:
        k_table_op<16, OP><<<grid, threads, 0, s>>>(d, t->dev, keys, offsets, n, totalWords, reps, out);
        break;
    case 32:
        k_table_op<32, OP><<<grid, threads, 0, s>>>(d, t->dev, keys, offsets, n, totalWords, reps, out);
        break;
    default:
        return SVDAG_ERR_INVALID;
    }
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

bool valid_table(const svdag_table* t) { return t && t->ctx && t->ready; }

} // namespace

extern "C" {

svdag_status svdag_level_table(svdag_ctx* ctx, uint32_t level, svdag_table** out)
{
    if (!ctx || !out || level > ctx->cfg.levels - 2)
        return SVDAG_ERR_INVALID;
    SVDAG_TRY(ensure_level_tables(ctx, nullptr));
    SVDAG_CUDA(cudaStreamSynchronize(nullptr));
    *out = &ctx->levelTables[level];
    return SVDAG_OK;
}

svdag_status svdag_table_create(svdag_ctx* ctx, uint32_t kind, const uint32_t* bucketsPerSize, svdag_table** out)
{
    if (!ctx || !out || !bucketsPerSize || kind > SVDAG_KIND_LEAF)
        return SVDAG_ERR_INVALID;
    auto* t = new svdag_table();
    const svdag_status st = alloc_table(ctx, t, kind, bucketsPerSize, nullptr);
    if (st != SVDAG_OK) {
        delete t;
        return st;
    }
    ctx->standalone.push_back(t);
    *out = t;
    return SVDAG_OK;
}

// The bucket arrays stay in the item region until the context is destroyed (the region is a bump
// allocator); the descriptor is released.
svdag_status svdag_table_destroy(svdag_table* t)
{
    if (!t || !t->ctx)
        return SVDAG_ERR_INVALID;
    if (t->level >= 0)
        return SVDAG_OK; // level tables belong to the context
    auto& v = t->ctx->standalone;
    v.erase(std::remove(v.begin(), v.end(), t), v.end());
    delete t;
    return SVDAG_OK;
}

svdag_status svdag_table_add(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    uint64_t totalWords, uint32_t* handles, uint32_t lanes, void* stream)
{
    if (!valid_table(t) || (n && (!keys || !offsets || !handles)))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    return launch_table_op<OP_ADD>(t, keys, offsets, n, totalWords, nullptr, handles, lanes, as_stream(stream));
}

svdag_status svdag_table_find(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    uint64_t totalWords, uint32_t* handles, uint32_t lanes, void* stream)
{
    if (!valid_table(t) || (n && (!keys || !offsets || !handles)))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    return launch_table_op<OP_FIND>(t, keys, offsets, n, totalWords, nullptr, handles, lanes, as_stream(stream));
}

svdag_status svdag_table_find_or_add(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    uint64_t totalWords, uint32_t* handles, uint32_t lanes, void* stream)
{
    if (!valid_table(t) || (n && (!keys || !offsets || !handles)))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    svdag_ctx* ctx = t->ctx;
    cudaStream_t s = as_stream(stream);
    uint32_t cap = 1;
    while (cap < 2ull * n)
        cap <<= 1;
    const unsigned long long need = (unsigned long long)cap * 8 + (unsigned long long)n * 4;
    if (need > ctx->scratchBytes)
        return SVDAG_ERR_OOM;
    auto* table = reinterpret_cast<unsigned long long*>(ctx->scratch);
    auto* reps = reinterpret_cast<uint32_t*>(ctx->scratch + (size_t)cap * 8);
    ctx->scratchHighWater = std::max(ctx->scratchHighWater, need);
    SVDAG_CUDA(cudaMemsetAsync(table, 0, (size_t)cap * 8, s));
    k_batch_dedup<<<grid_for(ctx, n, 256), 256, 0, s>>>(keys, offsets, n, totalWords, t->dev.kind, table, cap - 1, reps, ctx->ctl);
    SVDAG_CUDA(cudaGetLastError());
    SVDAG_TRY(launch_table_op<OP_FIND_OR_INSERT>(t, keys, offsets, n, totalWords, reps, handles, lanes, s));
    k_gather<<<grid_for(ctx, n, 256), 256, 0, s>>>(reps, n, handles);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

} // extern "C"

// ---------------------------------------------------------------- allocation-free find-or-add
// Some callers cannot allocate GPU memory while they run: code recording a CUDA graph, real-time
// loops that must not hit the driver's allocator, or hosts whose memory is owned by another runtime.
// This entry point does the same work as svdag_table_find_or_add, but its dedup scratch is a fixed
// array compiled into the library instead of the context's arena, so a call allocates nothing.
// The array lives in every GPU that loads the library until the process exits.

constexpr uint32_t kStaticMaxKeys = 65536; // largest batch the fixed scratch holds
constexpr uint32_t kStaticTableEntries = 2 * kStaticMaxKeys; // open-addressing entries (power of two)
constexpr size_t kStaticScratchBytes = kStaticTableEntries * sizeof(unsigned long long) + kStaticMaxKeys * sizeof(uint32_t);

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {
std::mutex g_static_mutex;
void* g_static_ptr[64] = {}; // device address of g_static_scratch, per device ordinal

// The symbol's device address, looked up once per device with that device current.
svdag_status static_scratch(int device, unsigned char** out)
{
    if (device < 0 || device >= 64)
        return SVDAG_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[device]) {
        int prev = 0;
        SVDAG_CUDA(cudaGetDevice(&prev));
        if (prev != device)
            SVDAG_CUDA(cudaSetDevice(device));
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (prev != device)
            cudaSetDevice(prev);
        if (e != cudaSuccess)
            return cuda_status(e);
        g_static_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_static_ptr[device]);
    return SVDAG_OK;
}
} // namespace

extern "C" svdag_status svdag_table_find_or_add_static(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    uint64_t totalWords, uint32_t* handles, uint32_t lanes, void* stream)
{
    if (!valid_table(t) || (n && (!keys || !offsets || !handles)))
        return SVDAG_ERR_INVALID;
    if (n > kStaticMaxKeys) {
        std::fprintf(stderr, "svdag_table_find_or_add_static: %u keys exceed the fixed scratch limit of %u keys\n", n, kStaticMaxKeys);
        return SVDAG_ERR_INVALID;
    }
    if (!n)
        return SVDAG_OK;
    svdag_ctx* ctx = t->ctx;
    // The kernels run on the calling thread's current device; the fixed array's address is that of
    // the table's device, so the two must be the same.
    int current = -1;
    SVDAG_CUDA(cudaGetDevice(&current));
    if (current != ctx->device)
        return SVDAG_ERR_INVALID;
    unsigned char* base = nullptr;
    SVDAG_TRY(static_scratch(ctx->device, &base));
    cudaStream_t s = as_stream(stream);
    uint32_t cap = 2;
    while (cap < 2ull * n)
        cap <<= 1; // <= kStaticTableEntries because n <= kStaticMaxKeys
    auto* table = reinterpret_cast<unsigned long long*>(base);
    auto* reps = reinterpret_cast<uint32_t*>(base + kStaticTableEntries * sizeof(unsigned long long));
    // The array keeps the previous call's contents: the probe table must start empty.
    SVDAG_CUDA(cudaMemsetAsync(table, 0, (size_t)cap * sizeof(unsigned long long), s));
    k_batch_dedup<<<grid_for(ctx, n, 256), 256, 0, s>>>(keys, offsets, n, totalWords, t->dev.kind, table, cap - 1, reps, ctx->ctl);
    SVDAG_CUDA(cudaGetLastError());
    SVDAG_TRY(launch_table_op<OP_FIND_OR_INSERT>(t, keys, offsets, n, totalWords, reps, handles, lanes, s));
    k_gather<<<grid_for(ctx, n, 256), 256, 0, s>>>(reps, n, handles);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

extern "C" {

svdag_status svdag_table_read(svdag_table* t, const uint32_t* handles, uint32_t n, uint32_t* out, void* stream)
{
    if (!valid_table(t) || (n && (!handles || !out)))
        return SVDAG_ERR_INVALID;
    if (!n)
        return SVDAG_OK;
    k_table_read<<<grid_for(t->ctx, n, 256), 256, 0, as_stream(stream)>>>(t->ctx->dag(), t->dev.kind, handles, n, out);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

svdag_status svdag_table_get_stats(svdag_table* t, svdag_table_stats* out, void* stream)
{
    if (!valid_table(t) || !out)
        return SVDAG_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    unsigned long long* counters = nullptr;
    SVDAG_CUDA(cudaMallocAsync(&counters, 3 * sizeof(unsigned long long), s));
    SVDAG_CUDA(cudaMemsetAsync(counters, 0, 3 * sizeof(unsigned long long), s));
    k_table_walk<<<grid_for(t->ctx, 1u << 20, 256), 256, 0, s>>>(t->ctx->dag(), t->dev, counters, nullptr, nullptr, 0);
    unsigned long long h[3];
    SVDAG_CUDA(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaFreeAsync(counters, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    out->items = h[0];
    out->overflow_slabs = h[1];
    unsigned long long buckets = 0, bytes = 0;
    for (uint32_t c = 0; c < kNumClasses; ++c) {
        buckets += t->dev.numBuckets[c];
        bytes += (unsigned long long)t->dev.numBuckets[c] * (body_words(c + 2) + kHeaderWords) * 4;
    }
    // Overflow slabs are counted per class by the walk only in total; bytes use the mean class size.
    out->buckets = buckets;
    out->bytes = bytes;
    return SVDAG_OK;
}

svdag_status svdag_export_level(svdag_ctx* ctx, uint32_t level, uint32_t* outHandles, uint32_t* outWords, uint64_t capacity,
    uint64_t* outCount, void* stream)
{
    if (!ctx || level > ctx->cfg.levels - 2 || !outCount)
        return SVDAG_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    svdag_table& t = ctx->levelTables[level];
    if (!t.ready) {
        *outCount = 0;
        return SVDAG_OK;
    }
    unsigned long long* counters = nullptr;
    SVDAG_CUDA(cudaMallocAsync(&counters, 3 * sizeof(unsigned long long), s));
    SVDAG_CUDA(cudaMemsetAsync(counters, 0, 3 * sizeof(unsigned long long), s));
    uint32_t *dh = nullptr, *dw = nullptr;
    if (capacity && outHandles && outWords) {
        SVDAG_CUDA(cudaMallocAsync(&dh, capacity * 4, s));
        SVDAG_CUDA(cudaMallocAsync(&dw, capacity * 4 * kItemStride, s));
    }
    k_table_walk<<<grid_for(ctx, 1u << 20, 256), 256, 0, s>>>(ctx->dag(), t.dev, counters, dh, dw, dh ? capacity : 0);
    SVDAG_CUDA(cudaGetLastError());
    unsigned long long h[3];
    SVDAG_CUDA(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    *outCount = h[0];
    if (dh) {
        const unsigned long long n = std::min<unsigned long long>(h[0], capacity);
        SVDAG_CUDA(cudaMemcpyAsync(outHandles, dh, n * 4, cudaMemcpyDeviceToHost, s));
        SVDAG_CUDA(cudaMemcpyAsync(outWords, dw, n * 4 * kItemStride, cudaMemcpyDeviceToHost, s));
        SVDAG_CUDA(cudaFreeAsync(dh, s));
        SVDAG_CUDA(cudaFreeAsync(dw, s));
    }
    SVDAG_CUDA(cudaFreeAsync(counters, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    return SVDAG_OK;
}

} // extern "C"

namespace svdag {

svdag_status table_add_lanes(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n, unsigned long long totalWords,
    uint32_t* out, uint32_t lanes, cudaStream_t s)
{
    return n ? launch_table_op<OP_ADD>(t, keys, offsets, n, totalWords, nullptr, out, lanes, s) : SVDAG_OK;
}
svdag_status table_find_lanes(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n, unsigned long long totalWords,
    uint32_t* out, uint32_t lanes, cudaStream_t s)
{
    return n ? launch_table_op<OP_FIND>(t, keys, offsets, n, totalWords, nullptr, out, lanes, s) : SVDAG_OK;
}

} // namespace svdag

// ---------------------------------------------------------------- helpers of the scene builder

namespace {

// Items per size class of a table: one thread per bucket walks its chain.
__global__ void k_table_class_counts(DevDag d, DevTable t, unsigned long long* perClass)
{
    for (uint32_t c = 0; c < kNumClasses; ++c) {
        unsigned long long items = 0;
        for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.numBuckets[c]; b += gridDim.x * blockDim.x) {
            uint32_t slab = t.bucketBase[c] + b;
            for (uint32_t steps = 0; steps < kMaxChain; ++steps) {
                const uint32_t* h = slab_ptr(d, slab);
                for (uint32_t s = 0; s < kSlots; ++s) {
                    const uint32_t tag = header_tag(h, s);
                    items += (tag != 0 && tag != kTagBusy) ? 1u : 0u;
                }
                const uint32_t next = h[7];
                if (next == kEnd)
                    break;
                if (!slab_ok(d, next)) {
                    set_status(d.ctl, SVDAG_ERR_CORRUPT);
                    break;
                }
                slab = next;
            }
        }
        if (items)
            atomicAdd(&perClass[c], items);
    }
}

} // namespace

namespace svdag {

svdag_status find_or_insert_distinct(svdag_ctx* ctx, uint32_t level, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    unsigned long long totalWords, uint32_t* out, cudaStream_t s)
{
    if (!n)
        return SVDAG_OK;
    return launch_table_op<OP_FIND_OR_INSERT>(&ctx->levelTables[level], keys, offsets, n, totalWords, nullptr, out, 1, s);
}

svdag_status table_class_counts(svdag_ctx* ctx, const svdag_table& t, unsigned long long* perClass, unsigned long long* scratch, cudaStream_t s)
{
    SVDAG_CUDA(cudaMemsetAsync(scratch, 0, kNumClasses * sizeof(unsigned long long), s));
    k_table_class_counts<<<grid_for(ctx, 1u << 20, 256), 256, 0, s>>>(ctx->dag(), t.dev, scratch);
    SVDAG_CUDA(cudaGetLastError());
    SVDAG_CUDA(cudaMemcpyAsync(perClass, scratch, kNumClasses * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    return SVDAG_OK;
}

} // namespace svdag
