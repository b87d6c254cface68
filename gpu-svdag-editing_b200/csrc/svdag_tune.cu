// svdag_tune.cu - the autotuner of the batched form: table load factor and lanes per key from a key
// sample, the launch form of small edits from an edit sample, both measured with CUDA events.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "svdag_edit.cuh"
#include "svdag_host.hpp"

using namespace svdag;

namespace {

// Words of a self-describing key (node: header + children; leaf: two mask words + materials).
uint32_t key_words(uint32_t kind, const uint32_t* p, unsigned long long avail)
{
    if (avail < 1)
        return 0;
    if (kind == SVDAG_KIND_NODE)
        return 1u + (uint32_t)__builtin_popcount(p[0] & 0xFFu);
    if (avail < 2)
        return 0;
    return leaf_words(p[0], p[1]);
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer()
    {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer()
    {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

svdag_status tune_tables(svdag_ctx* ctx, const uint32_t* keys, const uint32_t* offsets, uint32_t n, unsigned long long totalWords,
    uint32_t kind, svdag_tuning& out, cudaStream_t s)
{
    // Size classes of the sample (host copy of the keys).
    std::vector<uint32_t> hk(totalWords), ho(n);
    SVDAG_CUDA(cudaMemcpyAsync(hk.data(), keys, totalWords * 4, cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaMemcpyAsync(ho.data(), offsets, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    unsigned long long perClass[kNumClasses] = {};
    for (uint32_t i = 0; i < n; ++i) {
        if (ho[i] >= totalWords)
            return SVDAG_ERR_INVALID;
        const uint32_t k = key_words(kind, hk.data() + ho[i], totalWords - ho[i]);
        if (k < 2 || k > 10)
            return SVDAG_ERR_INVALID;
        ++perClass[k - 2];
    }
    uint32_t* handles = nullptr;
    SVDAG_CUDA(cudaMallocAsync(&handles, (size_t)n * 4, s));
    unsigned long long tops[2];
    SVDAG_CUDA(cudaMemcpyAsync(tops, &ctx->ctl->itemTop, sizeof(tops), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    Timer t0, t1;
    double best = 1e300;
    svdag_status st = SVDAG_OK;
    // Untimed warm-up of each lane count's kernels on a small scratch table: a kernel's first launch
    // also loads it (lazy module loading), which would count against the first load factor timed.
    for (uint32_t lanes : { 1u, 2u, 4u, 8u }) {
        uint32_t buckets[kNumClasses];
        for (auto& b : buckets)
            b = 1;
        svdag_table t;
        st = alloc_table(ctx, &t, kind, buckets, s);
        if (st != SVDAG_OK)
            break;
        const uint32_t wn = std::min(n, 256u);
        st = table_add_lanes(&t, keys, offsets, wn, totalWords, handles, lanes, s);
        if (st == SVDAG_OK)
            st = table_find_lanes(&t, keys, offsets, wn, totalWords, handles, lanes, s);
        SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->itemTop, tops, sizeof(tops), cudaMemcpyHostToDevice, s));
        SVDAG_CUDA(cudaStreamSynchronize(s));
        if (st != SVDAG_OK)
            break;
    }
    for (uint32_t lf : { 8u, 12u, 16u, 24u, 32u }) {
        if (st != SVDAG_OK)
            break;
        for (uint32_t lanes : { 1u, 2u, 4u, 8u }) {
            uint32_t buckets[kNumClasses];
            for (uint32_t c = 0; c < kNumClasses; ++c)
                buckets[c] = (uint32_t)std::max<unsigned long long>(1, perClass[c] / lf + 1);
            svdag_table t;
            st = alloc_table(ctx, &t, kind, buckets, s);
            if (st != SVDAG_OK)
                break;
            cudaEventRecord(t0.a, s);
            st = table_add_lanes(&t, keys, offsets, n, totalWords, handles, lanes, s);
            if (st == SVDAG_OK)
                st = table_find_lanes(&t, keys, offsets, n, totalWords, handles, lanes, s);
            cudaEventRecord(t0.b, s);
            if (st != SVDAG_OK)
                break;
            // Give the scratch table's space back (nothing else allocates during the call).
            SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->itemTop, tops, sizeof(tops), cudaMemcpyHostToDevice, s));
            SVDAG_CUDA(cudaStreamSynchronize(s));
            float ms = 0;
            cudaEventElapsedTime(&ms, t0.a, t0.b);
            ++out.trials;
            if (ms < best) {
                best = ms;
                out.load_factor = lf;
                out.probe_lanes = lanes;
            }
        }
        if (st != SVDAG_OK)
            break;
    }
    cudaFreeAsync(handles, s);
    SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->itemTop, tops, sizeof(tops), cudaMemcpyHostToDevice, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    SVDAG_TRY(st);
    SVDAG_TRY(read_status(ctx, s));
    out.table_ns_per_key = best * 1e6 / n;
    ctx->loadFactor = out.load_factor;
    ctx->probeLanes = out.probe_lanes;
    return SVDAG_OK;
}

svdag_status tune_edits(svdag_ctx* ctx, const svdag_edit* edits, uint32_t n, svdag_tuning& out, cudaStream_t s)
{
    SVDAG_TRY(ensure_level_tables(ctx, s));
    // Size buckets of the estimated SVO leaves: [0, 1K), [1K, 4K), [4K, 16K), [16K, 64K), [64K, inf).
    constexpr int kBuckets = 5;
    const double upper[kBuckets] = { 1024, 4096, 16384, 65536, 1e300 };
    double sum[kBuckets][2] = {}, cnt[kBuckets][2] = {};
    std::vector<Timer> timers(2 * (size_t)n);
    std::vector<int> bucketOf(2 * (size_t)n, -1), formOf(2 * (size_t)n, 0);
    // The first launch of a tool in a form may capture and instantiate its graph or load the kernel:
    // it is applied like the others but left out of the statistics (bucket -1).
    bool seen[2][SVDAG_NUM_TOOLS] = {};
    size_t used = 0;
    for (uint32_t i = 0; i < n; ++i) {
        DevEditor eds[2];
        const int m = expand_edit(ctx, edits[i], eds);
        for (int j = 0; j < m; ++j) {
            const int form = (int)((i + j) & 1u); // 0 graph, 1 persistent
            const double est = estimate_leaves(eds[j]);
            int b = 0;
            while (b < kBuckets - 1 && est >= upper[b])
                ++b;
            Timer& t = timers[used];
            cudaEventRecord(t.a, s);
            SVDAG_TRY(form ? launch_single_fused(ctx, eds[j], s) : launch_pipeline(ctx, eds[j], s, nullptr, true));
            cudaEventRecord(t.b, s);
            const uint32_t tool = eds[j].tool < SVDAG_NUM_TOOLS ? eds[j].tool : 0u;
            bucketOf[used] = seen[form][tool] ? b : -1;
            seen[form][tool] = true;
            formOf[used] = form;
            ++used;
        }
    }
    SVDAG_CUDA(cudaStreamSynchronize(s));
    for (size_t k = 0; k < used; ++k) {
        ++out.trials;
        if (bucketOf[k] < 0)
            continue;
        float ms = 0;
        cudaEventElapsedTime(&ms, timers[k].a, timers[k].b);
        sum[bucketOf[k]][formOf[k]] += ms * 1e3;
        cnt[bucketOf[k]][formOf[k]] += 1;
    }
    // Persistent kernel for the buckets, from the smallest up, where it is faster.
    double threshold = 0;
    for (int b = 0; b < kBuckets - 1; ++b) {
        if (!cnt[b][0] || !cnt[b][1])
            break;
        if (sum[b][1] / cnt[b][1] < sum[b][0] / cnt[b][0])
            threshold = upper[b];
        else
            break;
    }
    const double g = cnt[0][0] + cnt[1][0], p = cnt[0][1] + cnt[1][1];
    out.graph_us_small = g ? (sum[0][0] + sum[1][0]) / g : 0;
    out.persistent_us_small = p ? (sum[0][1] + sum[1][1]) / p : 0;
    out.persistent_leaves = (uint32_t)threshold;
    ctx->persistentLeaves = threshold;
    return read_status(ctx, s);
}

} // namespace

extern "C" {

svdag_status svdag_autotune(svdag_ctx* ctx, const svdag_edit* edits, uint32_t nEdits, const uint32_t* keys, const uint32_t* offsets,
    uint32_t nKeys, uint64_t totalWords, uint32_t kind, svdag_tuning* out, void* stream)
{
    if (!ctx || !out || (nEdits && !edits) || (nKeys && (!keys || !offsets || !totalWords)) || kind > SVDAG_KIND_LEAF)
        return SVDAG_ERR_INVALID;
    for (uint32_t i = 0; i < nEdits; ++i)
        if (!valid_edit(&edits[i]))
            return SVDAG_ERR_INVALID;
    svdag_tuning t {};
    SVDAG_TRY(svdag_get_tuning(ctx, &t));
    t.trials = 0;
    cudaStream_t s = as_stream(stream);
    if (nKeys)
        SVDAG_TRY(tune_tables(ctx, keys, offsets, nKeys, totalWords, kind, t, s));
    if (nEdits)
        SVDAG_TRY(tune_edits(ctx, edits, nEdits, t, s));
    *out = t;
    return SVDAG_OK;
}

svdag_status svdag_get_tuning(svdag_ctx* ctx, svdag_tuning* out)
{
    if (!ctx || !out)
        return SVDAG_ERR_INVALID;
    *out = svdag_tuning {};
    out->probe_lanes = ctx->probeLanes;
    out->load_factor = ctx->loadFactor;
    out->persistent_leaves = (uint32_t)ctx->persistentLeaves;
    return SVDAG_OK;
}

svdag_status svdag_set_tuning(svdag_ctx* ctx, const svdag_tuning* t)
{
    if (!ctx || !t || !t->load_factor)
        return SVDAG_ERR_INVALID;
    const uint32_t l = t->probe_lanes;
    if (l != 1 && l != 2 && l != 4 && l != 8 && l != 16 && l != 32)
        return SVDAG_ERR_INVALID;
    ctx->probeLanes = l;
    ctx->loadFactor = t->load_factor;
    ctx->persistentLeaves = t->persistent_leaves;
    return SVDAG_OK;
}

} // extern "C"
