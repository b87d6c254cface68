// svdag_io.cu - DAG import and export.
//
// Items of a DAG travel as per-level item lists ("item snapshots"): level l holds its items packed
// one after another (nodes: header + one word per child; leaves: 2 mask words + packed 4-bit
// materials), and a node's child words are ordinals into the item list of level l + 1. Item 0 of
// level 0 is the root. Snapshots are the portable form; the reference's own file
// (MyGPUHashDAG::writeTo/readFrom, my_gpu_hash_dag.cu:158-177, a dump of its raw hash tables)
// converts to and from them in svdag_v3.cu.
//
// The reference's BasicDAG geometry files (BasicDAGFactory::load_dag_from_file, basic_dag.cpp:
// 108-122) convert into a snapshot as MyGPUHashDAGFactory's create_dag_cpu converts them without
// colour import (my_gpu_hash_dag_factory.cpp:316-418): every voxel gets one material, and a node
// whose eight children are fully filled with one material carries the fully-filled header bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "svdag_device.cuh"
#include "svdag_snapshot.h"
#include "svdag_host.hpp"

using namespace svdag;

namespace {

uint32_t host_popc(uint32_t v) { return (uint32_t)__builtin_popcount(v); }

using snapshot::item_words;
using snapshot::split_level;

struct KeyRef {
    const std::vector<uint32_t>* words;
    uint64_t off;
    uint32_t n;
};
struct KeyHash {
    size_t operator()(const KeyRef& k) const
    {
        uint64_t h = 0x9E3779B97F4A7C15ull ^ k.n;
        for (uint32_t i = 0; i < k.n; ++i)
            h = (h ^ (*k.words)[k.off + i]) * 0xBF58476D1CE4E5B9ull;
        return (size_t)(h ^ (h >> 31));
    }
};
struct KeyEq {
    bool operator()(const KeyRef& a, const KeyRef& b) const
    {
        return a.n == b.n && std::equal(a.words->begin() + a.off, a.words->begin() + a.off + a.n, b.words->begin() + b.off);
    }
};

// Inserts the distinct keys of one level (packed in `keys`, offsets in `offs`) through the scratch
// arena in chunks; handles[i] receives the handle of key i.
svdag_status insert_level(svdag_ctx* ctx, uint32_t level, const std::vector<uint32_t>& keys, const std::vector<uint64_t>& offs,
    std::vector<uint32_t>& handles, cudaStream_t s)
{
    handles.assign(offs.size(), kNone);
    const unsigned long long budget = ctx->scratchBytes & ~255ull;
    size_t i = 0;
    while (i < offs.size()) {
        // as many keys as fit: words + offset + handle per key
        size_t j = i;
        unsigned long long bytes = 0;
        while (j < offs.size()) {
            const uint64_t end = j + 1 < offs.size() ? offs[j + 1] : keys.size();
            const unsigned long long add = (end - offs[j]) * 4ull + 8ull;
            if (bytes + add + 1024 > budget || j - i >= 0x7FFFFFFFull)
                break;
            bytes += add;
            ++j;
        }
        if (j == i)
            return SVDAG_ERR_OOM;
        const uint64_t w0 = offs[i], w1 = j < offs.size() ? offs[j] : keys.size();
        std::vector<uint32_t> relOffs(j - i);
        for (size_t k = i; k < j; ++k)
            relOffs[k - i] = (uint32_t)(offs[k] - w0);
        uint32_t* dw = reinterpret_cast<uint32_t*>(ctx->scratch);
        uint32_t* doff = reinterpret_cast<uint32_t*>(ctx->scratch + align256((w1 - w0) * 4));
        uint32_t* dout = reinterpret_cast<uint32_t*>(ctx->scratch + align256((w1 - w0) * 4) + align256(relOffs.size() * 4));
        ctx->scratchHighWater = std::max<unsigned long long>(ctx->scratchHighWater,
            align256((w1 - w0) * 4) + 2 * align256(relOffs.size() * 4));
        SVDAG_CUDA(cudaMemcpyAsync(dw, keys.data() + w0, (w1 - w0) * 4, cudaMemcpyHostToDevice, s));
        SVDAG_CUDA(cudaMemcpyAsync(doff, relOffs.data(), relOffs.size() * 4, cudaMemcpyHostToDevice, s));
        SVDAG_TRY(find_or_insert_distinct(ctx, level, dw, doff, (uint32_t)relOffs.size(), w1 - w0, dout, s));
        SVDAG_CUDA(cudaMemcpyAsync(handles.data() + i, dout, relOffs.size() * 4, cudaMemcpyDeviceToHost, s));
        SVDAG_CUDA(cudaStreamSynchronize(s));
        i = j;
    }
    return read_status(ctx, s);
}

// Replaces the context's DAG by a snapshot (already validated), bottom-up: the items of a level are
// deduplicated on the host, the level table is sized for them exactly (as a scene build sizes it),
// and its parents' child ordinals are rewritten to the handles the table returned.
svdag_status load_snapshot(svdag_ctx* ctx, const uint32_t* words, const uint64_t* levelWords, const uint64_t* levelItems,
    const std::vector<std::vector<uint64_t>>& offsets, cudaStream_t s)
{
    const uint32_t LL = ctx->cfg.levels - 2;
    SVDAG_TRY(reset_dag(ctx, s));
    std::vector<uint64_t> base(LL + 2, 0);
    for (uint32_t l = 0; l <= LL; ++l)
        base[l + 1] = base[l] + levelWords[l];
    std::vector<uint32_t> below; // handle of every item of the level below, by ordinal
    for (int level = (int)LL; level >= 0; --level) {
        const bool leaf = level == (int)LL;
        const uint32_t* w = words + base[level];
        const auto& offs = offsets[level];
        // rewritten keys, distinct ones packed; which[i] = distinct index of item i
        std::vector<uint32_t> keys;
        keys.reserve(levelWords[level]);
        std::vector<uint64_t> kOffs;
        std::vector<uint32_t> which(offs.size());
        std::unordered_map<KeyRef, uint32_t, KeyHash, KeyEq> index;
        index.reserve(offs.size() * 2);
        unsigned long long perClass[kNumClasses] = {};
        for (size_t i = 0; i < offs.size(); ++i) {
            const uint32_t n = item_words(leaf, w + offs[i], levelWords[level] - offs[i]);
            const uint64_t at = keys.size();
            keys.push_back(w[offs[i]]);
            for (uint32_t k = 1; k < n; ++k)
                keys.push_back(leaf ? w[offs[i] + k] : below[w[offs[i] + k]]);
            const KeyRef ref { &keys, at, n };
            auto it = index.find(ref);
            if (it != index.end()) {
                keys.resize(at);
                which[i] = it->second;
                continue;
            }
            which[i] = (uint32_t)kOffs.size();
            index.emplace(ref, which[i]);
            kOffs.push_back(at);
            perClass[n - 2]++;
        }
        uint32_t buckets[kNumClasses];
        for (uint32_t c = 0; c < kNumClasses; ++c)
            buckets[c] = (uint32_t)std::max<unsigned long long>(1, (perClass[c] + SVDAG_NUM_MATERIALS + ctx->loadFactor - 1) / ctx->loadFactor);
        svdag_table& t = ctx->levelTables[level];
        SVDAG_TRY(alloc_table(ctx, &t, leaf ? SVDAG_KIND_LEAF : SVDAG_KIND_NODE, buckets, s, true));
        t.level = (uint32_t)level;
        SVDAG_TRY(upload_tables(ctx, s));
        SVDAG_TRY(insert_canonical(ctx, (uint32_t)level, s));
        std::vector<uint32_t> distinct;
        SVDAG_TRY(insert_level(ctx, (uint32_t)level, keys, kOffs, distinct, s));
        below.resize(offs.size());
        for (size_t i = 0; i < offs.size(); ++i)
            below[i] = distinct[which[i]];
    }
    const uint32_t root = levelItems[0] ? below[0] : kNone;
    SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->root, &root, sizeof(root), cudaMemcpyHostToDevice, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    return read_status(ctx, s);
}

// BasicDAG -> snapshot conversion state: one item list per level, memoised by BasicDAG index.
struct BasicConverter {
    const uint32_t* data;
    uint64_t n;
    uint32_t levels, material;
    std::vector<std::vector<uint32_t>> words;
    std::vector<uint64_t> count;
    std::vector<std::unordered_map<uint32_t, std::pair<uint32_t, uint32_t>>> memo; // index -> (ordinal, fill)
    bool bad = false;

    // Returns (ordinal, fill material or kNone) of the subtree at (level, index).
    std::pair<uint32_t, uint32_t> visit(uint32_t level, uint32_t idx)
    {
        auto m = memo[level].find(idx);
        if (m != memo[level].end())
            return m->second;
        const uint32_t LL = levels - 2;
        std::pair<uint32_t, uint32_t> res { 0, kNone };
        if (level == LL) { // a 64-bit leaf mask: voxel i is bit i (low word first)
            if ((uint64_t)idx + 2 > n || (data[idx] == 0 && data[idx + 1] == 0)) {
                bad = true;
                return res;
            }
            const uint32_t lo = data[idx], hi = data[idx + 1];
            const uint32_t v = host_popc(lo) + host_popc(hi);
            auto& w = words[level];
            w.push_back(lo);
            w.push_back(hi);
            for (uint32_t nib = 0; nib < v; nib += 8) {
                const uint32_t k = std::min<uint32_t>(8, v - nib);
                w.push_back(k == 8 ? material * 0x11111111u : (material * 0x11111111u) & ((1u << (4 * k)) - 1u));
            }
            if (lo == 0xFFFFFFFFu && hi == 0xFFFFFFFFu)
                res.second = material;
        } else {
            if ((uint64_t)idx >= n) {
                bad = true;
                return res;
            }
            const uint32_t mask = data[idx] & 0xFFu;
            const uint32_t nc = host_popc(mask);
            if (!mask || (uint64_t)idx + 1 + nc > n) {
                bad = true;
                return res;
            }
            uint32_t kids[8];
            uint32_t fill = kNone;
            bool uniform = mask == 0xFFu;
            for (uint32_t c = 0, j = 0; c < 8; ++c) {
                if (!(mask >> c & 1u))
                    continue;
                const auto ch = visit(level + 1, data[idx + 1 + j]);
                if (bad)
                    return res;
                kids[j++] = ch.first;
                if (ch.second == kNone || (fill != kNone && ch.second != fill))
                    uniform = false;
                fill = ch.second;
            }
            auto& w = words[level];
            w.push_back(uniform ? (0xFFu | (1u << 8) | (fill << 9)) : mask);
            w.insert(w.end(), kids, kids + nc);
            if (uniform)
                res.second = fill;
        }
        res.first = (uint32_t)count[level]++;
        memo[level].emplace(idx, res);
        return res;
    }
};

} // namespace

extern "C" {

svdag_status svdag_basic_dag_to_items(const uint32_t* data, uint64_t nWords, uint32_t levels, uint32_t material, uint32_t* out,
    uint64_t capacity, uint64_t* levelWords, uint64_t* levelItems, uint64_t* totalWords)
{
    if (!data || !nWords || !levelWords || !levelItems || !totalWords || levels < SVDAG_MIN_LEVELS || levels > SVDAG_MAX_LEVELS
        || material >= SVDAG_NUM_MATERIALS || (capacity && !out))
        return SVDAG_ERR_INVALID;
    BasicConverter cv { data, nWords, levels, material, {}, {}, {} };
    cv.words.resize(levels - 1);
    cv.count.assign(levels - 1, 0);
    cv.memo.resize(levels - 1);
    cv.visit(0, 0); // the root is at index 0 (BasicDAG::get_first_node_index)
    if (cv.bad)
        return SVDAG_ERR_CORRUPT;
    uint64_t total = 0;
    for (uint32_t l = 0; l + 1 < levels; ++l) {
        levelWords[l] = cv.words[l].size();
        levelItems[l] = cv.count[l];
        if (out && total + cv.words[l].size() <= capacity)
            std::memcpy(out + total, cv.words[l].data(), cv.words[l].size() * 4);
        total += cv.words[l].size();
    }
    *totalWords = total;
    return total > capacity ? SVDAG_ERR_OOM : SVDAG_OK;
}

svdag_status svdag_load_items(svdag_ctx* ctx, const uint32_t* words, const uint64_t* levelWords, const uint64_t* levelItems, void* stream)
{
    if (!ctx || !levelWords || !levelItems)
        return SVDAG_ERR_INVALID;
    const uint32_t LL = ctx->cfg.levels - 2;
    uint64_t total = 0;
    for (uint32_t l = 0; l <= LL; ++l)
        total += levelWords[l];
    if (total && !words)
        return SVDAG_ERR_INVALID;
    // empty DAG: every level empty; otherwise one root and every level non-empty
    const bool empty = levelItems[0] == 0;
    if ((empty && total != 0) || (!empty && levelItems[0] != 1))
        return SVDAG_ERR_INVALID;
    std::vector<std::vector<uint64_t>> offsets(LL + 1);
    uint64_t at = 0;
    for (uint32_t l = 0; l <= LL; ++l) {
        const uint64_t below = l < LL ? levelItems[l + 1] : 0;
        if (!split_level(l == LL, words + at, levelWords[l], levelItems[l], below, offsets[l]))
            return SVDAG_ERR_INVALID;
        if (levelItems[l] > 0xFFFFFFF0ull)
            return SVDAG_ERR_INVALID;
        at += levelWords[l];
    }
    cudaStream_t s = as_stream(stream);
    SVDAG_CUDA(cudaSetDevice(ctx->device));
    if (empty) {
        SVDAG_TRY(reset_dag(ctx, s));
        return ensure_level_tables(ctx, s);
    }
    return load_snapshot(ctx, words, levelWords, levelItems, offsets, s);
}

svdag_status svdag_save_items(svdag_ctx* ctx, uint32_t* out, uint64_t capacity, uint64_t* levelWords, uint64_t* levelItems,
    uint64_t* totalWords, void* stream)
{
    if (!ctx || !levelWords || !levelItems || !totalWords || (capacity && !out))
        return SVDAG_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    SVDAG_CUDA(cudaSetDevice(ctx->device));
    SVDAG_TRY(ensure_level_tables(ctx, s));
    const uint32_t LL = ctx->cfg.levels - 2;
    uint32_t root = kNone;
    SVDAG_CUDA(cudaMemcpyAsync(&root, &ctx->ctl->root, sizeof(root), cudaMemcpyDeviceToHost, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    for (uint32_t l = 0; l <= LL; ++l)
        levelWords[l] = levelItems[l] = 0;
    *totalWords = 0;
    if (root == kNone)
        return SVDAG_OK;
    // breadth-first over the reachable items, one level at a time; a level's items are its
    // frontier's distinct handles in ascending order
    std::vector<uint32_t> frontier { root };
    uint64_t total = 0;
    const size_t perHandle = (ctx->scratchBytes / 4) / (1 + kItemStride);
    const size_t chunk = perHandle > 128 ? perHandle - 128 : 1;
    std::vector<uint32_t> itemWords;
    for (uint32_t l = 0; l <= LL; ++l) {
        const bool leaf = l == LL;
        itemWords.resize(frontier.size() * kItemStride);
        for (size_t i = 0; i < frontier.size(); i += chunk) {
            const size_t m = std::min(chunk, frontier.size() - i);
            uint32_t* dh = reinterpret_cast<uint32_t*>(ctx->scratch);
            uint32_t* dw = reinterpret_cast<uint32_t*>(ctx->scratch + align256(m * 4));
            SVDAG_CUDA(cudaMemcpyAsync(dh, frontier.data() + i, m * 4, cudaMemcpyHostToDevice, s));
            SVDAG_TRY(svdag_table_read(&ctx->levelTables[l], dh, (uint32_t)m, dw, s));
            SVDAG_CUDA(cudaMemcpyAsync(itemWords.data() + i * kItemStride, dw, m * kItemStride * 4, cudaMemcpyDeviceToHost, s));
            SVDAG_CUDA(cudaStreamSynchronize(s));
        }
        std::vector<uint32_t> next;
        if (!leaf) {
            for (size_t i = 0; i < frontier.size(); ++i) {
                const uint32_t* w = itemWords.data() + i * kItemStride;
                const uint32_t n = node_words(w[0]);
                next.insert(next.end(), w + 1, w + n);
            }
            std::sort(next.begin(), next.end());
            next.erase(std::unique(next.begin(), next.end()), next.end());
        }
        uint64_t lw = 0;
        for (size_t i = 0; i < frontier.size(); ++i) {
            const uint32_t* w = itemWords.data() + i * kItemStride;
            const uint32_t n = leaf ? leaf_words(w[0], w[1]) : node_words(w[0]);
            if (n < 2 || n > kItemStride)
                return SVDAG_ERR_CORRUPT;
            for (uint32_t k = 0; k < n; ++k) {
                uint32_t v = w[k];
                if (!leaf && k > 0)
                    v = (uint32_t)(std::lower_bound(next.begin(), next.end(), v) - next.begin());
                if (out && total + lw < capacity)
                    out[total + lw] = v;
                ++lw;
            }
        }
        levelWords[l] = lw;
        levelItems[l] = frontier.size();
        total += lw;
        frontier.swap(next);
    }
    *totalWords = total;
    SVDAG_TRY(read_status(ctx, s));
    return total > capacity ? SVDAG_ERR_OOM : SVDAG_OK;
}

} // extern "C"
