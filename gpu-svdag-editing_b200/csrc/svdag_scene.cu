// svdag_scene.cu - procedural scene construction (the GPU replacement of the factory's create_dag_cpu +
// setLoadFactor, my_gpu_hash_dag_factory.cpp:317-500, my_gpu_hash_dag.cu:139-155).
//
// Small scenes are built in one pass (build_scene_untiled). Large ones are cut at a tile level T:
// the host classifies the nodes above T, every node of level T that needs subdividing becomes a
// tile built on the GPU as a builder edit of its subtree, and the host assembles the few nodes above
// the tiles. Level tables must exist before the tiles insert into them, so the tiled build runs
// twice: a counting pass into provisional tables gives the number of distinct items per level and
// size class, and the final pass builds into tables sized exactly from those counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "svdag_edit.cuh"
#include "svdag_host.hpp"

namespace svdag {

namespace {

uint64_t splitmix64(uint64_t& state)
{
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct HostScene {
    SceneParams p {}; // host pointers
    std::vector<Structure> structures;
    std::vector<uint32_t> cellStart, cellList;
};

// Structures on the surface and their xz cell lists (the generator is specified with
// svdag_terrain_params).
void make_scene(uint32_t levels, const svdag_terrain_params& t, HostScene& hs)
{
    SceneParams& p = hs.p;
    p = SceneParams {};
    p.terrain = t;
    p.levels = levels;
    p.baseLog2 = levels - 2;
    p.numStructures = t.num_structures;
    p.cellLog2 = std::max<uint32_t>(levels > 8 ? levels - 8 : 0, 5);
    p.cellLog2 = std::min(p.cellLog2, levels);
    p.cellsPerAxis = 1u << (levels - p.cellLog2);
    const int64_t G = int64_t(1) << levels;
    uint64_t rng = t.structure_seed;
    hs.structures.resize(t.num_structures);
    int64_t ylo = INT64_MAX, yhi = INT64_MIN;
    for (uint32_t i = 0; i < t.num_structures; ++i) {
        const uint32_t x = (uint32_t)(splitmix64(rng) % (uint64_t)G);
        const uint32_t z = (uint32_t)(splitmix64(rng) % (uint64_t)G);
        const uint32_t kind = (uint32_t)(splitmix64(rng) & 1u);
        const uint32_t material = (uint32_t)(splitmix64(rng) % 16u);
        const uint64_t size = splitmix64(rng);
        const int32_t h = (int32_t)terrain_height(p, x, z);
        Structure s {};
        s.kind = kind;
        s.material = material;
        const int32_t c[3] = { (int32_t)x, h, (int32_t)z };
        if (kind == 0) {
            const int32_t side = 16 + (int32_t)(size % 497u);
            for (int a = 0; a < 3; ++a) {
                s.lo[a] = c[a] - side / 2;
                s.hi[a] = s.lo[a] + side;
            }
        } else {
            const int32_t r = 8 + (int32_t)(size % 249u);
            for (int a = 0; a < 3; ++a) {
                s.c[a] = c[a];
                s.lo[a] = c[a] - r;
                s.hi[a] = c[a] + r + 1;
            }
            s.r2 = (uint32_t)(r * r);
        }
        ylo = std::min<int64_t>(ylo, s.lo[1]);
        yhi = std::max<int64_t>(yhi, s.hi[1]);
        hs.structures[i] = s;
    }
    p.structYLo = t.num_structures ? (int32_t)ylo : 0;
    p.structYHi = t.num_structures ? (int32_t)yhi : 0;
    // CSR cell lists, structures in increasing index order within each cell.
    const uint32_t cpa = p.cellsPerAxis;
    std::vector<uint32_t> count((size_t)cpa * cpa + 1, 0);
    auto cell_range = [&](const Structure& s, uint32_t& x0, uint32_t& x1, uint32_t& z0, uint32_t& z1) {
        auto clampc = [&](int64_t v) { return (uint32_t)std::min<int64_t>(std::max<int64_t>(v, 0), cpa - 1); };
        x0 = clampc((int64_t)s.lo[0] >> p.cellLog2);
        x1 = clampc(((int64_t)s.hi[0] - 1) >> p.cellLog2);
        z0 = clampc((int64_t)s.lo[2] >> p.cellLog2);
        z1 = clampc(((int64_t)s.hi[2] - 1) >> p.cellLog2);
        return s.hi[0] > 0 && s.lo[0] < G && s.hi[2] > 0 && s.lo[2] < G;
    };
    for (const Structure& s : hs.structures) {
        uint32_t x0, x1, z0, z1;
        if (!cell_range(s, x0, x1, z0, z1))
            continue;
        for (uint32_t cz = z0; cz <= z1; ++cz)
            for (uint32_t cx = x0; cx <= x1; ++cx)
                ++count[(size_t)cz * cpa + cx + 1];
    }
    for (size_t i = 1; i < count.size(); ++i)
        count[i] += count[i - 1];
    hs.cellStart = count;
    hs.cellList.assign(count.back(), 0);
    std::vector<uint32_t> fill(count.begin(), count.end() - 1);
    for (uint32_t i = 0; i < t.num_structures; ++i) {
        uint32_t x0, x1, z0, z1;
        if (!cell_range(hs.structures[i], x0, x1, z0, z1))
            continue;
        for (uint32_t cz = z0; cz <= z1; ++cz)
            for (uint32_t cx = x0; cx <= x1; ++cx)
                hs.cellList[fill[(size_t)cz * cpa + cx]++] = i;
    }
    p.structures = hs.structures.data();
    p.cellStart = hs.cellStart.data();
    p.cellList = hs.cellList.data();
}

unsigned long long scene_device_bytes(const HostScene& hs)
{
    return align256(hs.structures.size() * sizeof(Structure)) + align256(hs.cellStart.size() * 4) + align256(hs.cellList.size() * 4 + 4);
}

// Copies the scene arrays to `dev` and returns the parameters with device pointers.
svdag_status upload_scene(const HostScene& hs, char* dev, SceneParams& out, cudaStream_t s)
{
    out = hs.p;
    char* at = dev;
    out.structures = reinterpret_cast<const Structure*>(at);
    if (!hs.structures.empty())
        SVDAG_CUDA(cudaMemcpyAsync(at, hs.structures.data(), hs.structures.size() * sizeof(Structure), cudaMemcpyHostToDevice, s));
    at += align256(hs.structures.size() * sizeof(Structure));
    out.cellStart = reinterpret_cast<const uint32_t*>(at);
    SVDAG_CUDA(cudaMemcpyAsync(at, hs.cellStart.data(), hs.cellStart.size() * 4, cudaMemcpyHostToDevice, s));
    at += align256(hs.cellStart.size() * 4);
    out.cellList = reinterpret_cast<const uint32_t*>(at);
    if (!hs.cellList.empty())
        SVDAG_CUDA(cudaMemcpyAsync(at, hs.cellList.data(), hs.cellList.size() * 4, cudaMemcpyHostToDevice, s));
    return SVDAG_OK;
}

// While a scene build runs, the top of the scratch arena holds the scene arrays and the tile results.
struct ScratchTop {
    svdag_ctx* ctx;
    unsigned long long saved;
    char* base = nullptr;
    ScratchTop(svdag_ctx* c, unsigned long long bytes) : ctx(c), saved(c->scratchBytes)
    {
        bytes = align256(bytes);
        if (bytes + (1ull << 20) <= saved) {
            ctx->scratchBytes = saved - bytes;
            base = ctx->scratch + ctx->scratchBytes;
        }
    }
    ~ScratchTop() { ctx->scratchBytes = saved; }
};

constexpr uint32_t kNoChild = 0xFFFFFFFFu;

// A node above the tile level (or a tile, at level T).
struct TopNode {
    uint32_t level;
    uint32_t path[3];
    uint32_t child[8]; // index into the next level's nodes, or kNoChild
    uint32_t handle = kNone; // resolved handle (kNone = empty)
    uint32_t fill = kNone; // material if the subtree is uniformly full
};

// The nodes above the tiles, by level, from the host classification of the scene.
void classify_top(const SceneParams& p, uint32_t T, std::vector<std::vector<TopNode>>& nodes, const uint32_t (*fullyFilled)[16])
{
    nodes.assign(T + 1, {});
    TopNode root {};
    root.level = 0;
    root.path[0] = root.path[1] = root.path[2] = 0;
    for (auto& c : root.child)
        c = kNoChild;
    nodes[0].push_back(root);
    for (uint32_t level = 0; level < T; ++level) {
        const uint32_t depth = p.levels - (level + 1);
        for (size_t i = 0; i < nodes[level].size(); ++i) {
            for (uint32_t c = 0; c < 8; ++c) {
                const TopNode& par = nodes[level][i];
                const uint32_t cx = (par.path[0] << 1) | ((c >> 2) & 1u), cy = (par.path[1] << 1) | ((c >> 1) & 1u),
                               cz = (par.path[2] << 1) | (c & 1u);
                uint32_t mat = 0;
                const uint32_t op = scene_classify(p, cx, cy, cz, depth, mat);
                if (op == 2)
                    continue;
                TopNode ch {};
                ch.level = level + 1;
                ch.path[0] = cx;
                ch.path[1] = cy;
                ch.path[2] = cz;
                for (auto& k : ch.child)
                    k = kNoChild;
                if (op == 1) {
                    ch.handle = fullyFilled[level + 1][mat];
                    ch.fill = mat;
                }
                nodes[level][i].child[c] = (uint32_t)nodes[level + 1].size();
                nodes[level + 1].push_back(ch);
            }
        }
    }
}

struct TiledBuild {
    svdag_ctx* ctx;
    const SceneParams& dev; // device pointers
    const SceneParams& host; // host pointers
    uint32_t T;
    char* top; // device: tile handles, then key staging for the top assembly
    unsigned long long topBytes;

    // Allocates the level tables (bottom-up, canonical items first) and makes them current.
    svdag_status alloc_tables(const std::vector<std::vector<uint32_t>>& buckets, cudaStream_t s)
    {
        const uint32_t LL = ctx->cfg.levels - 2;
        for (int level = (int)LL; level >= 0; --level) {
            svdag_table& t = ctx->levelTables[level];
            SVDAG_TRY(alloc_table(ctx, &t, level == (int)LL ? SVDAG_KIND_LEAF : SVDAG_KIND_NODE, buckets[level].data(), s, true));
            t.level = level;
            SVDAG_TRY(insert_canonical(ctx, (uint32_t)level, s));
        }
        return upload_tables(ctx, s);
    }

    // One pass: tiles on the GPU, then the nodes above them; returns the root handle.
    svdag_status build(uint32_t& root, cudaStream_t s)
    {
        uint32_t ff[kMaxLevels][16];
        SVDAG_CUDA(cudaMemcpyAsync(ff, ctx->ctl->fullyFilled, sizeof(ff), cudaMemcpyDeviceToHost, s));
        SVDAG_CUDA(cudaStreamSynchronize(s));
        std::vector<std::vector<TopNode>> nodes;
        classify_top(host, T, nodes, ff);
        // Tiles: the level-T nodes that need subdividing.
        std::vector<uint32_t> tileOf;
        std::vector<DevEditor> eds;
        uint32_t* tileOut = reinterpret_cast<uint32_t*>(top);
        for (uint32_t i = 0; i < nodes[T].size(); ++i) {
            if (nodes[T][i].handle != kNone)
                continue; // filled by classification
            DevEditor ed {};
            ed.tool = kToolTerrain;
            ed.scene = dev;
            ed.levels = ctx->cfg.levels;
            ed.builder = 1;
            ed.startLevel = T;
            for (int a = 0; a < 3; ++a)
                ed.startPath[a] = nodes[T][i].path[a];
            ed.tileOut = tileOut + eds.size();
            tileOf.push_back(i);
            eds.push_back(ed);
        }
        if (eds.size() * 4 > topBytes / 2)
            return SVDAG_ERR_OOM;
        if (!eds.empty()) {
            SVDAG_CUDA(cudaMemsetAsync(tileOut, 0xFF, eds.size() * 4, s));
            SVDAG_TRY(launch_scene_tiles(ctx, eds.data(), (uint32_t)eds.size(), s));
            SVDAG_TRY(read_status(ctx, s));
            std::vector<uint32_t> handles(eds.size());
            SVDAG_CUDA(cudaMemcpyAsync(handles.data(), tileOut, handles.size() * 4, cudaMemcpyDeviceToHost, s));
            SVDAG_CUDA(cudaStreamSynchronize(s));
            for (size_t k = 0; k < eds.size(); ++k) {
                TopNode& n = nodes[T][tileOf[k]];
                n.handle = handles[k];
                for (uint32_t m = 0; m < 16; ++m)
                    if (handles[k] != kNone && handles[k] == ff[T][m])
                        n.fill = m;
            }
        }
        // Levels above the tiles, bottom-up: build the node items (fully-filled discovery on every
        // level, as the factory does), find-or-insert the distinct ones.
        uint32_t* keysDev = tileOut + align256(eds.size() * 4) / 4;
        for (int level = (int)T - 1; level >= 0; --level) {
            std::vector<uint32_t> words, offsets, unique;
            std::map<std::vector<uint32_t>, uint32_t> index;
            std::vector<uint32_t> which(nodes[level].size(), kNoChild);
            for (size_t i = 0; i < nodes[level].size(); ++i) {
                TopNode& n = nodes[level][i];
                if (n.handle != kNone || n.fill != kNone)
                    continue; // filled by classification
                uint32_t mask = 0, fill = kNone;
                bool uniform = true;
                std::vector<uint32_t> key(1, 0);
                for (uint32_t c = 0; c < 8; ++c) {
                    const uint32_t ci = n.child[c];
                    const TopNode* ch = ci == kNoChild ? nullptr : &nodes[level + 1][ci];
                    if (!ch || ch->handle == kNone) {
                        uniform = false;
                        continue;
                    }
                    mask |= 1u << c;
                    key.push_back(ch->handle);
                    if (ch->fill == kNone || (fill != kNone && ch->fill != fill))
                        uniform = false;
                    fill = ch->fill;
                }
                if (!mask)
                    continue; // empty
                key[0] = uniform ? (0xFFu | (1u << 8) | (fill << 9)) : mask;
                if (uniform)
                    n.fill = fill;
                auto it = index.find(key);
                if (it == index.end()) {
                    it = index.emplace(key, (uint32_t)offsets.size()).first;
                    offsets.push_back((uint32_t)words.size());
                    words.insert(words.end(), key.begin(), key.end());
                }
                which[i] = it->second;
            }
            const uint32_t nu = (uint32_t)offsets.size();
            if (nu) {
                const unsigned long long bytes = (words.size() + 2ull * nu) * 4;
                if (align256(eds.size() * 4) + bytes > topBytes)
                    return SVDAG_ERR_OOM;
                uint32_t* dw = keysDev;
                uint32_t* doff = dw + words.size();
                uint32_t* dout = doff + nu;
                SVDAG_CUDA(cudaMemcpyAsync(dw, words.data(), words.size() * 4, cudaMemcpyHostToDevice, s));
                SVDAG_CUDA(cudaMemcpyAsync(doff, offsets.data(), nu * 4, cudaMemcpyHostToDevice, s));
                SVDAG_TRY(find_or_insert_distinct(ctx, (uint32_t)level, dw, doff, nu, words.size(), dout, s));
                std::vector<uint32_t> out(nu);
                SVDAG_CUDA(cudaMemcpyAsync(out.data(), dout, nu * 4, cudaMemcpyDeviceToHost, s));
                SVDAG_CUDA(cudaStreamSynchronize(s));
                for (size_t i = 0; i < nodes[level].size(); ++i)
                    if (which[i] != kNoChild)
                        nodes[level][i].handle = out[which[i]];
            }
        }
        root = nodes[0][0].handle;
        return read_status(ctx, s);
    }
};

} // namespace

svdag_status run_scene_build(svdag_ctx* ctx, const svdag_terrain_params* p, cudaStream_t s)
{
    const uint32_t levels = ctx->cfg.levels;
    HostScene hs;
    make_scene(levels, *p, hs);
    // Automatic tile level: the smallest whose tiles' intermediate SVO fits half the scratch arena,
    // at about 3 * 4^(depth of a tile - 2) leaves (a heightfield surface with structures) of ~200
    // bytes each with their work items and dedup entries.
    uint32_t T = p->tile_level;
    if (!T) {
        const double fit = std::log(std::max(1.0, (double)ctx->scratchBytes / 2.0 / (3.0 * 200.0))) / std::log(4.0);
        const double t = std::ceil((double)levels - 2.0 - fit);
        T = t <= 0.0 ? 0u : std::min<uint32_t>((uint32_t)t, std::min<uint32_t>(levels - 3, 6));
    }
    // Top of the scratch arena: scene arrays, tile results and key staging (at most 8^T tiles).
    const unsigned long long sceneBytes = scene_device_bytes(hs);
    const unsigned long long topBytes = T ? align256((1ull << (3 * T)) * 4) + (64ull << 10) * 4 * 11 : 0;
    ScratchTop reserve(ctx, sceneBytes + topBytes);
    if (!reserve.base)
        return SVDAG_ERR_OOM;
    SceneParams dev;
    SVDAG_TRY(upload_scene(hs, reserve.base, dev, s));
    if (T == 0) {
        DevEditor ed {};
        ed.tool = kToolTerrain;
        ed.scene = dev;
        ed.levels = levels;
        ed.builder = 1;
        return build_scene_untiled(ctx, ed, s);
    }
    TiledBuild tb { ctx, dev, hs.p, T, reserve.base + align256(sceneBytes), topBytes };
    const uint32_t LL = levels - 2;
    // Counting pass into provisional tables: about 3 * 4^level items per level, chains absorb the rest.
    std::vector<std::vector<uint32_t>> buckets(LL + 1, std::vector<uint32_t>(kNumClasses));
    for (uint32_t level = 0; level <= LL; ++level) {
        const unsigned long long expect = std::min<unsigned long long>(3ull << (2 * level), 1ull << 36);
        for (uint32_t c = 0; c < kNumClasses; ++c)
            buckets[level][c] = (uint32_t)std::min<unsigned long long>(std::max<unsigned long long>(16, expect / 256), 1u << 17);
    }
    uint32_t root = kNone;
    SVDAG_TRY(reset_dag(ctx, s));
    SVDAG_TRY(tb.alloc_tables(buckets, s));
    SVDAG_TRY(tb.build(root, s));
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(tb.top + topBytes - 256);
    for (uint32_t level = 0; level <= LL; ++level) {
        unsigned long long per[kNumClasses];
        SVDAG_TRY(table_class_counts(ctx, ctx->levelTables[level], per, counters, s));
        for (uint32_t c = 0; c < kNumClasses; ++c)
            buckets[level][c] = (uint32_t)std::max<unsigned long long>(1, (per[c] + ctx->loadFactor - 1) / ctx->loadFactor);
    }
    // Final pass into exactly sized tables.
    SVDAG_TRY(reset_dag(ctx, s));
    SVDAG_TRY(tb.alloc_tables(buckets, s));
    SVDAG_TRY(tb.build(root, s));
    SVDAG_CUDA(cudaMemcpyAsync(&ctx->ctl->root, &root, sizeof(root), cudaMemcpyHostToDevice, s));
    SVDAG_CUDA(cudaStreamSynchronize(s));
    return SVDAG_OK;
}

} // namespace svdag

extern "C" uint32_t svdag_scene_height(const svdag_terrain_params* params, uint32_t levels, uint32_t x, uint32_t z)
{
    if (!params || levels < SVDAG_MIN_LEVELS || levels > SVDAG_MAX_LEVELS || params->octaves == 0 || params->octaves > 16)
        return 0;
    svdag::SceneParams p {};
    p.terrain = *params;
    p.levels = levels;
    p.baseLog2 = levels - 2;
    return svdag::terrain_height(p, x, z);
}
