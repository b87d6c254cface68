// svdag_oracle.cpp - CPU oracle for the SVDAG editing pipeline and DAG tracer.
//
// TEST INFRASTRUCTURE ONLY: this file is the checker of the CUDA implementation, never part of
// the product. It restates, function by function, the reference's EDag::MyGpuDag path
// (mathijs727/GPU-SVDAG-Editing); each function cites the reference file:line it follows.
// Build flags: -O2 -ffp-contract=off, no fast-math (float predicates decide structure, so they
// must be the uncontracted IEEE forms; the CUDA side is built with -fmad=false for the same reason).
//
// Storage model: items of level l live in a flat word vector; an oracle handle is the word offset
// of the item inside its level. A content index per level gives find/add. This is deliberately the
// simplest correct container: the reference's slab hash tables only change where items live, not
// which items exist, so every structural comparison is made on contents.
#include "svdag_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <optional>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

constexpr uint32_t kSentinel = 0xFFFFFFFFu; // create_edit_svo.h:54 sentinel
constexpr uint32_t kMaterialBits = 4; // gpu_hash_dag_definitions.h:11
constexpr uint32_t kNumMaterials = 1u << kMaterialBits;
constexpr uint32_t kMaxNodeWords = 9; // my_gpu_base_dag.h:94
constexpr uint32_t kMaxLeafWords = 2 + (64 * kMaterialBits + 31) / 32; // my_gpu_base_dag.h:96 (= 10)

inline uint32_t popc(uint32_t v) { return (uint32_t)__builtin_popcount(v); }
inline uint32_t popcll(uint64_t v) { return (uint32_t)__builtin_popcountll(v); }

// ---------------------------------------------------------------- item encoding (my_gpu_base_dag.h)

// Header bits: 0-7 child mask, 8 hasFullyFilled, 9-12 material, 13-31 user payload
// (my_gpu_base_dag.h:344-351).
inline uint32_t header_child_mask(uint32_t h) { return h & 0xFFu; }
inline uint32_t header_payload(uint32_t h) { return h >> 13; }
inline bool header_fully_filled(uint32_t h, uint32_t& material)
{
    material = (h >> 9) & 0xFu; // get_node_is_fully_filled, my_gpu_base_dag.h:185-189
    return (h >> 8) & 1u;
}
inline uint32_t encode_header(uint32_t childMask) { return childMask & 0xFFu; } // :152-158
inline uint32_t encode_header_payload(uint32_t childMask, uint32_t payload) // :159-166
{
    return (childMask & 0xFFu) | (payload << 13);
}
inline uint32_t encode_header_filled(uint32_t childMask, uint32_t material) // :167-175
{
    return (childMask & 0xFFu) | (1u << 8) | ((material & 0xFu) << 9);
}
inline uint32_t node_size(const uint32_t* n) { return 1 + popc(header_child_mask(n[0])); } // :200-203
inline uint32_t leaf_size(const uint32_t* l) // get_leaf_size, :195-199
{
    const uint32_t voxels = popc(l[0]) + popc(l[1]);
    return 2 + ((voxels * kMaterialBits + 31) >> 5);
}
inline uint32_t child_offset(uint32_t childMask, uint32_t child) // :205-208
{
    return popc(childMask & ((1u << child) - 1u));
}
// get_material, my_gpu_base_dag.h:293-316 (32 % 4 == 0, so no material straddles two words).
inline bool leaf_material(const uint32_t* leaf, uint32_t voxel, uint32_t& out)
{
    const uint64_t mask = (uint64_t)leaf[0] | ((uint64_t)leaf[1] << 32);
    if (!(mask & (1ull << voxel)))
        return false;
    const uint32_t bit = popcll(mask & ((1ull << voxel) - 1ull)) * kMaterialBits;
    out = (leaf[2 + (bit >> 5)] >> (bit & 31)) & (kNumMaterials - 1u);
    return true;
}
// LeafBuilder, my_gpu_base_dag.h:102-150.
struct LeafBuilder {
    uint32_t* p;
    uint32_t voxelIndex = 0, voxelOffset = 0;
    explicit LeafBuilder(uint32_t* pLeaf)
        : p(pLeaf)
    {
        for (uint32_t i = 0; i < kMaxLeafWords; ++i)
            p[i] = 0;
    }
    void set(uint32_t value)
    {
        p[voxelIndex >> 5] |= 1u << (voxelIndex & 31);
        const uint32_t bits = voxelOffset * kMaterialBits;
        p[2 + (bits >> 5)] |= value << (bits & 31);
        ++voxelOffset;
    }
    void next() { ++voxelIndex; }
    uint32_t finalize() const { return 2 + (voxelOffset * kMaterialBits + 31) / 32; }
};

// ---------------------------------------------------------------- Path (path.h:7-101)

struct Path {
    uint32_t x = 0, y = 0, z = 0;
    void descend(uint32_t child) // path.h:27-35
    {
        x = (x << 1) | ((child & 4u) >> 2);
        y = (y << 1) | ((child & 2u) >> 1);
        z = (z << 1) | (child & 1u);
    }
    void ascend(uint32_t levels)
    {
        x >>= levels;
        y >>= levels;
        z >>= levels;
    }
    bool operator==(const Path& o) const { return x == o.x && y == o.y && z == o.z; }
    // child_index, path.h:54-59
    uint32_t child_index(uint32_t level, uint32_t totalLevels) const
    {
        const uint32_t s = totalLevels - level;
        return (((x >> s) & 1u) ? 4u : 0u) | (((y >> s) & 1u) ? 2u : 0u) | (((z >> s) & 1u) ? 1u : 0u);
    }
};
struct F3 {
    float x, y, z;
};
inline F3 as_position(const Path& p, uint32_t shift) // path.h:37-43
{
    return { float(p.x << shift), float(p.y << shift), float(p.z << shift) };
}
inline F3 add(F3 a, float s) { return { a.x + s, a.y + s, a.z + s }; }
inline F3 sub(F3 a, float s) { return { a.x - s, a.y - s, a.z - s }; }
inline F3 add(F3 a, F3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline F3 sub(F3 a, F3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline float sq(float f) { return f * f; } // cuda_math.h squared
// constexpr_max / constexpr_min, cuda_math.h:13-18
inline float cmax(float a, float b) { return a > b ? a : b; }
inline float cmin(float a, float b) { return a < b ? a : b; }
// voxel index of (x,y,z) inside its leaf, dag_utils.h:162-163
inline uint32_t leaf_bit_index(uint32_t x, uint32_t y, uint32_t z)
{
    return ((x & 1u) ? 4u : 0u) | ((y & 1u) ? 2u : 0u) | ((z & 1u) ? 1u : 0u) | ((x & 2u) ? 32u : 0u)
        | ((y & 2u) ? 16u : 0u) | ((z & 2u) ? 8u : 0u);
}

// ---------------------------------------------------------------- editors (my_gpu_dag_editors.h)

enum class State { Partial, Filled, Empty }; // my_gpu_dag_editors.h:7-11
enum class Op { Subdivide, Fill, Empty, Keep }; // :17-22
struct NodeDesc {
    State state;
    uint32_t fillMaterial;
};
struct EditDesc {
    Op op;
    uint32_t fillMaterial;
};

struct CopyParent {
    Path path;
    uint32_t handle;
};
struct CopyState { // MyGpuCopyEditor::State, my_gpu_dag_editors.h:139-145
    CopyParent parents[8];
};

struct Dag;

// Box tests shared by the box and copy tools (MyGpuBoxEditorBase, my_gpu_dag_editors.h:45-80).
struct BoxBase {
    float radius;
    F3 bmin, bmax;
    void init(F3 center, float r)
    {
        radius = r;
        bmin = sub(center, r);
        bmax = (r == 0) ? add(center, 1.0f) : add(center, r);
    }
    bool overlap(F3 nmin, F3 nmax) const // :64-67
    {
        return !(bmin.x >= nmax.x || bmin.y >= nmax.y || bmin.z >= nmax.z || bmax.x <= nmin.x || bmax.y <= nmin.y
            || bmax.z <= nmin.z || nmin.x >= bmax.x || nmin.y >= bmax.y || nmin.z >= bmax.z || nmax.x <= bmin.x
            || nmax.y <= bmin.y || nmax.z <= bmin.z);
    }
    bool contained(F3 nmin, F3 nmax) const // :76-79
    {
        return bmin.x <= nmin.x && bmin.y <= nmin.y && bmin.z <= nmin.z && bmax.x >= nmax.x && bmax.y >= nmax.y
            && bmax.z >= nmax.z;
    }
};
// Sphere tests (MyGpuSphereEditorBase, my_gpu_dag_editors.h:401-455).
struct SphereBase {
    F3 center;
    float radius, radiusSquared;
    void init(F3 c, float r)
    {
        center = add(c, 0.5f);
        radius = std::max(r, 0.1f);
        radiusSquared = radius * radius;
    }
    bool overlap(F3 nmin, F3 nmax) const // :420-440
    {
        float dist = radiusSquared;
        if (center.x < nmin.x)
            dist -= sq(center.x - nmin.x);
        else if (center.x > nmax.x)
            dist -= sq(center.x - nmax.x);
        if (center.y < nmin.y)
            dist -= sq(center.y - nmin.y);
        else if (center.y > nmax.y)
            dist -= sq(center.y - nmax.y);
        if (center.z < nmin.z)
            dist -= sq(center.z - nmin.z);
        else if (center.z > nmax.z)
            dist -= sq(center.z - nmax.z);
        return dist > 0;
    }
    bool contained(F3 nmin, F3 nmax) const // :442-454
    {
        return std::max(sq(nmin.x - center.x), sq(nmax.x - center.x)) + std::max(sq(nmin.y - center.y), sq(nmax.y - center.y))
            + std::max(sq(nmin.z - center.z), sq(nmax.z - center.z))
            < radiusSquared;
    }
};

uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// 3D value noise quantised to a 4-bit material (the BOX_PAINT_NOISE tool). Integer arithmetic only.
uint32_t lattice3(uint32_t seed, uint32_t x, uint32_t y, uint32_t z)
{
    uint32_t h = fmix32(seed * 0x9E3779B9u ^ 0x5bd1e995u);
    h = fmix32(h ^ (x * 0xC2B2AE35u));
    h = fmix32(h ^ (y * 0x27D4EB2Fu));
    h = fmix32(h ^ (z * 0x165667B1u));
    return h >> 16;
}
int64_t smooth16(int64_t t) { return (t * t * (3 * 65536 - 2 * t)) >> 32; }
int64_t lerp16(int64_t a, int64_t b, int64_t t) { return a + (((b - a) * t) >> 16); }
uint32_t noise_material(uint32_t seed, uint32_t cellLog2, uint32_t x, uint32_t y, uint32_t z)
{
    const uint32_t ix = x >> cellLog2, iy = y >> cellLog2, iz = z >> cellLog2;
    const uint32_t m = (1u << cellLog2) - 1u;
    const auto frac = [&](uint32_t v) -> int64_t {
        const uint32_t f = v & m;
        return cellLog2 <= 16 ? (int64_t)(f << (16 - cellLog2)) : (int64_t)(f >> (cellLog2 - 16));
    };
    const int64_t sx = smooth16(frac(x)), sy = smooth16(frac(y)), sz = smooth16(frac(z));
    int64_t c[2][2][2];
    for (uint32_t a = 0; a < 2; ++a)
        for (uint32_t b = 0; b < 2; ++b)
            for (uint32_t d = 0; d < 2; ++d)
                c[a][b][d] = lattice3(seed, ix + a, iy + b, iz + d);
    const int64_t x00 = lerp16(c[0][0][0], c[1][0][0], sx), x10 = lerp16(c[0][1][0], c[1][1][0], sx);
    const int64_t x01 = lerp16(c[0][0][1], c[1][0][1], sx), x11 = lerp16(c[0][1][1], c[1][1][1], sx);
    const int64_t y0 = lerp16(x00, x10, sy), y1 = lerp16(x01, x11, sy);
    const int64_t v = lerp16(y0, y1, sz);
    return (uint32_t)(v >> 12) & 0xFu;
}

struct Editor {
    svdag_edit e {};
    uint32_t tool = 0;
    BoxBase box {};
    SphereBase sphere {};
    // copy
    F3 fDestToSource {};
    int32_t iDestToSource[3] {};
    const Dag* dagCopy = nullptr;
    uint32_t copyRoot = kSentinel;
    const Dag* dagOld = nullptr; // erosion: the DAG the neighbour counts read (its root is unchanged until the merge)

    bool stateful() const { return tool == SVDAG_TOOL_COPY; }

    // Stateless should_edit of the tools; each branch cites its reference function.
    EditDesc should_edit(const Path& path, uint32_t depth, const NodeDesc& desc) const
    {
        const F3 nmin = as_position(path, depth);
        const F3 nmax = add(nmin, float(1u << depth));
        EditDesc out { Op::Keep, 0 };
        switch (tool) {
        case SVDAG_TOOL_BOX_ADD:
        case SVDAG_TOOL_BOX_REMOVE: { // MyGpuBoxEditor::should_edit, my_gpu_dag_editors.h:94-110
            if (box.contained(nmin, nmax)) {
                out.op = tool == SVDAG_TOOL_BOX_ADD ? Op::Fill : Op::Empty;
                out.fillMaterial = e.material;
            } else if (box.overlap(nmin, nmax)) {
                out.op = Op::Subdivide;
            }
        } break;
        case SVDAG_TOOL_SPHERE_ADD:
        case SVDAG_TOOL_SPHERE_REMOVE: { // MyGpuSphereEditor::should_edit, :467-487
            const bool overlaps = sphere.overlap(nmin, nmax);
            const bool fully = sphere.contained(add(nmin, 1.0f), sub(nmax, 1.0f));
            if (!overlaps)
                out.op = Op::Keep;
            else if (fully) {
                out.op = tool == SVDAG_TOOL_SPHERE_ADD ? Op::Fill : Op::Empty;
                out.fillMaterial = e.material;
            } else
                out.op = Op::Subdivide;
        } break;
        case SVDAG_TOOL_SPHERE_PAINT: { // MyGpuSpherePaintEditor::should_edit, :509-530
            const bool overlaps = sphere.overlap(nmin, nmax);
            const bool fully = sphere.contained(nmin, nmax);
            if (!overlaps)
                out.op = Op::Keep;
            else if (fully && desc.state == State::Filled) {
                out.op = Op::Fill;
                out.fillMaterial = e.material;
            } else if (desc.state == State::Empty)
                out.op = Op::Empty;
            else
                out.op = Op::Subdivide;
        } break;
        case SVDAG_TOOL_BOX_PAINT_NOISE: { // box form of the paint tool; the material varies per voxel
            if (!box.overlap(nmin, nmax))
                out.op = Op::Keep;
            else if (desc.state == State::Empty)
                out.op = Op::Empty;
            else
                out.op = Op::Subdivide;
        } break;
        case SVDAG_TOOL_COPY: { // stateless MyGpuCopyEditor::should_edit, :166-172
            out.op = box.overlap(nmin, nmax) ? Op::Subdivide : Op::Keep;
        } break;
        case SVDAG_TOOL_SPHERE_ERODE: { // MyGpuSphereErosionEditor::should_edit, :551-562
            if (!sphere.overlap(nmin, nmax))
                out.op = Op::Keep;
            else if (desc.state == State::Empty)
                out.op = Op::Empty;
            else
                out.op = Op::Subdivide;
        } break;
        default:
            break;
        }
        return out;
    }

    // get_new_value of the tools (create_edit_svo.cu:361-372 picks the overload).
    std::optional<uint32_t> new_value(const Path& voxel, std::optional<uint32_t> old, const CopyState* st) const;
    EditDesc should_edit_state(const Path& path, uint32_t depth, const NodeDesc& desc, const CopyState& in,
        CopyState& out, uint32_t maxLevels) const;
};

// ---------------------------------------------------------------- DAG container (my_gpu_hash_dag.h/.cu)

struct ItemKey {
    uint32_t n;
    uint32_t w[kMaxLeafWords];
    bool operator==(const ItemKey& o) const { return n == o.n && std::memcmp(w, o.w, n * 4) == 0; }
};
struct ItemKeyHash {
    size_t operator()(const ItemKey& k) const
    {
        uint64_t h = 1469598103934665603ull ^ k.n;
        for (uint32_t i = 0; i < k.n; ++i)
            h = (h ^ k.w[i]) * 1099511628211ull;
        return (size_t)(h ^ (h >> 29));
    }
};

struct Dag {
    uint32_t levels = 0;
    std::vector<std::vector<uint32_t>> words; // per level
    std::vector<std::unordered_map<ItemKey, uint32_t, ItemKeyHash>> index; // per level
    std::vector<std::array<uint32_t, kNumMaterials>> fullyFilled; // fullyFilledNodes[level][material]
    uint32_t root = kSentinel;
    // MyGPUHashDAGUndoRedo (my_gpu_base_dag.h:16-82)
    std::vector<uint32_t> undoFrames, redoFrames;

    uint32_t leaf_level() const { return levels - 2; } // base_dag.h:65-68
    const uint32_t* ptr(uint32_t level, uint32_t handle) const { return &words[level][handle]; }
    uint32_t item_size(uint32_t level, const uint32_t* p) const
    {
        return level == leaf_level() ? leaf_size(p) : node_size(p);
    }
    uint32_t find(uint32_t level, const uint32_t* item) const // find_node / find_leaf, my_gpu_hash_dag.h:168-262
    {
        ItemKey k {};
        k.n = item_size(level, item);
        std::memcpy(k.w, item, k.n * 4);
        auto it = index[level].find(k);
        return it == index[level].end() ? kSentinel : it->second;
    }
    // add_node / add_leaf (my_gpu_hash_dag.h:198-283). The reference's add never checks for an
    // existing copy; its callers only add items that a find just missed, so find-then-add is kept.
    uint32_t find_or_add(uint32_t level, const uint32_t* item, bool* added = nullptr)
    {
        ItemKey k {};
        k.n = item_size(level, item);
        std::memcpy(k.w, item, k.n * 4);
        auto it = index[level].find(k);
        if (it != index[level].end()) {
            if (added)
                *added = false;
            return it->second;
        }
        const uint32_t h = (uint32_t)words[level].size();
        words[level].insert(words[level].end(), k.w, k.w + k.n);
        index[level].emplace(k, h);
        if (added)
            *added = true;
        return h;
    }

    void init(uint32_t lv) // MyGPUHashDAG::allocate, my_gpu_hash_dag.cu:24-66
    {
        levels = lv;
        words.assign(levels, {});
        index.assign(levels, {});
        fullyFilled.assign(levels, {});
        for (auto& a : fullyFilled)
            a.fill(kSentinel);
        root = kSentinel;
        undoFrames.clear();
        redoFrames.clear();
        for (uint32_t m = 0; m < kNumMaterials; ++m) {
            uint32_t leaf[kMaxLeafWords];
            LeafBuilder b { leaf };
            for (uint32_t i = 0; i < 64; ++i) {
                b.set(m);
                b.next();
            }
            fullyFilled[leaf_level()][m] = find_or_add(leaf_level(), leaf);
        }
        for (int level = (int)leaf_level() - 1; level >= 0; --level) {
            for (uint32_t m = 0; m < kNumMaterials; ++m) {
                uint32_t node[kMaxNodeWords];
                node[0] = encode_header_filled(0xFF, m);
                for (uint32_t i = 0; i < 8; ++i)
                    node[1 + i] = fullyFilled[level + 1][m];
                fullyFilled[level][m] = find_or_add(level, node);
            }
        }
    }

    // MyGPUHashDAG::is_leaf_fully_filled, my_gpu_hash_dag.h:143-166
    bool leaf_fully_filled(const uint32_t* leaf, uint32_t& outMaterial) const
    {
        if (leaf[0] != 0xFFFFFFFFu || leaf[1] != 0xFFFFFFFFu)
            return false;
        const uint32_t first = leaf[2] & (kNumMaterials - 1u);
        const uint32_t* canon = ptr(leaf_level(), fullyFilled[leaf_level()][first]);
        for (uint32_t i = 2; i < kMaxLeafWords; ++i)
            if (canon[i] != leaf[i])
                return false;
        outMaterial = first;
        return true;
    }
};

std::optional<uint32_t> get_value(const Dag& dag, const Path& path) // DAGUtils::get_value, dag_utils.h:146-182
{
    if (dag.root == kSentinel)
        return std::nullopt;
    uint32_t index = dag.root;
    for (uint32_t level = 0; level < dag.levels; ++level) {
        if (level < dag.leaf_level()) {
            const uint32_t* node = dag.ptr(level, index);
            const uint32_t mask = header_child_mask(node[0]);
            const uint32_t child = path.child_index(level + 1, dag.levels);
            if (!(mask & (1u << child)))
                return std::nullopt;
            index = node[1 + child_offset(mask, child)];
        } else {
            const uint32_t v = leaf_bit_index(path.x, path.y, path.z);
            uint32_t m;
            if (leaf_material(dag.ptr(dag.leaf_level(), index), v, m))
                return m;
            return std::nullopt;
        }
    }
    return std::nullopt;
}

// MyGpuCopyEditor (the "#if 1" form, my_gpu_dag_editors.h:129-253).
EditDesc Editor::should_edit_state(const Path& path, uint32_t depth, const NodeDesc&, const CopyState& in,
    CopyState& out, uint32_t maxLevels) const
{
    const F3 nmin = as_position(path, depth);
    const float nodeSize = float(1u << depth);
    const F3 nmax = add(nmin, nodeSize);
    if (!box.overlap(nmin, nmax))
        return { Op::Keep, 0 };
    const F3 mx { cmax(nmin.x, box.bmin.x), cmax(nmin.y, box.bmin.y), cmax(nmin.z, box.bmin.z) };
    const F3 shiftedMin = add(mx, fDestToSource);
    const F3 a = add(shiftedMin, nodeSize);
    const F3 b = add(box.bmax, fDestToSource);
    const F3 shiftedMax { cmin(a.x, b.x), cmin(a.y, b.y), cmin(a.z, b.z) };
    const uint32_t parentLevel = maxLevels - depth - 1;
    int numOut = 0;
    for (const auto& parent : in.parents) {
        if (parent.handle == 0xFFFFFFFFu)
            break;
        const uint32_t* pNode = dagCopy->ptr(parentLevel, parent.handle);
        const uint32_t childMask = header_child_mask(pNode[0]);
        for (uint32_t c = 0; c < 8; ++c) {
            if (!(childMask & (1u << c)))
                continue;
            Path cp = parent.path;
            cp.descend(c);
            const F3 cmn = as_position(cp, depth);
            const F3 cmx = add(cmn, nodeSize);
            // aabbOverlap, my_gpu_dag_editors.h:121-125
            const bool ov = !(cmn.x >= shiftedMax.x || cmn.y >= shiftedMax.y || cmn.z >= shiftedMax.z || cmx.x <= shiftedMin.x
                || cmx.y <= shiftedMin.y || cmx.z <= shiftedMin.z || shiftedMin.x >= cmx.x || shiftedMin.y >= cmx.y
                || shiftedMin.z >= cmx.z || shiftedMax.x <= cmn.x || shiftedMax.y <= cmn.y || shiftedMax.z <= cmn.z);
            if (ov && numOut < 8) {
                out.parents[numOut].handle = pNode[1 + child_offset(childMask, c)];
                out.parents[numOut].path = cp;
                ++numOut;
            }
        }
    }
    if (numOut != 8)
        out.parents[numOut].handle = 0xFFFFFFFFu;
    return { numOut == 0 ? Op::Keep : Op::Subdivide, 0 };
}

std::optional<uint32_t> Editor::new_value(const Path& voxel, std::optional<uint32_t> old, const CopyState* st) const
{
    switch (tool) {
    case SVDAG_TOOL_BOX_ADD: // MyGpuBoxEditor::get_new_value, my_gpu_dag_editors.h:112-118
    case SVDAG_TOOL_SPHERE_ADD: // MyGpuSphereEditor::get_new_value, :489-495
        return e.material;
    case SVDAG_TOOL_BOX_REMOVE:
    case SVDAG_TOOL_SPHERE_REMOVE:
        return std::nullopt;
    case SVDAG_TOOL_SPHERE_PAINT: // :532-535
        return e.material;
    case SVDAG_TOOL_BOX_PAINT_NOISE:
        return noise_material(e.noise_seed, e.noise_cell_log2, voxel.x, voxel.y, voxel.z);
    case SVDAG_TOOL_SPHERE_ERODE: { // MyGpuSphereErosionEditor::get_new_value, :564-588
        uint32_t count = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (dx == 0 && dy == 0 && dz == 0)
                        continue;
                    // unsigned coordinates: -1 wraps around the grid as the reference's Path does
                    const Path nb { voxel.x + (uint32_t)dx, voxel.y + (uint32_t)dy, voxel.z + (uint32_t)dz };
                    count += get_value(*dagOld, nb).has_value() ? 1u : 0u;
                }
        if (count > e.noise_seed)
            return old;
        return std::nullopt;
    }
    case SVDAG_TOOL_COPY: { // get_new_value(uint3, optional, State), :225-252
        int32_t s[3] = { (int32_t)voxel.x + iDestToSource[0], (int32_t)voxel.y + iDestToSource[1],
            (int32_t)voxel.z + iDestToSource[2] };
        for (auto& v : s)
            v = std::max(v, 0);
        const Path src { (uint32_t)s[0], (uint32_t)s[1], (uint32_t)s[2] };
        const Path parentPath { src.x >> 2, src.y >> 2, src.z >> 2 };
        const CopyParent* pParent = nullptr;
        for (const auto& parent : st->parents) {
            if (parent.handle == 0xFFFFFFFFu)
                break;
            if (parent.path == parentPath)
                pParent = &parent;
        }
        if (!pParent)
            return old;
        uint32_t m;
        if (leaf_material(dagCopy->ptr(dagCopy->leaf_level(), pParent->handle), leaf_bit_index(src.x, src.y, src.z), m))
            old = m;
        return old;
    }
    default:
        return old;
    }
}

Editor make_editor(const svdag_edit& e, const Dag& dag)
{
    Editor ed;
    ed.e = e;
    ed.tool = e.tool;
    const F3 c { e.center[0], e.center[1], e.center[2] };
    switch (e.tool) {
    case SVDAG_TOOL_BOX_ADD:
    case SVDAG_TOOL_BOX_REMOVE:
    case SVDAG_TOOL_BOX_PAINT_NOISE:
        ed.box.init(c, e.radius);
        break;
    case SVDAG_TOOL_SPHERE_ADD:
    case SVDAG_TOOL_SPHERE_REMOVE:
    case SVDAG_TOOL_SPHERE_PAINT:
        ed.sphere.init(c, e.radius);
        break;
    case SVDAG_TOOL_SPHERE_ERODE: // MyGpuSphereErosionEditor constructor, :542-548
        ed.sphere.init(c, e.radius);
        ed.dagOld = &dag;
        break;
    case SVDAG_TOOL_COPY: { // MyGpuCopyEditor constructor, my_gpu_dag_editors.h:157-164
        const F3 src { e.src[0], e.src[1], e.src[2] };
        const F3 dst { e.dst[0], e.dst[1], e.dst[2] };
        ed.box.init(add(dst, sub(c, src)), e.radius);
        ed.fDestToSource = add(F3 { -dst.x, -dst.y, -dst.z }, src);
        ed.iDestToSource[0] = (int32_t)ed.fDestToSource.x;
        ed.iDestToSource[1] = (int32_t)ed.fDestToSource.y;
        ed.iDestToSource[2] = (int32_t)ed.fDestToSource.z;
        ed.dagCopy = &dag;
        ed.copyRoot = dag.root;
    } break;
    default:
        break;
    }
    return ed;
}

// ---------------------------------------------------------------- edit pipeline

struct WorkItem { // CreateIntermediateWorkItem, create_edit_svo.cu:55-65
    Path path;
    uint32_t handle;
    CopyState state;
};
struct SvoItem { // IntermediateSVO::Node / Leaf, create_edit_svo.h:10-61 (zero padded)
    uint32_t w[kMaxLeafWords];
    uint32_t size;
};

struct EditCounters {
    uint64_t svo[SVDAG_MAX_LEVELS] = {};
    uint64_t oldRead = 0, unique = 0, added = 0, edited = 0;
};

// Top-down construction of the intermediate SVO (createIntermediateSvoStructure_cuda and the
// per-level recursion, create_edit_svo.cu:548-630; inner nodes :168-303; leaves :321-426).
// Returns false when a level produced no work items (no leaves -> the DAG is not touched,
// my_gpu_hash_dag_edits.cu:651).
bool build_svo(const Dag& dag, const Editor& ed, std::vector<std::vector<SvoItem>>& svo, EditCounters& cnt)
{
    const uint32_t L = dag.levels;
    const uint32_t leafLevel = dag.leaf_level();
    svo.assign(leafLevel + 1, {});
    std::vector<WorkItem> work(1);
    work[0].path = Path {};
    work[0].handle = dag.root; // may be the sentinel for an empty DAG (create_edit_svo.cu:618)
    if (ed.stateful()) { // MyGpuCopyEditor::createInitialState, my_gpu_dag_editors.h:148-155
        for (auto& p : work[0].state.parents) {
            p.path = Path {};
            p.handle = 0;
        }
        work[0].state.parents[0].path = Path {};
        work[0].state.parents[0].handle = ed.copyRoot;
        work[0].state.parents[1].handle = 0xFFFFFFFFu;
    }
    for (uint32_t level = 0; level < leafLevel; ++level) {
        const uint32_t childLevel = level + 1;
        const uint32_t childDepth = L - childLevel;
        std::vector<WorkItem> next;
        auto& out = svo[level];
        out.resize(work.size());
        cnt.svo[level] = work.size();
        for (size_t wi = 0; wi < work.size(); ++wi) {
            const WorkItem& in = work[wi];
            uint32_t oldMask = 0;
            const uint32_t* oldNode = nullptr;
            if (in.handle != kSentinel) {
                oldNode = dag.ptr(level, in.handle);
                oldMask = header_child_mask(oldNode[0]);
                ++cnt.oldRead;
            }
            uint32_t childHandles[8];
            uint32_t intermediateMask = 0, outMask = 0;
            for (uint32_t c = 0; c < 8; ++c) {
                uint32_t childHandle = kSentinel;
                if (oldMask & (1u << c))
                    childHandle = oldNode[1 + child_offset(oldMask, c)];
                Path cp = in.path;
                cp.descend(c);
                NodeDesc desc { State::Empty, 0 };
                if (childHandle == kSentinel)
                    desc.state = State::Empty;
                else if (childLevel == leafLevel)
                    desc.state = State::Partial;
                else
                    desc.state = header_fully_filled(dag.ptr(childLevel, childHandle)[0], desc.fillMaterial) ? State::Filled
                                                                                                           : State::Partial;
                EditDesc ed_desc;
                CopyState childState {};
                if (ed.stateful())
                    ed_desc = ed.should_edit_state(cp, childDepth, desc, in.state, childState, L);
                else
                    ed_desc = ed.should_edit(cp, childDepth, desc);
                if (ed_desc.op == Op::Fill || ed_desc.op == Op::Empty)
                    cnt.edited += uint64_t(1) << (3 * childDepth);
                if (ed_desc.op == Op::Subdivide) {
                    WorkItem w;
                    w.path = cp;
                    w.handle = childHandle;
                    w.state = childState;
                    childHandle = (uint32_t)next.size();
                    next.push_back(w);
                    intermediateMask |= 1u << c;
                } else if (ed_desc.op == Op::Empty) {
                    childHandle = kSentinel;
                } else if (ed_desc.op == Op::Fill) {
                    childHandle = dag.fullyFilled[childLevel][ed_desc.fillMaterial];
                }
                childHandles[c] = childHandle;
                if (childHandle != kSentinel)
                    outMask |= 1u << c;
            }
            SvoItem& node = out[wi];
            std::memset(&node, 0, sizeof(node));
            if (outMask) {
                node.w[0] = encode_header_payload(outMask, intermediateMask);
                uint32_t k = 1;
                for (uint32_t c = 0; c < 8; ++c)
                    if (outMask & (1u << c))
                        node.w[k++] = childHandles[c];
                node.size = k;
            } else {
                node.size = 0;
            }
        }
        work.swap(next);
        if (work.empty())
            return false;
    }
    // Leaves: one voxel per "thread" (createIntermediateSvoStructure_leaf_workgroup, :321-426).
    auto& leaves = svo[leafLevel];
    leaves.resize(work.size());
    cnt.svo[leafLevel] = work.size();
    for (size_t wi = 0; wi < work.size(); ++wi) {
        const WorkItem& in = work[wi];
        const uint32_t* oldLeaf = nullptr;
        if (in.handle != kSentinel) {
            oldLeaf = dag.ptr(leafLevel, in.handle);
            ++cnt.oldRead;
        }
        SvoItem& leaf = leaves[wi];
        std::memset(&leaf, 0, sizeof(leaf));
        LeafBuilder b { leaf.w };
        for (uint32_t v = 0; v < 64; ++v) {
            std::optional<uint32_t> oldMat;
            uint32_t m;
            if (oldLeaf && leaf_material(oldLeaf, v, m))
                oldMat = m;
            Path vp = in.path;
            vp.descend(v >> 3);
            vp.descend(v & 7u);
            NodeDesc desc;
            desc.state = oldMat ? State::Filled : State::Empty;
            desc.fillMaterial = oldMat ? *oldMat : 0xFFFFFFFFu;
            const EditDesc d = ed.should_edit(vp, 0, desc); // stateless should_edit at depth 0
            std::optional<uint32_t> newMat;
            if (d.op == Op::Fill || d.op == Op::Subdivide)
                newMat = ed.new_value(vp, oldMat, ed.stateful() ? &in.state : nullptr);
            else if (d.op == Op::Keep)
                newMat = oldMat;
            if (d.op != Op::Keep)
                ++cnt.edited;
            if (newMat)
                b.set(*newMat);
            b.next();
        }
        leaf.size = b.finalize();
    }
    return true;
}

// Bottom-up merge (mergeDag_CUDA + doMergeDagHashing, my_gpu_hash_dag_edits.cu:313-631).
// `discoverAlways` disables the reference's fully-filled gating (:337-351); only the scene builder
// uses it, to reproduce the factory's full propagation of the fully-filled bits.
uint32_t merge_svo(Dag& dag, std::vector<std::vector<SvoItem>>& svo, EditCounters& cnt, bool discoverAlways)
{
    const uint32_t leafLevel = dag.leaf_level();
    std::vector<uint32_t> prevMapping, curMapping;
    bool hasFullyFilled = true; // :589
    for (int level = (int)leafLevel; level >= 0; --level) {
        auto& items = svo[level];
        curMapping.assign(items.size(), kSentinel);
        if (level != (int)leafLevel) { // updateChildPointers, :44-95
            for (auto& node : items) {
                uint32_t mask = header_child_mask(node.w[0]);
                const uint32_t interm = header_payload(node.w[0]);
                uint32_t in = 0, out = 0;
                uint32_t* ch = &node.w[1];
                for (uint32_t c = 0; c < 8; ++c) {
                    if (!(mask & (1u << c)))
                        continue;
                    uint32_t h = ch[in++];
                    if (interm & (1u << c))
                        h = prevMapping[h];
                    if (h != kSentinel)
                        ch[out++] = h;
                    else
                        mask ^= 1u << c;
                }
                node.w[0] = encode_header(mask);
                for (uint32_t i = 1 + out; i < node.size; ++i)
                    node.w[i] = 0;
                if (out != in)
                    node.size = 1 + out;
            }
        }
        if (hasFullyFilled || discoverAlways) { // discover_fully_filled, :96-150
            uint32_t count = 0;
            for (auto& item : items) {
                uint32_t material = kSentinel;
                bool full = false;
                if (level == (int)leafLevel) {
                    full = dag.leaf_fully_filled(item.w, material);
                } else if (header_child_mask(item.w[0]) == 0xFF) {
                    full = true;
                    for (uint32_t c = 0; c < 8 && full; ++c) {
                        const uint32_t h = item.w[1 + c];
                        uint32_t cm = kSentinel;
                        if ((uint32_t)level + 1 == leafLevel)
                            full &= dag.leaf_fully_filled(dag.ptr(leafLevel, h), cm);
                        else
                            full &= header_fully_filled(dag.ptr(level + 1, h)[0], cm);
                        if (c == 0)
                            material = cm;
                        full &= (cm == material);
                    }
                    if (full)
                        item.w[0] = encode_header_filled(0xFF, material);
                }
                count += full ? 1u : 0u;
            }
            hasFullyFilled = count > 0;
        }
        // Intra-SVO dedup, find in DAG, insert unique, gather (:353-429). Content identity gives
        // the same handle to every copy, which is what the three kernels compute together.
        std::unordered_map<ItemKey, uint32_t, ItemKeyHash> seen;
        for (size_t i = 0; i < items.size(); ++i) {
            const auto& item = items[i];
            const bool isEmpty = item.size == 0
                || (level == (int)leafLevel ? (item.w[0] == 0 && item.w[1] == 0) : header_child_mask(item.w[0]) == 0);
            if (isEmpty) {
                curMapping[i] = kSentinel;
                continue;
            }
            ItemKey k {};
            k.n = dag.item_size(level, item.w);
            std::memcpy(k.w, item.w, k.n * 4);
            auto it = seen.find(k);
            if (it != seen.end()) {
                curMapping[i] = it->second;
                continue;
            }
            bool added = false;
            const uint32_t h = dag.find_or_add(level, item.w, &added);
            ++cnt.unique;
            cnt.added += added ? 1 : 0;
            seen.emplace(k, h);
            curMapping[i] = h;
        }
        prevMapping.swap(curMapping);
    }
    return prevMapping.empty() ? kSentinel : prevMapping[0];
}

void add_undo_frame(Dag& dag, uint32_t root) // MyGPUHashDAGUndoRedo::add_frame, my_gpu_base_dag.h:23-34
{
    if (!dag.undoFrames.empty() && dag.undoFrames.back() == root)
        return;
    dag.redoFrames.clear();
    dag.undoFrames.push_back(root);
}

// ---------------------------------------------------------------- terrain

struct Terrain {
    svdag_terrain_params p;
    uint32_t levels;
    uint32_t baseLog2;
    mutable std::vector<uint32_t> cache; // lazily filled column heights (depth <= 12 only)

    uint32_t lattice(uint32_t ix, uint32_t iz, uint32_t octave) const
    {
        uint32_t h = fmix32(p.seed * 0x9E3779B9u ^ (octave * 0x85EBCA6Bu) ^ 0x68E31DA4u);
        h = fmix32(h ^ (ix * 0xC2B2AE35u));
        h = fmix32(h ^ (iz * 0x27D4EB2Fu));
        return h >> 16;
    }
    uint32_t cell_log2(uint32_t o) const { return baseLog2 > o ? baseLog2 - o : 0; }
    int64_t octave_value(uint32_t x, uint32_t z, uint32_t o) const
    {
        const uint32_t c = cell_log2(o);
        const uint32_t ix = x >> c, iz = z >> c, m = (1u << c) - 1u;
        const auto frac = [&](uint32_t v) -> int64_t {
            const uint32_t f = v & m;
            return c <= 16 ? (int64_t)(f << (16 - c)) : (int64_t)(f >> (c - 16));
        };
        const int64_t sx = smooth16(frac(x)), sz = smooth16(frac(z));
        const int64_t a = lerp16(lattice(ix, iz, o), lattice(ix + 1, iz, o), sx);
        const int64_t b = lerp16(lattice(ix, iz + 1, o), lattice(ix + 1, iz + 1, o), sx);
        return lerp16(a, b, sz);
    }
    uint32_t height_from_fbm(int64_t fbm) const
    {
        const int64_t G = int64_t(1) << levels;
        const int64_t base = G * p.min_height_pct / 100;
        const int64_t range = G * (p.max_height_pct - p.min_height_pct) / 100;
        const int64_t norm = ((int64_t(1) << p.octaves) - 1) * 65536;
        return (uint32_t)(base + (range * fbm) / norm);
    }
    uint32_t height(uint32_t x, uint32_t z) const
    {
        if (levels <= 12) {
            if (cache.empty())
                cache.assign(size_t(1) << (2 * levels), kSentinel);
            uint32_t& c = cache[((size_t)z << levels) | x];
            if (c == kSentinel)
                c = height_uncached(x, z);
            return c;
        }
        return height_uncached(x, z);
    }
    uint32_t height_uncached(uint32_t x, uint32_t z) const
    {
        int64_t f = 0;
        for (uint32_t o = 0; o < p.octaves; ++o)
            f += octave_value(x, z, o) << (p.octaves - 1 - o);
        return height_from_fbm(f);
    }
    // Conservative height bounds over the aligned footprint [x0, x0+s) x [z0, z0+s).
    void bounds(uint32_t x0, uint32_t z0, uint32_t s, uint32_t& hlo, uint32_t& hhi) const
    {
        int64_t lo = 0, hi = 0;
        for (uint32_t o = 0; o < p.octaves; ++o) {
            const uint32_t c = cell_log2(o);
            const uint32_t ix0 = x0 >> c, iz0 = z0 >> c;
            const uint32_t ix1 = ((x0 + s - 1) >> c) + 1, iz1 = ((z0 + s - 1) >> c) + 1;
            int64_t vlo = 65535, vhi = 0;
            if (s <= (1u << c)) {
                // Footprint inside one lattice cell: the field is bilinear in the (monotone) smoothstep
                // weights, so its extremes sit at the footprint corners; integer truncation of the
                // three lerps moves a value by at most 2 units below the real bilinear value.
                const uint32_t x1 = x0 + s - 1, z1 = z0 + s - 1;
                const int64_t v[4] = { octave_value(x0, z0, o), octave_value(x1, z0, o), octave_value(x0, z1, o), octave_value(x1, z1, o) };
                for (int64_t t : v) {
                    vlo = std::min(vlo, t);
                    vhi = std::max(vhi, t);
                }
                vlo = std::max<int64_t>(0, vlo - 2);
                vhi = std::min<int64_t>(65535, vhi + 2);
            } else if ((uint64_t)(ix1 - ix0 + 1) * (iz1 - iz0 + 1) > 64) {
                vlo = 0;
                vhi = 65535;
            } else {
                for (uint32_t iz = iz0; iz <= iz1; ++iz)
                    for (uint32_t ix = ix0; ix <= ix1; ++ix) {
                        const int64_t v = lattice(ix, iz, o);
                        vlo = std::min(vlo, v);
                        vhi = std::max(vhi, v);
                    }
            }
            lo += vlo << (p.octaves - 1 - o);
            hi += vhi << (p.octaves - 1 - o);
        }
        hlo = height_from_fbm(lo);
        hhi = height_from_fbm(hi);
    }
    uint32_t material(uint32_t y) const { return (uint32_t)(((uint64_t)y * p.num_materials) >> levels); }
};

// Boxes and spheres unioned on the terrain surface, drawn from one splitmix64 stream in the order
// the svdag_terrain_params documentation gives.
struct Scene {
    struct Structure {
        int64_t lo[3], hi[3]; // voxel bounding box [lo, hi)
        int64_t c[3];
        int64_t r2;
        bool sphere;
        uint32_t material;
    };
    Terrain t;
    std::vector<Structure> s;
    bool clipped = false; // restrict the scene to the voxel box [rlo, rhi)
    int64_t rlo[3] = {}, rhi[3] = {};
    // 0 = node outside the region, 1 = partly inside, 2 = inside (always 2 without a region)
    int region(int64_t x0, int64_t y0, int64_t z0, int64_t n) const
    {
        if (!clipped)
            return 2;
        const int64_t b[3] = { x0, y0, z0 };
        bool inside = true;
        for (int a = 0; a < 3; ++a) {
            if (b[a] + n <= rlo[a] || b[a] >= rhi[a])
                return 0;
            inside = inside && b[a] >= rlo[a] && b[a] + n <= rhi[a];
        }
        return inside ? 2 : 1;
    }

    static uint64_t splitmix(uint64_t& x)
    {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    Scene(const svdag_terrain_params& p, uint32_t levels) : t { p, levels, levels - 2, {} }
    {
        const uint64_t G = uint64_t(1) << levels;
        uint64_t st = p.structure_seed;
        for (uint32_t i = 0; i < p.num_structures; ++i) {
            const uint64_t x = splitmix(st) % G, z = splitmix(st) % G;
            const bool sphere = splitmix(st) & 1u;
            const uint32_t material = (uint32_t)(splitmix(st) % 16);
            const uint64_t size = splitmix(st);
            const int64_t c[3] = { (int64_t)x, (int64_t)t.height((uint32_t)x, (uint32_t)z), (int64_t)z };
            Structure q {};
            q.sphere = sphere;
            q.material = material;
            if (!sphere) {
                const int64_t side = 16 + (int64_t)(size % 497);
                for (int a = 0; a < 3; ++a) {
                    q.lo[a] = c[a] - side / 2;
                    q.hi[a] = q.lo[a] + side;
                }
            } else {
                const int64_t r = 8 + (int64_t)(size % 249);
                q.r2 = r * r;
                for (int a = 0; a < 3; ++a) {
                    q.c[a] = c[a];
                    q.lo[a] = c[a] - r;
                    q.hi[a] = c[a] + r + 1;
                }
            }
            s.push_back(q);
        }
    }
    bool contains(const Structure& q, int64_t x, int64_t y, int64_t z) const
    {
        if (q.sphere) {
            const int64_t dx = x - q.c[0], dy = y - q.c[1], dz = z - q.c[2];
            return dx * dx + dy * dy + dz * dz <= q.r2;
        }
        return x >= q.lo[0] && x < q.hi[0] && y >= q.lo[1] && y < q.hi[1] && z >= q.lo[2] && z < q.hi[2];
    }
    bool touches(const Structure& q, int64_t x0, int64_t y0, int64_t z0, int64_t n) const
    {
        return x0 < q.hi[0] && x0 + n > q.lo[0] && y0 < q.hi[1] && y0 + n > q.lo[1] && z0 < q.hi[2] && z0 + n > q.lo[2];
    }
    // Material of a voxel (kSentinel = empty), among the structures listed in `active`.
    uint32_t voxel(uint32_t x, uint32_t y, uint32_t z, uint32_t height, const std::vector<uint32_t>& active) const
    {
        for (size_t k = active.size(); k-- > 0;)
            if (contains(s[active[k]], x, y, z))
                return s[active[k]].material;
        return y < height ? t.material(y) : kSentinel;
    }
};

struct BuildResult {
    uint32_t handle;
    uint32_t fillMaterial; // kSentinel unless uniformly filled
};

// Factory-style recursive construction (create_dag_cpu, my_gpu_hash_dag_factory.cpp:317-409):
// children first, fully-filled bits wherever all 8 children are filled with one material,
// find-then-add per item. Height bounds only prune uniform subtrees (they are conservative).
// Structures only add subdivision: a node that any structure's bounding box touches is subdivided
// down to the leaves, where every voxel is evaluated.
BuildResult build_terrain_rec(Dag& dag, const Scene& sc, uint32_t level, const Path& path, const std::vector<uint32_t>& parentActive)
{
    const Terrain& t = sc.t;
    const uint32_t depth = dag.levels - level;
    const uint32_t s = 1u << depth;
    const uint32_t x0 = path.x << depth, y0 = path.y << depth, z0 = path.z << depth;
    const int inRegion = sc.region(x0, y0, z0, s);
    if (inRegion == 0)
        return { kSentinel, kSentinel };
    std::vector<uint32_t> active;
    for (uint32_t i : parentActive)
        if (sc.touches(sc.s[i], x0, y0, z0, s))
            active.push_back(i);
    if (active.empty() && inRegion == 2) {
        uint32_t hlo, hhi;
        t.bounds(x0, z0, s, hlo, hhi);
        if (y0 >= hhi)
            return { kSentinel, kSentinel };
        if (y0 + s <= hlo) {
            const uint32_t m0 = t.material(y0), m1 = t.material(y0 + s - 1);
            if (m0 == m1)
                return { dag.fullyFilled[level][m0], m0 };
        }
    }
    if (level == dag.leaf_level()) {
        uint32_t h[4][4];
        for (uint32_t dx = 0; dx < 4; ++dx)
            for (uint32_t dz = 0; dz < 4; ++dz)
                h[dx][dz] = t.height(x0 + dx, z0 + dz);
        uint32_t leaf[kMaxLeafWords];
        LeafBuilder b { leaf };
        bool allSame = true;
        uint32_t prev = kSentinel;
        uint64_t mask = 0;
        for (uint32_t v = 0; v < 64; ++v) {
            const uint32_t c = v >> 3, f = v & 7u;
            const uint32_t dx = ((c >> 2) & 1u) * 2 + ((f >> 2) & 1u);
            const uint32_t dy = ((c >> 1) & 1u) * 2 + ((f >> 1) & 1u);
            const uint32_t dz = (c & 1u) * 2 + (f & 1u);
            const uint32_t m = sc.region(x0 + dx, y0 + dy, z0 + dz, 1) ? sc.voxel(x0 + dx, y0 + dy, z0 + dz, h[dx][dz], active) : kSentinel;
            if (m != kSentinel) {
                b.set(m);
                mask |= 1ull << v;
                if (v == 0)
                    prev = m;
                allSame &= (m == prev);
                prev = m;
            }
            b.next();
        }
        b.finalize();
        if (mask == 0)
            return { kSentinel, kSentinel };
        const uint32_t handle = dag.find_or_add(level, leaf);
        return { handle, (allSame && mask == ~0ull) ? prev : kSentinel };
    }
    uint32_t node[kMaxNodeWords];
    uint32_t mask = 0, k = 1;
    uint32_t fills[8];
    for (uint32_t c = 0; c < 8; ++c) {
        Path cp = path;
        cp.descend(c);
        const BuildResult r = build_terrain_rec(dag, sc, level + 1, cp, active);
        fills[c] = r.fillMaterial;
        if (r.handle != kSentinel) {
            mask |= 1u << c;
            node[k++] = r.handle;
        }
    }
    if (!mask)
        return { kSentinel, kSentinel };
    bool uniform = fills[0] != kSentinel;
    for (uint32_t c = 1; c < 8; ++c)
        uniform &= fills[c] == fills[0];
    node[0] = uniform ? encode_header_filled(mask, fills[0]) : encode_header(mask);
    return { dag.find_or_add(level, node), uniform ? fills[0] : kSentinel };
}

// createBoxDag, reference test gpu_hash_dag_tests.cpp:35-89.
uint32_t build_box_rec(Dag& dag, const Path& path, uint32_t level, F3 bmin, F3 bmax, uint32_t material)
{
    BoxBase box;
    box.bmin = bmin;
    box.bmax = bmax;
    const uint32_t childLevel = level + 1;
    const uint32_t childDepth = dag.levels - childLevel;
    if (level == dag.leaf_level()) {
        uint32_t leaf[kMaxLeafWords];
        LeafBuilder b { leaf };
        for (uint32_t v = 0; v < 64; ++v) {
            Path vp = path;
            vp.descend(v >> 3);
            vp.descend(v & 7u);
            const F3 p = as_position(vp, 0);
            if (box.overlap(p, add(p, 1.0f)))
                b.set(material);
            b.next();
        }
        b.finalize();
        return dag.find_or_add(level, leaf);
    }
    uint32_t node[kMaxNodeWords];
    uint32_t mask = 0, k = 1;
    for (uint32_t c = 0; c < 8; ++c) {
        Path cp = path;
        cp.descend(c);
        const F3 mn = as_position(cp, childDepth);
        const F3 mx = add(mn, float(1u << childDepth));
        if (box.contained(mn, mx)) {
            node[k++] = dag.fullyFilled[childLevel][material];
            mask |= 1u << c;
        } else if (box.overlap(mn, mx)) {
            node[k++] = build_box_rec(dag, cp, level + 1, bmin, bmax, material);
            mask |= 1u << c;
        }
    }
    node[0] = encode_header(mask);
    return dag.find_or_add(level, node);
}

// ---------------------------------------------------------------- tracer (tracer.cu:28-411)

struct Ray {
    F3 o, d, inv;
    float tmin, tmax;
};
inline float vmax3(F3 v) { return cmax(v.x, cmax(v.y, v.z)); } // cuda_math.h max(float3)
inline float vmin3(F3 v) { return cmin(v.x, cmin(v.y, v.z)); }

uint32_t next_child(uint32_t order, uint32_t mask) // tracer.cu:45-54
{
    for (uint32_t c = 0; c < 8; ++c) {
        const uint32_t ci = c ^ order;
        if (mask & (1u << ci))
            return ci;
    }
    return 0;
}

// compute_intersection_mask, tracer.cu:56-173. The device `max(float,float)` / `min` builtins are
// fmaxf / fminf; the vector max/min of cuda_math.h are the ternary forms above.
uint32_t intersection_mask(bool isRoot, uint32_t level, const Path& path, uint32_t levels, const Ray& ray)
{
    const uint32_t shift = levels - level;
    const float radius = float(1u << (shift - 1));
    const F3 pos = as_position(path, shift);
    const F3 center { radius + pos.x, radius + pos.y, radius + pos.z };
    const F3 crel = sub(center, ray.o);
    const F3 tmid { crel.x * ray.inv.x, crel.y * ray.inv.y, crel.z * ray.inv.z };
    float tmin, tmax;
    {
        const F3 slab { radius * std::fabs(ray.inv.x), radius * std::fabs(ray.inv.y), radius * std::fabs(ray.inv.z) };
        const F3 pmin = sub(tmid, slab);
        tmin = std::fmax(vmax3(pmin), 0.0f);
        const F3 pmax = add(tmid, slab);
        tmax = vmin3(pmax);
    }
    tmin = std::fmax(tmin, ray.tmin);
    tmax = std::fmin(tmax, ray.tmax);
    if (isRoot && (tmin >= tmax))
        return 0;
    uint32_t mask = 0;
    {
        const float tm = 0.5f * (tmin + tmax);
        const F3 p { tm * ray.d.x, tm * ray.d.y, tm * ray.d.z };
        const uint32_t first = ((p.x >= crel.x) ? 4u : 0u) + ((p.y >= crel.y) ? 2u : 0u) + ((p.z >= crel.z) ? 1u : 0u);
        mask |= 1u << first;
    }
    const float eps = 1e-4f;
    if (tmin <= tmid.x && tmid.x <= tmax) {
        const F3 p { tmid.x * ray.d.x, tmid.x * ray.d.y, tmid.x * ray.d.z };
        uint32_t A = 0, B = 0;
        if (p.y >= crel.y - eps)
            A |= 0xCC;
        if (p.y <= crel.y + eps)
            A |= 0x33;
        if (p.z >= crel.z - eps)
            B |= 0xAA;
        if (p.z <= crel.z + eps)
            B |= 0x55;
        mask |= A & B;
    }
    if (tmin <= tmid.y && tmid.y <= tmax) {
        const F3 p { tmid.y * ray.d.x, tmid.y * ray.d.y, tmid.y * ray.d.z };
        uint32_t C = 0, D = 0;
        if (p.x >= crel.x - eps)
            C |= 0xF0;
        if (p.x <= crel.x + eps)
            C |= 0x0F;
        if (p.z >= crel.z - eps)
            D |= 0xAA;
        if (p.z <= crel.z + eps)
            D |= 0x55;
        mask |= C & D;
    }
    if (tmin <= tmid.z && tmid.z <= tmax) {
        const F3 p { tmid.z * ray.d.x, tmid.z * ray.d.y, tmid.z * ray.d.z };
        uint32_t E = 0, F = 0;
        if (p.x >= crel.x - eps)
            E |= 0xF0;
        if (p.x <= crel.x + eps)
            E |= 0x0F;
        if (p.y >= crel.y - eps)
            F |= 0xCC;
        if (p.y <= crel.y + eps)
            F |= 0x33;
        mask |= E & F;
    }
    return mask & 0xFFu;
}

uint32_t leaf_first_child_mask(uint32_t lo, uint32_t hi) // Leaf::get_first_child_mask, base_dag.h:16-52
{
    const uint64_t m = (uint64_t)lo | ((uint64_t)hi << 32);
    uint32_t out = 0;
    for (uint32_t i = 0; i < 8; ++i)
        if ((m >> (8 * i)) & 0xFFull)
            out |= 1u << i;
    return out;
}
uint32_t leaf_second_child_mask(uint32_t lo, uint32_t hi, uint32_t first) // base_dag.h:53-58
{
    const uint32_t shift = (first & 3u) * 8;
    const uint32_t m = (first & 4u) ? hi : lo;
    return (m >> shift) & 0xFFu;
}

struct TraceCounters {
    uint64_t nodes = 0, leaves = 0;
};

// intersect_ray, tracer.cu:186-273.
Path intersect_ray(const Dag& dag, Ray& ray, uint32_t& materialId, TraceCounters* tc)
{
    struct Entry {
        uint32_t index;
        uint32_t childMask;
        uint32_t visitMask;
    };
    const uint32_t order = (ray.d.x < 0.f ? 4u : 0u) + (ray.d.y < 0.f ? 2u : 0u) + (ray.d.z < 0.f ? 1u : 0u);
    uint32_t level = 0, addr = 0;
    Path path {};
    Entry stack[SVDAG_MAX_LEVELS];
    Entry cache;
    uint32_t leafLo = 0, leafHi = 0;
    if (dag.root == kSentinel) { // an empty DAG hits nothing
        materialId = 0xFFFFFFFFu;
        return Path {};
    }
    cache.index = dag.root;
    cache.childMask = header_child_mask(dag.ptr(0, cache.index)[0]);
    cache.visitMask = cache.childMask & intersection_mask(true, 0, path, dag.levels, ray);
    if (tc)
        tc->nodes++;
    for (;;) {
        {
            uint32_t newLevel = level;
            while (newLevel > 0 && !cache.visitMask) {
                newLevel--;
                cache = stack[newLevel];
            }
            if (newLevel == 0 && !cache.visitMask) {
                path = Path {};
                break;
            }
            path.ascend(level - newLevel);
            level = newLevel;
        }
        const uint32_t nextChild = next_child(order, cache.visitMask);
        cache.visitMask &= ~(1u << nextChild);
        path.descend(nextChild);
        stack[level] = cache;
        level++;
        if (level == dag.levels) {
            const uint32_t voxel = leaf_bit_index(path.x, path.y, path.z); // mortonU32() & 63
            if (!leaf_material(dag.ptr(dag.leaf_level(), addr), voxel, materialId))
                materialId = 0xFFFFFFFFu;
            break;
        }
        if (level < dag.leaf_level()) {
            const uint32_t* node = dag.ptr(level - 1, cache.index);
            cache.index = node[1 + child_offset(cache.childMask, nextChild)];
            cache.childMask = header_child_mask(dag.ptr(level, cache.index)[0]);
            cache.visitMask = cache.childMask & intersection_mask(false, level, path, dag.levels, ray);
            if (tc)
                tc->nodes++;
        } else {
            uint32_t childMask;
            if (level == dag.leaf_level()) {
                const uint32_t* node = dag.ptr(level - 1, cache.index);
                addr = node[1 + child_offset(cache.childMask, nextChild)];
                const uint32_t* leaf = dag.ptr(level, addr);
                leafLo = leaf[0];
                leafHi = leaf[1];
                childMask = leaf_first_child_mask(leafLo, leafHi);
                if (tc)
                    tc->leaves++;
            } else {
                childMask = leaf_second_child_mask(leafLo, leafHi, nextChild);
            }
            cache.childMask = childMask;
            cache.visitMask = cache.childMask & intersection_mask(false, level, path, dag.levels, ray);
        }
    }
    return path;
}

// createSurfaceInteraction, tracer.cu:353-389.
void surface_interaction(const Ray& ray, const Path& path, uint32_t materialId, svdag_hit& out)
{
    const F3 bmin = as_position(path, 0);
    const F3 bmax = add(bmin, 1.0f);
    const F3 t1 { (bmin.x - ray.o.x) * ray.inv.x, (bmin.y - ray.o.y) * ray.inv.y, (bmin.z - ray.o.z) * ray.inv.z };
    const F3 t2 { (bmax.x - ray.o.x) * ray.inv.x, (bmax.y - ray.o.y) * ray.inv.y, (bmax.z - ray.o.z) * ray.inv.z };
    const F3 dists { cmin(t1.x, t2.x), cmin(t1.y, t2.y), cmin(t1.z, t2.z) };
    const int axis = dists.x > dists.y ? (dists.x > dists.z ? 0 : 2) : (dists.y > dists.z ? 1 : 2);
    std::memset(&out, 0, sizeof(out));
    out.path[0] = path.x;
    out.path[1] = path.y;
    out.path[2] = path.z;
    out.material = (uint8_t)materialId;
    float t = 0.0f;
    if (axis == 0) {
        out.normal[0] = ray.d.x < 0.0f ? +1.0f : -1.0f;
        out.dpdu[2] = 1.0f;
        out.dpdv[1] = 1.0f;
        t = dists.x;
    } else if (axis == 1) {
        out.normal[1] = ray.d.y < 0.0f ? +1.0f : -1.0f;
        out.dpdu[0] = 1.0f;
        out.dpdv[2] = 1.0f;
        t = dists.y;
    } else {
        out.normal[2] = ray.d.z < 0.0f ? +1.0f : -1.0f;
        out.dpdu[0] = 1.0f;
        out.dpdv[1] = 1.0f;
        t = dists.z;
    }
    out.position[0] = ray.o.x + t * ray.d.x;
    out.position[1] = ray.o.y + t * ray.d.y;
    out.position[2] = ray.o.z + t * ray.d.z;
}

// trace_paths, tracer.cu:391-411 (ray setup in double, normalize = (1/length) * v, cuda_math.h:118).
Ray make_ray(const svdag_trace_params& p, uint32_t px, uint32_t py)
{
    const double dpx = (double)px, dpy = (double)py;
    double v[3];
    for (int i = 0; i < 3; ++i)
        v[i] = ((p.ray_min[i] + dpx * p.ray_ddx[i]) + dpy * p.ray_ddy[i]) - p.camera[i];
    const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double inv = 1 / len;
    Ray r;
    r.o = { (float)p.camera[0], (float)p.camera[1], (float)p.camera[2] };
    r.d = { (float)(inv * v[0]), (float)(inv * v[1]), (float)(inv * v[2]) };
    r.inv = { 1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z };
    r.tmin = 0.0f;
    r.tmax = std::numeric_limits<float>::max();
    return r;
}

// ---------------------------------------------------------------- canonicalisation

uint64_t mix64(uint64_t h)
{
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h;
}

// Merkle digests per reachable item, bottom-up; an item's digest covers its header/leaf words and
// its children's digests, so equal digests mean equal subtrees whatever the handles are.
struct Canon {
    uint32_t levels;
    std::function<const uint32_t*(uint32_t, uint32_t)> fetch;
    std::vector<std::unordered_map<uint32_t, uint64_t>> digest;
    std::vector<std::unordered_map<uint32_t, __uint128_t>> voxels;

    uint64_t visit(uint32_t level, uint32_t handle, __uint128_t& vox)
    {
        auto it = digest[level].find(handle);
        if (it != digest[level].end()) {
            vox = voxels[level][handle];
            return it->second;
        }
        const uint32_t* p = fetch(level, handle);
        uint64_t h = mix64(0x1234567ull + level);
        __uint128_t v = 0;
        if (level == levels - 2) {
            const uint32_t n = leaf_size(p);
            for (uint32_t i = 0; i < n; ++i)
                h = mix64(h ^ p[i]);
            v = popc(p[0]) + popc(p[1]);
        } else {
            const uint32_t mask = header_child_mask(p[0]);
            h = mix64(h ^ p[0]);
            const uint32_t n = popc(mask);
            std::vector<uint32_t> ch(p + 1, p + 1 + n);
            for (uint32_t i = 0; i < n; ++i) {
                __uint128_t cv = 0;
                h = mix64(h ^ visit(level + 1, ch[i], cv));
                v += cv;
            }
        }
        digest[level][handle] = h;
        voxels[level][handle] = v;
        vox = v;
        return h;
    }
    void run(uint32_t root, oracle_canon* out, uint32_t startLevel = 0)
    {
        std::memset(out, 0, sizeof(*out));
        digest.assign(levels, {});
        voxels.assign(levels, {});
        if (root == kSentinel)
            return;
        __uint128_t total = 0;
        out->root_digest = visit(startLevel, root, total);
        out->voxel_count_lo = (uint64_t)total;
        out->voxel_count_hi = (uint64_t)(total >> 64);
        for (uint32_t l = 0; l + 1 < levels; ++l) {
            std::unordered_set<uint64_t> uniq;
            for (auto& [hnd, d] : digest[l])
                uniq.insert(d);
            out->unique_per_level[l] = uniq.size();
            uint64_t acc = 0;
            for (uint64_t d : uniq)
                acc += mix64(d ^ 0x9E3779B97F4A7C15ull);
            out->digest_per_level[l] = acc;
        }
    }
};

} // namespace

struct oracle_dag {
    Dag dag;
};

extern "C" {

oracle_dag* oracle_create(uint32_t levels)
{
    if (levels < SVDAG_MIN_LEVELS || levels > SVDAG_MAX_LEVELS)
        return nullptr;
    auto* o = new oracle_dag();
    o->dag.init(levels);
    return o;
}
void oracle_destroy(oracle_dag* dag) { delete dag; }
uint32_t oracle_levels(const oracle_dag* d) { return d->dag.levels; }
uint32_t oracle_root(const oracle_dag* d) { return d->dag.root; }
int oracle_is_empty(const oracle_dag* d) { return d->dag.root == kSentinel; }

int oracle_build_terrain(oracle_dag* d, const svdag_terrain_params* params)
{
    if (!d || !params || params->octaves == 0 || params->num_materials == 0 || params->num_materials > kNumMaterials
        || params->max_height_pct > 100 || params->min_height_pct > params->max_height_pct)
        return SVDAG_ERR_INVALID;
    d->dag.init(d->dag.levels);
    const Scene sc(*params, d->dag.levels);
    std::vector<uint32_t> all(sc.s.size());
    for (uint32_t i = 0; i < all.size(); ++i)
        all[i] = i;
    d->dag.root = build_terrain_rec(d->dag, sc, 0, Path {}, all).handle;
    return SVDAG_OK;
}

int oracle_build_scene_subtree(oracle_dag* d, const svdag_terrain_params* params, uint32_t level, const uint32_t path[3], uint32_t* out_handle)
{
    if (!d || !params || !path || !out_handle || level >= d->dag.leaf_level() || params->octaves == 0 || params->num_materials == 0)
        return SVDAG_ERR_INVALID;
    d->dag.init(d->dag.levels);
    const Scene sc(*params, d->dag.levels);
    std::vector<uint32_t> all(sc.s.size());
    for (uint32_t i = 0; i < all.size(); ++i)
        all[i] = i;
    Path p {};
    p.x = path[0];
    p.y = path[1];
    p.z = path[2];
    *out_handle = build_terrain_rec(d->dag, sc, level, p, all).handle;
    return SVDAG_OK;
}

int oracle_build_scene_region(oracle_dag* d, const svdag_terrain_params* params, const int64_t lo[3], const int64_t hi[3])
{
    if (!d || !params || !lo || !hi || params->octaves == 0 || params->num_materials == 0)
        return SVDAG_ERR_INVALID;
    d->dag.init(d->dag.levels);
    Scene sc(*params, d->dag.levels);
    sc.clipped = true;
    for (int a = 0; a < 3; ++a) {
        sc.rlo[a] = lo[a];
        sc.rhi[a] = hi[a];
    }
    std::vector<uint32_t> all(sc.s.size());
    for (uint32_t i = 0; i < all.size(); ++i)
        all[i] = i;
    d->dag.root = build_terrain_rec(d->dag, sc, 0, Path {}, all).handle;
    return SVDAG_OK;
}

uint32_t oracle_node_at(const oracle_dag* d, uint32_t level, const uint32_t path[3])
{
    uint32_t h = d->dag.root;
    for (uint32_t l = 0; l < level && h != kSentinel; ++l) {
        const uint32_t* n = d->dag.ptr(l, h);
        const uint32_t sh = level - l - 1;
        const uint32_t c = (((path[0] >> sh) & 1u) << 2) | (((path[1] >> sh) & 1u) << 1) | ((path[2] >> sh) & 1u);
        const uint32_t mask = header_child_mask(n[0]);
        if (!((mask >> c) & 1u))
            return kSentinel;
        h = n[1 + child_offset(mask, c)];
    }
    return h;
}

int oracle_scene_voxels(const svdag_terrain_params* params, uint32_t levels, const uint32_t* xyz, uint64_t count, uint32_t* out)
{
    if (!params || !xyz || !out || params->octaves == 0 || params->num_materials == 0)
        return SVDAG_ERR_INVALID;
    const Scene sc(*params, levels);
    std::vector<uint32_t> all(sc.s.size());
    for (uint32_t i = 0; i < all.size(); ++i)
        all[i] = i;
    for (uint64_t i = 0; i < count; ++i) {
        const uint32_t x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        out[i] = sc.voxel(x, y, z, sc.t.height_uncached(x, z), all);
    }
    return SVDAG_OK;
}

int oracle_build_box(oracle_dag* d, float bmin, float bmax, uint32_t material)
{
    d->dag.init(d->dag.levels);
    d->dag.root = build_box_rec(d->dag, Path {}, 0, F3 { bmin, bmin, bmin }, F3 { bmax, bmax, bmax }, material);
    return SVDAG_OK;
}

static int edit_impl(oracle_dag* d, const svdag_edit* e, svdag_edit_stats* out, uint32_t sourceRoot);

int oracle_edit(oracle_dag* d, const svdag_edit* e, svdag_edit_stats* out)
{
    if (!d || !e || e->tool >= SVDAG_NUM_TOOLS || e->material >= kNumMaterials)
        return SVDAG_ERR_INVALID;
    Dag& dag = d->dag;
    if (e->tool == SVDAG_TOOL_MOVE) { // clear the source box, then paste from the pre-move DAG
        const uint32_t sourceRoot = dag.root;
        svdag_edit rm = *e;
        rm.tool = SVDAG_TOOL_BOX_REMOVE;
        svdag_edit_stats s1 {}, s2 {};
        int r = oracle_edit(d, &rm, &s1);
        if (r)
            return r;
        svdag_edit c = *e;
        c.tool = SVDAG_TOOL_COPY;
        r = edit_impl(d, &c, &s2, sourceRoot);
        if (out) {
            *out = s2;
            out->root_before = s1.root_before;
            out->edited_voxels += s1.edited_voxels;
        }
        return r;
    }
    return edit_impl(d, e, out, dag.root);
}

static int edit_impl(oracle_dag* d, const svdag_edit* e, svdag_edit_stats* out, uint32_t sourceRoot)
{
    Dag& dag = d->dag;
    add_undo_frame(dag, dag.root); // my_gpu_hash_dag_edits.cu:638-640
    Editor ed = make_editor(*e, dag);
    ed.copyRoot = sourceRoot;
    std::vector<std::vector<SvoItem>> svo;
    EditCounters cnt;
    const uint32_t before = dag.root;
    if (build_svo(dag, ed, svo, cnt)) {
        if (!svo[dag.leaf_level()].empty())
            dag.root = merge_svo(dag, svo, cnt, false);
    }
    if (out) {
        std::memset(out, 0, sizeof(*out));
        for (uint32_t l = 0; l < SVDAG_MAX_LEVELS; ++l)
            out->svo_nodes[l] = cnt.svo[l];
        out->old_items_read = cnt.oldRead;
        out->unique_items = cnt.unique;
        out->new_items = cnt.added;
        out->edited_voxels = cnt.edited;
        out->root_before = before;
        out->root_after = dag.root;
    }
    return SVDAG_OK;
}

int oracle_undo(oracle_dag* d) // my_gpu_base_dag.h:35-49
{
    Dag& dag = d->dag;
    if (dag.undoFrames.empty())
        return SVDAG_OK;
    const uint32_t f = dag.undoFrames.back();
    dag.undoFrames.pop_back();
    dag.redoFrames.push_back(dag.root);
    dag.root = f;
    return SVDAG_OK;
}
int oracle_redo(oracle_dag* d) // my_gpu_base_dag.h:50-64
{
    Dag& dag = d->dag;
    if (dag.redoFrames.empty())
        return SVDAG_OK;
    const uint32_t f = dag.redoFrames.back();
    dag.redoFrames.pop_back();
    dag.undoFrames.push_back(dag.root);
    dag.root = f;
    return SVDAG_OK;
}
// garbageCollect (my_gpu_base_dag.h:66-77, my_gpu_hash_dag.cu:305-362): clears the history and keeps
// what is reachable from the root and from the canonical fully-filled nodes. Re-packing the oracle's
// storage keeps its structure identical, which is all the GC may change.
int oracle_gc(oracle_dag* d)
{
    Dag& dag = d->dag;
    dag.undoFrames.clear();
    dag.redoFrames.clear();
    Dag fresh;
    fresh.init(dag.levels);
    std::vector<std::unordered_map<uint32_t, uint32_t>> remap(dag.levels);
    std::function<uint32_t(uint32_t, uint32_t)> copy = [&](uint32_t level, uint32_t h) -> uint32_t {
        auto it = remap[level].find(h);
        if (it != remap[level].end())
            return it->second;
        const uint32_t* p = dag.ptr(level, h);
        uint32_t buf[kMaxLeafWords] = {};
        const uint32_t n = dag.item_size(level, p);
        std::memcpy(buf, p, n * 4);
        if (level != dag.leaf_level())
            for (uint32_t i = 1; i < n; ++i)
                buf[i] = copy(level + 1, p[i]);
        const uint32_t nh = fresh.find_or_add(level, buf);
        remap[level][h] = nh;
        return nh;
    };
    if (dag.root != kSentinel)
        fresh.root = copy(0, dag.root);
    dag = std::move(fresh);
    return SVDAG_OK;
}
uint32_t oracle_undo_count(const oracle_dag* d) { return (uint32_t)d->dag.undoFrames.size(); }
uint32_t oracle_redo_count(const oracle_dag* d) { return (uint32_t)d->dag.redoFrames.size(); }

int oracle_sample_voxels(const oracle_dag* d, const uint32_t* xyz, uint64_t count, uint32_t* out)
{
    for (uint64_t i = 0; i < count; ++i) {
        const Path p { xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2] };
        const auto v = get_value(d->dag, p);
        out[i] = v ? *v : SVDAG_NO_MATERIAL;
    }
    return SVDAG_OK;
}

int oracle_export_items(const oracle_dag* d, uint32_t* out, uint64_t capacity, uint64_t* count)
{
    const Dag& g = d->dag;
    *count = 0;
    if (g.root == kSentinel)
        return 0;
    // Breadth first, level by level: ids are assigned in order of first appearance.
    std::vector<std::vector<uint32_t>> order(g.levels - 1);
    std::vector<std::unordered_map<uint32_t, uint64_t>> id(g.levels - 1);
    order[0].push_back(g.root);
    id[0][g.root] = 0;
    uint64_t next = 1;
    for (uint32_t level = 0; level < g.leaf_level(); ++level) {
        for (uint32_t h : order[level]) {
            const uint32_t* p = g.ptr(level, h);
            const uint32_t n = (uint32_t)__builtin_popcount(header_child_mask(p[0]));
            for (uint32_t j = 0; j < n; ++j)
                if (id[level + 1].emplace(p[1 + j], 0).second)
                    order[level + 1].push_back(p[1 + j]);
        }
        uint64_t base = next;
        for (uint32_t c : order[level + 1])
            id[level + 1][c] = base++;
        next = base;
    }
    *count = next;
    if (capacity < next)
        return 1;
    for (uint32_t level = 0; level <= g.leaf_level(); ++level) {
        for (uint32_t h : order[level]) {
            uint32_t* o = out + id[level][h] * 10ull;
            for (uint32_t j = 0; j < 10; ++j)
                o[j] = 0;
            const uint32_t* p = g.ptr(level, h);
            const uint32_t n = g.item_size(level, p);
            for (uint32_t j = 0; j < n; ++j)
                o[j] = p[j];
            if (level < g.leaf_level()) {
                const uint32_t k = (uint32_t)__builtin_popcount(header_child_mask(p[0]));
                for (uint32_t j = 0; j < k; ++j)
                    o[1 + j] = (uint32_t)id[level + 1][p[1 + j]];
            }
        }
    }
    return 0;
}

int oracle_trace(const oracle_dag* d, const svdag_trace_params* p, svdag_hit* out, int threads)
{
    const uint32_t W = p->width, H = p->height;
    const auto work = [&](uint32_t y0, uint32_t y1) {
        for (uint32_t y = y0; y < y1; ++y)
            for (uint32_t x = 0; x < W; ++x) {
                Ray ray = make_ray(*p, x, y);
                uint32_t mat = 0xFFFFFFFFu;
                const Path path = intersect_ray(d->dag, ray, mat, nullptr);
                if (path.x == 0 && path.y == 0 && path.z == 0)
                    mat = 0xFFFFFFFFu; // a miss carries no material (the reference leaves it unset)
                surface_interaction(ray, path, mat, out[(size_t)(H - 1 - y) * W + x]);
            }
    };
    if (threads <= 1) {
        work(0, H);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
            pool.emplace_back(work, H * t / threads, H * (t + 1) / threads);
        for (auto& th : pool)
            th.join();
    }
    return SVDAG_OK;
}

int oracle_trace_counts(const oracle_dag* d, const svdag_trace_params* p, uint64_t* nodes, uint64_t* leaves, uint64_t* hits)
{
    TraceCounters tc;
    uint64_t h = 0;
    for (uint32_t y = 0; y < p->height; ++y)
        for (uint32_t x = 0; x < p->width; ++x) {
            Ray ray = make_ray(*p, x, y);
            uint32_t mat = 0;
            const Path path = intersect_ray(d->dag, ray, mat, &tc);
            h += !(path.x == 0 && path.y == 0 && path.z == 0);
        }
    *nodes = tc.nodes;
    *leaves = tc.leaves;
    *hits = h;
    return SVDAG_OK;
}

// ---------------------------------------------------------------- shading (tracer.cu:413-730)

namespace {

// intersect_ray_node_out_of_order, tracer.cu:275-352: any voxel on the ray within [tmin, tmax].
bool any_hit(const Dag& dag, const Ray& ray)
{
    struct Entry {
        uint32_t index;
        uint32_t childMask;
        uint32_t visitMask;
    };
    if (dag.root == kSentinel)
        return false;
    uint32_t level = 0;
    Path path {};
    Entry stack[SVDAG_MAX_LEVELS];
    Entry cache;
    uint32_t leafLo = 0, leafHi = 0;
    cache.index = dag.root;
    cache.childMask = header_child_mask(dag.ptr(0, cache.index)[0]);
    cache.visitMask = cache.childMask & intersection_mask(true, 0, path, dag.levels, ray);
    for (;;) {
        {
            uint32_t newLevel = level;
            while (newLevel > 0 && !cache.visitMask) {
                newLevel--;
                cache = stack[newLevel];
            }
            if (newLevel == 0 && !cache.visitMask)
                return false;
            path.ascend(level - newLevel);
            level = newLevel;
        }
        const uint32_t nextChild = 31u - (uint32_t)__builtin_clz(cache.visitMask);
        cache.visitMask &= ~(1u << nextChild);
        path.descend(nextChild);
        stack[level] = cache;
        level++;
        if (level == dag.levels)
            return true;
        if (level < dag.leaf_level()) {
            const uint32_t* node = dag.ptr(level - 1, cache.index);
            cache.index = node[1 + child_offset(cache.childMask, nextChild)];
            cache.childMask = header_child_mask(dag.ptr(level, cache.index)[0]);
            cache.visitMask = cache.childMask & intersection_mask(false, level, path, dag.levels, ray);
        } else {
            uint32_t childMask;
            if (level == dag.leaf_level()) {
                const uint32_t* node = dag.ptr(level - 1, cache.index);
                const uint32_t* leaf = dag.ptr(level, node[1 + child_offset(cache.childMask, nextChild)]);
                leafLo = leaf[0];
                leafHi = leaf[1];
                childMask = leaf_first_child_mask(leafLo, leafHi);
            } else {
                childMask = leaf_second_child_mask(leafLo, leafHi, nextChild);
            }
            cache.childMask = childMask;
            cache.visitMask = cache.childMask & intersection_mask(false, level, path, dag.levels, ray);
        }
    }
}

Ray ray_create(F3 o, F3 dir, float tmax) // Ray::create, tracer.cu:32-41
{
    Ray r;
    r.o = o;
    r.d = dir;
    r.inv = { 1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z };
    r.tmin = 0.0f;
    r.tmax = tmax;
    return r;
}

struct Pcg { // Utils::PCG_RNG, utils.h:45-78
    uint64_t state = 0x853c49e6748fea9bull, inc;
    explicit Pcg(uint64_t stream)
        : inc(stream)
    {
        next();
        next();
    }
    uint32_t next()
    {
        const uint64_t old = state;
        state = old * 6364136223846793005ull + (inc | 1ull);
        const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((0xFFFFFFFFu - rot + 1u) & 31u));
    }
    float next_float() { return float(next()) / 4294967296.0f; }
};

// sin and cos of x in [0, 2 pi] by quadrant reduction and Taylor polynomials (the library evaluates
// the same operations, so sample directions agree exactly).
void sincos_quadrant(float x, float& s, float& c)
{
    const float k = std::rint(x * 0.63661975f);
    const float r = (float)((double)x - (double)k * 1.5707963267948966);
    const float r2 = r * r;
    const float sp = r + (r * r2) * (-0.16666667f + r2 * (0.008333334f + r2 * (-0.0001984127f + r2 * 2.7557319e-06f)));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (0.041666668f + r2 * (-0.0013888889f + r2 * 2.4801588e-05f)));
    switch ((int)k & 3) {
    case 0:
        s = sp;
        c = cp;
        break;
    case 1:
        s = cp;
        c = -sp;
        break;
    case 2:
        s = -sp;
        c = -cp;
        break;
    default:
        s = -cp;
        c = sp;
        break;
    }
}

float srgb_to_linear(float v) // ColorUtils::accurateSRGBToLinear, color_utils.h:233-242
{
    const float lo = v / 12.92f;
    const float hi = std::pow((v + 0.055f) / 1.055f, 2.4f);
    return (v <= 0.04045f) ? lo : hi;
}
float linear_to_srgb(float v) // ColorUtils::accurateLinearToSRGB, :243-252
{
    const float lo = v * 12.92f;
    const float hi = (std::pow(std::fabs(v), 1.0f / 2.4f) * 1.055f) - 0.055f;
    return (v <= 0.0031308f) ? lo : hi;
}
uint32_t to_rgb888(float r, float g, float b) // ColorUtils::float3_to_rgb888, :31-37
{
    r = std::fmax(0.f, std::fmin(r, 1.f));
    g = std::fmax(0.f, std::fmin(g, 1.f));
    b = std::fmax(0.f, std::fmin(b, 1.f));
    return (uint32_t(r * 255.0f) << 0) | (uint32_t(g * 255.0f) << 8) | (uint32_t(b * 255.0f) << 16) | 0xff000000u;
}

void shade_pixel(const Dag& dag, const svdag_trace_params& tp, const svdag_shade_params& sp, uint32_t x, uint32_t y, svdag_hit& si,
    uint32_t& rgba, float& sunOut, float& aoOut)
{
    const bool hit = si.path[0] != 0 || si.path[1] != 0 || si.path[2] != 0;
    uint32_t diffuse; // computeColorAtSurface, tracer.cu:413-445
    if (!hit) {
        diffuse = to_rgb888(0.f, 0.f, 0.f);
    } else if (si.material < SVDAG_NUM_MATERIALS) {
        diffuse = (sp.material_srgb8[si.material] & 0x00FFFFFFu) | 0xff000000u;
    } else {
        const float b = float((si.path[0] ^ si.path[1] ^ si.path[2]) & 1u);
        diffuse = to_rgb888(1.f, b, 1.f - b);
    }
    si.color = diffuse;
    const F3 pos { si.position[0], si.position[1], si.position[2] };
    const F3 n { si.normal[0], si.normal[1], si.normal[2] };
    const F3 sun { sp.sun_direction[0], sp.sun_direction[1], sp.sun_direction[2] };
    float sunVis = 0.f, ao = 0.f;
    if (hit && (sp.flags & SVDAG_SHADE_SHADOWS)) { // trace_shadows, tracer.cu:609-628
        const Ray r = ray_create({ pos.x + sp.shadow_bias * sun.x, pos.y + sp.shadow_bias * sun.y, pos.z + sp.shadow_bias * sun.z }, sun,
            std::numeric_limits<float>::max());
        const bool occluded = any_hit(dag, r);
        const float ndotl = std::fmax((n.x * r.d.x + n.y * r.d.y) + n.z * r.d.z, 0.0f);
        sunVis = occluded ? 0.0f : ndotl;
    }
    if (hit && (sp.flags & SVDAG_SHADE_AO) && sp.ao_samples) { // trace_ambient_occlusion, tracer.cu:654-683
        const uint64_t seed = (uint64_t)(y * tp.width + x) * (sp.random_seed > 1ull ? sp.random_seed : 1ull);
        Pcg rng(seed);
        uint32_t samples = 0, open = 0;
        const F3 o { pos.x + n.x * sp.shadow_bias, pos.y + n.y * sp.shadow_bias, pos.z + n.z * sp.shadow_bias };
        for (uint32_t k = 0; k < sp.ao_samples; ++k) {
            const float ux = rng.next_float();
            const float uy = rng.next_float();
            const float rr = std::sqrt(ux);
            const float theta = 6.2831855f * uy;
            float sn, cs;
            sincos_quadrant(theta, sn, cs);
            const float lx = rr * cs, ly = rr * sn, lz = std::sqrt(std::fmax(0.0f, 1 - ux));
            const F3 w { (lx * si.dpdu[0] + ly * si.dpdv[0]) + lz * n.x, (lx * si.dpdu[1] + ly * si.dpdv[1]) + lz * n.y,
                (lx * si.dpdu[2] + ly * si.dpdv[2]) + lz * n.z };
            if (!any_hit(dag, ray_create(o, w, sp.ao_ray_length)))
                open += 1;
            samples += 1;
        }
        ao = (float)open / (float)samples;
    }
    sunOut = sunVis;
    aoOut = ao;
    const float skyR = 187.f / 255.f, skyG = 242.f / 255.f, skyB = 250.f / 255.f; // trace_lighting, tracer.cu:701-730
    float sr, sg, sb;
    if (!hit) {
        sr = skyR;
        sg = skyG;
        sb = skyB;
    } else {
        const float kr = srgb_to_linear(float((diffuse >> 0) & 0xFFu) / 255.0f);
        const float kg = srgb_to_linear(float((diffuse >> 8) & 0xFFu) / 255.0f);
        const float kb = srgb_to_linear(float((diffuse >> 16) & 0xFFu) / 255.0f);
        const float occl = (sp.flags & SVDAG_SHADE_AO) && sp.ao_samples ? ao : 1.0f;
        const float vis = (sp.flags & SVDAG_SHADE_SHADOWS) ? sunVis : 1.0f;
        const float a = occl * 0.5f;
        sr = ((a * skyR) + ((vis * 0.95f) * sp.sun_brightness)) * kr;
        sg = ((a * skyG) + ((vis * 0.94f) * sp.sun_brightness)) * kg;
        sb = ((a * skyB) + ((vis * 0.47f) * sp.sun_brightness)) * kb;
        if (sp.fog_density > 0.0f) { // applyFog, tracer.cu:685-699
            double v[3];
            for (int i = 0; i < 3; ++i)
                v[i] = ((tp.ray_min[i] + (double)x * tp.ray_ddx[i]) + (double)y * tp.ray_ddy[i]) - tp.camera[i];
            const double inv = 1.0 / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            const float dx = (float)(v[0] * inv), dy = (float)(v[1] * inv), dz = (float)(v[2] * inv);
            const float ex = (float)tp.camera[0] - pos.x, ey = (float)tp.camera[1] - pos.y, ez = (float)tp.camera[2] - pos.z;
            const float density = sp.fog_density * 0.00001f;
            const float amount = 1.0f - std::exp(-std::sqrt((ex * ex + ey * ey) + ez * ez) * density);
            const float sunAmount = 1.01f * std::fmax((dx * sun.x + dy * sun.y) + dz * sun.z, 0.0f);
            const float t = std::pow(sunAmount, 30.0f);
            const float fr = skyR + t * (1.0f - skyR), fg = skyG + t * (1.0f - skyG), fb = skyB + t * (1.0f - skyB);
            const float f = std::fmax(0.0f, std::fmin(amount, 1.0f));
            sr = sr + f * (fr - sr);
            sg = sg + f * (fg - sg);
            sb = sb + f * (fb - sb);
        }
    }
    rgba = to_rgb888(linear_to_srgb(sr), linear_to_srgb(sg), linear_to_srgb(sb));
}

} // namespace

void oracle_sincos(float x, float* s, float* c) { sincos_quadrant(x, *s, *c); }

int oracle_shade(const oracle_dag* d, const svdag_trace_params* tp, const svdag_shade_params* sp, svdag_hit* hits, uint32_t* rgba, float* sun,
    float* ao, int threads)
{
    const uint32_t W = tp->width, H = tp->height;
    const auto work = [&](uint32_t y0, uint32_t y1) {
        for (uint32_t y = y0; y < y1; ++y)
            for (uint32_t x = 0; x < W; ++x) {
                const size_t i = (size_t)y * W + x;
                shade_pixel(d->dag, *tp, *sp, x, y, hits[i], rgba[i], sun[i], ao[i]);
            }
    };
    if (threads <= 1) {
        work(0, H);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
            pool.emplace_back(work, H * t / threads, H * (t + 1) / threads);
        for (auto& th : pool)
            th.join();
    }
    return SVDAG_OK;
}

int oracle_canonicalize(const oracle_dag* d, oracle_canon* out)
{
    Canon c;
    c.levels = d->dag.levels;
    const Dag* dag = &d->dag;
    c.fetch = [dag](uint32_t level, uint32_t h) { return dag->ptr(level, h); };
    c.run(d->dag.root, out);
    return SVDAG_OK;
}

int oracle_canonicalize_at(const oracle_dag* d, uint32_t level, uint32_t handle, oracle_canon* out)
{
    Canon c;
    c.levels = d->dag.levels;
    const Dag* dag = &d->dag;
    c.fetch = [dag](uint32_t l, uint32_t h) { return dag->ptr(l, h); };
    c.run(handle, out, level);
    return SVDAG_OK;
}

int oracle_canonicalize_dump_at(uint32_t levels, uint32_t level, uint32_t root, const uint32_t* const* handles,
    const uint32_t* const* words, const uint64_t* counts, oracle_canon* out);

int oracle_canonicalize_dump(uint32_t levels, uint32_t root, const uint32_t* const* handles, const uint32_t* const* words,
    const uint64_t* counts, oracle_canon* out)
{
    return oracle_canonicalize_dump_at(levels, 0, root, handles, words, counts, out);
}

int oracle_canonicalize_dump_at(uint32_t levels, uint32_t level, uint32_t root, const uint32_t* const* handles,
    const uint32_t* const* words, const uint64_t* counts, oracle_canon* out)
{
    std::vector<std::unordered_map<uint32_t, uint64_t>> where(levels);
    for (uint32_t l = 0; l + 1 < levels; ++l)
        for (uint64_t i = 0; i < counts[l]; ++i)
            where[l][handles[l][i]] = i;
    bool bad = false;
    Canon c;
    c.levels = levels;
    static const uint32_t zeros[kMaxLeafWords] = {};
    c.fetch = [&](uint32_t level, uint32_t h) -> const uint32_t* {
        auto it = where[level].find(h);
        if (it == where[level].end()) {
            bad = true;
            return zeros;
        }
        return &words[level][it->second * SVDAG_MAX_ITEM_WORDS];
    };
    c.run(root, out, level);
    return bad ? SVDAG_ERR_CORRUPT : SVDAG_OK;
}

uint32_t oracle_encode_node_header(uint32_t child_mask, uint32_t user_payload)
{
    return encode_header_payload(child_mask, user_payload);
}
uint32_t oracle_header_child_mask(uint32_t header) { return header_child_mask(header); }
uint32_t oracle_header_user_payload(uint32_t header) { return header_payload(header); }
uint32_t oracle_build_leaf(uint64_t mask, const uint32_t* materials, uint32_t* out_words)
{
    LeafBuilder b { out_words };
    for (uint32_t i = 0; i < 64; ++i) {
        if ((mask >> i) & 1u)
            b.set(materials[i] & (kNumMaterials - 1u));
        b.next();
    }
    return b.finalize();
}
uint32_t oracle_leaf_size(const uint32_t* leaf) { return leaf_size(leaf); }
int oracle_leaf_material(const uint32_t* leaf, uint32_t voxel, uint32_t* out) { return leaf_material(leaf, voxel, *out) ? 1 : 0; }
uint32_t oracle_terrain_height(const svdag_terrain_params* params, uint32_t levels, uint32_t x, uint32_t z)
{
    Terrain t { *params, levels, levels - 2, {} };
    return t.height_uncached(x, z);
}
uint32_t oracle_noise_material(uint32_t seed, uint32_t cell_log2, uint32_t x, uint32_t y, uint32_t z)
{
    return noise_material(seed, cell_log2, x, y, z);
}
int oracle_should_edit(const svdag_edit* e, const uint32_t path[3], uint32_t depth, uint32_t state, uint32_t fill,
    uint32_t* out_fill)
{
    Dag empty;
    const Editor ed = make_editor(*e, empty);
    const Path p { path[0], path[1], path[2] };
    const NodeDesc desc { state == 0 ? State::Partial : state == 1 ? State::Filled : State::Empty, fill };
    const EditDesc d = ed.should_edit(p, depth, desc);
    if (out_fill)
        *out_fill = d.fillMaterial;
    return (int)d.op;
}

int oracle_should_edit_many(const svdag_edit* e, const uint32_t* paths, const uint32_t* depths, const uint32_t* states,
    const uint32_t* fills, uint64_t n, int32_t* ops, uint32_t* out_fills)
{
    for (uint64_t i = 0; i < n; ++i)
        ops[i] = oracle_should_edit(e, paths + 3 * i, depths[i], states[i], fills[i], out_fills + i);
    return 0;
}

void oracle_camera_params(const double pos[3], const double target[3], double fovDeg, uint32_t W, uint32_t H,
    svdag_trace_params* out)
{
    double f[3] = { target[0] - pos[0], target[1] - pos[1], target[2] - pos[2] };
    double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (double& v : f)
        v /= fl;
    double wu[3] = { 0, 1, 0 };
    if (std::fabs(f[1]) > 0.999)
        wu[0] = 0, wu[1] = 0, wu[2] = 1;
    double r[3] = { f[1] * wu[2] - f[2] * wu[1], f[2] * wu[0] - f[0] * wu[2], f[0] * wu[1] - f[1] * wu[0] };
    double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (double& v : r)
        v /= rl;
    double u[3] = { r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0] };
    const double fov = fovDeg / 2.0 * (3.14159265358979323846 / 180.);
    const double aspect = double(W) / double(H);
    double X[3], Y[3], Z[3], bl[3], br[3], tl[3];
    for (int i = 0; i < 3; ++i) {
        X[i] = r[i] * std::sin(fov) * aspect;
        Y[i] = u[i] * std::sin(fov);
        Z[i] = f[i] * std::cos(fov);
        bl[i] = pos[i] + Z[i] - Y[i] - X[i];
        br[i] = pos[i] + Z[i] - Y[i] + X[i];
        tl[i] = pos[i] + Z[i] + Y[i] - X[i];
    }
    for (int i = 0; i < 3; ++i) {
        out->camera[i] = pos[i];
        out->ray_min[i] = bl[i];
        out->ray_ddx[i] = (br[i] - bl[i]) * (1.0 / W);
        out->ray_ddy[i] = (tl[i] - bl[i]) * (1.0 / H);
    }
    out->width = W;
    out->height = H;
}

} // extern "C"
