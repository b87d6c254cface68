// svdag_v3.cu - the reference's own DAG file: MyGPUHashDAG::writeTo / readFrom, format version 3
// (my_gpu_hash_dag.cu:158-177), converted to and from item snapshots on the host.
//
// The file is the raw state of the reference's hash tables as its BinaryWriter serialises them
// (binary_writer.h:84-116: a trivially copyable field as its bytes; array.h:30-53: a StaticArray as
// its size, its EMemoryType and its elements; array.h:311-315: a DynamicArray adds its allocated
// size), in the reference's default configuration (configuration/gpu_hash_dag_definitions.h:
// CompactAccelerationHash tables, SlabHashXor buckets, the first slab of every bucket stored in the
// table; 4 material bits; CAPTURE_MEMORY_STATS_SLOW off), all little-endian:
//
//   u32 version = 3
//   fullyFilledNodes, StaticArray2D<u32> (array2d.h:113-118): {u64 n, u32 memory type, n words},
//       u32 width = the scene depth, u32 height = 16 materials; word [material * width + level] is
//       the handle of the item of that level fully filled with that material
//   u32 firstNodeIndex: the root's handle (0xFFFFFFFF for an empty DAG)
//   hashTables: {u64 9, u32 memory type}, then per item size 2..10 words (gpu_hash_table_base.cu:
//       117-137):
//     u32 itemSizeInU32, u32 slabSizeInU32 = 10 + 32 * item size, u32 numBuckets
//     m_table, StaticArray<u32, u32 size>: {u32 n = numBuckets * slab size, u32 memory type, n words}
//     DynamicSlabAllocator (dynamic_slab_alloc.cu:172-179): u32 memUnitSizeInU32 = slab size,
//       u32 superBlockSizeInU32 = 512 + 16384 * slab size, superBlocksCPU {u64 n, u32 memory type,
//       n x {u64 super block words, u32 memory type, words}, u64 n}, u32 allocated units
//     u32 numItems, u32 numSlabs
//
// A slab (compact_acceleration_hash_table.h:510-531) is 8 words of 8-bit tags (slot j in word j/4
// at bit 8 * (j % 4), 0 = empty; the tag is computeAccelerationHash, :478-489), the next-slab
// pointer (0xFFFFFFFF ends the chain), the collector's active mask, then 32 item slots. A super
// block (dynamic_slab_alloc.h:355-369) is 512 bitmap words, one bit per memory unit, then 16384
// units of one slab each; a unit pointer is super block << 14 | unit. An item pointer
// (gpu_hash_table_base.h:310-321) is slab << 6 | in-table << 5 | slot, where the slab is the bucket
// for a first slab and the unit pointer otherwise. A DAG handle (my_gpu_base_dag.h:334-342) is
// (item size - 2 for a node, - 3 for a leaf) << 29 | item pointer; the table of an item is its
// size - 2, so a node and a leaf of equal words are one item. The bucket of an item is xorHash32xN
// (utils.h:386-403) modulo the bucket count.
//
// Reading follows the handles from the root and emits each level's items in first-visit order.
// Writing lays every distinct item out as the reference's host insert (compact_acceleration_hash_
// table.h:27-57) would place it: the fully-filled items first (MyGPUHashDAG::allocate,
// my_gpu_hash_dag.cu:29-65), then the snapshot bottom-up, tables sized to 96 items per bucket
// (TARGET_LOAD_FACTOR, applied by setLoadFactor, my_gpu_hash_dag.cu:138-155), overflow slabs taken
// from the allocator in order.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "svdag_hash.h"
#include "svdag_snapshot.h"

#include "../../include/svdag.h"

namespace {

using svdag::leaf_words;
using svdag::node_words;

constexpr uint32_t kVersion = 3;
constexpr uint32_t kMinItem = 2, kTables = 9; // item sizes 2..10
constexpr uint32_t kMaterials = 16;
constexpr uint32_t kTagWords = 8, kNextWord = 8, kItemsAt = 10, kSlots = 32;
static_assert(kTagWords * 4 == kSlots && kNextWord == kTagWords, "one tag byte per slot, then the next pointer");
constexpr uint32_t kEnd = 0xFFFFFFFFu; // next_sentinel; also the empty DAG's root
constexpr uint32_t kBitmapWords = 512, kUnitsPerSuper = 16384;
constexpr uint32_t kPtrBits = 29, kPtrMask = (1u << kPtrBits) - 1u;
constexpr uint32_t kMaxSlab = 1u << (kPtrBits - 6); // slab field of a pointer that fits a handle
constexpr uint32_t kLoadFactor = 96;
constexpr uint32_t kMemCPU = 3, kMemTypes = 4; // EMemoryType: GPU_Managed, GPU_Malloc, GPU_Async, CPU

uint32_t slab_words(uint32_t itemWords) { return kItemsAt + kSlots * itemWords; }

// Utils::xorHash32xN (utils.h:395-403): 32-bit products and sums, a 32-bit modulo by the largest
// 32-bit prime.
uint32_t bucket_hash(const uint32_t* w, uint32_t n)
{
    uint32_t seed = 0;
    for (uint32_t i = 0; i < n; ++i)
        seed ^= (2717583853u * w[i] + i * 1117415409u) % 4294967291u;
    return seed;
}
// CompactAccelerationHashTable::computeAccelerationHash (compact_acceleration_hash_table.h:478-489).
uint32_t tag_hash(const uint32_t* w, uint32_t n)
{
    uint32_t t = 0;
    for (uint32_t i = 0; i < n; ++i)
        t ^= (32u - i) * w[i];
    t &= 0xFFu;
    return t == 0 ? 1u : t;
}

// ------------------------------------------------------------------ reading

struct Cursor {
    const uint8_t* p;
    uint64_t n, at = 0;
    bool bad = false;
    template <class T>
    T get()
    {
        T v {};
        if (bad || n - at < sizeof(T)) {
            bad = true;
            return v;
        }
        std::memcpy(&v, p + at, sizeof(T));
        at += sizeof(T);
        return v;
    }
    const uint32_t* words(uint64_t count)
    {
        if (bad || (n - at) / 4 < count) {
            bad = true;
            return nullptr;
        }
        const uint32_t* q = reinterpret_cast<const uint32_t*>(p + at);
        at += count * 4;
        return q;
    }
    bool memory_type() { return get<uint32_t>() < kMemTypes; }
};

struct Table {
    uint32_t itemWords = 0, slabWords = 0, buckets = 0;
    const uint32_t* first = nullptr; // buckets * slabWords
    std::vector<const uint32_t*> supers; // 512 bitmap words + 16384 slabs each
};

// Address of the item at pointer `ptr` of table t, or null when the pointer does not name an
// occupied slot (the reference's isValidSlab plus the slot's tag).
const uint32_t* locate(const Table& t, uint32_t ptr)
{
    const uint32_t slot = ptr & 31u, slab = ptr >> 6;
    const uint32_t* s;
    if (ptr >> 5 & 1u) {
        if (slab >= t.buckets)
            return nullptr;
        s = t.first + (uint64_t)slab * t.slabWords;
    } else {
        const uint32_t sb = slab / kUnitsPerSuper, unit = slab % kUnitsPerSuper;
        if (sb >= t.supers.size() || !(t.supers[sb][unit >> 5] >> (unit & 31u) & 1u))
            return nullptr;
        s = t.supers[sb] + kBitmapWords + (uint64_t)unit * t.slabWords;
    }
    if (!(s[slot >> 2] >> ((slot & 3u) * 8u) & 0xFFu))
        return nullptr;
    return s + kItemsAt + (uint64_t)slot * t.itemWords;
}

svdag_status parse(Cursor& c, uint32_t levels, uint32_t& root, Table (&tables)[kTables])
{
    if (c.get<uint32_t>() != kVersion)
        return c.bad ? SVDAG_ERR_CORRUPT : SVDAG_ERR_UNSUPPORTED;
    const uint64_t ffCount = c.get<uint64_t>();
    if (!c.memory_type())
        return SVDAG_ERR_CORRUPT;
    c.words(ffCount);
    const uint32_t width = c.get<uint32_t>(), height = c.get<uint32_t>();
    if (c.bad)
        return SVDAG_ERR_CORRUPT;
    if (height != kMaterials || ffCount != (uint64_t)width * height)
        return SVDAG_ERR_UNSUPPORTED;
    if (width != levels)
        return SVDAG_ERR_INVALID;
    root = c.get<uint32_t>();
    if (c.get<uint64_t>() != kTables)
        return c.bad ? SVDAG_ERR_CORRUPT : SVDAG_ERR_UNSUPPORTED;
    if (!c.memory_type())
        return SVDAG_ERR_CORRUPT;
    for (uint32_t i = 0; i < kTables; ++i) {
        Table& t = tables[i];
        t.itemWords = c.get<uint32_t>();
        t.slabWords = c.get<uint32_t>();
        t.buckets = c.get<uint32_t>();
        if (c.bad)
            return SVDAG_ERR_CORRUPT;
        if (t.itemWords != kMinItem + i || t.slabWords != slab_words(t.itemWords))
            return SVDAG_ERR_UNSUPPORTED;
        const uint32_t tableWords = c.get<uint32_t>();
        if (!c.memory_type() || t.buckets == 0 || tableWords != (uint64_t)t.buckets * t.slabWords)
            return SVDAG_ERR_CORRUPT;
        t.first = c.words(tableWords);
        const uint32_t unitWords = c.get<uint32_t>(), superWords = c.get<uint32_t>();
        if (unitWords != t.slabWords || superWords != kBitmapWords + (uint64_t)kUnitsPerSuper * t.slabWords)
            return SVDAG_ERR_CORRUPT;
        const uint64_t nSuper = c.get<uint64_t>();
        if (!c.memory_type() || nSuper > (1u << 18))
            return SVDAG_ERR_CORRUPT;
        t.supers.resize(nSuper);
        for (uint64_t s = 0; s < nSuper; ++s) {
            if (c.get<uint64_t>() != superWords || !c.memory_type())
                return SVDAG_ERR_CORRUPT;
            t.supers[s] = c.words(superWords);
        }
        c.get<uint64_t>(); // allocated size of the super block list
        c.get<uint32_t>(); // allocated units
        c.get<uint32_t>(); // numItems
        c.get<uint32_t>(); // numSlabs
        if (c.bad)
            return SVDAG_ERR_CORRUPT;
    }
    return SVDAG_OK;
}

// ------------------------------------------------------------------ writing

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
using KeyMap = std::unordered_map<KeyRef, uint32_t, KeyHash, KeyEq>;

// Distinct items in insertion order. A node's key is its header, its children's ids and whether
// those children are leaves (their handles, and so the node's words, depend on it); a leaf's key is
// its words.
struct Registry {
    std::vector<uint32_t> keys; // key words, one item after another
    std::vector<uint64_t> off; // per id
    std::vector<uint8_t> leaf; // per id: a leaf item
    std::vector<uint32_t> perTable; // ids per table
    KeyMap map;

    Registry() : perTable(kTables, 0) {}

    uint32_t add(const uint32_t* w, uint32_t n, bool isLeaf, uint32_t itemWords)
    {
        const uint64_t at = keys.size();
        keys.insert(keys.end(), w, w + n);
        auto [it, fresh] = map.emplace(KeyRef { &keys, at, n }, (uint32_t)off.size());
        if (!fresh) {
            keys.resize(at);
            return it->second;
        }
        off.push_back(at);
        leaf.push_back(isLeaf);
        ++perTable[itemWords - kMinItem];
        return it->second;
    }
};

struct Writer {
    std::FILE* f;
    bool bad = false;
    template <class T>
    void put(T v)
    {
        bad |= std::fwrite(&v, sizeof(T), 1, f) != 1;
    }
    void put_words(const uint32_t* w, uint64_t n)
    {
        if (n)
            bad |= std::fwrite(w, 4, n, f) != n;
    }
};

struct Placed {
    uint32_t buckets = 1;
    std::vector<uint32_t> first; // buckets * slab words
    std::vector<uint32_t> units; // overflow slabs, one after another
    std::vector<uint32_t> fill, last; // per bucket: items, last slab of the chain (kEnd = the first)
    KeyMap words; // real words -> item pointer
    std::vector<uint32_t> real; // real words of the placed items
};

} // namespace

extern "C" {

svdag_status svdag_v3_to_items(const void* data, uint64_t nBytes, uint32_t levels, uint32_t* out, uint64_t capacity,
    uint64_t* levelWords, uint64_t* levelItems, uint64_t* totalWords)
{
    if (!data || !levelWords || !levelItems || !totalWords || levels < SVDAG_MIN_LEVELS || levels > SVDAG_MAX_LEVELS
        || (capacity && !out) || reinterpret_cast<uintptr_t>(data) % 4)
        return SVDAG_ERR_INVALID;
    Cursor c { static_cast<const uint8_t*>(data), nBytes };
    uint32_t root = kEnd;
    Table tables[kTables];
    if (svdag_status st = parse(c, levels, root, tables))
        return st;
    const uint32_t LL = levels - 2;
    std::vector<std::vector<uint32_t>> words(LL + 1);
    std::vector<uint32_t> frontier, next;
    if (root != kEnd)
        frontier.push_back(root);
    for (uint32_t l = 0; l <= LL; ++l) {
        const bool leaf = l == LL;
        std::unordered_map<uint32_t, uint32_t> ordinal; // child handle -> ordinal at level l + 1
        next.clear();
        for (const uint32_t h : frontier) {
            const uint32_t n = (h >> kPtrBits) + (leaf ? 3u : 2u);
            if (n - kMinItem >= kTables)
                return SVDAG_ERR_CORRUPT;
            const uint32_t* w = locate(tables[n - kMinItem], h & kPtrMask);
            if (!w || svdag::snapshot::item_words(leaf, w, n) != n)
                return SVDAG_ERR_CORRUPT;
            auto& lw = words[l];
            lw.push_back(w[0]);
            if (leaf) {
                lw.insert(lw.end(), w + 1, w + n);
                continue;
            }
            for (uint32_t i = 1; i < n; ++i) {
                auto [it, fresh] = ordinal.emplace(w[i], (uint32_t)next.size());
                if (fresh)
                    next.push_back(w[i]);
                lw.push_back(it->second);
            }
        }
        levelItems[l] = frontier.size();
        frontier.swap(next);
    }
    uint64_t total = 0;
    for (uint32_t l = 0; l <= LL; ++l) {
        levelWords[l] = words[l].size();
        if (out && total + words[l].size() <= capacity)
            std::memcpy(out + total, words[l].data(), words[l].size() * 4);
        total += words[l].size();
    }
    *totalWords = total;
    return total > capacity ? SVDAG_ERR_OOM : SVDAG_OK;
}

svdag_status svdag_items_to_v3(const uint32_t* words, const uint64_t* levelWords, const uint64_t* levelItems, uint32_t levels,
    uint32_t memoryType, const char* path)
{
    if (!levelWords || !levelItems || !path || levels < SVDAG_MIN_LEVELS || levels > SVDAG_MAX_LEVELS || memoryType >= kMemTypes)
        return SVDAG_ERR_INVALID;
    const uint32_t LL = levels - 2;
    uint64_t total = 0;
    for (uint32_t l = 0; l <= LL; ++l)
        total += levelWords[l];
    if (total && !words)
        return SVDAG_ERR_INVALID;
    const bool empty = levelItems[0] == 0;
    if ((empty && total != 0) || (!empty && levelItems[0] != 1))
        return SVDAG_ERR_INVALID;
    std::vector<std::vector<uint64_t>> offs(LL + 1);
    for (uint64_t l = 0, at = 0; l <= LL; at += levelWords[l], ++l)
        if (!svdag::snapshot::split_level(l == LL, words + at, levelWords[l], levelItems[l], l < LL ? levelItems[l + 1] : 0, offs[l])
            || levelItems[l] > 0xFFFFFFF0ull)
            return SVDAG_ERR_INVALID;

    // ids of the fully-filled items (MyGPUHashDAG::allocate), then of the snapshot, bottom-up
    Registry reg;
    std::vector<uint32_t> fullId((uint64_t)levels * kMaterials, kEnd);
    uint32_t key[11];
    for (uint32_t m = 0; m < kMaterials; ++m) {
        key[0] = key[1] = 0xFFFFFFFFu;
        for (uint32_t i = 2; i < 10; ++i)
            key[i] = m * 0x11111111u;
        fullId[m * levels + LL] = reg.add(key, 10, true, 10);
    }
    for (int l = (int)LL - 1; l >= 0; --l)
        for (uint32_t m = 0; m < kMaterials; ++m) {
            key[0] = 0xFFu | 1u << 8 | m << 9;
            for (uint32_t i = 1; i <= 8; ++i)
                key[i] = fullId[m * levels + l + 1];
            key[9] = (uint32_t)l + 1 == LL;
            fullId[m * levels + l] = reg.add(key, 10, false, 9);
        }
    std::vector<uint64_t> levelAt(LL + 1, 0);
    for (uint32_t l = 1; l <= LL; ++l)
        levelAt[l] = levelAt[l - 1] + levelWords[l - 1];
    std::vector<uint32_t> below, here;
    for (int l = (int)LL; l >= 0 && !empty; --l) {
        const uint64_t at = levelAt[l];
        here.assign(offs[l].size(), 0);
        for (size_t i = 0; i < offs[l].size(); ++i) {
            const uint32_t* w = words + at + offs[l][i];
            if (l == (int)LL) {
                const uint32_t n = leaf_words(w[0], w[1]);
                here[i] = reg.add(w, n, true, n);
            } else {
                const uint32_t n = node_words(w[0]);
                key[0] = w[0];
                for (uint32_t j = 1; j < n; ++j)
                    key[j] = below[w[j]];
                key[n] = (uint32_t)l + 1 == LL;
                here[i] = reg.add(key, n + 1, false, n);
            }
        }
        below.swap(here);
    }
    const uint32_t rootId = empty ? kEnd : below[0];

    // placement in id order: children are placed before their parents
    std::vector<Placed> tabs(kTables);
    for (uint32_t t = 0; t < kTables; ++t) {
        Placed& p = tabs[t];
        const uint64_t buckets = reg.perTable[t] / kLoadFactor + 1;
        if (buckets >= kMaxSlab || buckets * slab_words(kMinItem + t) > 0xFFFFFFFFull)
            return SVDAG_ERR_OOM;
        p.buckets = (uint32_t)buckets;
        p.first.assign(buckets * slab_words(kMinItem + t), 0);
        for (uint32_t b = 0; b < buckets; ++b)
            p.first[(uint64_t)b * slab_words(kMinItem + t) + kNextWord] = kEnd;
        p.fill.assign(buckets, 0);
        p.last.assign(buckets, kEnd);
    }
    const size_t ids = reg.off.size();
    std::vector<uint32_t> ptrOf(ids);
    uint32_t w[10];
    for (size_t id = 0; id < ids; ++id) {
        const uint32_t* k = reg.keys.data() + reg.off[id];
        uint32_t n;
        if (reg.leaf[id]) {
            n = leaf_words(k[0], k[1]);
            std::memcpy(w, k, n * 4);
        } else {
            n = node_words(k[0]);
            const uint32_t sizeBase = k[n] ? 3u : 2u; // children are leaves / nodes
            w[0] = k[0];
            for (uint32_t j = 1; j < n; ++j) {
                const uint32_t cn = reg.leaf[k[j]] ? leaf_words(reg.keys[reg.off[k[j]]], reg.keys[reg.off[k[j]] + 1])
                                                   : node_words(reg.keys[reg.off[k[j]]]);
                w[j] = (cn - sizeBase) << kPtrBits | ptrOf[k[j]];
            }
        }
        Placed& p = tabs[n - kMinItem];
        const uint64_t at = p.real.size();
        p.real.insert(p.real.end(), w, w + n);
        auto [it, fresh] = p.words.emplace(KeyRef { &p.real, at, n }, 0u);
        if (!fresh) { // a leaf and a node of equal words: one item
            p.real.resize(at);
            ptrOf[id] = it->second;
            continue;
        }
        const uint32_t sw = slab_words(n);
        const uint32_t b = bucket_hash(w, n) % p.buckets;
        const uint32_t slot = p.fill[b] % kSlots;
        uint32_t* slab;
        uint32_t ptr;
        if (p.fill[b] < kSlots) {
            slab = p.first.data() + (uint64_t)b * sw;
            ptr = b << 6 | 1u << 5 | slot;
        } else {
            if (slot == 0) { // chain a new slab from the allocator
                const uint32_t unit = (uint32_t)(p.units.size() / sw);
                if (unit >= kMaxSlab)
                    return SVDAG_ERR_OOM;
                p.units.resize(p.units.size() + sw, 0);
                p.units[(uint64_t)unit * sw + kNextWord] = kEnd;
                uint32_t* prev = p.last[b] == kEnd ? p.first.data() + (uint64_t)b * sw : p.units.data() + (uint64_t)p.last[b] * sw;
                prev[kNextWord] = unit;
                p.last[b] = unit;
            }
            slab = p.units.data() + (uint64_t)p.last[b] * sw;
            ptr = p.last[b] << 6 | slot;
        }
        slab[slot >> 2] |= tag_hash(w, n) << ((slot & 3u) * 8u);
        std::memcpy(slab + kItemsAt + (uint64_t)slot * n, w, n * 4);
        ++p.fill[b];
        ptrOf[id] = ptr;
        it->second = ptr;
    }
    auto handle = [&](uint32_t id, bool leaf) {
        const uint32_t* k = reg.keys.data() + reg.off[id];
        const uint32_t n = reg.leaf[id] ? leaf_words(k[0], k[1]) : node_words(k[0]);
        return (n - (leaf ? 3u : 2u)) << kPtrBits | ptrOf[id];
    };

    std::FILE* f = std::fopen(path, "wb");
    if (!f)
        return SVDAG_ERR_INVALID;
    std::vector<char> buffer(1 << 22);
    std::setvbuf(f, buffer.data(), _IOFBF, buffer.size());
    Writer wr { f };
    wr.put(kVersion);
    wr.put((uint64_t)levels * kMaterials);
    wr.put(memoryType);
    for (uint32_t m = 0; m < kMaterials; ++m)
        for (uint32_t l = 0; l < levels; ++l)
            wr.put(l <= LL ? handle(fullId[m * levels + l], l == LL) : kEnd);
    wr.put(levels);
    wr.put(kMaterials);
    wr.put(rootId == kEnd ? kEnd : handle(rootId, false));
    wr.put((uint64_t)kTables);
    wr.put(memoryType);
    std::vector<uint32_t> super;
    for (uint32_t t = 0; t < kTables; ++t) {
        const Placed& p = tabs[t];
        const uint32_t n = kMinItem + t, sw = slab_words(n);
        const uint64_t units = p.units.size() / sw;
        const uint64_t nSuper = units ? (units + kUnitsPerSuper - 1) / kUnitsPerSuper : 1;
        const uint32_t superWords = kBitmapWords + kUnitsPerSuper * sw;
        wr.put(n);
        wr.put(sw);
        wr.put(p.buckets);
        wr.put((uint32_t)p.first.size());
        wr.put(memoryType);
        wr.put_words(p.first.data(), p.first.size());
        wr.put(sw);
        wr.put(superWords);
        wr.put(nSuper);
        wr.put(kMemCPU); // superBlocksCPU lives in host memory whatever the table's memory type
        for (uint64_t s = 0; s < nSuper; ++s) {
            super.assign(superWords, 0);
            const uint64_t lo = s * kUnitsPerSuper, hi = std::min<uint64_t>(units, lo + kUnitsPerSuper);
            for (uint64_t u = lo; u < hi; ++u)
                super[(u - lo) >> 5] |= 1u << ((u - lo) & 31u);
            if (hi > lo)
                std::memcpy(super.data() + kBitmapWords, p.units.data() + lo * sw, (hi - lo) * sw * 4);
            wr.put((uint64_t)superWords);
            wr.put(memoryType);
            wr.put_words(super.data(), super.size());
        }
        wr.put(nSuper);
        wr.put((uint32_t)units);
        wr.put(0u); // numItems, numSlabs: written only with CAPTURE_MEMORY_STATS_SLOW
        wr.put(0u);
    }
    const bool closed = std::fclose(f) == 0;
    return wr.bad || !closed ? SVDAG_ERR_INVALID : SVDAG_OK;
}

} // extern "C"
