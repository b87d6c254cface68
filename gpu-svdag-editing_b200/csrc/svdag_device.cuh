// svdag_device.cuh - device-side data layout and the slab hash table probes.
//
// Item region: one array inside the context's HBM pool. A handle is the index of an item in 16-byte
// units (items are 16-byte aligned), so decoding a handle is a shift and an add and 32-bit handles
// reach 64 GiB (the reference decodes through a table descriptor and the slab allocator's super-block
// table, gpu_hash_table_base.h:275-294). Slabs are 32-byte aligned and named by their index in
// 32-byte units (the "slab id").
//
// Hash tables: one table per DAG level. A level table holds keys of 2..10 words; keys of one length
// share a slab family (the "size class"), so slots have a fixed stride and the slot index gives the
// item address. A slab is a 32-byte header in the header region plus a body of 24 items in the item
// region:
//   header words 0..5 : 24 one-byte tags, slot s at word s / 4, byte s % 4; 0 = free, 0xFF = being written
//   header word 6     : handle of the body (item of slot 0)
//   header word 7     : header id of the next slab in the bucket's chain, 0 = end (header 0 is unused)
//   body              : 24 items of k words at a stride of k rounded up to a multiple of 4 (slot s at body + s*stride)
// A probe reads one 32-byte header sector per slab plus the candidate item. Headers are dense (a
// table's headers are about a tenth of its bytes), so the headers a lookup stream touches stay in
// the 126 MB L2 while the items it compares are read once; the reference interleaves a 10-word
// header with each slab's items (compact_acceleration_hash_table.h:519-541). The first slab of each
// bucket is allocated with the table (HASH_TABLE_STORE_SLABS_IN_TABLE, gpu_hash_table_base.h:30-49);
// overflow slabs come from bump allocators over the two regions and are linked at the chain's tail.
//
// Free list (DynamicSlabAllocator::free, dynamic_slab_alloc.h:187-208, and the sweep's unlinking of
// empty slabs, gpu_hash_table_base.cu:265-281,320-336): garbage collection unlinks every overflow
// slab of a level table that it leaves empty and pushes it on the free list of its size class, a
// stack of header ids linked through header word 7 whose head carries a 32-bit version count beside
// the id (so a pop racing a push cannot take a stale link). Overflow allocations of level tables pop
// from that list before they bump. Tables whose space is given back by rewinding the bump pointers
// (the autotuner's scratch tables) neither pop nor push.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>
#include <cstddef>
#include <cstdint>

#include "../../include/svdag.h"
#include "svdag_hash.h"

namespace svdag {

constexpr uint32_t kNone = 0xFFFFFFFFu; // empty child / missing handle
constexpr uint32_t kEnd = 0u; // end of a slab chain
constexpr uint32_t kFillMarker = 0xFFFFFF00u; // SVO child "canonical fully-filled node of material m" = kFillMarker | m
constexpr uint32_t kUnitWords = 4; // a handle counts 16-byte units
constexpr unsigned long long kMaxItemWords = (unsigned long long)kUnitWords * 0xFFFFFF00ull - 64; // item region limit (just under 64 GiB)
constexpr uint32_t kSlots = 24;
constexpr uint32_t kHeaderWords = 8;
constexpr uint32_t kTagBusy = 0xFFu;
constexpr uint32_t kMaxLevels = SVDAG_MAX_LEVELS;
constexpr uint32_t kItemStride = 10; // padded stride of items in scratch arrays
constexpr uint32_t kNumClasses = 9; // item sizes 2..10

__host__ __device__ constexpr uint32_t item_stride(uint32_t k) { return (k + kUnitWords - 1u) & ~(kUnitWords - 1u); } // words
__host__ __device__ constexpr uint32_t body_words(uint32_t k) { return kSlots * item_stride(k); } // a multiple of 32
// Handle of slot s of the slab whose body starts at handle `body`, for items of k words.
__host__ __device__ constexpr uint32_t slot_handle(uint32_t body, uint32_t s, uint32_t k) { return body + s * (item_stride(k) / kUnitWords); }
__host__ __device__ inline uint32_t header_tag(const uint32_t* h, uint32_t s) { return (h[s >> 2] >> (8u * (s & 3u))) & 0xFFu; }

// Per-table descriptor, passed by value to kernels.
struct DevTable {
    uint32_t kind; // svdag_item_kind
    uint32_t numBuckets[kNumClasses];
    uint32_t bucketBase[kNumClasses]; // header id of bucket 0
    uint32_t bodyBase[kNumClasses]; // body handle of bucket 0 (bucket b's body follows at b * body size)
    uint32_t recycle; // overflow slabs come from and go back to the free lists (level tables)
};

// Device control block (lives at the start of the scratch side of the pool).
struct EditCounters {
    uint32_t count[kMaxLevels]; // intermediate SVO items per level
    uint32_t ffCount[kMaxLevels]; // fully-filled items found per level
    uint32_t ffRan[kMaxLevels]; // discovery ran at this level
    uint32_t repCount[kMaxLevels]; // items left after intra-level dedup
    uint32_t repPerClass[kMaxLevels][kNumClasses];
    unsigned long long oldRead, added, edited;
    unsigned long long offW[kMaxLevels]; // scratch byte offset of each level's work items
    unsigned long long offN[kMaxLevels]; // scratch byte offset of each level's SVO items
    unsigned long long buildTop; // end of the top-down allocations
    uint32_t rootBefore, rootAfter;
    uint32_t overflow; // scratch arena exhausted
    uint32_t builder; // scene build: merge even without leaves, discovery on every level
    uint32_t startLevel;
    uint32_t err; // first error status raised while this edit ran (0 = none)
};

struct Control {
    unsigned long long itemTop; // bump pointer of the item region, in words
    unsigned long long headerTop; // bump pointer of the header region, in headers (0 is never used)
    uint32_t status; // latched svdag_status
    uint32_t root; // current root handle (kNone = empty DAG)
    unsigned long long freeBytes; // bytes (headers and bodies) of the slabs on the free lists
    uint32_t undo[64];
    uint32_t redo[64];
    uint32_t undoHead, undoCount, redoCount, undoDepth;
    uint32_t savedRoot; // source root of a move (the DAG before its removal step)
    uint32_t pad0;
    uint32_t fullyFilled[kMaxLevels][SVDAG_NUM_MATERIALS];
    DevTable tables[kMaxLevels]; // the level tables (copied here by the host whenever they change)
    EditCounters edit;
    unsigned long long phaseTimes[64]; // GPU global-timer stamps at the phase barriers of the last fused edit
    uint32_t phaseCount;
    uint32_t pad1;
    unsigned long long freeHead[kNumClasses]; // per size class: version << 32 | header id of the first free slab (0 = none)
    unsigned long long freeSlabs[kNumClasses]; // slabs on each free list
    unsigned long long gcFreedItems; // items the last collection freed
    unsigned long long gcFreedSlabs; // overflow slabs the last collection put on the free lists
    unsigned long long gcLiveItems; // items the last collection marked (reachable from its roots)
};

// The first 32 bytes of the control block, copied to the host after every served launch.
struct MemSnapshot {
    unsigned long long itemTop, headerTop;
    uint32_t status, root;
    unsigned long long freeBytes;
};
static_assert(offsetof(Control, itemTop) == offsetof(MemSnapshot, itemTop) && offsetof(Control, headerTop) == offsetof(MemSnapshot, headerTop)
        && offsetof(Control, status) == offsetof(MemSnapshot, status) && offsetof(Control, root) == offsetof(MemSnapshot, root)
        && offsetof(Control, freeBytes) == offsetof(MemSnapshot, freeBytes),
    "MemSnapshot mirrors the head of Control");

// Bytes of item and header region a slab of k-word items occupies.
__host__ __device__ constexpr unsigned long long slab_bytes(uint32_t k) { return 32ull + 4ull * body_words(k); }

struct DevDag {
    uint32_t* items;
    unsigned long long itemWords; // capacity of the item region
    uint32_t* headers; // slab headers, 8 words each
    unsigned long long headerCount; // capacity of the header region
    Control* ctl;
    uint32_t levels;
    uint32_t leafLevel;
    EditCounters* edit; // counters of the running edit: &ctl->edit, or a subtree edit's own
    uint32_t solo; // each block runs an edit of its own (a subtree edit): phases see one block of a one-block grid
    uint32_t* locks; // kLockStripes bucket lock words of a group of subtree edits (null otherwise)
};
constexpr uint32_t kLockStripes = 1u << 16;

// Block index and block count of an edit phase: the launch's own, or 0 of 1 for a block that runs an
// edit of its own.
__device__ __forceinline__ uint32_t ph_block(const DevDag& d) { return d.solo ? 0u : blockIdx.x; }
__device__ __forceinline__ uint32_t ph_grid(const DevDag& d) { return d.solo ? 1u : gridDim.x; }

// Release fence at GPU scope: stores before it are visible to other SMs before stores after it (the
// writers' half of publishing data through a flag or table entry; readers depend on the published
// value's address, which orders their loads).
__device__ __forceinline__ void fence_release() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Latches the first error of the context (reported by svdag_sync) and of the running edit (which
// then leaves the root unchanged).
__device__ __forceinline__ void set_status(Control* ctl, uint32_t code)
{
    atomicCAS(&ctl->status, 0u, code);
    atomicCAS(&ctl->edit.err, 0u, code);
}

// Every handle read from memory is checked before it is dereferenced: a bad handle (which only a
// bug could produce) latches SVDAG_ERR_CORRUPT and reads a zero item instead of faulting.
__device__ const uint32_t kZeroItem[16] = {};
__device__ __forceinline__ bool handle_ok(const DevDag& d, uint32_t h)
{
    return (unsigned long long)kUnitWords * h + 16ull <= d.itemWords;
}
__device__ __forceinline__ const uint32_t* item_ptr(const DevDag& d, uint32_t h)
{
    if (handle_ok(d, h))
        return d.items + (unsigned long long)kUnitWords * h;
    set_status(d.ctl, SVDAG_ERR_CORRUPT);
    return kZeroItem;
}
__device__ __forceinline__ bool slab_ok(const DevDag& d, uint32_t slab) { return slab != 0 && slab < d.headerCount; }
__device__ __forceinline__ uint32_t* slab_ptr(const DevDag& d, uint32_t slab) { return d.headers + 8ull * slab; }
__device__ __forceinline__ uint32_t* handle_ptr(const DevDag& d, uint32_t h) { return d.items + (unsigned long long)kUnitWords * h; }

// ---------------------------------------------------------------- hashing: svdag_hash.h

__device__ __forceinline__ uint32_t bucket_of(uint32_t ha, uint32_t numBuckets) { return __umulhi(ha, numBuckets); }

// Key length from the first words: node_words / leaf_words in svdag_hash.h.
__device__ __forceinline__ uint32_t dev_node_words(uint32_t header) { return 1u + __popc(header & 0xFFu); }
__device__ __forceinline__ uint32_t dev_leaf_words(uint32_t lo, uint32_t hi) { return 2u + (((__popc(lo) + __popc(hi)) * 4u + 31u) >> 5); }

// ---------------------------------------------------------------- cooperative groups of G lanes

template <int G>
struct Grp {
    static constexpr int KW = (int(kItemStride) + G - 1) / G; // key words per lane
    uint32_t lane; // 0..G-1
    uint32_t mask; // warp lanes of this group
    __device__ __forceinline__ Grp()
    {
        const uint32_t wl = threadIdx.x & 31u;
        lane = wl % G;
        mask = (G == 32) ? 0xFFFFFFFFu : (((1u << G) - 1u) << (wl / G * G));
    }
    __device__ __forceinline__ uint32_t bcast(uint32_t v, uint32_t src) const
    {
        if constexpr (G == 1)
            return v;
        else
            return __shfl_sync(mask, v, src, G);
    }
    __device__ __forceinline__ uint32_t reduce_or(uint32_t v) const
    {
        if constexpr (G > 1) {
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1)
                v |= __shfl_xor_sync(mask, v, o, G);
        }
        return v;
    }
    __device__ __forceinline__ uint32_t reduce_xor(uint32_t v) const
    {
        if constexpr (G > 1) {
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1)
                v ^= __shfl_xor_sync(mask, v, o, G);
        }
        return v;
    }
    __device__ __forceinline__ bool all(bool p) const
    {
        if constexpr (G == 1)
            return p;
        else
            return __all_sync(mask, p);
    }
    __device__ __forceinline__ void sync() const
    {
        if constexpr (G > 1)
            __syncwarp(mask);
    }
};

// A key spread over the lanes of a group: lane j holds words j, j+G, j+2G, ...
template <int G>
struct Key {
    uint32_t w[Grp<G>::KW];
    uint32_t n; // words
    uint32_t ha, hb; // bucket hash, tag hash
};

// Load flavours: default caching, L2 only (__ldcg: coherent with other SMs' stores of the same
// launch) and streaming (__ldcs: evict-first in L1 and L2, for data read once).
enum : int { LD_DEFAULT = 0, LD_L2 = 1, LD_STREAM = 2 };
template <int MODE>
__device__ __forceinline__ uint32_t ld(const uint32_t* p)
{
    if constexpr (MODE == LD_L2)
        return __ldcg(p);
    else if constexpr (MODE == LD_STREAM)
        return __ldcs(p);
    else
        return *p;
}

// Loads a self-describing key (node or leaf) of at most 10 words; `limit` bounds the readable words.
template <int G, int MODE = LD_DEFAULT>
__device__ __forceinline__ void load_key(const Grp<G>& g, const uint32_t* p, unsigned long long limit, uint32_t kind, Key<G>& key)
{
    if constexpr (G == 1) {
        // All ten words are requested at once (one memory round trip instead of two: the length is
        // only known from the first words) and trimmed to the key's length afterwards.
        uint32_t v[kItemStride];
        if (limit >= kItemStride) { // all but the last keys of an array: no per-word bound
#pragma unroll
            for (uint32_t i = 0; i < kItemStride; ++i)
                v[i] = ld<MODE>(p + i);
        } else {
#pragma unroll
            for (uint32_t i = 0; i < kItemStride; ++i)
                v[i] = i < limit ? ld<MODE>(p + i) : 0u;
        }
        key.n = kind == SVDAG_KIND_NODE ? dev_node_words(v[0]) : dev_leaf_words(v[0], v[1]);
        uint32_t a = 0;
#pragma unroll
        for (uint32_t i = 0; i < kItemStride; ++i) {
            key.w[i] = i < key.n ? v[i] : 0u;
            a ^= i < key.n ? word_term(v[i], i) : 0u;
        }
        key.ha = bucket_hash(a);
        key.hb = tag_hash(a);
        return;
    }
    uint32_t w0 = 0, w1 = 0;
    if constexpr (G == 1) {
        w0 = limit > 0 ? ld<MODE>(p) : 0u;
        w1 = limit > 1 ? ld<MODE>(p + 1) : 0u;
    } else {
        uint32_t v = (g.lane < 2 && g.lane < limit) ? ld<MODE>(p + g.lane) : 0u;
        w0 = g.bcast(v, 0);
        w1 = g.bcast(v, 1);
    }
    key.n = kind == SVDAG_KIND_NODE ? dev_node_words(w0) : dev_leaf_words(w0, w1);
    uint32_t a = 0;
#pragma unroll
    for (int i = 0; i < Grp<G>::KW; ++i) {
        const uint32_t idx = g.lane + uint32_t(i) * G;
        uint32_t v = 0;
        if (idx < key.n && idx < limit)
            v = (G == 1 && idx < 2) ? (idx == 0 ? w0 : w1) : ld<MODE>(p + idx);
        key.w[i] = v;
        if (idx < key.n)
            a ^= word_term(v, idx);
    }
    a = g.reduce_xor(a);
    key.ha = bucket_hash(a);
    key.hb = tag_hash(a);
}

// Sets up a key already held in registers of a single thread (G == 1 paths of the pipeline).
__device__ __forceinline__ void hash_words(const uint32_t* w, uint32_t n, uint32_t& ha, uint32_t& hb)
{
    uint32_t a = 0;
#pragma unroll
    for (uint32_t i = 0; i < kItemStride; ++i) // fixed trip count keeps w[] in registers
        if (i < n)
            a ^= word_term(w[i], i);
    ha = bucket_hash(a);
    hb = tag_hash(a);
}

// The tag words of a probed header as the lanes of a group loaded them: with G lanes, lane l holds
// words first(l) .. first(l) + N - 1 (G = 1: all six; G >= 8: word l). A claim starts its
// compare-and-swap from the probed value instead of reading the word again.
template <int G>
struct HdrSnap {
    static constexpr int N = G == 1 ? 6 : (G == 2 ? 4 : (G == 4 ? 2 : 1));
    uint32_t w[N];
    static __device__ __forceinline__ uint32_t first(uint32_t lane) { return G == 1 ? 0u : (G == 2 ? 4u * lane : (G == 4 ? 2u * lane : lane)); }
    static __device__ __forceinline__ uint32_t owner(uint32_t word) { return G == 1 ? 0u : (G == 2 ? word / 4u : (G == 4 ? word / 2u : word)); }
    __device__ __forceinline__ uint32_t get(uint32_t word, uint32_t lane) const
    {
        const uint32_t j = word - first(lane);
        uint32_t v = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
            v = j == uint32_t(i) ? w[i] : v;
        return v;
    }
};

// Loads the 8 header words of a slab. Returns the candidate mask of slots whose tag byte equals
// `tag` (24 bits), with the body handle, the next header id and (EMPTY) the mask of free slots;
// `snap` (optional) receives the tag words. A single thread reads the 32-byte header with one
// 256-bit load (headers are 32-byte aligned).
template <int G, bool CG = false, bool EMPTY = true>
__device__ __forceinline__ uint32_t probe_header(const Grp<G>& g, const uint32_t* hdr, uint32_t tag, uint32_t& next, uint32_t& body,
    uint32_t& emptyMask, HdrSnap<G>* snap = nullptr)
{
    const uint32_t tag4 = tag * 0x01010101u;
    uint32_t cand = 0, empty = 0;
    // bit 7 of each byte set exactly where that byte of v is zero (the adds carry within a byte only)
    auto zero_bytes = [](uint32_t v) { return ~(((v & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | v | 0x7F7F7F7Fu); };
    // bits 7, 15, 23, 31 -> bits 28..31: the partial products of the multiply never overlap
    auto gather = [](uint32_t m) { return (m * 0x00204081u) >> 28; };
    auto account = [&](uint32_t word, uint32_t x) {
        if (word < 6) {
            cand |= gather(zero_bytes(x ^ tag4)) << (4 * word);
            if constexpr (EMPTY)
                empty |= gather(zero_bytes(x)) << (4 * word);
        }
    };
    uint32_t nx = 0, bd = 0;
    if constexpr (G == 1) {
        uint4 a, b;
        if constexpr (CG) {
            a = __ldcg(reinterpret_cast<const uint4*>(hdr));
            b = __ldcg(reinterpret_cast<const uint4*>(hdr) + 1);
        } else {
            asm("ld.global.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
                : "l"(hdr));
        }
        account(0, a.x);
        account(1, a.y);
        account(2, a.z);
        account(3, a.w);
        account(4, b.x);
        account(5, b.y);
        bd = b.z;
        nx = b.w;
        if (snap) {
            snap->w[0] = a.x;
            snap->w[1] = a.y;
            snap->w[2] = a.z;
            snap->w[3] = a.w;
            snap->w[4] = b.x;
            snap->w[5] = b.y;
        }
    } else if constexpr (G == 2) {
        const uint4 a = CG ? __ldcg(reinterpret_cast<const uint4*>(hdr) + g.lane) : reinterpret_cast<const uint4*>(hdr)[g.lane];
        account(4 * g.lane + 0, a.x);
        account(4 * g.lane + 1, a.y);
        account(4 * g.lane + 2, a.z);
        account(4 * g.lane + 3, a.w);
        bd = g.bcast(a.z, 1);
        nx = g.bcast(a.w, 1);
        if (snap) {
            snap->w[0] = a.x;
            snap->w[1] = a.y;
            snap->w[2 % HdrSnap<G>::N] = a.z;
            snap->w[3 % HdrSnap<G>::N] = a.w;
        }
    } else if constexpr (G == 4) {
        const uint2 a = CG ? __ldcg(reinterpret_cast<const uint2*>(hdr) + g.lane) : reinterpret_cast<const uint2*>(hdr)[g.lane];
        account(2 * g.lane + 0, a.x);
        account(2 * g.lane + 1, a.y);
        bd = g.bcast(a.x, 3);
        nx = g.bcast(a.y, 3);
        if (snap) {
            snap->w[0] = a.x;
            snap->w[1 % HdrSnap<G>::N] = a.y;
        }
    } else {
        uint32_t x = 0;
        if (g.lane < 8)
            x = CG ? __ldcg(hdr + g.lane) : hdr[g.lane];
        if (g.lane < 8)
            account(g.lane, x);
        bd = g.bcast(x, 6);
        nx = g.bcast(x, 7);
        if (snap)
            snap->w[0] = x;
    }
    next = nx;
    body = bd;
    emptyMask = g.reduce_or(empty);
    return g.reduce_or(cand);
}

template <int MODE>
__device__ __forceinline__ uint4 ld4(const uint4* p)
{
    if constexpr (MODE == LD_L2)
        return __ldcg(p);
    else if constexpr (MODE == LD_STREAM)
        return __ldcs(p);
    else
        return *p;
}

// Word i of a single thread's key (zero past its ten words).
__device__ __forceinline__ uint32_t key_word(const Key<1>& key, uint32_t i) { return i < kItemStride ? key.w[i] : 0u; }

// Compares the key with the item at `item`; all lanes of the group get the same answer. A single
// thread compares 16-byte chunks (items are 16-byte aligned; words past the key's length are not
// compared).
template <int G, int MODE = LD_DEFAULT>
__device__ __forceinline__ bool item_equals(const Grp<G>& g, const uint32_t* item, const Key<G>& key)
{
    if constexpr (G == 1) {
        bool eq = true;
#pragma unroll
        for (uint32_t c = 0; c < 3; ++c) {
            if (4u * c < key.n) {
                const uint4 v = ld4<MODE>(reinterpret_cast<const uint4*>(item) + c);
                eq &= (4u * c + 0 >= key.n || v.x == key_word(key, 4u * c + 0)) && (4u * c + 1 >= key.n || v.y == key_word(key, 4u * c + 1))
                    && (4u * c + 2 >= key.n || v.z == key_word(key, 4u * c + 2)) && (4u * c + 3 >= key.n || v.w == key_word(key, 4u * c + 3));
            }
        }
        return eq;
    }
    bool eq = true;
#pragma unroll
    for (int i = 0; i < Grp<G>::KW; ++i) {
        const uint32_t idx = g.lane + uint32_t(i) * G;
        if (idx < key.n)
            eq &= ld<MODE>(item + idx) == key.w[i];
    }
    return g.all(eq);
}

template <int G>
__device__ __forceinline__ void write_item(const Grp<G>& g, uint32_t* item, const Key<G>& key)
{
    if constexpr (G == 1) { // 16-byte chunks; pad words (inside the slot's stride) are written as zero
#pragma unroll
        for (uint32_t c = 0; c < 3; ++c)
            if (4u * c < key.n) {
                auto word = [&](uint32_t i) { return i < key.n ? key_word(key, i) : 0u; };
                *reinterpret_cast<uint4*>(item + 4u * c) = make_uint4(word(4u * c), word(4u * c + 1), word(4u * c + 2), word(4u * c + 3));
            }
    } else {
#pragma unroll
        for (int i = 0; i < Grp<G>::KW; ++i) {
            const uint32_t idx = g.lane + uint32_t(i) * G;
            if (idx < key.n)
                item[idx] = key.w[i];
        }
    }
}

__device__ __forceinline__ uint32_t first_slab(const DevTable& t, uint32_t cls, uint32_t ha)
{
    return t.bucketBase[cls] + bucket_of(ha, t.numBuckets[cls]);
}

constexpr uint32_t kFreeListTries = 64; // pops that lose this many races fall back to the bump allocator

// Takes a slab off the free list of size class `cls`; kNone when the list is empty (or contended).
// The head's version count changes with every pop and push, so a pop whose head is stale fails its
// compare-and-swap even when the same id is back on top.
__device__ __forceinline__ uint32_t pop_free_slab(const DevDag& d, uint32_t cls)
{
    unsigned long long* head = &d.ctl->freeHead[cls];
    unsigned long long cur = __ldcg(head);
    for (uint32_t tries = 0; tries < kFreeListTries; ++tries) {
        const uint32_t id = (uint32_t)cur;
        if (id == kEnd)
            return kNone;
        if (!slab_ok(d, id)) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        const uint32_t next = __ldcg(slab_ptr(d, id) + 7);
        const unsigned long long want = (((cur >> 32) + 1ull) << 32) | next;
        const unsigned long long old = atomicCAS(head, cur, want);
        if (old == cur) {
            atomicAdd(&d.ctl->freeSlabs[cls], ~0ull); // minus one (two's complement)
            atomicAdd(&d.ctl->freeBytes, 0ull - slab_bytes(cls + 2));
            return id;
        }
        cur = old;
    }
    return kNone;
}

// Pushes a chain of `count` free slabs (first .. last, linked through header word 7) on the free
// list of size class `cls`.
__device__ __forceinline__ void push_free_chain(const DevDag& d, uint32_t cls, uint32_t first, uint32_t last, uint32_t count)
{
    unsigned long long* head = &d.ctl->freeHead[cls];
    unsigned long long cur = __ldcg(head);
    for (uint32_t tries = 0; tries < (1u << 20); ++tries) {
        slab_ptr(d, last)[7] = (uint32_t)cur;
        __threadfence(); // the link is visible before the slab is reachable from the head
        const unsigned long long want = (((cur >> 32) + 1ull) << 32) | first;
        const unsigned long long old = atomicCAS(head, cur, want);
        if (old == cur) {
            atomicAdd(&d.ctl->freeSlabs[cls], (unsigned long long)count);
            atomicAdd(&d.ctl->freeBytes, (unsigned long long)count * slab_bytes(cls + 2));
            return;
        }
        cur = old;
    }
    set_status(d.ctl, SVDAG_ERR_TIMEOUT); // the chain stays allocated (lost to reuse, never corrupt)
}

// Allocates and initialises an overflow slab of class k (a header and a cleared body); returns its
// header id, or kNone when a region is full. `recycle`: try the free list of class k first.
template <int G>
__device__ __forceinline__ uint32_t alloc_slab(const Grp<G>& g, const DevDag& d, uint32_t k, uint32_t recycle)
{
    uint32_t id = kNone, body = 0;
    if (g.lane == 0 && recycle) {
        id = pop_free_slab(d, k - 2u);
        if (id != kNone) {
            body = __ldcg(slab_ptr(d, id) + 6); // a free slab keeps its body
            if ((unsigned long long)kUnitWords * body + body_words(k) > d.itemWords) {
                set_status(d.ctl, SVDAG_ERR_CORRUPT);
                id = kNone; // dropped from the list: never handed out
            }
        }
    }
    if (g.lane == 0 && id == kNone) {
        // The groups of a warp that allocate at the same time share one atomic per region (the
        // bump pointers are single addresses every allocation in the launch goes through).
        namespace cg = cooperative_groups;
        const cg::coalesced_group leaders = cg::coalesced_threads();
        const unsigned long long w = body_words(k);
        const unsigned long long before = cg::exclusive_scan(leaders, w);
        const unsigned long long total = leaders.shfl(before + w, leaders.num_threads() - 1);
        unsigned long long hbase = 0, obase = 0;
        if (leaders.thread_rank() == 0) {
            hbase = atomicAdd(&d.ctl->headerTop, (unsigned long long)leaders.num_threads());
            obase = atomicAdd(&d.ctl->itemTop, total);
        }
        const unsigned long long hid = leaders.shfl(hbase, 0) + leaders.thread_rank();
        const unsigned long long o = leaders.shfl(obase, 0) + before;
        if (hid < d.headerCount && o + w <= d.itemWords) {
            id = (uint32_t)hid;
            body = (uint32_t)(o / kUnitWords); // itemTop stays a multiple of 32 words
        } else {
            set_status(d.ctl, SVDAG_ERR_OOM);
        }
    }
    id = g.bcast(id, 0);
    body = g.bcast(body, 0);
    if (id != kNone) {
        // Free slots keep zero words (a valid key is never all zero), so the whole body is cleared.
        const uint32_t bw = body_words(k);
        uint32_t* p = handle_ptr(d, body);
        for (uint32_t i = g.lane * 4; i < bw; i += G * 4)
            *reinterpret_cast<uint4*>(p + i) = make_uint4(0, 0, 0, 0);
        if (g.lane == 0) {
            uint32_t* h = slab_ptr(d, id);
            reinterpret_cast<uint4*>(h)[0] = make_uint4(0, 0, 0, 0);
            reinterpret_cast<uint4*>(h)[1] = make_uint4(0, 0, body, kEnd);
        }
        __threadfence();
        g.sync();
    }
    return id;
}

// Links `fresh` behind `slab`; returns the slab that follows `slab` afterwards (ours or a racer's).
__device__ __forceinline__ uint32_t link_slab(const DevDag& d, uint32_t slab, uint32_t fresh)
{
    const uint32_t prev = atomicCAS(slab_ptr(d, slab) + 7, kEnd, fresh);
    return prev == kEnd ? fresh : prev;
}

// An overflow slab allocated by a group that lost the race to link it; it may only be linked into a
// chain of the same size class later.
struct Spare {
    uint32_t slab = kNone;
    uint32_t k = 0;
};

// Gives an unused spare back: a level table's goes on its class's free list; other tables' spares
// stay allocated (their space comes back when the bump pointers are rewound or never).
template <int G>
__device__ __forceinline__ void release_spare(const Grp<G>& g, const DevDag& d, const DevTable& t, Spare& spare)
{
    if (spare.slab != kNone && t.recycle && g.lane == 0)
        push_free_chain(d, spare.k - 2u, spare.slab, spare.slab, 1);
    spare.slab = kNone;
}
// A spare of another size class than `k` is released before a new one is allocated.
template <int G>
__device__ __forceinline__ void take_spare(const Grp<G>& g, const DevDag& d, const DevTable& t, Spare& spare, uint32_t k)
{
    if (spare.slab == kNone || spare.k != k) {
        release_spare<G>(g, d, t, spare);
        spare.slab = alloc_slab<G>(g, d, k, t.recycle);
        spare.k = k;
    }
}

constexpr uint32_t kMaxChain = 1u << 14; // bound on chain walks (16K slabs in one bucket only happens on a corrupt chain)

// Read-only lookup (CompactAccelerationHashTable::findAsWarp, compact_acceleration_hash_table.h:233-280).
// Candidate items are streamed (read once) so that the slab header sectors stay resident in L2.
template <int G>
__device__ __forceinline__ uint32_t table_find(const Grp<G>& g, const DevDag& d, const DevTable& t, const Key<G>& key)
{
    const uint32_t cls = key.n - 2u;
    if (key.n < 2u || key.n > 10u || t.numBuckets[cls] == 0)
        return kNone;
    const uint32_t tag = tag_of(key.hb);
    uint32_t slab = first_slab(t, cls, key.ha);
    for (uint32_t steps = 0;; ++steps) {
        if (steps >= kMaxChain) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        uint32_t next, body, empty;
        uint32_t cand = probe_header<G, false, false>(g, slab_ptr(d, slab), tag, next, body, empty);
        while (cand) {
            const uint32_t s = __ffs(cand) - 1u;
            cand &= cand - 1u;
            const uint32_t item = slot_handle(body, s, key.n);
            if (item_equals<G, LD_DEFAULT>(g, handle_ptr(d, item), key))
                return item;
        }
        if (next == kEnd)
            return kNone;
        if (!slab_ok(d, next)) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        slab = next;
    }
}

// Claims a free slot of `slab` for the key; returns the item offset or kNone when the slab is full.
// `busy` claims with the in-flight tag (published later), otherwise with the final tag.
template <int G>
__device__ __forceinline__ uint32_t claim_in_slab(const Grp<G>& g, const DevDag& d, uint32_t slab, uint32_t body, uint32_t emptyMask,
    uint32_t tag, uint32_t n, bool busy, uint32_t& slot, uint32_t spread, const HdrSnap<G>* snap = nullptr)
{
    // Claimants of one slab start at different free slots (`spread` is a hash of the key), so that
    // they do not all race for the first free slot of the same snapshot.
    const uint32_t start = spread % kSlots;
    while (emptyMask) {
        const uint32_t up = emptyMask >> start;
        const uint32_t s = up ? start + (uint32_t)__ffs(up) - 1u : (uint32_t)__ffs(emptyMask) - 1u;
        const uint32_t word = s >> 2, shift = 8u * (s & 3u);
        uint32_t got = 0;
        // The lane that probed the tag word claims (its probed value is the first guess; a stale
        // guess only costs one failed compare-and-swap, which returns the current word).
        const uint32_t claimer = snap ? HdrSnap<G>::owner(word) : 0u;
        if (g.lane == claimer) {
            uint32_t* p = slab_ptr(d, slab) + word;
            uint32_t cur = snap ? snap->get(word, g.lane) : *reinterpret_cast<volatile uint32_t*>(p);
            for (;;) {
                if ((cur >> shift) & 0xFFu)
                    break; // taken meanwhile
                const uint32_t want = cur | ((busy ? kTagBusy : tag) << shift);
                const uint32_t old = atomicCAS(p, cur, want);
                if (old == cur) {
                    got = 1;
                    break;
                }
                cur = old;
            }
        }
        got = g.bcast(got, claimer);
        if (got) {
            slot = s;
            return slot_handle(body, s, n);
        }
        emptyMask &= ~(1u << s);
    }
    return kNone;
}

// Unconditional insert (CompactAccelerationHashTable::addAsWarp, compact_acceleration_hash_table.h:63-121):
// the key gets a fresh slot even when an equal key is stored already.
template <int G>
__device__ __forceinline__ uint32_t table_add(const Grp<G>& g, const DevDag& d, const DevTable& t, const Key<G>& key, Spare& spare)
{
    const uint32_t cls = key.n - 2u;
    if (key.n < 2u || key.n > 10u || t.numBuckets[cls] == 0) {
        set_status(d.ctl, SVDAG_ERR_INVALID);
        return kNone;
    }
    const uint32_t tag = tag_of(key.hb);
    uint32_t slab = first_slab(t, cls, key.ha);
    for (uint32_t steps = 0; steps < kMaxChain; ++steps) {
        uint32_t next, body, empty, slot;
        HdrSnap<G> snap;
        probe_header<G>(g, slab_ptr(d, slab), tag, next, body, empty, &snap);
        const uint32_t item = claim_in_slab<G>(g, d, slab, body, empty, tag, key.n, false, slot, key.ha >> 8, &snap);
        if (item != kNone) {
            write_item<G>(g, handle_ptr(d, item), key);
            return item;
        }
        if (next == kEnd) {
            take_spare<G>(g, d, t, spare, key.n);
            if (spare.slab == kNone)
                return kNone;
            uint32_t linked = kNone;
            if (g.lane == 0)
                linked = link_slab(d, slab, spare.slab);
            linked = g.bcast(linked, 0);
            if (linked == spare.slab)
                spare.slab = kNone;
            next = linked;
        }
        if (!slab_ok(d, next)) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        slab = next;
    }
    set_status(d.ctl, SVDAG_ERR_TIMEOUT);
    return kNone;
}

constexpr uint32_t kLockTries = 1u << 20; // bound on waiting for a bucket lock (about 30 ms)

// Find-or-insert for keys that no other group of the same launch looks up (the DAG merge inserts
// each distinct item once). A slot is claimed with the in-flight tag, the item written, then the
// final tag published, so concurrent probes of other keys never compare a half-written item.
template <int G>
__device__ __forceinline__ uint32_t table_find_or_insert_one(const Grp<G>& g, const DevDag& d, const DevTable& t, const Key<G>& key,
    Spare& spare, bool& inserted);

// Insert modes of table_find_or_insert: the default (keys that no other group of the launch looks
// up) and shared (several threads may insert the same key at once: under the bucket lock).
enum : int { kInsertLaunch = 0, kInsertShared = 1 };

// Find-or-insert. In the shared mode (one thread per key, G = 1), several threads may look up and
// insert the same key at once (the blocks and the path threads of a group of subtree edits): the
// lookup and insert then run under the bucket's lock (a striped lock word in d.locks), so the
// second of two equal keys finds the first's published item. A holder only probes and inserts into its own chain, so no lock waits on
// another; the wait for a lock is bounded and ends with SVDAG_ERR_TIMEOUT.
template <int G, int MODE = kInsertLaunch>
__device__ __forceinline__ uint32_t table_find_or_insert(const Grp<G>& g, const DevDag& d, const DevTable& t, const Key<G>& key,
    Spare& spare, bool& inserted)
{
    if constexpr (MODE == kInsertShared && G == 1) {
        inserted = false;
        const uint32_t cls = key.n - 2u;
        if (key.n < 2u || key.n > 10u || t.numBuckets[cls] == 0 || !d.locks) {
            set_status(d.ctl, SVDAG_ERR_INVALID);
            return kNone;
        }
        uint32_t* lock = d.locks + (first_slab(t, cls, key.ha) & (kLockStripes - 1u));
        uint32_t tries = 0;
        while (atomicCAS(lock, 0u, 1u) != 0u) {
            if (++tries >= kLockTries) {
                set_status(d.ctl, SVDAG_ERR_TIMEOUT);
                return kNone;
            }
            __nanosleep(32);
        }
        __threadfence(); // acquire: the previous holder's item and tag are visible
        const uint32_t h = table_find_or_insert_one<G>(g, d, t, key, spare, inserted);
        __threadfence(); // release: this holder's item and tag are visible before the lock is free
        atomicExch(lock, 0u);
        return h;
    } else {
        return table_find_or_insert_one<G>(g, d, t, key, spare, inserted);
    }
}

template <int G>
__device__ __forceinline__ uint32_t table_find_or_insert_one(const Grp<G>& g, const DevDag& d, const DevTable& t, const Key<G>& key,
    Spare& spare, bool& inserted)
{
    inserted = false;
    const uint32_t cls = key.n - 2u;
    if (key.n < 2u || key.n > 10u || t.numBuckets[cls] == 0) {
        set_status(d.ctl, SVDAG_ERR_INVALID);
        return kNone;
    }
    const uint32_t tag = tag_of(key.hb);
    uint32_t slab = first_slab(t, cls, key.ha);
    uint32_t tail = slab, tailEmpty = 0, tailBody = 0;
    uint32_t open = kNone, openEmpty = 0, openBody = 0; // first slab of the chain with a free slot
    HdrSnap<G> snap;
    for (uint32_t steps = 0;; ++steps) {
        if (steps >= kMaxChain) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        uint32_t next, body, empty;
        uint32_t cand = probe_header<G, true>(g, slab_ptr(d, slab), tag, next, body, empty, &snap);
        while (cand) {
            const uint32_t s = __ffs(cand) - 1u;
            cand &= cand - 1u;
            const uint32_t item = slot_handle(body, s, key.n);
            if (item_equals<G, LD_L2>(g, handle_ptr(d, item), key))
                return item;
        }
        tail = slab;
        tailEmpty = empty;
        tailBody = body;
        if (open == kNone && empty) {
            open = slab;
            openEmpty = empty;
            openBody = body;
        }
        if (next == kEnd)
            break;
        if (!slab_ok(d, next)) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        slab = next;
    }
    // Not present: claim a slot in the first slab that had one free (slots freed by garbage
    // collection are reused before the chain grows), else at the tail of the chain.
    const bool atTail = open == kNone || open == tail;
    slab = atTail ? tail : open;
    uint32_t empty = atTail ? tailEmpty : openEmpty, body = atTail ? tailBody : openBody;
    bool snapValid = atTail; // `snap` holds the tag words of the tail, the last slab probed
    for (uint32_t steps = 0; steps < kMaxChain; ++steps) {
        uint32_t s = 0;
        const uint32_t item = claim_in_slab<G>(g, d, slab, body, empty, tag, key.n, true, s, key.ha >> 8, snapValid ? &snap : nullptr);
        snapValid = true;
        if (item != kNone) {
            write_item<G>(g, handle_ptr(d, item), key);
            if constexpr (G == 1)
                fence_release(); // the writer publishes: a release orders its item before the tag
            else
                __threadfence();
            g.sync();
            if (g.lane == 0)
                atomicXor(slab_ptr(d, slab) + (s >> 2), (kTagBusy ^ tag) << (8u * (s & 3u)));
            inserted = true;
            return item;
        }
        uint32_t next;
        probe_header<G, true>(g, slab_ptr(d, slab), tag, next, body, empty, &snap);
        if (empty)
            continue; // a slot was freed up meanwhile (cannot happen during edits, kept for safety)
        if (next == kEnd) {
            take_spare<G>(g, d, t, spare, key.n);
            if (spare.slab == kNone)
                return kNone;
            uint32_t linked = kNone;
            if (g.lane == 0)
                linked = link_slab(d, slab, spare.slab);
            linked = g.bcast(linked, 0);
            if (linked == spare.slab)
                spare.slab = kNone;
            next = linked;
        }
        if (!slab_ok(d, next)) {
            set_status(d.ctl, SVDAG_ERR_CORRUPT);
            return kNone;
        }
        slab = next;
        probe_header<G, true>(g, slab_ptr(d, slab), tag, next, body, empty, &snap);
    }
    set_status(d.ctl, SVDAG_ERR_TIMEOUT);
    return kNone;
}

} // namespace svdag
