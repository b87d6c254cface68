// svdag_alt_tables.cuh - the reference's alternative table layouts for fixed-size items, as tables
// of their own: TicketBoard (ticket_board_hash_table.h), Atomic64 (atomic64_hash_table.h),
// Acceleration (acceleration_hash_table.h) and IndividualChaining (individual_chaining_hash_table.h).
// The compact 8-bit-tag layout is the level tables' (svdag_device.cuh). These serve the fixed-size
// hashmap workload of the reference's table benchmark (extras/hashmap_bench/src/main.cu) so the
// layouts can be measured against each other.
//
// One table is one device allocation: a control block and an arena of equal-sized slabs. Slabs
// 0..numBuckets-1 are the buckets' first slabs; overflow slabs are taken from a bump counter and
// linked at the tail of a chain. The arena is zeroed when the table is created and a slab is never
// given back to the counter (slots freed by garbage collection are reused in place), so a fresh
// slab needs no initialisation and a next word of 0 ends a chain (no overflow slab has id 0;
// kLinkBusy marks a link being made). A handle is slab * 32 + slot.
//
// Slab layouts (32-bit words; a slab's stride is rounded up to 8 words, 32 bytes):
//   TicketBoard : [0] occupied-slot mask, [1] next, [2..7] unused, items of slots 0..31 from word 8.
//                 A slot is claimed by an atomic OR of its bit, then the item is written.
//   Atomic64    : words 2s, 2s+1 = the first 8 bytes of slot s's item (s = 0..30, 0 = free),
//                 [62] next, [63] unused, the other k-2 words of slot s's item from word 64.
//                 A slot is claimed by a 64-bit CAS of its first 8 bytes; items whose first two
//                 words are both 0 cannot be stored (the reference requires the same).
//   Acceleration: [0] next, [s] = 32-bit tag of slot s (s = 1..31, 0 = free), items of slots
//                 1..31 from word 32. A slot is claimed by a CAS of its tag.
// IndividualChaining (individual_chaining_hash_table.h) has no slabs: a head word per bucket and an
// arena of nodes of k + 1 words (the item, then the next node's id + 1, 0 = end), taken from a bump
// counter and pushed onto the bucket's head by CAS. Its handle is the node's id.
//
// The thread-per-key functions below compile for the device and, unchanged, for the host (the
// atomics are GCC builtins there), so their claim and chain logic can be exercised by host threads.
// Adds and finds must not overlap in time (the reference's bulk phases do the same): a finder may
// see a claimed slot before its item is written.
#pragma once
#include <cstdint>

#include "../../include/svdag.h"
#include "svdag_hash.h"

namespace svdag {
namespace alt {

enum Layout : uint32_t { kTicketBoard = 1, kAtomic64 = 2, kAcceleration = 3, kIndividualChaining = 4 };

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kNoSlab = 0xFFFFFFFFu;
constexpr uint32_t kMaxItemWords = 32;
constexpr uint32_t kMaxSlabs = 1u << 27; // handles slab * 32 + slot stay below 2^32 - 1
constexpr uint32_t kMaxNodes = 1u << 30; // IndividualChaining nodes (handles are node ids)
constexpr uint32_t kMaxSteps = 1u << 22; // slabs one add or find may visit before it gives up
constexpr uint32_t kLinkBusy = 0xFFFFFFFFu; // next word of a slab whose successor is being linked
constexpr uint32_t kMaxSpin = 1u << 20; // reads of a busy next word before a wait gives up

// Control block words.
enum Ctl : uint32_t { kCtlNextSlab = 0, kCtlStatus = 1, kCtlWords = 8 };

struct AltTable {
    uint32_t layout;
    uint32_t k; // item words
    uint32_t numBuckets;
    uint32_t slabWords; // stride of a slab in words, a multiple of 8 (IndividualChaining: of a node, k + 1)
    uint32_t slabCount; // slabs in the arena (IndividualChaining: nodes)
    uint32_t pad;
    uint32_t* slabs; // the arena (IndividualChaining: the nodes)
    uint32_t* ctl;
    uint32_t* heads; // IndividualChaining: first node id + 1 of each bucket (0 = empty); else null
    uint32_t* active; // garbage-collection flags: bit (h & 31) of word (h >> 5) for handle h
};

SVDAG_HD uint32_t round8(uint32_t w) { return (w + 7u) & ~7u; }
SVDAG_HD uint32_t slab_words(uint32_t layout, uint32_t k)
{
    return layout == kTicketBoard ? round8(8u + 32u * k) : layout == kAtomic64 ? round8(64u + 31u * (k - 2u)) : round8(32u + 31u * k);
}
SVDAG_HD uint32_t slots_per_slab(uint32_t layout) { return layout == kTicketBoard ? 32u : 31u; }
SVDAG_HD uint32_t next_word(uint32_t layout) { return layout == kTicketBoard ? 1u : layout == kAtomic64 ? 62u : 0u; }
SVDAG_HD bool layout_ok(uint32_t layout, uint32_t k)
{
    return (layout == kTicketBoard || layout == kAcceleration || layout == kIndividualChaining) ? (k >= 1 && k <= kMaxItemWords)
         : layout == kAtomic64 ? (k >= 2 && k <= kMaxItemWords) : false;
}
// Slabs of a table's arena: the bucket slabs and overflow slabs for `reserved` more items, or 0 when
// that exceeds kMaxSlabs.
inline uint32_t arena_slabs(uint32_t layout, uint32_t numBuckets, uint64_t reserved)
{
    const uint64_t overflow = (reserved + slots_per_slab(layout) - 1) / slots_per_slab(layout);
    const uint64_t slabs = (uint64_t)numBuckets + overflow;
    return slabs > kMaxSlabs ? 0u : (uint32_t)slabs;
}
// Words of a table's active-flag bitmap: one per slab, or one per 32 nodes.
SVDAG_HD uint32_t active_words(const AltTable& t) { return t.layout == kIndividualChaining ? (t.slabCount + 31u) / 32u : t.slabCount; }

// Bytes of a table's single allocation, 0 when the sizes exceed the handle space. With `base` set,
// *t becomes the descriptor of a table in that allocation: a 256-byte control block, then the
// IndividualChaining heads (rounded to 256 bytes), the arena (rounded to 256 bytes) and the
// active-flag bitmap.
inline uint64_t table_layout(uint32_t layout, uint32_t k, uint32_t numBuckets, uint64_t reserved, void* base, AltTable* t)
{
    AltTable d {};
    d.layout = layout;
    d.k = k;
    d.numBuckets = numBuckets;
    uint64_t headBytes = 0, count = 0;
    if (layout == kIndividualChaining) {
        count = reserved ? reserved : 1;
        if (count > kMaxNodes)
            return 0;
        headBytes = ((uint64_t)numBuckets * 4u + 255u) & ~255ull;
        d.slabWords = k + 1;
    } else {
        count = arena_slabs(layout, numBuckets, reserved);
        if (!count)
            return 0;
        d.slabWords = slab_words(layout, k);
    }
    d.slabCount = (uint32_t)count;
    const uint64_t arenaBytes = (count * d.slabWords * 4ull + 255u) & ~255ull;
    const uint64_t activeBytes = active_words(d) * 4ull;
    if (base) {
        d.ctl = (uint32_t*)base;
        d.heads = headBytes ? (uint32_t*)((char*)base + 256) : nullptr;
        d.slabs = (uint32_t*)((char*)base + 256 + headBytes);
        d.active = (uint32_t*)((char*)base + 256 + headBytes + arenaBytes);
        *t = d;
    }
    return 256 + headBytes + arenaBytes + activeBytes;
}
// Initial value of the control block's bump counter: overflow slabs follow the bucket slabs; nodes
// start at 0.
inline uint32_t initial_counter(uint32_t layout, uint32_t numBuckets) { return layout == kIndividualChaining ? 0u : numBuckets; }

// Slot numbers a layout uses: 0..31, 0..30 or 1..31.
SVDAG_HD bool slot_ok(uint32_t layout, uint32_t slot)
{
    return layout == kTicketBoard ? slot < 32u : layout == kAtomic64 ? slot < 31u : (slot >= 1u && slot < 32u);
}
// Word offset (in its slab) of the stored part of slot s's item: all k words, or the last k-2 for Atomic64.
SVDAG_HD uint32_t body_word(uint32_t layout, uint32_t k, uint32_t s)
{
    return layout == kTicketBoard ? 8u + s * k : layout == kAtomic64 ? 64u + s * (k - 2u) : 32u + (s - 1u) * k;
}

// ---------------------------------------------------------------- atomics (device / host builtins)

#ifdef __CUDA_ARCH__
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ uint64_t ld_relaxed64(const uint64_t* p) { return *(const volatile uint64_t*)p; }
__device__ __forceinline__ uint32_t cas32(uint32_t* p, uint32_t cmp, uint32_t v) { return atomicCAS(p, cmp, v); }
__device__ __forceinline__ uint64_t cas64(uint64_t* p, uint64_t cmp, uint64_t v)
{
    return atomicCAS((unsigned long long*)p, (unsigned long long)cmp, (unsigned long long)v);
}
__device__ __forceinline__ uint32_t or32(uint32_t* p, uint32_t v) { return atomicOr(p, v); }
__device__ __forceinline__ uint32_t add32(uint32_t* p, uint32_t v) { return atomicAdd(p, v); }
__device__ __forceinline__ uint32_t exch32(uint32_t* p, uint32_t v) { return atomicExch(p, v); }
__device__ __forceinline__ uint32_t ctz32(uint32_t v) { return __ffs(v) - 1u; }
__device__ __forceinline__ uint32_t popc32(uint32_t v) { return __popc(v); }
#else
inline uint32_t ld_relaxed(const uint32_t* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline uint64_t ld_relaxed64(const uint64_t* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline uint32_t cas32(uint32_t* p, uint32_t cmp, uint32_t v)
{
    __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE);
    return cmp;
}
inline uint64_t cas64(uint64_t* p, uint64_t cmp, uint64_t v)
{
    __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE);
    return cmp;
}
inline uint32_t or32(uint32_t* p, uint32_t v) { return __atomic_fetch_or(p, v, __ATOMIC_ACQ_REL); }
inline uint32_t add32(uint32_t* p, uint32_t v) { return __atomic_fetch_add(p, v, __ATOMIC_ACQ_REL); }
inline uint32_t exch32(uint32_t* p, uint32_t v) { return __atomic_exchange_n(p, v, __ATOMIC_ACQ_REL); }
inline uint32_t ctz32(uint32_t v) { return (uint32_t)__builtin_ctz(v); }
inline uint32_t popc32(uint32_t v) { return (uint32_t)__builtin_popcount(v); }
#endif

SVDAG_HD void set_status(const AltTable& t, uint32_t st) { cas32(&t.ctl[kCtlStatus], 0u, st); }
SVDAG_HD uint32_t* slab_at(const AltTable& t, uint32_t slab) { return t.slabs + (uint64_t)slab * t.slabWords; }

// Key hash over the k words (the level tables' hash, svdag_hash.h).
SVDAG_HD uint32_t key_acc(const uint32_t* key, uint32_t k)
{
    uint32_t acc = 0;
    for (uint32_t i = 0; i < k; ++i)
        acc ^= word_term(key[i], i);
    return acc;
}
SVDAG_HD uint32_t acc_tag32(uint32_t acc)
{
    const uint32_t t = tag_hash(acc);
    return t ? t : 1u;
}
SVDAG_HD uint64_t key_prefix(const uint32_t* key) { return (uint64_t)key[0] | ((uint64_t)key[1] << 32); }
SVDAG_HD bool words_equal(const uint32_t* a, const uint32_t* b, uint32_t n)
{
    bool eq = true;
    for (uint32_t i = 0; i < n; ++i)
        eq &= a[i] == b[i];
    return eq;
}

// Claims a free slot of slab s for the key (tag / prefix already computed); the slot or kInvalid if
// the slab is full. Each failed claim is a slot another thread took, so the loops are bounded by 32.
SVDAG_HD uint32_t try_claim(const AltTable& t, uint32_t* s, uint32_t tag, uint64_t prefix)
{
    if (t.layout == kTicketBoard) {
        uint32_t m = ld_relaxed(&s[0]);
        while (m != 0xFFFFFFFFu) {
            const uint32_t slot = ctz32(~m);
            const uint32_t old = or32(&s[0], 1u << slot);
            if (!(old & (1u << slot)))
                return slot;
            m = old | (1u << slot);
        }
        return kInvalid;
    }
    if (t.layout == kAtomic64) {
        uint64_t* pre = (uint64_t*)s;
        for (uint32_t slot = 0; slot < 31u; ++slot)
            if (ld_relaxed64(&pre[slot]) == 0 && cas64(&pre[slot], 0, prefix) == 0)
                return slot;
        return kInvalid;
    }
    for (uint32_t slot = 1; slot < 32u; ++slot)
        if (ld_relaxed(&s[slot]) == 0 && cas32(&s[slot], 0u, tag) == 0)
            return slot;
    return kInvalid;
}

// Slot of slab s holding the key, or kInvalid.
SVDAG_HD uint32_t match_slab(const AltTable& t, const uint32_t* s, const uint32_t* key, uint32_t tag, uint64_t prefix)
{
    const uint32_t k = t.k;
    if (t.layout == kTicketBoard) {
        uint32_t m = s[0];
        while (m) {
            const uint32_t slot = ctz32(m);
            m &= m - 1u;
            if (words_equal(s + body_word(kTicketBoard, k, slot), key, k))
                return slot;
        }
        return kInvalid;
    }
    if (t.layout == kAtomic64) {
        const uint64_t* pre = (const uint64_t*)s;
        for (uint32_t slot = 0; slot < 31u; ++slot)
            if (pre[slot] == prefix && words_equal(s + body_word(kAtomic64, k, slot), key + 2, k - 2u))
                return slot;
        return kInvalid;
    }
    for (uint32_t slot = 1; slot < 32u; ++slot)
        if (s[slot] == tag && words_equal(s + body_word(kAcceleration, k, slot), key, k))
            return slot;
    return kInvalid;
}

// Next slab of a chain after slab s, linking a new one when the chain ends there. The thread that
// turns the next word from 0 to kLinkBusy takes a slab from the bump counter and stores its id;
// threads that meet kLinkBusy wait for the id (the holder waits for nothing in between, so the wait
// is short; it is bounded all the same). One slab is taken per link and none is lost, where taking
// a slab before the race for the link would strand the losers' slabs (the reference frees them,
// gpu_hash_table_base.h:128-219). kNoSlab with the status latched on exhaustion, a bad link or a
// wait that gave up.
SVDAG_HD uint32_t next_or_link(const AltTable& t, uint32_t* s)
{
    uint32_t* link = &s[next_word(t.layout)];
    uint32_t nx = ld_relaxed(link);
    for (uint32_t spin = 0; nx == 0 || nx == kLinkBusy; ++spin) {
        if (spin >= kMaxSpin) {
            set_status(t, SVDAG_ERR_TIMEOUT);
            return kNoSlab;
        }
        if (nx == 0) {
            nx = cas32(link, 0u, kLinkBusy);
            if (nx == 0) {
                const uint32_t fresh = add32(&t.ctl[kCtlNextSlab], 1u);
                if (fresh >= t.slabCount) {
                    exch32(link, 0u); // the chain ends here again; later arrivals fail the same way
                    set_status(t, SVDAG_ERR_OOM);
                    return kNoSlab;
                }
                exch32(link, fresh);
                return fresh;
            }
        } else {
#ifdef __CUDA_ARCH__
            __nanosleep(32); // yield: the link's holder may be a thread of this warp
#endif
            nx = ld_relaxed(link);
        }
    }
    if (nx < t.numBuckets || nx >= t.slabCount) {
        set_status(t, SVDAG_ERR_CORRUPT);
        return kNoSlab;
    }
    return nx;
}

// IndividualChaining add (individual_chaining_hash_table.h:271-296): a node from the counter, the
// item written, then pushed onto the bucket's head by CAS with its next word set to the head it
// replaces. Each failed CAS is another push that succeeded; the loop is bounded all the same.
SVDAG_HD uint32_t chain_add(const AltTable& t, const uint32_t* key)
{
    const uint32_t k = t.k;
    uint32_t* head = &t.heads[bucket_index(bucket_hash(key_acc(key, k)), t.numBuckets)];
    const uint32_t id = add32(&t.ctl[kCtlNextSlab], 1u);
    if (id >= t.slabCount) {
        set_status(t, SVDAG_ERR_OOM);
        return kInvalid;
    }
    uint32_t* node = slab_at(t, id);
    for (uint32_t i = 0; i < k; ++i)
        node[i] = key[i];
    uint32_t old = ld_relaxed(head);
    for (uint32_t spin = 0; spin < kMaxSpin; ++spin) {
        node[k] = old;
        const uint32_t seen = cas32(head, old, id + 1u);
        if (seen == old)
            return id;
        old = seen;
    }
    set_status(t, SVDAG_ERR_TIMEOUT);
    return kInvalid;
}

// IndividualChaining find (individual_chaining_hash_table.h:236-248): the first node of the chain
// holding the key (the most recently added copy).
SVDAG_HD uint32_t chain_find(const AltTable& t, const uint32_t* key)
{
    const uint32_t k = t.k;
    uint32_t cur = t.heads[bucket_index(bucket_hash(key_acc(key, k)), t.numBuckets)];
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
        if (cur == 0)
            return kInvalid;
        if (cur > t.slabCount) {
            set_status(t, SVDAG_ERR_CORRUPT);
            return kInvalid;
        }
        const uint32_t* node = slab_at(t, cur - 1u);
        if (words_equal(node, key, k))
            return cur - 1u;
        cur = node[k];
    }
    set_status(t, SVDAG_ERR_TIMEOUT);
    return kInvalid;
}

// add (ticket_board_hash_table.h:24-60, atomic64_hash_table.h:36-64, acceleration_hash_table.h:31-72):
// stores the key in a fresh slot, duplicates included, and returns its handle.
SVDAG_HD uint32_t add(const AltTable& t, const uint32_t* key)
{
    if (t.layout == kIndividualChaining)
        return chain_add(t, key);
    const uint32_t k = t.k;
    const uint32_t acc = key_acc(key, k);
    const uint32_t tag = acc_tag32(acc);
    const uint64_t prefix = t.layout == kAtomic64 ? key_prefix(key) : 0;
    if (t.layout == kAtomic64 && prefix == 0) {
        set_status(t, SVDAG_ERR_INVALID);
        return kInvalid;
    }
    uint32_t slab = bucket_index(bucket_hash(acc), t.numBuckets);
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
        uint32_t* s = slab_at(t, slab);
        const uint32_t slot = try_claim(t, s, tag, prefix);
        if (slot != kInvalid) {
            const uint32_t first = t.layout == kAtomic64 ? 2u : 0u;
            uint32_t* dst = s + body_word(t.layout, k, slot);
            for (uint32_t i = first; i < k; ++i)
                dst[i - first] = key[i];
            return slab * 32u + slot;
        }
        slab = next_or_link(t, s);
        if (slab == kNoSlab)
            return kInvalid;
    }
    set_status(t, SVDAG_ERR_TIMEOUT);
    return kInvalid;
}

// find (ticket_board_hash_table.h:176-197, atomic64_hash_table.h:194-214, acceleration_hash_table.h):
// handle of a stored copy of the key, or kInvalid.
SVDAG_HD uint32_t find(const AltTable& t, const uint32_t* key)
{
    if (t.layout == kIndividualChaining)
        return chain_find(t, key);
    const uint32_t k = t.k;
    const uint32_t acc = key_acc(key, k);
    const uint32_t tag = acc_tag32(acc);
    const uint64_t prefix = t.layout == kAtomic64 ? key_prefix(key) : 0;
    if (t.layout == kAtomic64 && prefix == 0)
        return kInvalid;
    uint32_t slab = bucket_index(bucket_hash(acc), t.numBuckets);
    for (uint32_t step = 0; step < kMaxSteps; ++step) {
        const uint32_t* s = slab_at(t, slab);
        const uint32_t slot = match_slab(t, s, key, tag, prefix);
        if (slot != kInvalid)
            return slab * 32u + slot;
        const uint32_t nx = s[next_word(t.layout)];
        if (nx == 0)
            return kInvalid;
        if (nx < t.numBuckets || nx >= t.slabCount) {
            set_status(t, SVDAG_ERR_CORRUPT);
            return kInvalid;
        }
        slab = nx;
    }
    set_status(t, SVDAG_ERR_TIMEOUT);
    return kInvalid;
}

// Whether slot `slot` of slab s is occupied.
SVDAG_HD bool slot_used(uint32_t layout, const uint32_t* s, uint32_t slot)
{
    return layout == kTicketBoard ? ((s[0] >> slot) & 1u) != 0
         : layout == kAtomic64 ? ((const uint64_t*)s)[slot] != 0 : s[slot] != 0;
}

// decodePointer: the k words of a handle's item into out[0..k); false for a handle that names no
// stored item (out is then zeroed).
SVDAG_HD bool read(const AltTable& t, uint32_t h, uint32_t* out)
{
    if (t.layout == kIndividualChaining) {
        const bool ok = h < t.slabCount && h < ld_relaxed(&t.ctl[kCtlNextSlab]);
        for (uint32_t i = 0; i < t.k; ++i)
            out[i] = ok ? slab_at(t, h)[i] : 0u;
        return ok;
    }
    const uint32_t slab = h >> 5, slot = h & 31u, k = t.k;
    const bool ok = h != kInvalid && slab < t.slabCount && slot_ok(t.layout, slot) && slot_used(t.layout, slab_at(t, slab), slot);
    if (!ok) {
        for (uint32_t i = 0; i < k; ++i)
            out[i] = 0;
        return false;
    }
    const uint32_t* s = slab_at(t, slab);
    const uint32_t* body = s + body_word(t.layout, k, slot);
    if (t.layout == kAtomic64) {
        out[0] = s[2 * slot];
        out[1] = s[2 * slot + 1];
        for (uint32_t i = 2; i < k; ++i)
            out[i] = body[i - 2];
    } else {
        for (uint32_t i = 0; i < k; ++i)
            out[i] = body[i];
    }
    return true;
}

// Occupied slots of slab s.
SVDAG_HD uint32_t slab_items(uint32_t layout, const uint32_t* s)
{
    uint32_t n = 0;
    for (uint32_t slot = 0; slot < 32u; ++slot)
        n += slot_ok(layout, slot) && slot_used(layout, s, slot);
    return n;
}

// ---------------------------------------------------------------- garbage collection
//
// clearActiveFlags / markAsActive / freeInactiveItems (gpu_hash_table_base.h:102-112,
// gpu_hash_table_base.cu:231-330): the caller clears the flags, marks the handles it keeps, and the
// table frees every stored item left unmarked. A freed slot is free for later adds; the reference
// also unlinks overflow slabs left empty and returns them to its allocator, which this bump
// allocator has no use for: they stay linked and their slots are reused in place. Freed
// IndividualChaining nodes are unlinked from their lists (the reference's node allocator does not
// free either). These phases must not overlap adds or finds.

// markAsActive: sets the flag of handle h (handles outside the table are ignored).
SVDAG_HD void mark_active(const AltTable& t, uint32_t h)
{
    if (h != kInvalid && (h >> 5) < active_words(t))
        or32(&t.active[h >> 5], 1u << (h & 31u));
}

// Frees the unmarked items of slab `slab` (a slab layout); returns how many.
SVDAG_HD uint32_t free_inactive_slab(const AltTable& t, uint32_t slab)
{
    uint32_t* s = slab_at(t, slab);
    const uint32_t act = t.active[slab];
    if (t.layout == kTicketBoard) {
        const uint32_t dead = s[0] & ~act;
        s[0] &= ~dead;
        return popc32(dead);
    }
    uint32_t freed = 0;
    if (t.layout == kAtomic64) {
        uint64_t* pre = (uint64_t*)s;
        for (uint32_t slot = 0; slot < 31u; ++slot)
            if (!((act >> slot) & 1u) && pre[slot] != 0) {
                pre[slot] = 0;
                ++freed;
            }
        return freed;
    }
    for (uint32_t slot = 1; slot < 32u; ++slot)
        if (!((act >> slot) & 1u) && s[slot] != 0) {
            s[slot] = 0;
            ++freed;
        }
    return freed;
}

// Unlinks the unmarked nodes of bucket b's list (IndividualChaining); returns how many.
SVDAG_HD uint32_t free_inactive_chain(const AltTable& t, uint32_t b)
{
    uint32_t* link = &t.heads[b];
    uint32_t freed = 0;
    for (uint32_t steps = 0; steps < t.slabCount; ++steps) {
        const uint32_t cur = *link;
        if (cur == 0 || cur > t.slabCount)
            break;
        const uint32_t id = cur - 1u;
        uint32_t* node = slab_at(t, id);
        if ((t.active[id >> 5] >> (id & 31u)) & 1u) {
            link = &node[t.k];
        } else {
            *link = node[t.k];
            ++freed;
        }
    }
    return freed;
}

// ---------------------------------------------------------------- warp-hybrid forms
//
// addAsWarpHybrid / findAsWarpHybrid (atomic64_hash_table.h:125-185, 245-300 and the same pair in
// ticket_board_hash_table.h and acceleration_hash_table.h): every lane of a warp holds a key (or
// none), and the warp serves the lanes' keys one at a time, each lane inspecting one slot of the
// slab, so a slab's slot words are read by one coalesced load. W supplies the collectives lane(),
// ballot(p, site), shfl(v, src, site) and shfl64(v, src, site); every lane takes part in every call,
// in the same order (the loop conditions below are warp-uniform). `site` names the call (its source
// line): the CUDA kernels pass the warp intrinsics, which ignore it; the host tests pass an emulated
// warp that checks that all lanes of a warp stand at the same site.
#ifdef __CUDACC__
#define SVDAG_WARP_FN __device__ __forceinline__
#else
#define SVDAG_WARP_FN inline
#endif

// Whether slot `lane` of slab s holds the broadcast key.
template <uint32_t L>
SVDAG_HD bool lane_match(const AltTable& t, const uint32_t* s, uint32_t lane, const uint32_t* key, uint32_t tag, uint64_t prefix)
{
    const uint32_t k = t.k;
    if (L == kTicketBoard)
        return ((s[0] >> lane) & 1u) && words_equal(s + body_word(L, k, lane), key, k);
    if (L == kAtomic64)
        return lane < 31u && ((const uint64_t*)s)[lane] == prefix && words_equal(s + body_word(L, k, lane), key + 2, k - 2u);
    return lane >= 1u && s[lane] == tag && words_equal(s + body_word(L, k, lane), key, k);
}

template <class W>
SVDAG_WARP_FN const uint32_t* shfl_ptr(const W& w, const uint32_t* p, uint32_t src, uint32_t site)
{
    return (const uint32_t*)(uintptr_t)w.shfl64((uint64_t)(uintptr_t)p, src, site);
}

// This lane's result: the handle of a stored copy of its key, or kInvalid (a miss or no key).
template <uint32_t L, class W>
SVDAG_WARP_FN uint32_t warp_find(const W& w, const AltTable& t, const uint32_t* key, bool valid)
{
    const uint32_t lane = w.lane();
    uint32_t tag = 0, slab = 0, result = kInvalid;
    uint64_t prefix = 0;
    if (valid) {
        const uint32_t acc = key_acc(key, t.k);
        tag = acc_tag32(acc);
        prefix = L == kAtomic64 ? key_prefix(key) : 0;
        slab = bucket_index(bucket_hash(acc), t.numBuckets);
        valid = !(L == kAtomic64 && prefix == 0);
    }
    bool active = valid;
    uint32_t steps = 0;
    for (uint32_t mask; (mask = w.ballot(active, __LINE__)) != 0;) {
        if (++steps > kMaxSteps) { // warp-uniform
            if (active)
                set_status(t, SVDAG_ERR_TIMEOUT);
            break;
        }
        const uint32_t src = ctz32(mask);
        const uint32_t sSlab = w.shfl(slab, src, __LINE__);
        const uint32_t sTag = w.shfl(tag, src, __LINE__);
        const uint64_t sPrefix = w.shfl64(prefix, src, __LINE__);
        const uint32_t* sKey = shfl_ptr(w, key, src, __LINE__);
        const uint32_t* s = slab_at(t, sSlab);
        const uint32_t hits = w.ballot(lane_match<L>(t, s, lane, sKey, sTag, sPrefix), __LINE__);
        if (lane == src) {
            if (hits) {
                result = sSlab * 32u + ctz32(hits);
                active = false;
            } else {
                const uint32_t nx = s[next_word(L)];
                if (nx == 0) {
                    active = false;
                } else if (nx < t.numBuckets || nx >= t.slabCount) {
                    set_status(t, SVDAG_ERR_CORRUPT);
                    active = false;
                } else {
                    slab = nx;
                }
            }
        }
    }
    return result;
}

// This lane's handle: its key stored in a fresh slot (kInvalid for no key or on failure).
template <uint32_t L, class W>
SVDAG_WARP_FN uint32_t warp_add(const W& w, const AltTable& t, const uint32_t* key, bool valid)
{
    const uint32_t lane = w.lane();
    const uint32_t k = t.k;
    uint32_t tag = 0, slab = 0, result = kInvalid;
    uint64_t prefix = 0;
    if (valid) {
        const uint32_t acc = key_acc(key, k);
        tag = acc_tag32(acc);
        prefix = L == kAtomic64 ? key_prefix(key) : 0;
        slab = bucket_index(bucket_hash(acc), t.numBuckets);
        if (L == kAtomic64 && prefix == 0) {
            set_status(t, SVDAG_ERR_INVALID);
            valid = false;
        }
    }
    bool active = valid;
    uint32_t steps = 0;
    for (uint32_t mask; (mask = w.ballot(active, __LINE__)) != 0;) {
        if (++steps > kMaxSteps) { // warp-uniform
            if (active)
                set_status(t, SVDAG_ERR_TIMEOUT);
            break;
        }
        const uint32_t src = ctz32(mask);
        const uint32_t sSlab = w.shfl(slab, src, __LINE__);
        const uint32_t sTag = w.shfl(tag, src, __LINE__);
        const uint64_t sPrefix = w.shfl64(prefix, src, __LINE__);
        const uint32_t* sKey = shfl_ptr(w, key, src, __LINE__);
        uint32_t* s = slab_at(t, sSlab);
        uint32_t slot = kInvalid;
        if (L == kTicketBoard) {
            // one lane claims on the slot mask (at most 32 failed ORs)
            if (lane == src)
                slot = try_claim(t, s, sTag, sPrefix);
            slot = w.shfl(slot, src, __LINE__);
        } else {
            // every lane reads its slot word; the free ones are tried in order (each failed CAS is a
            // slot another warp took)
            const bool mine = L == kAtomic64 ? lane < 31u : lane >= 1u;
            const bool isFree = mine && (L == kAtomic64 ? ld_relaxed64((const uint64_t*)s + lane) == 0 : ld_relaxed(s + lane) == 0);
            uint32_t freeMask = w.ballot(isFree, __LINE__);
            while (freeMask) {
                const uint32_t d = ctz32(freeMask);
                uint32_t won = 0;
                if (lane == d)
                    won = L == kAtomic64 ? cas64((uint64_t*)s + d, 0, sPrefix) == 0 : cas32(s + d, 0u, sTag) == 0;
                if (w.shfl(won, d, __LINE__)) {
                    slot = d;
                    break;
                }
                freeMask &= freeMask - 1u;
            }
        }
        if (slot != kInvalid) {
            const uint32_t first = L == kAtomic64 ? 2u : 0u;
            if (lane < k - first)
                s[body_word(L, k, slot) + lane] = sKey[first + lane];
            if (lane == src) {
                result = sSlab * 32u + slot;
                active = false;
            }
        } else if (lane == src) {
            const uint32_t nx = next_or_link(t, s);
            if (nx == kNoSlab)
                active = false;
            else
                slab = nx;
        }
    }
    return result;
}

} // namespace alt
} // namespace svdag
