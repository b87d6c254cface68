// Host build of the alternative table layouts (gpu-svdag-editing_b200/csrc/svdag_alt_tables.cuh)
// for the CPU tests: the same thread-per-key add / find / read functions the CUDA kernels run, driven
// by std::threads that take keys round-robin, so that claims and chain links race as they do on the
// GPU; and the same warp-hybrid functions, run by emulated warps (32 lanes as coroutines on one
// thread per warp, switching at every collective). Test infrastructure only; the library's tables
// run on the GPU.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

#include <ucontext.h>

#include "../gpu-svdag-editing_b200/csrc/svdag_alt_tables.cuh"

using namespace svdag::alt;

namespace {

struct HostTable {
    AltTable t {};
    void* mem = nullptr;
};

template <class F>
void run_threads(uint32_t n, uint32_t threads, F&& f)
{
    if (threads <= 1) {
        for (uint32_t i = 0; i < n; ++i)
            f(i);
        return;
    }
    std::vector<std::thread> pool;
    for (uint32_t tid = 0; tid < threads; ++tid)
        pool.emplace_back([&, tid] {
            for (uint32_t i = tid; i < n; i += threads)
                f(i);
        });
    for (auto& th : pool)
        th.join();
}

// An emulated warp: one OS thread runs the 32 lanes as coroutines (ucontext), each lane running until
// its next collective, where it posts its value and its call site and yields. A pass of the scheduler
// over the lanes completes one collective; results are read from the posted values (two buffers by
// collective parity, so a lane that runs ahead cannot overwrite values another lane has yet to read).
// Lanes that stand at different call sites after a pass, or a lane that finishes while others wait at
// a collective, are divergent warp code: the process aborts with a message. Warps are separate OS threads, so they
// race on the table as warps do on the GPU.
struct CoWarp;

struct EmuWarp {
    CoWarp* cw;
    uint32_t ln;
    uint32_t lane() const { return ln; }
    uint32_t ballot(bool p, uint32_t site) const;
    uint32_t shfl(uint32_t v, uint32_t src, uint32_t site) const { return (uint32_t)exchange(v, src, site); }
    uint64_t shfl64(uint64_t v, uint32_t src, uint32_t site) const { return exchange(v, src, site); }
    uint64_t exchange(uint64_t v, uint32_t src, uint32_t site) const;
};

struct CoWarp {
    ucontext_t sched {};
    ucontext_t lane[32] {};
    std::vector<char> stack[32];
    uint64_t vals[2][32] = {};
    uint64_t seq[32] = {}; // collectives each lane has entered
    uint32_t site[32] = {}; // call site (source line) of each lane's current collective
    bool finished[32] = {};
    std::function<void(const EmuWarp&)> body;

    void post(uint32_t ln, uint64_t v, uint32_t at)
    {
        site[ln] = at;
        vals[seq[ln] & 1][ln] = v;
        ++seq[ln];
        swapcontext(&lane[ln], &sched);
    }
    static void entry(uint32_t hi, uint32_t lo, uint32_t ln)
    {
        CoWarp* cw = (CoWarp*)(((uintptr_t)hi << 32) | lo);
        cw->body(EmuWarp { cw, ln });
        cw->finished[ln] = true;
        // returning switches to uc_link (the scheduler)
    }
    void run()
    {
        for (uint32_t ln = 0; ln < 32; ++ln) {
            stack[ln].resize(256 * 1024);
            getcontext(&lane[ln]);
            lane[ln].uc_stack.ss_sp = stack[ln].data();
            lane[ln].uc_stack.ss_size = stack[ln].size();
            lane[ln].uc_link = &sched;
            const uintptr_t self = (uintptr_t)this;
            makecontext(&lane[ln], (void (*)())entry, 3, (uint32_t)(self >> 32), (uint32_t)self, ln);
        }
        for (;;) {
            uint32_t live = 0;
            for (uint32_t ln = 0; ln < 32; ++ln)
                if (!finished[ln]) {
                    swapcontext(&sched, &lane[ln]);
                    live += !finished[ln];
                }
            if (live == 0)
                return;
            for (uint32_t ln = 0; ln < 32; ++ln)
                if (finished[ln] || seq[ln] != seq[0] || site[ln] != site[0]) {
                    std::fprintf(stderr, "emulated warp: lanes diverged at a collective (lane %u)\n", ln);
                    std::abort();
                }
        }
    }
};

uint64_t EmuWarp::exchange(uint64_t v, uint32_t src, uint32_t at) const
{
    const uint64_t s = cw->seq[ln];
    cw->post(ln, v, at);
    return cw->vals[s & 1][src & 31u];
}

uint32_t EmuWarp::ballot(bool p, uint32_t at) const
{
    const uint64_t s = cw->seq[ln];
    cw->post(ln, p ? 1u : 0u, at);
    uint32_t m = 0;
    for (uint32_t i = 0; i < 32; ++i)
        m |= (cw->vals[s & 1][i] ? 1u : 0u) << i;
    return m;
}

// The warp-hybrid kernels' loop (k_alt_warp in svdag_alt_tables.cu) over `warps` emulated warps.
template <uint32_t L, bool ADD>
void run_warps(const AltTable& t0, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t warps)
{
    AltTable t = t0;
    t.layout = L;
    std::vector<std::unique_ptr<CoWarp>> cws;
    std::vector<std::thread> pool;
    for (uint32_t g = 0; g < warps; ++g) {
        cws.emplace_back(new CoWarp());
        cws.back()->body = [&, g](const EmuWarp& w) {
            for (uint64_t base = 32ull * g; base < n; base += 32ull * warps) {
                const uint64_t i = base + w.lane();
                const bool valid = i < n;
                const uint32_t* key = keys + (valid ? i : 0) * t.k;
                const uint32_t h = ADD ? warp_add<L>(w, t, key, valid) : warp_find<L>(w, t, key, valid);
                if (valid)
                    handles[i] = h;
            }
        };
    }
    for (uint32_t g = 0; g < warps; ++g)
        pool.emplace_back([&, g] { cws[g]->run(); });
    for (auto& th : pool)
        th.join();
}

} // namespace

extern "C" {

void* alt_host_create(uint32_t layout, uint32_t k, uint32_t numBuckets, uint64_t reserved)
{
    if (!layout_ok(layout, k) || numBuckets == 0)
        return nullptr;
    const uint64_t bytes = table_layout(layout, k, numBuckets, reserved, nullptr, nullptr);
    if (!bytes)
        return nullptr;
    void* mem = std::aligned_alloc(256, (bytes + 255) & ~(uint64_t)255);
    if (!mem)
        return nullptr;
    std::memset(mem, 0, bytes);
    auto* h = new HostTable();
    h->mem = mem;
    table_layout(layout, k, numBuckets, reserved, mem, &h->t);
    h->t.ctl[kCtlNextSlab] = initial_counter(layout, numBuckets);
    return h;
}

void alt_host_destroy(void* p)
{
    auto* h = (HostTable*)p;
    std::free(h->mem);
    delete h;
}

void alt_host_add(void* p, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t threads)
{
    const AltTable t = ((HostTable*)p)->t;
    run_threads(n, threads, [&](uint32_t i) { handles[i] = add(t, keys + (uint64_t)i * t.k); });
}

void alt_host_find(void* p, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t threads)
{
    const AltTable t = ((HostTable*)p)->t;
    run_threads(n, threads, [&](uint32_t i) { handles[i] = find(t, keys + (uint64_t)i * t.k); });
}

void alt_host_read(void* p, const uint32_t* handles, uint32_t n, uint32_t* out)
{
    const AltTable t = ((HostTable*)p)->t;
    for (uint32_t i = 0; i < n; ++i)
        read(t, handles[i], out + (uint64_t)i * t.k);
}

void alt_host_warp_op(void* p, const uint32_t* keys, uint32_t n, uint32_t* handles, uint32_t warps, int add)
{
    const AltTable& t = ((HostTable*)p)->t;
    switch (t.layout) {
    case kTicketBoard: add ? run_warps<kTicketBoard, true>(t, keys, n, handles, warps) : run_warps<kTicketBoard, false>(t, keys, n, handles, warps); break;
    case kAtomic64: add ? run_warps<kAtomic64, true>(t, keys, n, handles, warps) : run_warps<kAtomic64, false>(t, keys, n, handles, warps); break;
    default: add ? run_warps<kAcceleration, true>(t, keys, n, handles, warps) : run_warps<kAcceleration, false>(t, keys, n, handles, warps); break;
    }
}

void alt_host_clear_active(void* p)
{
    const AltTable& t = ((HostTable*)p)->t;
    std::memset(t.active, 0, (size_t)active_words(t) * 4u);
}

void alt_host_mark_active(void* p, const uint32_t* handles, uint32_t n, uint32_t threads)
{
    const AltTable t = ((HostTable*)p)->t;
    run_threads(n, threads, [&](uint32_t i) { mark_active(t, handles[i]); });
}

// freeInactiveItems over every slab taken (or every bucket list); returns the items freed.
uint64_t alt_host_free_inactive(void* p)
{
    const AltTable& t = ((HostTable*)p)->t;
    uint64_t n = 0;
    if (t.layout == kIndividualChaining) {
        for (uint32_t b = 0; b < t.numBuckets; ++b)
            n += free_inactive_chain(t, b);
    } else {
        const uint32_t used = t.ctl[kCtlNextSlab] < t.slabCount ? t.ctl[kCtlNextSlab] : t.slabCount;
        for (uint32_t s = 0; s < used; ++s)
            n += free_inactive_slab(t, s);
    }
    return n;
}

uint32_t alt_host_status(void* p) { return ((HostTable*)p)->t.ctl[kCtlStatus]; }

// Nodes reachable from the IndividualChaining heads.
static uint64_t chain_nodes(const AltTable& t)
{
    uint64_t n = 0;
    for (uint32_t b = 0; b < t.numBuckets; ++b)
        for (uint32_t cur = t.heads[b]; cur != 0 && cur <= t.slabCount; cur = slab_at(t, cur - 1u)[t.k])
            ++n;
    return n;
}

// Occupied slots over the slabs taken so far, and the overflow slabs taken (IndividualChaining:
// linked nodes, and 0).
void alt_host_stats(void* p, uint64_t* items, uint64_t* overflow)
{
    const AltTable t = ((HostTable*)p)->t;
    if (t.layout == kIndividualChaining) {
        *items = chain_nodes(t);
        *overflow = 0;
        return;
    }
    const uint32_t used = t.ctl[kCtlNextSlab] < t.slabCount ? t.ctl[kCtlNextSlab] : t.slabCount;
    uint64_t n = 0;
    for (uint32_t s = 0; s < used; ++s)
        n += slab_items(t.layout, slab_at(t, s));
    *items = n;
    *overflow = used - t.numBuckets;
}

// Overflow slabs reachable from the buckets' chains (every slab taken from the counter should be).
uint64_t alt_host_linked_overflow(void* p)
{
    const AltTable t = ((HostTable*)p)->t;
    if (t.layout == kIndividualChaining)
        return 0;
    uint64_t n = 0;
    for (uint32_t b = 0; b < t.numBuckets; ++b)
        for (uint32_t s = slab_at(t, b)[next_word(t.layout)]; s != 0 && s < t.slabCount; s = slab_at(t, s)[next_word(t.layout)])
            ++n;
    return n;
}

} // extern "C"
