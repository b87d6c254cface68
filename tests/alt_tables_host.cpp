// Host build of the alternative table layouts (gpu-svdag-editing_b200/csrc/svdag_alt_tables.cuh)
// for the CPU tests: the same thread-per-key add / find / read functions the CUDA kernels run, driven
// by std::threads that take keys round-robin, so that claims and chain links race as they do on the
// GPU. Test infrastructure only; the library's tables run on the GPU.
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

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

} // namespace

extern "C" {

void* alt_host_create(uint32_t layout, uint32_t k, uint32_t numBuckets, uint64_t reserved)
{
    if (!layout_ok(layout, k) || numBuckets == 0)
        return nullptr;
    const uint32_t slabs = arena_slabs(layout, numBuckets, reserved);
    if (!slabs)
        return nullptr;
    const uint32_t sw = slab_words(layout, k);
    const size_t bytes = 256 + (size_t)slabs * sw * 4;
    void* mem = std::aligned_alloc(256, (bytes + 255) & ~(size_t)255);
    if (!mem)
        return nullptr;
    std::memset(mem, 0, bytes);
    auto* h = new HostTable();
    h->mem = mem;
    h->t.layout = layout;
    h->t.k = k;
    h->t.numBuckets = numBuckets;
    h->t.slabWords = sw;
    h->t.slabCount = slabs;
    h->t.ctl = (uint32_t*)mem;
    h->t.slabs = (uint32_t*)((char*)mem + 256);
    h->t.ctl[kCtlNextSlab] = numBuckets;
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

uint32_t alt_host_status(void* p) { return ((HostTable*)p)->t.ctl[kCtlStatus]; }

// Occupied slots over the slabs taken so far, and the overflow slabs taken.
void alt_host_stats(void* p, uint64_t* items, uint64_t* overflow)
{
    const AltTable t = ((HostTable*)p)->t;
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
    uint64_t n = 0;
    for (uint32_t b = 0; b < t.numBuckets; ++b)
        for (uint32_t s = slab_at(t, b)[next_word(t.layout)]; s != 0 && s < t.slabCount; s = slab_at(t, s)[next_word(t.layout)])
            ++n;
    return n;
}

} // extern "C"
