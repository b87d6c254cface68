// memory_host.cu - a host-memory-only stand-in for the reference's Memory singleton (memory.h).
//
// TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libref.so in place of the reference's memory.cu,
// which the reference's MyGPUHashDAG<EMemoryType::CPU> needs for every StaticArray allocation.
// memory.cu itself is not used because (a) it replaces the global operator new/delete when
// TRACK_GLOBAL_NEWDELETE is set and links NVML, neither wanted inside a library loaded into a test
// process, and (b) on this machine's glibc its CPU path calls std::aligned_alloc with sizes that
// are not multiples of the alignment, which returns null. This stand-in keeps the interface of
// memory.h (the allocation table, the counters) and serves EMemoryType::CPU only: a device memory
// type gets a null pointer and a message, which the callers in the harness never request.
#include "memory.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

Memory Memory::singleton;

Memory::~Memory() = default;

void Memory::cuda_memcpy_impl(uint8* dst, const uint8* src, uint64 size, cudaMemcpyKind memcpyKind)
{
    if (memcpyKind == cudaMemcpyHostToHost || memcpyKind == cudaMemcpyDefault) {
        std::memcpy(dst, src, size);
        return;
    }
    std::fprintf(stderr, "memory_host: device copy requested in a host-only build\n");
}

void* Memory::malloc_impl(size_t size, size_t alignment, const char* name, EMemoryType type)
{
    if (type != EMemoryType::CPU) {
        std::fprintf(stderr, "memory_host: device allocation '%s' requested in a host-only build\n", name);
        return nullptr;
    }
    void* ptr;
    if (alignment == 0) {
        ptr = std::malloc(size);
    } else {
        // aligned_alloc wants a size that is a multiple of the alignment
        const size_t rounded = (size + alignment - 1) / alignment * alignment;
        ptr = std::aligned_alloc(alignment, rounded);
    }
    if (!ptr)
        return nullptr;
    totalAllocatedCPUMemory += size;
    allocations[ptr] = { name, type, size };
    return ptr;
}

void Memory::free_impl(void* ptr)
{
    if (!ptr)
        return;
    auto it = allocations.find(ptr);
    if (it != allocations.end()) {
        totalAllocatedCPUMemory -= it->second.size;
        allocations.erase(it);
    }
    std::free(ptr);
}

void Memory::realloc_impl(void*& ptr, size_t newSize, size_t newAlignment)
{
    auto it = allocations.find(ptr);
    const char* name = it != allocations.end() ? it->second.name : "realloc";
    const size_t oldSize = it != allocations.end() ? it->second.size : 0;
    void* fresh = malloc_impl(newSize, newAlignment, name, EMemoryType::CPU);
    if (fresh && ptr)
        std::memcpy(fresh, ptr, oldSize < newSize ? oldSize : newSize);
    free_impl(ptr);
    ptr = fresh;
}

const char* Memory::get_alloc_name_impl(void* ptr) const
{
    auto it = allocations.find(ptr);
    return it != allocations.end() ? it->second.name : "unknown";
}

std::string Memory::get_stats_string_impl() const
{
    std::ostringstream s;
    s << allocations.size() << " host allocations, " << totalAllocatedCPUMemory << " bytes";
    return s.str();
}

size_t Memory::availableDeviceMemory() const
{
    return 0;
}
