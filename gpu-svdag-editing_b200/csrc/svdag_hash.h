// svdag_hash.h - the key hash shared by every table layout and the length of a self-describing key,
// for device code and plain C++ alike.
//
// The hash is ours; the bucket function of the reference is xorHash32xN (utils.h:395-403), which uses
// a 32-bit modulo per word. Compiles under nvcc (host + device) and under a host C++ compiler.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define SVDAG_HD __host__ __device__ __forceinline__
#else
#define SVDAG_HD inline
#endif

namespace svdag {

SVDAG_HD uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
// Per-word term of the key hash: an odd multiply of the word offset by a position constant (a
// bijection of the word; the terms of a key are combined by XOR, so lanes that hold different words
// of one key can combine theirs). The finalisers below turn the sum into the bucket and tag hashes.
SVDAG_HD uint32_t word_term(uint32_t w, uint32_t i)
{
    return (w ^ (i * 0x9E3779B9u + 0x7F4A7C15u)) * (0x85EBCA6Bu + 2u * i);
}
SVDAG_HD uint32_t bucket_hash(uint32_t acc) { return fmix32(acc); }
SVDAG_HD uint32_t tag_hash(uint32_t acc) { return fmix32(acc ^ 0x5BD1E995u); }
SVDAG_HD uint32_t tag_of(uint32_t hb)
{
    uint32_t t = hb >> 24;
    return t == 0 ? 1u : (t == 0xFFu ? 0xFEu : t);
}
// Key length from the first words (my_gpu_base_dag.h:195-203): a node is its header and one child
// per bit of the child mask; a leaf is its two mask words and 4 material bits per voxel, in words.
SVDAG_HD uint32_t node_words(uint32_t header) { return 1u + __builtin_popcount(header & 0xFFu); }
SVDAG_HD uint32_t leaf_words(uint32_t lo, uint32_t hi)
{
    const uint32_t v = __builtin_popcount(lo) + __builtin_popcount(hi);
    return 2u + ((v * 4u + 31u) >> 5);
}
// Bucket of a bucket hash among numBuckets: the high half of the 64-bit product (no modulo).
SVDAG_HD uint32_t bucket_index(uint32_t ha, uint32_t numBuckets) { return (uint32_t)(((uint64_t)ha * numBuckets) >> 32); }

} // namespace svdag
