// ref_v3_harness.cu - the reference's own DAG, MyGPUHashDAG<EMemoryType::CPU>, and its file
// format (writeTo / readFrom, my_gpu_hash_dag.cu:158-177) behind a C API, to check the library's
// version-3 reader and writer against the reference's code.
//
// TEST INFRASTRUCTURE ONLY (like the rest of oracle/): nothing in the product loads the built
// library. Compiled by oracle/build_ref.py together with the reference's own my_gpu_hash_dag.cu,
// gpu_hash_table_base.cu, compact_acceleration_hash_table.cu, dynamic_slab_alloc.cu and the cub
// wrappers, from the reference sources where they lie, into oracle/_ref/libref.so; oracle/ref_shim
// stands in for gsl-lite, TBB and the reference's memory.cu (host memory only).
//
// What runs here is the reference's code: MyGPUHashDAG::allocate, find_leaf / add_leaf / find_node
// / add_node (the host insert of CompactAccelerationHashTable), setLoadFactor, writeTo through
// BinaryWriter, readFrom through BinaryReader, get_node_ptr / get_leaf_ptr, and DAGUtils::get_value.
// The reference's host DAG copies its arrays with cudaMemcpy(cudaMemcpyDefault) (array.h:90-99), so
// these functions need a CUDA driver even though all their data is in host memory.
#include "configuration/script_definitions.h"
#include "typedefs.h"

#include "binary_reader.h"
#include "binary_writer.h"
#include "dags/dag_utils.h"
#include "dags/my_gpu_dags/my_gpu_hash_dag/my_gpu_hash_dag.h"
#include "path.h"
#include "stats.h"

#include <cstdint>
#include <fstream>
#include <optional>
#include <unordered_map>
#include <vector>

// MyGPUHashDAG::report is compiled into my_gpu_hash_dag.cu; the harness never calls it. These two
// empty definitions stand in for stats.cpp, which needs the reference's engine and its libraries.
void StatsRecorder::report(std::string, const my_units::bytes, Device) {}
void StatsRecorder::reportInt(std::string, int64_t, std::string, Device) {}

namespace {

using Dag = MyGPUHashDAG<EMemoryType::CPU>;

uint32_t popc(uint32_t v) { return (uint32_t)__builtin_popcount(v); }
uint32_t leaf_words(const uint32_t* w) { return 2u + (((popc(w[0]) + popc(w[1])) * 4u + 31u) >> 5); }
uint32_t node_words(const uint32_t* w) { return 1u + popc(w[0] & 0xFFu); }

struct Loaded {
    Dag dag;
};

} // namespace

extern "C" {

// The scene depth the reference was compiled with (SCENE_DEPTH = MAX_LEVELS); its DAG has exactly
// these levels.
uint32_t ref_v3_levels() { return MAX_LEVELS; }

// Builds the reference's host DAG from an item snapshot the way its factory fills one
// (my_gpu_hash_dag_factory.cpp:427-470): allocate with an initial table size, every leaf and node
// inserted bottom-up through find_* then add_*, the root set, setLoadFactor(TARGET_LOAD_FACTOR);
// then writes it with MyGPUHashDAG::writeTo. Returns 0, or 1 for a snapshot that does not parse.
int ref_v3_write(const uint32_t* words, const uint64_t* levelWords, const uint64_t* levelItems, const char* path)
{
    const uint32_t LL = MAX_LEVELS - 2;
    uint64_t items = 0;
    for (uint32_t l = 0; l <= LL; ++l)
        items += levelItems[l];
    Dag dag = Dag::allocate((uint32_t)(items / 64 + 1));
    std::vector<uint32_t> below, here;
    uint64_t at = 0;
    std::vector<uint64_t> levelAt(LL + 1, 0);
    for (uint32_t l = 1; l <= LL; ++l)
        levelAt[l] = levelAt[l - 1] + levelWords[l - 1];
    bool bad = false;
    for (int l = (int)LL; l >= 0 && items; --l) {
        here.clear();
        at = levelAt[l];
        const uint64_t end = at + levelWords[l];
        while (at < end) {
            const uint32_t* w = words + at;
            uint32_t buffer[Dag::maxItemSizeInU32] = {};
            uint32_t n, h;
            if (l == (int)LL) {
                n = leaf_words(w);
                std::copy(w, w + n, buffer);
                h = dag.find_leaf(buffer);
                if (h == Dag::invalid_handle)
                    h = dag.add_leaf(buffer);
            } else {
                n = node_words(w);
                buffer[0] = w[0];
                for (uint32_t i = 1; i < n; ++i) {
                    if (w[i] >= below.size()) {
                        bad = true;
                        break;
                    }
                    buffer[i] = below[w[i]];
                }
                if (bad)
                    break;
                h = dag.find_node(buffer);
                if (h == Dag::invalid_handle)
                    h = dag.add_node(buffer);
            }
            here.push_back(h);
            at += n;
        }
        if (bad || here.size() != levelItems[l])
            break;
        below.swap(here);
    }
    if (bad || (items && below.size() != 1)) {
        dag.free();
        return 1;
    }
    dag.firstNodeIndex = items ? below[0] : Dag::invalid_handle;
    if (items)
        dag.setLoadFactor(TARGET_LOAD_FACTOR);
    {
        std::ofstream create(path, std::ios::binary); // BinaryWriter wants an existing file
    }
    {
        BinaryWriter writer(path);
        writer.write(dag);
    }
    dag.free();
    return 0;
}

// Reads a file with MyGPUHashDAG::readFrom. The handle owns the reference's DAG until ref_v3_close.
void* ref_v3_open(const char* path)
{
    auto* h = new Loaded;
    BinaryReader reader(path);
    reader.read(h->dag);
    return h;
}

void ref_v3_close(void* handle)
{
    auto* h = static_cast<Loaded*>(handle);
    h->dag.free();
    delete h;
}

uint32_t ref_v3_root(const void* handle) { return static_cast<const Loaded*>(handle)->dag.firstNodeIndex; }

// The items reachable from the root through the reference's get_node_ptr / get_leaf_ptr, each
// level's in first-visit order (a snapshot, children as ordinals); *found counts the reachable items
// that the reference's find_node / find_leaf locate at the handle they were reached through.
// Returns 0, or 2 when capacity (words) is too small (*total holds the words needed).
int ref_v3_items(const void* handle, uint32_t* out, uint64_t capacity, uint64_t* levelWords, uint64_t* levelItems,
    uint64_t* total, uint64_t* found)
{
    const Dag& dag = static_cast<const Loaded*>(handle)->dag;
    const uint32_t LL = MAX_LEVELS - 2;
    std::vector<std::vector<uint32_t>> words(LL + 1);
    std::vector<uint32_t> frontier, next;
    if (dag.firstNodeIndex != Dag::invalid_handle)
        frontier.push_back(dag.firstNodeIndex);
    *found = 0;
    for (uint32_t l = 0; l <= LL; ++l) {
        std::unordered_map<uint32_t, uint32_t> ordinal;
        next.clear();
        for (const uint32_t h : frontier) {
            if (l == LL) {
                const uint32_t* w = dag.get_leaf_ptr(h);
                const uint32_t n = Dag::get_leaf_size(w);
                words[l].insert(words[l].end(), w, w + n);
                *found += dag.find_leaf(w) == h;
                continue;
            }
            const uint32_t* w = dag.get_node_ptr(l, h);
            const uint32_t n = Dag::get_node_size(w);
            *found += dag.find_node(w) == h;
            words[l].push_back(w[0]);
            for (uint32_t i = 1; i < n; ++i) {
                auto [it, fresh] = ordinal.emplace(w[i], (uint32_t)next.size());
                if (fresh)
                    next.push_back(w[i]);
                words[l].push_back(it->second);
            }
        }
        levelItems[l] = frontier.size();
        frontier.swap(next);
    }
    uint64_t t = 0;
    for (uint32_t l = 0; l <= LL; ++l) {
        levelWords[l] = words[l].size();
        if (out && t + words[l].size() <= capacity)
            std::copy(words[l].begin(), words[l].end(), out + t);
        t += words[l].size();
    }
    *total = t;
    return t > capacity ? 2 : 0;
}

// DAGUtils::get_value (dag_utils.h:146-182) on the loaded DAG: the material of each voxel, or
// 0xFFFFFFFF where it is empty.
int ref_v3_get_values(const void* handle, const uint32_t* xyz, uint64_t n, uint32_t* out)
{
    const Dag& dag = static_cast<const Loaded*>(handle)->dag;
    for (uint64_t i = 0; i < n; ++i) {
        if (dag.firstNodeIndex == Dag::invalid_handle) {
            out[i] = 0xFFFFFFFFu;
            continue;
        }
        const std::optional<uint32_t> v = DAGUtils::get_value(dag, Path(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
        out[i] = v ? *v : 0xFFFFFFFFu;
    }
    return 0;
}

} // extern "C"
