// svdag_edit.cuh - device editors and the per-edit scratch layout.
//
// The editors restate the reference tools' predicates with the same float expressions
// (my_gpu_dag_editors.h). The library is built with -fmad=false so no expression is contracted:
// Fill/Empty/Subdivide decisions, and so the DAG structure, are then bit-identical to the
// uncontracted IEEE evaluation the oracle performs on the CPU.
#pragma once
#include "svdag_device.cuh"
#include "svdag_scene.cuh"

namespace svdag {

enum : uint32_t { OP_SUBDIVIDE = 0, OP_FILL = 1, OP_EMPTY = 2, OP_KEEP = 3 };
enum : uint32_t { ST_PARTIAL = 0, ST_FILLED = 1, ST_EMPTY = 2 };
constexpr uint32_t kToolTerrain = 100; // internal: the procedural scene builder
constexpr uint32_t kEmptyRep = 0xFFFFFFFEu; // dedup result of an empty SVO item
constexpr int kNumGraphs = 10; // CUDA graphs of the phase launches: one per tool, the last for the scene builder

struct EditRecord;

struct DevEditor {
    uint32_t tool;
    uint32_t material;
    float bmin[3], bmax[3]; // box, copy destination box, noise box (MyGpuBoxEditorBase)
    float center[3]; // sphere centre (+0.5 applied)
    float radius, radiusSquared;
    float fDestToSource[3];
    int32_t iDestToSource[3];
    uint32_t noiseSeed, noiseCellLog2;
    SceneParams scene; // scene builder: heightfield and structures
    uint32_t levels;
    uint32_t startLevel; // the edit covers the subtree of the node (startLevel, startPath); 0 = whole DAG
    uint32_t startPath[3];
    uint32_t* tileOut; // scene builder tiles: the subtree's handle goes here instead of the root
    EditRecord* record; // per-edit record of a batch (or null)
    uint32_t useSavedSource; // copy: read the source from the saved root (move)
    uint32_t saveRoot; // remember the root before this edit as the source of a later copy (move)
    uint32_t builder; // scene build: fully-filled discovery on every level, no undo frame
    // Subtree edit: the edit covers the subtree of the node (startLevel, startPath) of the DAG as the
    // batch found it (that node's region holds the edit's whole footprint and no other edit of its
    // group touches it); no undo frame; the subtree's new handle goes to *tileOut (kNone when it
    // empties, kKeep while the edit has changed nothing), and the path above is rebuilt afterwards
    // with the edits before it in the group applied.
    uint32_t subtree;
};
constexpr uint32_t kKeep = 0xFFFFFFFDu; // subtree edit: nothing committed

// Summary of one edit of a batch (written on the device, read by the host after the batch).
struct EditRecord {
    uint32_t rootBefore, rootAfter, status, pad;
    unsigned long long edited, added, unique, svoItems;
};

// Editor of the running edit for the one-launch-per-phase form (and its CUDA graphs): the phase
// kernels read `slot`; with `eds` set, the first phase copies eds[cursor] into the slot and the
// last one advances the cursor, so one captured graph per tool serves every edit of a batch.
struct EditQueue {
    const DevEditor* eds;
    uint32_t cursor;
    uint32_t pad;
    DevEditor slot;
};

struct WorkItem { // CreateIntermediateWorkItem (create_edit_svo.cu:55-65)
    uint32_t x, y, z, handle;
};
struct CopyParent {
    uint32_t x, y, z, handle;
};

__host__ __device__ inline unsigned long long align256(unsigned long long v) { return (v + 255ull) & ~255ull; }

struct MergeLayout {
    unsigned long long rep, handle, table, end;
    uint32_t cap;
};

// Scratch layout of the bottom-up phase; every thread recomputes it from the final level counts
// (count has kMaxLevels entries). The counts are all loaded before the walk over the levels, and the
// walk is unrolled, so the counts stay in registers and cost one round trip.
__host__ __device__ inline MergeLayout merge_layout(const uint32_t* count, unsigned long long buildTop, uint32_t level, uint32_t leafLevel)
{
    uint32_t c[kMaxLevels];
#pragma unroll
    for (uint32_t l = 0; l < kMaxLevels; ++l)
        c[l] = count[l];
    unsigned long long off = buildTop;
    MergeLayout m {};
#pragma unroll
    for (int l = (int)kMaxLevels - 1; l >= 0; --l) {
        if (l > (int)leafLevel)
            continue;
        const unsigned long long n = c[l];
        uint32_t cap = 2;
        while (cap < 2ull * n)
            cap <<= 1;
        m.rep = off;
        m.handle = align256(m.rep + 4 * n);
        m.table = align256(m.handle + 4 * n);
        m.end = align256(m.table + 8ull * cap);
        m.cap = cap;
        if ((uint32_t)l == level)
            return m;
        off = m.end;
    }
    return m;
}

} // namespace svdag
