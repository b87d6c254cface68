// svdag_host.hpp - host-side context of libsvdag (shared by the .cu translation units).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "svdag_device.cuh"
#include "svdag_edit.cuh"

struct svdag_table {
    svdag_ctx* ctx = nullptr;
    svdag::DevTable dev {};
    int level = -1; // -1 for standalone tables
    bool ready = false;
    unsigned long long words = 0; // words of the bucket arrays
};

struct svdag_ctx {
    svdag_config cfg {};
    int device = 0;
    char* pool = nullptr;
    size_t poolBytes = 0;
    svdag::Control* ctl = nullptr; // device control block
    char* scratch = nullptr; // per-edit arena
    unsigned long long scratchBytes = 0;
    char* batch = nullptr; // editors and per-edit records of a persistent batch launch
    unsigned long long batchBytes = 0;
    svdag::EditQueue* queue = nullptr; // editor slot of the one-launch-per-phase form (end of the batch region)
    cudaGraphExec_t graphs[svdag::kNumGraphs] = {}; // per tool: the phase launches of one edit
    uint32_t lastBatch = 0;
    uint32_t* items = nullptr; // item region
    unsigned long long itemWords = 0;
    uint32_t* headers = nullptr; // slab header region
    unsigned long long headerCount = 0;
    svdag_table levelTables[svdag::kMaxLevels];
    std::vector<svdag_table*> standalone;
    uint32_t probeLanes = 8;
    double persistentLeaves = 0; // edits estimated at or below this many SVO leaves run in the persistent kernel (0 = none)
    uint32_t loadFactor = 16;
    unsigned long long scratchHighWater = 0;
    svdag::DevDag dag() const { return svdag::DevDag { items, itemWords, headers, headerCount, ctl, cfg.levels, cfg.levels - 2, &ctl->edit, 0u, nullptr }; }
};

namespace svdag {

// Maps a CUDA error to a status (and remembers nothing: CUDA errors are reported where they occur).
inline svdag_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess)
        return SVDAG_OK;
    std::fprintf(stderr, "libsvdag: CUDA error %s\n", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? SVDAG_ERR_OOM : SVDAG_ERR_CUDA;
}

#define SVDAG_CUDA(call)                                      \
    do {                                                      \
        const cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess)                                \
            return ::svdag::cuda_status(e_);                  \
    } while (0)
#define SVDAG_TRY(call)                                       \
    do {                                                      \
        const svdag_status s_ = (call);                       \
        if (s_ != SVDAG_OK)                                   \
            return s_;                                        \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Item and header region bytes in use: what the bump pointers handed out (a failed allocation may
// leave a pointer past the end), less the slabs on the free lists.
inline unsigned long long used_region_bytes(const svdag_ctx* ctx, unsigned long long itemTop, unsigned long long headerTop,
    unsigned long long freeBytes)
{
    const unsigned long long used = (itemTop < ctx->itemWords ? itemTop : ctx->itemWords) * 4ull
        + (headerTop < ctx->headerCount ? headerTop : ctx->headerCount) * 32ull;
    return used > freeBytes ? used - freeBytes : 0ull;
}

// Number of resident-CTA-sized grid for grid-stride kernels: a multiple of the SM count.
int grid_for(const svdag_ctx* ctx, unsigned long long work, int threadsPerBlock, int blocksPerSm = 8);

// Table management (svdag_tables.cu).
// `recycle`: a level table, whose overflow slabs come from and go back to the free lists.
svdag_status alloc_table(svdag_ctx* ctx, svdag_table* t, uint32_t kind, const uint32_t* bucketsPerClass, cudaStream_t s, bool recycle = false);
svdag_status ensure_level_tables(svdag_ctx* ctx, cudaStream_t s);
svdag_status insert_canonical(svdag_ctx* ctx, uint32_t level, cudaStream_t s);
svdag_status upload_tables(svdag_ctx* ctx, cudaStream_t s);
svdag_status read_status(svdag_ctx* ctx, cudaStream_t s);
void reset_level_tables(svdag_ctx* ctx);
// Find-or-insert of keys that are pairwise distinct (no batch dedup) into a level table.
svdag_status find_or_insert_distinct(svdag_ctx* ctx, uint32_t level, const uint32_t* keys, const uint32_t* offsets, uint32_t n,
    unsigned long long totalWords, uint32_t* out, cudaStream_t s);
// Items per size class of a table (`scratch`: 9 device words).
svdag_status table_class_counts(svdag_ctx* ctx, const svdag_table& t, unsigned long long* perClass, unsigned long long* scratch, cudaStream_t s);

// Edit machinery (svdag_edit.cu).
svdag_status run_edit(svdag_ctx* ctx, const svdag_edit* e, cudaStream_t s);
svdag_status run_edit_batch(svdag_ctx* ctx, const svdag_edit* edits, uint32_t count, cudaStream_t s);
struct DevEditor;
// Resets the DAG to empty: no items, no tables, empty history.
svdag_status reset_dag(svdag_ctx* ctx, cudaStream_t s);
// Scene build in one pass over the whole grid, level tables sized exactly per level (svdag_edit.cu).
svdag_status build_scene_untiled(svdag_ctx* ctx, const DevEditor& ed, cudaStream_t s);
// Builds the subtrees of scene tiles, one builder editor per tile (svdag_edit.cu).
svdag_status launch_scene_tiles(svdag_ctx* ctx, const DevEditor* eds, uint32_t n, cudaStream_t s);
// Edit validation, expansion into device editors (a move gives two) and the persistent launch of
// expanded editors with their editors and records in `region` (svdag_edit.cu).
bool valid_edit(const svdag_edit* e);
int expand_edit(const svdag_ctx* ctx, const svdag_edit& e, DevEditor* out);
double estimate_leaves(const DevEditor& e);
svdag_status launch_single_fused(svdag_ctx* ctx, const DevEditor& ed, cudaStream_t s);
svdag_status launch_pipeline(svdag_ctx* ctx, const DevEditor& ed, cudaStream_t s, EditRecord* record, bool graphOk);
// The batched table operations of the public API, by lane count (svdag_tables.cu).
svdag_status table_add_lanes(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n, unsigned long long totalWords,
    uint32_t* out, uint32_t lanes, cudaStream_t s);
svdag_status table_find_lanes(svdag_table* t, const uint32_t* keys, const uint32_t* offsets, uint32_t n, unsigned long long totalWords,
    uint32_t* out, uint32_t lanes, cudaStream_t s);
svdag_status launch_edits_at(svdag_ctx* ctx, const DevEditor* eds, uint32_t n, char* region, size_t regionBytes, cudaStream_t s);
// A frame of the root stored at `root` (device word) instead of the current one (svdag_trace.cu).
svdag_status trace_frame(svdag_ctx* ctx, const svdag_trace_params* p, svdag_hit* out, const uint32_t* root, cudaStream_t s);
// The same frame over the previous frame of the same camera in `out`: only pixels whose ray meets one
// of the boxes (6 floats each: min xyz, max xyz) are traced again.
svdag_status trace_frame_incremental(svdag_ctx* ctx, const svdag_trace_params* p, svdag_hit* out, const uint32_t* root, const float* boxes,
    uint32_t nBoxes, cudaStream_t s);
// Procedural scene construction (svdag_scene.cu).
svdag_status run_scene_build(svdag_ctx* ctx, const svdag_terrain_params* p, cudaStream_t s);

} // namespace svdag
