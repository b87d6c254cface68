/*
 * svdag.h - C ABI of libsvdag, a B200-native (sm_100a) SVDAG editing back-end and DAG ray tracer.
 *
 * The entry points replace the C++ template interface of the reference's EDag::MyGpuDag path
 * (mathijs727/GPU-SVDAG-Editing). Each declaration names the reference interface it stands in for.
 *
 * Conventions
 *  - Every function returns an svdag_status (0 = SVDAG_OK) and never aborts the process.
 *  - Device pointers are marked *_dev; everything else is host memory owned by the caller.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Calls on one context are not thread-safe; the serving loop (svdag_serve_*) is the
 *    thread-safe way to feed a context from several producers.
 *  - Asynchronous failures (device-side capacity or iteration-limit errors) are latched in a
 *    device status word; svdag_sync() and every call that synchronises report them.
 */
#ifndef SVDAG_H
#define SVDAG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SVDAG_ABI_VERSION 2u

typedef enum svdag_status {
    SVDAG_OK = 0,
    SVDAG_ERR_INVALID = 1, /* bad argument */
    SVDAG_ERR_OOM = 2, /* pool, slab region or scratch arena exhausted */
    SVDAG_ERR_TIMEOUT = 3, /* a bounded device-side wait or retry loop gave up */
    SVDAG_ERR_CORRUPT = 4, /* structural invariant violated (bad handle, bad size) */
    SVDAG_ERR_CUDA = 5, /* CUDA runtime error */
    SVDAG_ERR_NO_DEVICE = 6, /* no usable sm_100 device */
    SVDAG_ERR_UNSUPPORTED = 7,
    SVDAG_ERR_BUSY = 8 /* serving queue full / admission refused */
} svdag_status;

/* Item handles are 32-bit indices of items in 16-byte units of the context's item region (up to 64 GiB). */
#define SVDAG_INVALID_HANDLE 0xFFFFFFFFu
/* Voxel sampling and hit records use this value for "no voxel". */
#define SVDAG_NO_MATERIAL 0xFFFFFFFFu

#define SVDAG_MAX_LEVELS 17u /* total octree depth (reference MAX_LEVELS) */
#define SVDAG_MIN_LEVELS 4u
#define SVDAG_MATERIAL_BITS 4u /* reference HASH_DAG_MATERIAL_BITS */
#define SVDAG_NUM_MATERIALS 16u
#define SVDAG_MIN_ITEM_WORDS 2u /* node: header + 1 child */
#define SVDAG_MAX_ITEM_WORDS 10u /* leaf: 2 mask words + 8 material words */
#define SVDAG_NUM_SIZE_CLASSES 9u /* item sizes 2..10 words */

/* Table kinds: a node key's length is 1 + popcount(child mask); a leaf key's length is
 * 2 + ceil(4 * popcount(64-bit voxel mask) / 32). Keys are self-describing. */
typedef enum svdag_item_kind { SVDAG_KIND_NODE = 0, SVDAG_KIND_LEAF = 1 } svdag_item_kind;

/* Launch every edit phase directly instead of replaying the tool's captured CUDA graph of the phase
 * launches (for profiling single phases). */
#define SVDAG_FLAG_PHASE_KERNELS 1u
/* Run edits whose intermediate SVO is estimated small (up to 16384 leaves) in the persistent kernel
 * (one CTA, block barriers between phases; a run of such edits is one launch) instead of the tool's
 * CUDA graph of the phase launches. svdag_autotune chooses the threshold by measurement. */
#define SVDAG_FLAG_PERSISTENT 2u

typedef struct svdag_config {
    uint32_t levels; /* octree depth, SVDAG_MIN_LEVELS..SVDAG_MAX_LEVELS (1 << levels voxels per axis) */
    int32_t device; /* CUDA device ordinal */
    uint64_t pool_bytes; /* the single preallocated HBM pool (item region + scratch arena) */
    uint64_t scratch_bytes; /* part of the pool reserved for per-edit temporaries */
    uint32_t target_load_factor; /* items per bucket when a level table is sized; 0 = default (16) */
    uint32_t probe_lanes; /* lanes cooperating on one key: 1, 2, 4, 8, 16 or 32; 0 = default (1) */
    uint32_t undo_depth; /* undo history ring size; 0 = default (32) */
    uint32_t flags; /* SVDAG_FLAG_* */
} svdag_config;

typedef struct svdag_ctx svdag_ctx;
typedef struct svdag_table svdag_table;

/* ---------------------------------------------------------------- context */

/* Replaces MyGPUHashDAG<GPU_Malloc>::allocate (my_gpu_hash_dag.cu:24-66): one HBM pool, one table
 * per level, the canonical fully-filled node of every (level, material) inserted up front. */
svdag_status svdag_create(const svdag_config* config, svdag_ctx** out_ctx);
/* Replaces MyGPUHashDAG::free (my_gpu_hash_dag.cu:68-76). */
svdag_status svdag_destroy(svdag_ctx* ctx);
/* Waits for all work of the context on `stream` and returns the latched device status (then clears it). */
svdag_status svdag_sync(svdag_ctx* ctx, void* stream);
const char* svdag_status_string(svdag_status status);
uint32_t svdag_abi_version(void);

/* ---------------------------------------------------------------- scene construction */

typedef struct svdag_terrain_params {
    uint32_t seed; /* lattice hash seed */
    uint32_t octaves; /* fBm octaves */
    uint32_t num_materials; /* height bands -> materials [0, num_materials) (8 or 16) */
    uint32_t min_height_pct; /* surface height range, in percent of the grid height */
    uint32_t max_height_pct;
    uint32_t num_structures; /* random boxes/spheres unioned on the surface (0 = none), at most 65536 */
    uint32_t structure_seed;
    uint32_t tile_level; /* level (at most min(levels - 3, 6)) at which the build is cut into
                            independently built tiles; 0 = automatic (the smallest level whose
                            tiles fit the scratch arena; untiled when the whole scene fits) */
} svdag_terrain_params;

/* The scene. Voxel (x, y, z) of a 2^levels grid is solid when y < height(x, z) or when a structure
 * contains it; its material is that of the highest-index structure containing it, else the height
 * band (y * num_materials) >> levels. height(x, z) is integer value-noise fBm: octave o has lattice
 * cells of 2^max(levels-2-o, 0) voxels, lattice values fmix32-hashed from (seed, o, ix, iz) in
 * [0, 65535], smoothstep-weighted bilinear interpolation in 16.16 fixed point, weight 2^(octaves-1-o);
 * the sum maps linearly onto [min_height_pct, max_height_pct] of the grid height.
 *
 * Structure i (i = 0 .. num_structures-1) draws from one splitmix64 stream seeded with
 * structure_seed, in this order: x = next % 2^levels, z = next % 2^levels, kind = next & 1
 * (0 box, 1 sphere), material = next % 16, size = next; with h = height(x, z):
 *   box: side = 16 + size % 497, voxels [x - side/2, x - side/2 + side) (same for y around h, z);
 *   sphere: radius r = 8 + size % 249, voxels v with |v - (x, h, z)|^2 <= r^2. */

/* Builds a procedural heightfield terrain into an empty context; stands in for the reference's
 * scene load MyGPUHashDAGFactory::load_from_DAG (my_gpu_hash_dag_factory.cpp:427-500). Every
 * uniformly filled node carries the fully-filled header bits, as the factory's create_dag_cpu does. */
svdag_status svdag_build_terrain(svdag_ctx* ctx, const svdag_terrain_params* params, void* stream);
/* Surface height of column (x, z) of the terrain of a 2^levels grid (host function, for placing
 * edits on the surface). No counterpart in the reference, whose scenes are loaded from files. */
uint32_t svdag_scene_height(const svdag_terrain_params* params, uint32_t levels, uint32_t x, uint32_t z);

/* ---------------------------------------------------------------- edits */

typedef enum svdag_tool {
    SVDAG_TOOL_SPHERE_ADD = 0, /* MyGpuSphereEditor<true>   (my_gpu_dag_editors.h:457-496) */
    SVDAG_TOOL_SPHERE_REMOVE = 1, /* MyGpuSphereEditor<false> */
    SVDAG_TOOL_BOX_ADD = 2, /* MyGpuBoxEditor<true>      (my_gpu_dag_editors.h:82-119) */
    SVDAG_TOOL_BOX_REMOVE = 3, /* MyGpuBoxEditor<false> */
    SVDAG_TOOL_SPHERE_PAINT = 4, /* MyGpuSpherePaintEditor    (my_gpu_dag_editors.h:498-536) */
    SVDAG_TOOL_COPY = 5, /* MyGpuCopyEditor           (my_gpu_dag_editors.h:129-253) */
    SVDAG_TOOL_BOX_PAINT_NOISE = 6, /* box paint with a per-voxel material from 3D value noise */
    SVDAG_TOOL_MOVE = 7, /* copy followed by removal of the source box */
    SVDAG_TOOL_SPHERE_ERODE = 8, /* MyGpuSphereErosionEditor (my_gpu_dag_editors.h:538-589): inside the
                                    sphere a filled voxel stays when more than noise_seed of its 26
                                    neighbours are filled in the DAG before the edit, else it is removed */
    SVDAG_NUM_TOOLS = 9
} svdag_tool;

typedef struct svdag_edit {
    uint32_t tool; /* svdag_tool */
    uint32_t material; /* fill / paint material, < SVDAG_NUM_MATERIALS */
    float center[3]; /* voxel coordinates; sphere centre or box centre */
    float radius; /* sphere radius, or box half extent */
    float src[3]; /* copy/move: source anchor */
    float dst[3]; /* copy/move: destination anchor */
    uint32_t noise_seed; /* BOX_PAINT_NOISE: lattice seed; SPHERE_ERODE: neighbour threshold */
    uint32_t noise_cell_log2; /* BOX_PAINT_NOISE: lattice cell size = 1 << noise_cell_log2 voxels */
} svdag_edit;

/* Per-edit counters (exact, from the device) used for the algorithmic-byte roofline. */
typedef struct svdag_edit_stats {
    uint64_t svo_nodes[SVDAG_MAX_LEVELS]; /* intermediate SVO items per level (leaf level = leaves) */
    uint64_t old_items_read; /* existing DAG nodes read by the top-down pass */
    uint64_t unique_items; /* items left after intra-SVO dedup */
    uint64_t new_items; /* items inserted into the DAG tables */
    uint64_t edited_voxels; /* voxels whose operation is not Keep (Fill/Empty regions count fully) */
    uint32_t root_before;
    uint32_t root_after;
    uint32_t status;
    uint32_t reserved;
} svdag_edit_stats;

/* Replaces editMyHashDag<Editor>(editor, dag, undoRedo, stats, memPool, stream)
 * (my_gpu_hash_dag_edits.h:12-13, body my_gpu_hash_dag_edits.cu:633-671). Asynchronous on
 * `stream`; the root handle, undo history and counters stay on the device. */
svdag_status svdag_edit_apply(svdag_ctx* ctx, const svdag_edit* edit, void* stream);
/* Batched form: applies the edits in order with no host round trip between them, all reading their
 * editors from device memory. Consecutive small sphere/box add, remove and paint edits whose
 * footprints lie in pairwise disjoint subtrees are built side by side (one block each) and committed
 * in order; other small edits run one after another in one persistent launch; the others are
 * replayed through the tool's CUDA graph. The result, the undo frames and the records equal applying
 * the edits one by one. Each edit gets an svdag_edit_record. A move counts as two records (removal,
 * then paste). */
svdag_status svdag_edit_apply_many(svdag_ctx* ctx, const svdag_edit* edits, uint32_t count, void* stream);

typedef struct svdag_edit_record {
    uint32_t root_before;
    uint32_t root_after;
    uint32_t status;
    uint32_t reserved;
    uint64_t edited_voxels;
    uint64_t new_items;
    uint64_t unique_items;
    uint64_t svo_items;
} svdag_edit_record;
/* Copies the records of the first `count` edits of the most recent svdag_edit_apply_many (synchronises `stream`). */
svdag_status svdag_edit_records(svdag_ctx* ctx, svdag_edit_record* out, uint32_t count, void* stream);
/* Copies the counters of the most recent edit to the host (synchronises `stream`). */
svdag_status svdag_last_edit_stats(svdag_ctx* ctx, svdag_edit_stats* out, void* stream);

/* Profiling: GPU global-timer stamps (ns) taken at the phase barriers of the most recent edit run by
 * the persistent kernel: start, after begin, after each top-down level, after the leaves, after each
 * bottom-up level, after the end. Plays the role of the reference's GPUTimingsManager scopes
 * (timings.h). Synchronises `stream`. */
svdag_status svdag_last_edit_phase_times(svdag_ctx* ctx, uint64_t* out_ns, uint32_t capacity, uint32_t* out_count,
    void* stream);

/* Convenience forms mirroring the reference tool constructors. */
svdag_status svdag_edit_sphere(svdag_ctx* ctx, float cx, float cy, float cz, float radius,
    uint32_t material, int add, void* stream);
svdag_status svdag_edit_box(svdag_ctx* ctx, float cx, float cy, float cz, float half_extent,
    uint32_t material, int add, void* stream);
svdag_status svdag_edit_paint(svdag_ctx* ctx, float cx, float cy, float cz, float radius,
    uint32_t material, void* stream);
svdag_status svdag_edit_paint_noise(svdag_ctx* ctx, float cx, float cy, float cz, float half_extent,
    uint32_t seed, uint32_t cell_log2, void* stream);
svdag_status svdag_edit_copy(svdag_ctx* ctx, const float src[3], const float dst[3],
    const float center[3], float radius, void* stream);

/* MyGPUHashDAGUndoRedo::undo / redo (my_gpu_base_dag.h:35-64): swap the root with the history. */
svdag_status svdag_undo(svdag_ctx* ctx, void* stream);
svdag_status svdag_redo(svdag_ctx* ctx, void* stream);
/* MyGPUHashDAGUndoRedo::garbageCollect (my_gpu_base_dag.h:66-77) -> MyGPUHashDAG::garbageCollect
 * (my_gpu_hash_dag.cu:365-475) and freeInactiveItems (gpu_hash_table_base.cu:265-374): clears the
 * history, marks everything reachable from the root and the canonical fully-filled nodes, frees the
 * rest and puts every overflow slab it leaves empty on the free list of its size class, from which
 * later overflow allocations are served. Synchronous. The collection first clears the context's
 * latched status (errors of earlier calls were reported by those calls or their edit records) and
 * returns only its own errors; when marking fails (SVDAG_ERR_OOM: the scratch arena cannot hold a
 * level's frontier) nothing is freed and the history is kept. No other work on the context (edits,
 * traces) may run while it does. */
svdag_status svdag_gc(svdag_ctx* ctx, void* stream);
/* MyGPUHashDAG::garbageCollect(activeRootNodes) (my_gpu_hash_dag.cu:373-463) with the active roots
 * = the current root and every root of the undo and redo history: the same collection as svdag_gc,
 * but undo and redo keep working afterwards. The serving loop runs it when its memory fills. */
svdag_status svdag_gc_keep_history(svdag_ctx* ctx, void* stream);
/* MyGPUHashDAG::get_first_node_index (my_gpu_hash_dag.h:290-293); synchronises `stream`. */
svdag_status svdag_get_root(svdag_ctx* ctx, uint32_t* out_root, void* stream);

/* ---------------------------------------------------------------- tracing and sampling */

/* Tracer::TracePathsParams (tracer.h:112-121) as produced by get_trace_params (dag_tracer.cu:59-101),
 * already in voxel coordinates of the [0, 2^levels)^3 grid. */
typedef struct svdag_trace_params {
    double camera[3];
    double ray_min[3];
    double ray_ddx[3];
    double ray_ddy[3];
    uint32_t width;
    uint32_t height;
} svdag_trace_params;

/* Layout-compatible with Tracer::SurfaceInteraction (tracer.h:95-110): 68 bytes. A miss has
 * path (0,0,0); material 0xFF means "no material". */
typedef struct svdag_hit {
    uint32_t path[3];
    uint8_t material;
    uint8_t pad[3];
    float position[3];
    float normal[3];
    float dpdu[3];
    float dpdv[3];
    uint32_t color;
} svdag_hit;

/* Replaces DAGTracer::resolve_paths -> Tracer::trace_paths<MyGPUHashDAG> (dag_tracer.cu:112-134,
 * tracer.cu:391-411). Writes width*height hit records, row (height-1-y) for pixel row y. */
svdag_status svdag_trace_primary(svdag_ctx* ctx, const svdag_trace_params* params,
    svdag_hit* out_dev, void* stream);

/* Replaces DAGTracer::get_voxel_values -> getVoxelValues_kernel (dag_tracer.cu:361-390): material of
 * each voxel (x,y,z triplets) or SVDAG_NO_MATERIAL. */
svdag_status svdag_sample_voxels(svdag_ctx* ctx, const uint32_t* xyz_dev, uint32_t count,
    uint32_t* out_dev, void* stream);

/* Post-hit shading of a hit buffer, all four of the reference's passes in one kernel: the diffuse
 * colour (Tracer::trace_colors, tracer.cu:413-593), the sun shadow ray (trace_shadows, :609-628),
 * ambient occlusion (trace_ambient_occlusion, :654-683) and lighting (trace_lighting, :701-730). The
 * output pixel (x, y) is hit record y * width + x, as the reference's surfaces index them. Material
 * textures are files the reference loads; here each material has one sRGB8 diffuse colour. Shadow
 * and AO rays use the any-hit traversal intersect_ray_node_out_of_order (tracer.cu:275-352). */
#define SVDAG_SHADE_SHADOWS 1u
#define SVDAG_SHADE_AO 2u

typedef struct svdag_shade_params {
    uint32_t material_srgb8[SVDAG_NUM_MATERIALS]; /* diffuse colour per material, 0x00BBGGRR */
    float sun_direction[3]; /* unit vector towards the sun (the reference: normalize(0.3, 1, 0.5)) */
    float shadow_bias; /* offset of shadow and AO ray origins (engine.h: 1) */
    float ao_ray_length; /* AO ray tmax (engine.h: 2^(depth - 10)) */
    float sun_brightness; /* direct light scale (the reference's resolve_lighting leaves it 0, dag_tracer.cu:232-245) */
    float fog_density; /* 0 = no fog */
    uint32_t ao_samples; /* cosine-weighted hemisphere samples per pixel */
    uint32_t flags; /* SVDAG_SHADE_* */
    uint32_t pad;
    uint64_t random_seed; /* PCG stream of pixel i = i * max(random_seed, 1) */
} svdag_shade_params;

/* `hits_dev` holds the trace of `trace` (svdag_trace_primary); each hit's `color` receives its
 * diffuse colour (SurfaceInteraction::diffuseColorSRGB8). Writes width*height packed sRGB8 pixels
 * (0xFFBBGGRR) to out_rgba_dev and, when not NULL, the sun visibility (trace_shadows' sunLight
 * surface) and the AO fraction per pixel; misses write 0 there. */
svdag_status svdag_shade(svdag_ctx* ctx, const svdag_trace_params* trace, const svdag_shade_params* shade,
    svdag_hit* hits_dev, uint32_t* out_rgba_dev, float* out_sun_dev, float* out_ao_dev, void* stream);

/* ---------------------------------------------------------------- hash tables */

/* The table of one DAG level (level leaf_level = levels-2 holds leaves). The handle stays owned by
 * the context. Mirrors MyGPUHashDAG::find_/add_{node,leaf}[_as_warp] (my_gpu_hash_dag.h:168-283). */
svdag_status svdag_level_table(svdag_ctx* ctx, uint32_t level, svdag_table** out_table);
/* A standalone table (microbenchmarks, tests): buckets_per_size[i] = bucket count for keys of
 * 2+i words (0 = no keys of that size). Replaces CompactAccelerationHashTable::allocate
 * (compact_acceleration_hash_table.cu:10). */
svdag_status svdag_table_create(svdag_ctx* ctx, uint32_t kind, const uint32_t* buckets_per_size,
    svdag_table** out_table);
svdag_status svdag_table_destroy(svdag_table* table);

/* Batched add (CompactAccelerationHashTable::add / addAsWarp, compact_acceleration_hash_table.h:27-121):
 * every key is stored in a fresh slot, duplicates included, as the reference does. keys_dev holds
 * the packed key words; offsets_dev[i] is the word offset of key i; total_words bounds the reads.
 * lanes = lanes cooperating on one key (1 = thread per key, 8, 32 = warp per key; 0 = default). */
svdag_status svdag_table_add(svdag_table* table, const uint32_t* keys_dev, const uint32_t* offsets_dev,
    uint32_t count, uint64_t total_words, uint32_t* handles_dev, uint32_t lanes, void* stream);
/* Batched find (find / findAsWarp, compact_acceleration_hash_table.h:205-280): handle of a stored
 * copy of each key, or SVDAG_INVALID_HANDLE. */
svdag_status svdag_table_find(svdag_table* table, const uint32_t* keys_dev, const uint32_t* offsets_dev,
    uint32_t count, uint64_t total_words, uint32_t* handles_dev, uint32_t lanes, void* stream);
/* Find-or-add: one slot per distinct key even when a batch holds duplicates (the DAG insert path). */
svdag_status svdag_table_find_or_add(svdag_table* table, const uint32_t* keys_dev,
    const uint32_t* offsets_dev, uint32_t count, uint64_t total_words, uint32_t* handles_dev,
    uint32_t lanes, void* stream);
/* Allocation-free form of svdag_table_find_or_add, with no counterpart in the reference. It is for
 * callers that must not allocate GPU memory during the call (for example while recording a CUDA graph,
 * or inside a real-time loop that may not reach the driver's allocator): its dedup scratch is a fixed
 * 1.25 MiB array compiled into the library, which every GPU that loads the library keeps until the
 * process exits. At most 65536 keys per call; larger batches are rejected with SVDAG_ERR_INVALID.
 * The first call on a device looks up the array's address (with that device made current), so make
 * that first call before any stream capture. All calls share the one array: calls whose work
 * overlaps on the GPU (different streams, or different contexts on the same device) race on it and
 * must be serialised by the caller. The calling thread's current device must be the table's device
 * (else SVDAG_ERR_INVALID). Results are the same as svdag_table_find_or_add's. */
svdag_status svdag_table_find_or_add_static(svdag_table* table, const uint32_t* keys_dev,
    const uint32_t* offsets_dev, uint32_t count, uint64_t total_words, uint32_t* handles_dev,
    uint32_t lanes, void* stream);
/* decodePointer (compact_acceleration_hash_table.h:398-402): copies the words of each handle into
 * out_words_dev[i * SVDAG_MAX_ITEM_WORDS ...], zero padded. */
svdag_status svdag_table_read(svdag_table* table, const uint32_t* handles_dev, uint32_t count,
    uint32_t* out_words_dev, void* stream);

typedef struct svdag_table_stats {
    uint64_t items; /* occupied slots */
    uint64_t buckets; /* base slabs */
    uint64_t overflow_slabs; /* chained slabs taken from the slab allocator */
    uint64_t bytes; /* bytes of slab storage (base + overflow) */
} svdag_table_stats;
svdag_status svdag_table_get_stats(svdag_table* table, svdag_table_stats* out, void* stream);

/* ---------------------------------------------------------------- alternative table layouts */

/* The reference's other slab layouts, for items of a fixed size (the workload of its table benchmark,
 * extras/hashmap_bench/src/main.cu): the DAG's level tables keep the compact 8-bit-tag layout above.
 * TICKET_BOARD: 32 slots per slab, a slot-occupancy mask claimed by atomic OR
 * (TicketBoardHashTable, ticket_board_hash_table.h:10-347). ATOMIC64: 31 slots, each claimed by a
 * 64-bit CAS of its item's first 8 bytes, which makes items with two zero first words unstorable
 * (Atomic64HashTable, atomic64_hash_table.h:11-414). ACCELERATION: 31 slots with a 32-bit tag each,
 * claimed by CAS (AccelerationHashTable, acceleration_hash_table.h:17-491). INDIVIDUAL_CHAINING: no
 * slabs; a node per item pushed onto its bucket's list by CAS, found by walking the list
 * (IndividualChainingHashTable, individual_chaining_hash_table.h:181-336); it has no warp form, so
 * lanes 32 runs a thread per key too, and a find returns the most recently added copy. */
#define SVDAG_TABLE_LAYOUT_TICKET_BOARD 1u
#define SVDAG_TABLE_LAYOUT_ATOMIC64 2u
#define SVDAG_TABLE_LAYOUT_ACCELERATION 3u
#define SVDAG_TABLE_LAYOUT_INDIVIDUAL_CHAINING 4u
typedef struct svdag_alt_table svdag_alt_table;
/* Table::allocate(numBuckets, numReservedElements, itemSizeInU32) (gpu_hash_table_base.h,
 * ticket_board_hash_table.h:19): one device allocation on the context's GPU holding num_buckets
 * first slabs and overflow slabs for reserved_items more items (INDIVIDUAL_CHAINING: num_buckets
 * heads and reserved_items nodes). item_words 1..32 (2..32 for ATOMIC64). More than 2^27 slabs or
 * 2^30 nodes gives SVDAG_ERR_INVALID. */
svdag_status svdag_alt_table_create(svdag_ctx* ctx, uint32_t layout, uint32_t item_words, uint32_t num_buckets,
    uint64_t reserved_items, svdag_alt_table** out_table);
svdag_status svdag_alt_table_destroy(svdag_alt_table* table);
/* add / addAsWarpHybrid: keys_dev holds count items of item_words words back to back; each is stored
 * in a fresh slot, duplicates included. lanes 1 = a thread per key; 32 or 0 = warp-hybrid (every lane
 * holds a key and the warp inspects one slab for one lane's key at a time). Asynchronous: exhausted
 * overflow slabs (SVDAG_ERR_OOM), an unstorable ATOMIC64 item (SVDAG_ERR_INVALID) or a bad link
 * (SVDAG_ERR_CORRUPT) give that key SVDAG_INVALID_HANDLE and are latched for svdag_alt_table_sync.
 * Adds and finds on one table must not overlap in time. */
svdag_status svdag_alt_table_add(svdag_alt_table* table, const uint32_t* keys_dev, uint32_t count, uint32_t* handles_dev,
    uint32_t lanes, void* stream);
/* find / findAsWarpHybrid: handle of a stored copy of each key, or SVDAG_INVALID_HANDLE. */
svdag_status svdag_alt_table_find(svdag_alt_table* table, const uint32_t* keys_dev, uint32_t count, uint32_t* handles_dev,
    uint32_t lanes, void* stream);
/* decodePointer: the item_words words of each handle to out_words_dev[i * item_words ...]; a handle
 * that names no stored item reads as zeros. */
svdag_status svdag_alt_table_read(svdag_alt_table* table, const uint32_t* handles_dev, uint32_t count,
    uint32_t* out_words_dev, void* stream);
/* Waits for the stream and returns (and clears) the first latched device-side error. */
svdag_status svdag_alt_table_sync(svdag_alt_table* table, void* stream);
/* Occupied slots, bucket slabs, overflow slabs linked, bytes of those slabs; synchronous, returns like
 * svdag_alt_table_sync. */
svdag_status svdag_alt_table_get_stats(svdag_alt_table* table, svdag_table_stats* out, void* stream);

/* The table half of garbage collection: clearActiveFlags / markAsActive / freeInactiveItems
 * (gpu_hash_table_base.h:102-112, gpu_hash_table_base.cu:231-330). Clear the flags, mark the handles
 * to keep (handles that name nothing are ignored), then free every stored item left unmarked:
 * *freed (may be NULL) receives how many. Kept items keep their handles; freed slots are reused by
 * later adds (overflow slabs stay linked; IndividualChaining unlinks freed nodes). Must not overlap
 * adds or finds. free_inactive is synchronous and returns like svdag_alt_table_sync. */
svdag_status svdag_alt_table_clear_active(svdag_alt_table* table, void* stream);
svdag_status svdag_alt_table_mark_active(svdag_alt_table* table, const uint32_t* handles_dev, uint32_t count, void* stream);
svdag_status svdag_alt_table_free_inactive(svdag_alt_table* table, uint64_t* freed, void* stream);

/* One measured candidate of svdag_alt_table_tune. */
typedef struct svdag_alt_tuning {
    uint32_t layout; /* SVDAG_TABLE_LAYOUT_* */
    uint32_t lanes; /* 1 or 32 */
    float add_ms; /* bulk add of the sample into a fresh table; < 0: the layout cannot hold the sample */
    float find_ms; /* find of every sample key afterwards */
} svdag_alt_tuning;
#define SVDAG_ALT_TUNING_CANDIDATES 7u
/* Measured choice among the alternative layouts for fixed-size items, with no counterpart in the
 * reference (which compares them offline, extras/hashmap_bench). For each slab layout and launch form
 * (lanes 1 and 32) and for INDIVIDUAL_CHAINING (lanes 1) a fresh table of count / items_per_bucket + 1 buckets (items_per_bucket 0 = 64)
 * is filled with the count keys of keys_dev and searched for all of them, timed with CUDA events on
 * `stream`. *best receives the candidate with the least add + find time; all[] (NULL, or room for
 * SVDAG_ALT_TUNING_CANDIDATES) every candidate. Synchronous; the tables are freed again. */
svdag_status svdag_alt_table_tune(svdag_ctx* ctx, const uint32_t* keys_dev, uint32_t count, uint32_t item_words,
    uint32_t items_per_bucket, svdag_alt_tuning* best, svdag_alt_tuning* all, void* stream);

/* ---------------------------------------------------------------- inspection */

typedef struct svdag_stats {
    uint32_t levels;
    uint32_t root;
    uint64_t pool_bytes;
    uint64_t item_region_bytes; /* items and slab headers */
    uint64_t item_region_used_bytes;
    uint64_t scratch_bytes;
    uint64_t scratch_high_water_bytes;
    uint64_t level_items[SVDAG_MAX_LEVELS];
    uint64_t level_buckets[SVDAG_MAX_LEVELS];
    uint32_t undo_count;
    uint32_t redo_count;
    uint64_t free_list_bytes; /* slabs on the free lists (counted as not in use above) */
    uint64_t free_list_slabs;
    uint64_t gc_freed_items; /* items the last collection freed */
    uint64_t gc_freed_slabs; /* overflow slabs the last collection put on the free lists */
    uint64_t gc_live_items; /* items the last collection found reachable */
} svdag_stats;
/* MyGPUHashDAG::report (my_gpu_hash_dag.cu:217-230). Synchronises `stream`. */
svdag_status svdag_get_stats(svdag_ctx* ctx, svdag_stats* out, void* stream);

/* Dumps every occupied item of a level table: out_handles[i] and out_words[i*SVDAG_MAX_ITEM_WORDS..]
 * (zero padded). With capacity 0 only *out_count is written. Synchronous; used for structural
 * comparison (MyGPUHashDAG::copy<CPU>, my_gpu_hash_dag.h:106-127). */
svdag_status svdag_export_level(svdag_ctx* ctx, uint32_t level, uint32_t* out_handles, uint32_t* out_words,
    uint64_t capacity, uint64_t* out_count, void* stream);

/* ---------------------------------------------------------------- import and export */

/* An item snapshot: level l (0 .. levels-2) holds level_items[l] items packed in level_words[l]
 * words (nodes: header + one word per child; leaves: 2 mask words + packed 4-bit materials), the
 * levels one after another. A node's child words are ordinals into the item list of the level below
 * and item 0 of level 0 is the root; all counts 0 is the empty DAG. Snapshots are the portable
 * form; the reference's own file (MyGPUHashDAG::writeTo / readFrom, my_gpu_hash_dag.cu:158-177)
 * converts to and from them with svdag_v3_to_items / svdag_items_to_v3 below. */

/* Writes the items reachable from the current root, each level in ascending handle order. Fills
 * level_words and level_items (levels - 1 entries each) and *total_words; writes the words when
 * capacity suffices, else returns SVDAG_ERR_OOM (call again with capacity >= *total_words).
 * Synchronous. */
svdag_status svdag_save_items(svdag_ctx* ctx, uint32_t* out_words, uint64_t capacity, uint64_t* level_words,
    uint64_t* level_items, uint64_t* total_words, void* stream);
/* Replaces the DAG by a snapshot: history cleared, each level table sized for its distinct items,
 * fully-filled items deduplicated against the canonical ones. A snapshot that does not parse (item
 * sizes, counts, child ordinals) gives SVDAG_ERR_INVALID and leaves the DAG unchanged. Synchronous. */
svdag_status svdag_load_items(svdag_ctx* ctx, const uint32_t* words, const uint64_t* level_words, const uint64_t* level_items,
    void* stream);
/* Host function: converts the node array of a BasicDAG (BasicDAG::data, basic_dag.h: root at index
 * 0, inner nodes [child mask in bits 0-7 | child indices], 64-bit leaves {low, high} at level
 * levels - 2) into a snapshot as create_dag_cpu converts it without colour import
 * (my_gpu_hash_dag_factory.cpp:316-418): every voxel gets `material`, and a node whose 8 children are
 * fully filled with one material carries the fully-filled header. Output as svdag_save_items; an
 * index out of range or an empty item gives SVDAG_ERR_CORRUPT. */
svdag_status svdag_basic_dag_to_items(const uint32_t* data, uint64_t n_words, uint32_t levels, uint32_t material,
    uint32_t* out_words, uint64_t capacity, uint64_t* level_words, uint64_t* level_items, uint64_t* total_words);

/* The reference's own DAG file: what MyGPUHashDAG::writeTo writes and readFrom reads, format
 * version 3 (my_gpu_hash_dag.cu:158-177), in the reference's default configuration
 * (configuration/gpu_hash_dag_definitions.h: CompactAccelerationHash tables, SlabHashXor buckets,
 * first slabs stored in the table, 4 material bits). Values of EMemoryType (memory.h:17-23) as the
 * file records them: */
#define SVDAG_V3_GPU_MANAGED 0u
#define SVDAG_V3_GPU_MALLOC 1u /* the engine's MyGPUHashDAG<EMemoryType::GPU_Malloc> */
#define SVDAG_V3_GPU_ASYNC 2u
#define SVDAG_V3_CPU 3u /* MyGPUHashDAG<EMemoryType::CPU> */
/* Host function: converts a version-3 file held in `data` (n_bytes, 4-byte aligned) into a snapshot,
 * following the handles from its root; output as svdag_save_items. The file's scene depth (the
 * width of its fully-filled node array, the reference's SCENE_DEPTH) must equal `levels`
 * (SVDAG_ERR_INVALID otherwise); another version or table configuration gives
 * SVDAG_ERR_UNSUPPORTED; a truncated file or a handle that does not name an occupied slot holding an
 * item of the handle's size gives SVDAG_ERR_CORRUPT. An empty DAG (root 0xFFFFFFFF) gives all
 * counts 0. */
svdag_status svdag_v3_to_items(const void* data, uint64_t n_bytes, uint32_t levels, uint32_t* out_words,
    uint64_t capacity, uint64_t* level_words, uint64_t* level_items, uint64_t* total_words);
/* Host function: writes a snapshot (as svdag_load_items takes it) to `path` as a version-3 file
 * whose arrays record `memory_type` (SVDAG_V3_*): the fully-filled items of every level and material
 * that MyGPUHashDAG::allocate inserts (my_gpu_hash_dag.cu:29-65), then the snapshot's distinct
 * items, each table sized to 96 items per bucket (TARGET_LOAD_FACTOR) and every item in a slot of
 * its bucket's slab chain, where the reference's find looks for it. The tables are laid out in host
 * memory before they are written (about the file's size). A snapshot that does not parse gives
 * SVDAG_ERR_INVALID; one whose handles would not fit the reference's 29-bit index SVDAG_ERR_OOM. */
svdag_status svdag_items_to_v3(const uint32_t* words, const uint64_t* level_words, const uint64_t* level_items,
    uint32_t levels, uint32_t memory_type, const char* path);

/* ---------------------------------------------------------------- autotuner
 *
 * Picks the settings of the batched form by measuring them on the device (no counterpart in the
 * reference, whose table sizes, slab layout and thread mapping are compile-time constants):
 *  - with a key sample: for each load factor (items per bucket of the tables sized from then on:
 *    8, 12, 16, 24, 32) and lane count per key (1, 2, 4, 8), a scratch table sized for the sample is
 *    filled with it and searched for it, timed with CUDA events; the fastest pair is kept. The
 *    scratch tables' space is given back afterwards.
 *  - with an edit sample: the edits are applied in order (for real, each pushing its undo frame),
 *    alternately through the per-tool CUDA graph of the phase launches and through the persistent
 *    single-CTA kernel, each timed with CUDA events; the persistent kernel is kept for the size
 *    buckets of the estimated SVO leaves, from the smallest up, where it is faster.
 * Synchronous; no other call may use the context meanwhile. */
typedef struct svdag_tuning {
    uint32_t probe_lanes; /* lanes per key of the table kernels */
    uint32_t load_factor; /* items per bucket of tables sized from now on */
    uint32_t persistent_leaves; /* edits estimated at or below this many SVO leaves use the persistent kernel (0 = none) */
    uint32_t trials; /* measurements taken */
    double table_ns_per_key; /* best fill + search time per key of the key sample */
    double graph_us_small; /* mean time of the sample's edits estimated below 4096 leaves: graph form */
    double persistent_us_small; /* the same through the persistent kernel */
} svdag_tuning;
svdag_status svdag_autotune(svdag_ctx* ctx, const svdag_edit* edits, uint32_t n_edits, const uint32_t* keys_dev,
    const uint32_t* offsets_dev, uint32_t n_keys, uint64_t total_words, uint32_t kind, svdag_tuning* out, void* stream);
svdag_status svdag_get_tuning(svdag_ctx* ctx, svdag_tuning* out);
svdag_status svdag_set_tuning(svdag_ctx* ctx, const svdag_tuning* tuning);

/* ---------------------------------------------------------------- serving form
 *
 * A request loop on its own host thread keeps the DAG, its tables and the undo history resident and
 * serves edit and frame requests as they arrive. Edits that arrive while earlier launches are on the
 * GPU are coalesced into the next batched launch (continuous batching: up to max_inflight launches
 * are queued on the GPU ahead of their completion). Frames run on a second stream, one at a time,
 * each behind every batch launched before it: its completion makes those edits visible and answers
 * the frame requests pending when it started, and the next batch edits while it renders.
 * An edit is admitted when the memory pressure (item-region bytes in use, less the slots the last
 * collection freed) plus the bytes reserved by admitted, unfinished edits (an upper estimate from
 * the tool's footprint) stays under the memory cap; a queue head that does not fit waits until
 * launches complete. Memory is reclaimed in the loop: once the pressure passes gc_threshold_bytes,
 * or when the queue head does not fit with nothing in flight, the loop lets
 * the launches and the frame in flight finish, then runs svdag_gc_keep_history (the undo history
 * survives) before it admits more. An edit that does not fit even after a collection fails with
 * SVDAG_ERR_OOM without being launched. With SVDAG_SERVE_PLAIN the same loop serves one request
 * at a time, synchronously, as the reference's engine does (an edit, then a frame: engine.h:104-163,
 * engine.cpp:627-629): the per-edit baseline. No counterpart in the reference beyond that loop. */

#define SVDAG_SERVE_PLAIN 1u /* one request per launch, synchronously */
#define SVDAG_SERVE_COPY_FRAMES 2u /* copy every rendered frame to host memory (svdag_server_frame) */
/* Trace every frame whole. Without it, a frame of the same camera as the one before is traced only
 * where a ray meets the bounding box of an edit made since (the other pixels keep their records,
 * which a whole frame would reproduce bit for bit); undo and redo, a new camera and the first frame
 * are traced whole. SVDAG_SERVE_PLAIN always traces whole frames, as the reference's loop does. */
#define SVDAG_SERVE_FULL_FRAMES 4u
/* Never collect garbage in the loop (edits that do not fit then fail with SVDAG_ERR_OOM). */
#define SVDAG_SERVE_NO_GC 8u

typedef struct svdag_server_config {
    uint32_t max_batch; /* edits per launch; 0 = 256 */
    uint32_t max_inflight; /* launches queued on the GPU; 0 = 2 */
    uint64_t memory_cap_bytes; /* item-region bytes that admitted edits may fill; 0 = the whole item region */
    svdag_trace_params frame; /* camera and resolution of the frames rendered after each launch */
    uint32_t flags; /* SVDAG_SERVE_* */
    uint32_t reserved;
    /* Memory pressure that starts a collection; 0 = the cap less 1/32 of it (at least 1 GiB, at most
     * an eighth). Pressure = item and header bytes in use less the slot bytes the last collection
     * freed and inserts have not filled yet (16 bytes per freed item, less 50 per item inserted). */
    uint64_t gc_threshold_bytes;
} svdag_server_config;

typedef struct svdag_server svdag_server;

typedef struct svdag_request_result {
    uint64_t ticket;
    uint32_t kind; /* 0 edit, 1 frame */
    uint32_t status; /* svdag_status of the edit (frames: 0) */
    uint32_t root_after; /* edits: root after this edit */
    uint32_t launch; /* sequence number of the launch that carried the request */
    uint64_t edited_voxels;
    double submit_s; /* host clock, seconds since the server started */
    double visible_s; /* completion of the frame that shows the request */
} svdag_request_result;

svdag_status svdag_server_create(svdag_ctx* ctx, const svdag_server_config* config, svdag_server** out);
/* Serves every request submitted so far, then stops the loop and frees the server (not the context). */
svdag_status svdag_server_destroy(svdag_server* server);
svdag_status svdag_submit_edit(svdag_server* server, const svdag_edit* edit, uint64_t* out_ticket);
/* `params` may be NULL (the configured camera). */
svdag_status svdag_submit_frame(svdag_server* server, const svdag_trace_params* params, uint64_t* out_ticket);
/* Result of a request: with wait = 0 returns SVDAG_ERR_BUSY while it is not visible yet. A result is
 * handed out once. */
svdag_status svdag_poll(svdag_server* server, uint64_t ticket, int wait, svdag_request_result* out);
/* Frames launched so far, traced whole and incrementally, and the bytes of frames copied to host
 * memory (SVDAG_SERVE_COPY_FRAMES). Any pointer may be NULL. No counterpart in the reference. */
svdag_status svdag_server_counters(svdag_server* server, uint64_t* frames_whole, uint64_t* frames_incremental,
    uint64_t* frame_bytes_to_host);
/* Memory accounting of the loop. No counterpart in the reference. */
typedef struct svdag_server_memory {
    uint64_t used_bytes; /* item and header region in use after the last finished launch (free lists excluded) */
    uint64_t cap_bytes; /* admission cap */
    uint64_t gc_threshold_bytes;
    uint64_t gc_runs; /* collections the loop ran */
    uint64_t gc_freed_bytes; /* drop of used_bytes over those collections */
    double gc_seconds; /* host time they took (the loop admits nothing meanwhile) */
    uint64_t rejected_edits; /* failed with SVDAG_ERR_OOM before launch: they did not fit after a collection */
    uint64_t failed_edits; /* launched edits whose record reported an error */
    uint64_t reuse_credit_bytes; /* freed slot bytes counted as available (see gc_threshold_bytes) */
} svdag_server_memory;
svdag_status svdag_server_memory_stats(svdag_server* server, svdag_server_memory* out);
/* Copies the most recent frame (SVDAG_SERVE_COPY_FRAMES) to `out` (width * height hits). */
svdag_status svdag_server_frame(svdag_server* server, svdag_hit* out, uint64_t capacity);
/* Replays a timed request stream (the reference's replay of recorded edits, replay.h): edit i is
 * submitted edit_times[i] seconds after the call starts, frame j at frame_times[j]; returns when all
 * are visible, with results[0 .. n_edits) for the edits and results[n_edits ..) for the frames. */
svdag_status svdag_server_replay(svdag_server* server, const svdag_edit* edits, const double* edit_times, uint32_t n_edits,
    const double* frame_times, uint32_t n_frames, svdag_request_result* results);
/* An undo (redo = 0) or redo (redo = 1) request: MyGPUHashDAGUndoRedo::undo/redo
 * (my_gpu_base_dag.h:35-64) applied after every edit submitted before it and before every edit
 * submitted after it. Its result has kind 2 (undo) or 3 (redo) and the root it left. */
svdag_status svdag_submit_undo(svdag_server* server, int redo, uint64_t* out_ticket);

/* ---------------------------------------------------------------- recorded edit sessions */

/* The reference's replay files (ReplayManager::load_csv, replay.h:650-683): one action per line, the
 * action name then comma-separated values, trailing empty cells ignored; text after the last newline
 * is ignored, as load_csv ignores it. */
typedef enum svdag_replay_kind {
    SVDAG_REPLAY_OTHER = 0, /* SetToolParameters, EditFill (CPU HashDAG only): no GPU request */
    SVDAG_REPLAY_EDIT = 1, /* EditSphere, EditCube, EditPaint, EditCopy */
    SVDAG_REPLAY_UNDO = 2,
    SVDAG_REPLAY_REDO = 3,
    SVDAG_REPLAY_END_FRAME = 4,
    SVDAG_REPLAY_CAMERA_LOCATION = 5, /* SetLocation: camera[0..3) world position */
    SVDAG_REPLAY_CAMERA_ROTATION = 6 /* SetRotation: camera[0..9) rows D00..D22 of the view matrix */
} svdag_replay_kind;

typedef struct svdag_replay_action {
    uint32_t kind; /* svdag_replay_kind */
    svdag_edit edit; /* SVDAG_REPLAY_EDIT: the editor the reference's apply() builds (replay.cpp:52-134) */
    float camera[9];
} svdag_replay_action;

/* Parses a replay file held in memory. Edit positions and radii are multiplied by `scale` (the
 * reference's scalingFactor = 2^SCENE_DEPTH / 2^REPLAY_DEPTH, replay.cpp:10), colours are dropped
 * (the DAG stores materials), materials default to 1 as in the reference's loaders (replay.h:288-541).
 * Writes min(count, capacity) actions; *count is the number parsed. A line the reference's loaders
 * would reject (unknown action, wrong cell count, a number or boolean that does not parse) or a
 * material >= SVDAG_NUM_MATERIALS gives SVDAG_ERR_INVALID with its 0-based index in *bad_line (may
 * be NULL); more actions than a nonzero capacity gives SVDAG_ERR_OOM. */
svdag_status svdag_replay_parse(const char* text, uint64_t length, float scale, svdag_replay_action* out, uint64_t capacity,
    uint64_t* count, uint64_t* bad_line);
/* Serves a parsed replay: the actions of recorded frame f (those before its EndFrame) are submitted
 * f * frame_period_s seconds after the call starts, in order (edits, undos, redos), and each EndFrame
 * submits a frame request (the camera frames[f] when frames is not NULL, one per EndFrame, else the
 * configured one), as ReplayManager::replay_frame does (replay.h:583-596). Returns when every request
 * is visible; results[i] belongs to actions[i] (ticket 0 for actions that are not requests). */
svdag_status svdag_server_replay_actions(svdag_server* server, const svdag_replay_action* actions, uint64_t n_actions,
    double frame_period_s, const svdag_trace_params* frames, svdag_request_result* results);

#ifdef __cplusplus
}
#endif

#endif /* SVDAG_H */
