/*
 * svdag_oracle.h - C API of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is a plain C++ restatement of the reference's
 * EDag::MyGpuDag algorithms (mathijs727/GPU-SVDAG-Editing). It is the checker of the
 * CUDA implementation: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it. It is compiled with -ffp-contract=off and without fast-math so that its
 * float predicates are the IEEE-exact, uncontracted forms of the reference's expressions.
 *
 * Handles inside the oracle are per-level item indices; they are never compared with the
 * CUDA implementation's handles. Structure is compared canonically (per-level distinct
 * content counts and Merkle digests), voxels through sampling, and hits per pixel.
 */
#ifndef SVDAG_ORACLE_H
#define SVDAG_ORACLE_H

#include "../include/svdag.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_dag oracle_dag;

typedef struct oracle_canon {
    uint64_t unique_per_level[SVDAG_MAX_LEVELS]; /* distinct contents reachable from the root */
    uint64_t digest_per_level[SVDAG_MAX_LEVELS]; /* order-independent digest of the level's content set */
    uint64_t root_digest; /* Merkle digest of the whole DAG (0 for an empty DAG) */
    uint64_t voxel_count_lo; /* number of solid voxels (low 64 bits) */
    uint64_t voxel_count_hi;
} oracle_canon;

oracle_dag* oracle_create(uint32_t levels);
void oracle_destroy(oracle_dag* dag);
uint32_t oracle_levels(const oracle_dag* dag);
uint32_t oracle_root(const oracle_dag* dag);
int oracle_is_empty(const oracle_dag* dag);

int oracle_build_terrain(oracle_dag* dag, const svdag_terrain_params* params);
/* The reference test scene of gpu_hash_dag_tests.cpp:35-89 (createBoxDag): an axis-aligned box. */
int oracle_build_box(oracle_dag* dag, float bmin, float bmax, uint32_t material);
/* Builds only the subtree of the scene node (level, path) into an emptied DAG; *out_handle is its
 * handle at `level` (0xFFFFFFFF = empty). */
int oracle_build_scene_subtree(oracle_dag* dag, const svdag_terrain_params* params, uint32_t level, const uint32_t path[3],
    uint32_t* out_handle);
/* Builds the scene with every voxel outside [lo, hi) left empty (regions of scenes too large for
 * the oracle; nodes wholly inside the region equal those of the full scene). */
int oracle_build_scene_region(oracle_dag* dag, const svdag_terrain_params* params, const int64_t lo[3], const int64_t hi[3]);
/* Handle of the node (level, path), 0xFFFFFFFF where the DAG is empty there. */
uint32_t oracle_node_at(const oracle_dag* dag, uint32_t level, const uint32_t path[3]);
/* The scene's voxels straight from its definition (no DAG): material or 0xFFFFFFFF. */
int oracle_scene_voxels(const svdag_terrain_params* params, uint32_t levels, const uint32_t* xyz, uint64_t count, uint32_t* out);

int oracle_edit(oracle_dag* dag, const svdag_edit* edit, svdag_edit_stats* out_stats);
int oracle_undo(oracle_dag* dag);
int oracle_redo(oracle_dag* dag);
int oracle_gc(oracle_dag* dag);
uint32_t oracle_undo_count(const oracle_dag* dag);
uint32_t oracle_redo_count(const oracle_dag* dag);

int oracle_sample_voxels(const oracle_dag* dag, const uint32_t* xyz, uint64_t count, uint32_t* out);
/* The items reachable from the root as one array of items at a stride of 10 words (zero padded),
 * level by level, every child word rewritten to the index of the child's item in that array; item 0
 * is the root. Writes *count items when capacity (in items) suffices, else only sets *count and
 * returns 1. An empty DAG gives *count = 0. For feeding the reference's own decoding code. */
/* oracle_should_edit over n nodes of one edit (paths: 3 words each). */
int oracle_should_edit_many(const svdag_edit* e, const uint32_t* paths, const uint32_t* depths, const uint32_t* states,
    const uint32_t* fills, uint64_t n, int32_t* ops, uint32_t* out_fills);
int oracle_export_items(const oracle_dag* dag, uint32_t* out, uint64_t capacity, uint64_t* count);
int oracle_trace(const oracle_dag* dag, const svdag_trace_params* params, svdag_hit* out, int threads);
/* Shading of a hit buffer (trace_colors, trace_shadows, trace_ambient_occlusion, trace_lighting,
 * tracer.cu:413-730); hits[i].color receives the diffuse colour; rgba, sun and ao get width*height values. */
/* sin and cos of the AO sample angle (quadrant reduction, Taylor polynomials), as the library computes them. */
void oracle_sincos(float x, float* s, float* c);
int oracle_shade(const oracle_dag* dag, const svdag_trace_params* trace, const svdag_shade_params* shade, svdag_hit* hits,
    uint32_t* rgba, float* sun, float* ao, int threads);
/* Node-visit counters of the trace (for the tracer's algorithmic bytes). */
int oracle_trace_counts(const oracle_dag* dag, const svdag_trace_params* params, uint64_t* out_node_visits,
    uint64_t* out_leaf_visits, uint64_t* out_hits);

int oracle_canonicalize(const oracle_dag* dag, oracle_canon* out);
/* Canonicalises a DAG given as per-level dumps of (handle, 10 padded words) records, as produced
 * by svdag_export_level. handles[l]/words[l] have counts[l] entries. */
/* Canonical form of the subtree under the item `handle` of `level`. */
int oracle_canonicalize_at(const oracle_dag* dag, uint32_t level, uint32_t handle, oracle_canon* out);
int oracle_canonicalize_dump_at(uint32_t levels, uint32_t level, uint32_t root, const uint32_t* const* handles,
    const uint32_t* const* words, const uint64_t* counts, oracle_canon* out);
int oracle_canonicalize_dump(uint32_t levels, uint32_t root, const uint32_t* const* handles,
    const uint32_t* const* words, const uint64_t* counts, oracle_canon* out);

/* Item encodings (my_gpu_base_dag.h) exposed for known-answer tests. */
uint32_t oracle_encode_node_header(uint32_t child_mask, uint32_t user_payload);
uint32_t oracle_header_child_mask(uint32_t header);
uint32_t oracle_header_user_payload(uint32_t header);
/* LeafBuilder: voxel i is set when (mask >> i) & 1, with material materials[i]; returns size. */
uint32_t oracle_build_leaf(uint64_t mask, const uint32_t* materials, uint32_t* out_words);
uint32_t oracle_leaf_size(const uint32_t* leaf);
int oracle_leaf_material(const uint32_t* leaf, uint32_t voxel, uint32_t* out_material);
uint32_t oracle_terrain_height(const svdag_terrain_params* params, uint32_t levels, uint32_t x, uint32_t z);
uint32_t oracle_noise_material(uint32_t seed, uint32_t cell_log2, uint32_t x, uint32_t y, uint32_t z);
/* should_edit of a tool for the node at `path` of size 2^depth, with the given node state
 * (0 Partial, 1 Filled, 2 Empty). Returns op (0 Subdivide, 1 Fill, 2 Empty, 3 Keep). Stateless tools only. */
int oracle_should_edit(const svdag_edit* edit, const uint32_t path[3], uint32_t depth, uint32_t state,
    uint32_t fill_material, uint32_t* out_fill_material);
/* get_trace_params (dag_tracer.cu:59-101) for a look-at camera in voxel coordinates. */
void oracle_camera_params(const double position[3], const double target[3], double fov_degrees,
    uint32_t width, uint32_t height, svdag_trace_params* out);

#ifdef __cplusplus
}
#endif

#endif
