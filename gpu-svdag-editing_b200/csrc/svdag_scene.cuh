// svdag_scene.cuh - the procedural scene used as input data: an integer value-noise fBm heightfield
// with optional boxes and spheres unioned on its surface. Host and device share this code (the host
// places the structures on the surface); everything is integer arithmetic, so the GPU builder and the
// CPU oracle's own restatement agree exactly.
//
// Voxel (x, y, z) is solid when y < height(x, z) or when a structure contains it. Its material is that
// of the highest-index structure containing it, else the height band (y * num_materials) >> levels.
#pragma once
#include <cstdint>

#include "../../include/svdag.h"

namespace svdag {

struct Structure {
    int32_t lo[3], hi[3]; // voxel bounds [lo, hi) of a box, bounding box of a sphere
    int32_t c[3]; // sphere centre
    uint32_t r2; // sphere radius squared
    uint32_t kind; // 0 box, 1 sphere
    uint32_t material;
};

struct SceneParams {
    svdag_terrain_params terrain;
    uint32_t levels;
    uint32_t baseLog2; // lattice cell of octave 0 = 2^baseLog2 voxels
    const Structure* structures;
    const uint32_t* cellStart; // CSR over an xz grid of 2^cellLog2-voxel cells: structures overlapping each cell
    const uint32_t* cellList;
    uint32_t numStructures;
    uint32_t cellLog2;
    uint32_t cellsPerAxis;
    int32_t structYLo, structYHi; // y range [lo, hi) covered by any structure
    uint32_t pad;
};

__host__ __device__ inline uint32_t scene_fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
__host__ __device__ inline uint32_t terrain_lattice(const SceneParams& p, uint32_t ix, uint32_t iz, uint32_t o)
{
    uint32_t h = scene_fmix32(p.terrain.seed * 0x9E3779B9u ^ (o * 0x85EBCA6Bu) ^ 0x68E31DA4u);
    h = scene_fmix32(h ^ (ix * 0xC2B2AE35u));
    h = scene_fmix32(h ^ (iz * 0x27D4EB2Fu));
    return h >> 16;
}
__host__ __device__ inline long long smooth16(long long t) { return (t * t * (3 * 65536 - 2 * t)) >> 32; }
__host__ __device__ inline long long lerp16(long long a, long long b, long long t) { return a + (((b - a) * t) >> 16); }
__host__ __device__ inline uint32_t terrain_cell_log2(const SceneParams& p, uint32_t o) { return p.baseLog2 > o ? p.baseLog2 - o : 0u; }
__host__ __device__ inline uint32_t terrain_height_from_fbm(const SceneParams& p, long long f)
{
    const long long G = 1ll << p.levels;
    const long long base = G * p.terrain.min_height_pct / 100;
    const long long range = G * (long long)(p.terrain.max_height_pct - p.terrain.min_height_pct) / 100;
    const long long norm = ((1ll << p.terrain.octaves) - 1) * 65536;
    return (uint32_t)(base + (range * f) / norm);
}
__host__ __device__ inline long long terrain_octave(const SceneParams& p, uint32_t x, uint32_t z, uint32_t o)
{
    const uint32_t c = terrain_cell_log2(p, o);
    const uint32_t ix = x >> c, iz = z >> c, m = (1u << c) - 1u;
    const long long fx = c <= 16 ? (long long)((x & m) << (16 - c)) : (long long)((x & m) >> (c - 16));
    const long long fz = c <= 16 ? (long long)((z & m) << (16 - c)) : (long long)((z & m) >> (c - 16));
    const long long sx = smooth16(fx), sz = smooth16(fz);
    const long long a = lerp16(terrain_lattice(p, ix, iz, o), terrain_lattice(p, ix + 1, iz, o), sx);
    const long long b = lerp16(terrain_lattice(p, ix, iz + 1, o), terrain_lattice(p, ix + 1, iz + 1, o), sx);
    return lerp16(a, b, sz);
}
__host__ __device__ inline uint32_t terrain_height(const SceneParams& p, uint32_t x, uint32_t z)
{
    long long f = 0;
    for (uint32_t o = 0; o < p.terrain.octaves; ++o)
        f += terrain_octave(p, x, z, o) << (p.terrain.octaves - 1 - o);
    return terrain_height_from_fbm(p, f);
}
// Conservative height bounds over the aligned footprint [x0, x0+s) x [z0, z0+s).
__host__ __device__ inline void terrain_bounds(const SceneParams& p, uint32_t x0, uint32_t z0, uint32_t s, uint32_t& hlo, uint32_t& hhi)
{
    long long lo = 0, hi = 0;
    for (uint32_t o = 0; o < p.terrain.octaves; ++o) {
        const uint32_t c = terrain_cell_log2(p, o);
        const uint32_t ix0 = x0 >> c, iz0 = z0 >> c;
        const uint32_t ix1 = ((x0 + s - 1) >> c) + 1, iz1 = ((z0 + s - 1) >> c) + 1;
        long long vlo = 65535, vhi = 0;
        if (s <= (1u << c)) {
            // Inside one lattice cell the field is bilinear in the (monotone) smoothstep weights, so
            // the extremes sit at the footprint corners; integer truncation of the three lerps moves a
            // value at most 2 units below the real bilinear value.
            const uint32_t x1 = x0 + s - 1, z1 = z0 + s - 1;
            const long long v0 = terrain_octave(p, x0, z0, o), v1 = terrain_octave(p, x1, z0, o);
            const long long v2 = terrain_octave(p, x0, z1, o), v3 = terrain_octave(p, x1, z1, o);
            vlo = v0 < v1 ? v0 : v1;
            vlo = vlo < v2 ? vlo : v2;
            vlo = vlo < v3 ? vlo : v3;
            vhi = v0 > v1 ? v0 : v1;
            vhi = vhi > v2 ? vhi : v2;
            vhi = vhi > v3 ? vhi : v3;
            vlo = vlo - 2 < 0 ? 0 : vlo - 2;
            vhi = vhi + 2 > 65535 ? 65535 : vhi + 2;
        } else if ((unsigned long long)(ix1 - ix0 + 1) * (iz1 - iz0 + 1) > 64) {
            vlo = 0;
            vhi = 65535;
        } else {
            for (uint32_t iz = iz0; iz <= iz1; ++iz)
                for (uint32_t ix = ix0; ix <= ix1; ++ix) {
                    const long long v = terrain_lattice(p, ix, iz, o);
                    vlo = v < vlo ? v : vlo;
                    vhi = v > vhi ? v : vhi;
                }
        }
        lo += vlo << (p.terrain.octaves - 1 - o);
        hi += vhi << (p.terrain.octaves - 1 - o);
    }
    hlo = terrain_height_from_fbm(p, lo);
    hhi = terrain_height_from_fbm(p, hi);
}
__host__ __device__ inline uint32_t terrain_material(const SceneParams& p, uint32_t y)
{
    return (uint32_t)(((unsigned long long)y * p.terrain.num_materials) >> p.levels);
}

// ---- structures

__host__ __device__ inline bool structure_contains(const Structure& s, int32_t x, int32_t y, int32_t z)
{
    if (x < s.lo[0] || x >= s.hi[0] || y < s.lo[1] || y >= s.hi[1] || z < s.lo[2] || z >= s.hi[2])
        return false;
    if (s.kind == 0)
        return true;
    const long long dx = x - s.c[0], dy = y - s.c[1], dz = z - s.c[2];
    return (unsigned long long)(dx * dx + dy * dy + dz * dz) <= s.r2;
}

// Relation of a structure to the voxel box [b0, b0+n)^3 (voxel coordinates b0 .. b0+n-1):
// 0 disjoint, 1 partial, 2 contains every voxel.
__host__ __device__ inline uint32_t structure_vs_box(const Structure& s, const int32_t* b0, int32_t n)
{
    for (int a = 0; a < 3; ++a)
        if (b0[a] + n <= s.lo[a] || b0[a] >= s.hi[a])
            return 0;
    if (s.kind == 0) {
        for (int a = 0; a < 3; ++a)
            if (b0[a] < s.lo[a] || b0[a] + n > s.hi[a])
                return 1;
        return 2;
    }
    long long dmin = 0, dmax = 0;
    for (int a = 0; a < 3; ++a) {
        const long long lo = b0[a], hi = (long long)b0[a] + n - 1;
        const long long c = s.c[a];
        const long long near = c < lo ? lo - c : (c > hi ? c - hi : 0);
        const long long far = (c - lo > hi - c) ? c - lo : hi - c;
        dmin += near * near;
        dmax += far * far;
    }
    if ((unsigned long long)dmin > s.r2)
        return 0;
    return (unsigned long long)dmax <= s.r2 ? 2 : 1;
}

// Material of voxel (x, y, z) or SVDAG_NO_MATERIAL; `h` is height(x, z).
__host__ __device__ inline uint32_t scene_voxel(const SceneParams& p, uint32_t x, uint32_t y, uint32_t z, uint32_t h)
{
    if (p.numStructures) {
        const uint32_t cx = x >> p.cellLog2, cz = z >> p.cellLog2;
        const uint32_t cell = cz * p.cellsPerAxis + cx;
        uint32_t best = 0xFFFFFFFFu;
        for (uint32_t i = p.cellStart[cell]; i < p.cellStart[cell + 1]; ++i) {
            const uint32_t j = p.cellList[i];
            if ((best == 0xFFFFFFFFu || j > best) && structure_contains(p.structures[j], (int32_t)x, (int32_t)y, (int32_t)z))
                best = j;
        }
        if (best != 0xFFFFFFFFu)
            return p.structures[best].material;
    }
    return y < h ? terrain_material(p, y) : SVDAG_NO_MATERIAL;
}

// Classification of the node [p << depth, +2^depth)^3: 0 = Subdivide, 1 = Fill (*material), 2 = Empty.
__host__ __device__ inline uint32_t scene_classify(const SceneParams& p, uint32_t px, uint32_t py, uint32_t pz, uint32_t depth,
    uint32_t& material)
{
    const uint32_t s = 1u << depth;
    const uint32_t x0 = px << depth, y0 = py << depth, z0 = pz << depth;
    uint32_t hlo, hhi;
    terrain_bounds(p, x0, z0, s, hlo, hhi);
    uint32_t terrainOp = 0, terrainMat = 0;
    if (y0 >= hhi) {
        terrainOp = 2;
    } else if (y0 + s <= hlo) {
        const uint32_t m0 = terrain_material(p, y0), m1 = terrain_material(p, y0 + s - 1);
        if (m0 == m1) {
            terrainOp = 1;
            terrainMat = m0;
        }
    }
    if (p.numStructures && (long long)y0 + s > p.structYLo && (long long)y0 < p.structYHi) {
        const uint32_t c0x = x0 >> p.cellLog2, c0z = z0 >> p.cellLog2;
        const uint32_t c1x = (x0 + s - 1) >> p.cellLog2, c1z = (z0 + s - 1) >> p.cellLog2;
        if ((c1x - c0x + 1) * (c1z - c0z + 1) > 16)
            return 0; // large nodes: subdividing is always correct
        const int32_t b0[3] = { (int32_t)x0, (int32_t)y0, (int32_t)z0 };
        uint32_t best = 0xFFFFFFFFu, bestRel = 0;
        for (uint32_t cz = c0z; cz <= c1z; ++cz)
            for (uint32_t cx = c0x; cx <= c1x; ++cx) {
                const uint32_t cell = cz * p.cellsPerAxis + cx;
                for (uint32_t i = p.cellStart[cell]; i < p.cellStart[cell + 1]; ++i) {
                    const uint32_t j = p.cellList[i];
                    if (best != 0xFFFFFFFFu && j <= best)
                        continue;
                    const uint32_t rel = structure_vs_box(p.structures[j], b0, (int32_t)s);
                    if (rel) {
                        best = j;
                        bestRel = rel;
                    }
                }
            }
        if (best != 0xFFFFFFFFu) {
            if (bestRel == 2) { // the topmost intersecting structure covers the node
                material = p.structures[best].material;
                return 1;
            }
            return 0;
        }
    }
    material = terrainMat;
    return terrainOp;
}

} // namespace svdag
