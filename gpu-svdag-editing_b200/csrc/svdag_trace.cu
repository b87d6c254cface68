// svdag_trace.cu - primary-ray DAG traversal writing the per-pixel hit buffer, and voxel sampling.
//
// Reference: Tracer::trace_paths / intersect_ray / compute_intersection_mask / createSurfaceInteraction
// (tracer.cu:28-411), ray setup from DAGTracer::resolve_paths (dag_tracer.cu:112-134), voxel queries
// from getVoxelValues_kernel -> DAGUtils::get_value (dag_tracer.cu:361-372, dag_utils.h:146-182).
// Float and double arithmetic follow the reference expression by expression; with -fmad=false nothing
// is contracted, so hits equal the oracle's bit for bit. A child fetch is one load: handles are
// offsets of the items (8-byte units), so the traversal reads the header and the child handle without
// a slab-table decode.
#include <cuda_runtime.h>

#include "svdag_host.hpp"

namespace svdag {
namespace {

struct RayF {
    float ox, oy, oz, dx, dy, dz, ix, iy, iz;
};

__device__ __forceinline__ float cmaxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float cminf(float a, float b) { return a < b ? a : b; }

// compute_intersection_mask, tracer.cu:56-173 (device max/min of two floats are fmaxf/fminf; the
// vector max/min of cuda_math.h are the ternary forms).
__device__ __forceinline__ uint32_t intersection_mask(bool isRoot, uint32_t level, uint32_t px, uint32_t py, uint32_t pz, uint32_t levels,
    const RayF& r)
{
    const uint32_t shift = levels - level;
    const float radius = float(1u << (shift - 1));
    const float cx = radius + float(px << shift), cy = radius + float(py << shift), cz = radius + float(pz << shift);
    const float rx = cx - r.ox, ry = cy - r.oy, rz = cz - r.oz;
    const float tmx = rx * r.ix, tmy = ry * r.iy, tmz = rz * r.iz;
    float tmin, tmax;
    {
        const float sx = radius * fabsf(r.ix), sy = radius * fabsf(r.iy), sz = radius * fabsf(r.iz);
        tmin = fmaxf(cmaxf(tmx - sx, cmaxf(tmy - sy, tmz - sz)), 0.0f);
        tmax = cminf(tmx + sx, cminf(tmy + sy, tmz + sz));
    }
    tmin = fmaxf(tmin, 0.0f); // ray.tmin
    tmax = fminf(tmax, 3.402823466e+38f); // ray.tmax
    if (isRoot && (tmin >= tmax))
        return 0;
    uint32_t mask;
    {
        const float tm = 0.5f * (tmin + tmax);
        const float x = tm * r.dx, y = tm * r.dy, z = tm * r.dz;
        mask = 1u << (((x >= rx) ? 4u : 0u) + ((y >= ry) ? 2u : 0u) + ((z >= rz) ? 1u : 0u));
    }
    const float eps = 1e-4f;
    // The three plane tests as selects (no divergent branches; same comparisons and operands).
    {
        const float y = tmx * r.dy, z = tmx * r.dz;
        const uint32_t A = ((y >= ry - eps) ? 0xCCu : 0u) | ((y <= ry + eps) ? 0x33u : 0u);
        const uint32_t B = ((z >= rz - eps) ? 0xAAu : 0u) | ((z <= rz + eps) ? 0x55u : 0u);
        mask |= (tmin <= tmx && tmx <= tmax) ? (A & B) : 0u;
    }
    {
        const float x = tmy * r.dx, z = tmy * r.dz;
        const uint32_t C = ((x >= rx - eps) ? 0xF0u : 0u) | ((x <= rx + eps) ? 0x0Fu : 0u);
        const uint32_t D = ((z >= rz - eps) ? 0xAAu : 0u) | ((z <= rz + eps) ? 0x55u : 0u);
        mask |= (tmin <= tmy && tmy <= tmax) ? (C & D) : 0u;
    }
    {
        const float x = tmz * r.dx, y = tmz * r.dy;
        const uint32_t E = ((x >= rx - eps) ? 0xF0u : 0u) | ((x <= rx + eps) ? 0x0Fu : 0u);
        const uint32_t F = ((y >= ry - eps) ? 0xCCu : 0u) | ((y <= ry + eps) ? 0x33u : 0u);
        mask |= (tmin <= tmz && tmz <= tmax) ? (E & F) : 0u;
    }
    return mask & 0xFFu;
}

// The first child ci = c ^ order (c = 0, 1, ...) whose bit is set (tracer.cu:45-54; mask != 0): the
// mask is permuted so that bit c holds bit c ^ order, then the lowest set bit is taken.
__device__ __forceinline__ uint32_t next_child(uint32_t order, uint32_t mask)
{
    uint32_t m = mask;
    m = (order & 1u) ? (((m & 0x55u) << 1) | ((m >> 1) & 0x55u)) : m;
    m = (order & 2u) ? (((m & 0x33u) << 2) | ((m >> 2) & 0x33u)) : m;
    m = (order & 4u) ? (((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu)) : m;
    return ((uint32_t)__ffs(m) - 1u) ^ order;
}

__device__ __forceinline__ uint32_t first_child_mask(uint32_t lo, uint32_t hi) // Leaf::get_first_child_mask, base_dag.h:16-52
{
    uint32_t out = 0;
#pragma unroll
    for (uint32_t i = 0; i < 4; ++i) {
        out |= ((lo >> (8 * i)) & 0xFFu) ? (1u << i) : 0u;
        out |= ((hi >> (8 * i)) & 0xFFu) ? (1u << (i + 4)) : 0u;
    }
    return out;
}

__global__ void __launch_bounds__(256) k_trace(DevDag d, svdag_trace_params p, svdag_hit* out, const uint32_t* rootPtr)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.width || y >= p.height)
        return;
    // Ray setup in double (trace_paths, tracer.cu:403-405; normalize = (1 / length) * v).
    const double dpx = (double)x, dpy = (double)y;
    const double vx = ((p.ray_min[0] + dpx * p.ray_ddx[0]) + dpy * p.ray_ddy[0]) - p.camera[0];
    const double vy = ((p.ray_min[1] + dpx * p.ray_ddx[1]) + dpy * p.ray_ddy[1]) - p.camera[1];
    const double vz = ((p.ray_min[2] + dpx * p.ray_ddx[2]) + dpy * p.ray_ddy[2]) - p.camera[2];
    const double len = sqrt(vx * vx + vy * vy + vz * vz);
    const double inv = 1 / len;
    RayF r;
    r.ox = (float)p.camera[0];
    r.oy = (float)p.camera[1];
    r.oz = (float)p.camera[2];
    r.dx = (float)(inv * vx);
    r.dy = (float)(inv * vy);
    r.dz = (float)(inv * vz);
    r.ix = 1.0f / r.dx;
    r.iy = 1.0f / r.dy;
    r.iz = 1.0f / r.dz;

    // intersect_ray, tracer.cu:186-273.
    const uint32_t levels = d.levels, LL = d.leafLevel;
    const uint32_t order = (r.dx < 0.f ? 4u : 0u) + (r.dy < 0.f ? 2u : 0u) + (r.dz < 0.f ? 1u : 0u);
    // Traversal stack in shared memory, [level][thread] so that a warp's accesses hit distinct banks.
    __shared__ uint32_t sIndex[kMaxLevels][256];
    __shared__ uint32_t sMasks[kMaxLevels][256]; // childMask | visitMask << 8
    const uint32_t tix = threadIdx.y * blockDim.x + threadIdx.x;
    uint32_t level = 0, addr = 0, px = 0, py = 0, pz = 0, leafLo = 0, leafHi = 0;
    uint32_t material = 0xFFFFFFFFu;
    const uint32_t root = rootPtr ? *rootPtr : d.ctl->root;
    if (root != kNone) {
        uint32_t cIndex = root;
        uint32_t cChild = item_ptr(d, root)[0] & 0xFFu;
        uint32_t cVisit = cChild & intersection_mask(true, 0, 0, 0, 0, levels, r);
        for (;;) {
            {
                uint32_t newLevel = level;
                while (newLevel > 0 && !cVisit) {
                    newLevel--;
                    cIndex = sIndex[newLevel][tix];
                    cChild = sMasks[newLevel][tix] & 0xFFu;
                    cVisit = sMasks[newLevel][tix] >> 8;
                }
                if (newLevel == 0 && !cVisit) {
                    px = py = pz = 0;
                    break;
                }
                const uint32_t up = level - newLevel;
                px >>= up;
                py >>= up;
                pz >>= up;
                level = newLevel;
            }
            const uint32_t nextChild = next_child(order, cVisit);
            cVisit &= ~(1u << nextChild);
            px = (px << 1) | ((nextChild >> 2) & 1u);
            py = (py << 1) | ((nextChild >> 1) & 1u);
            pz = (pz << 1) | (nextChild & 1u);
            sIndex[level][tix] = cIndex;
            sMasks[level][tix] = cChild | (cVisit << 8);
            level++;
            if (level == levels) {
                const uint32_t voxel = ((px & 1u) ? 4u : 0u) | ((py & 1u) ? 2u : 0u) | ((pz & 1u) ? 1u : 0u) | ((px & 2u) ? 32u : 0u)
                    | ((py & 2u) ? 16u : 0u) | ((pz & 2u) ? 8u : 0u); // mortonU32() & 63
                const uint32_t* leaf = item_ptr(d, addr);
                const unsigned long long m = (unsigned long long)leafLo | ((unsigned long long)leafHi << 32);
                if ((m >> voxel) & 1ull) {
                    const uint32_t bit = __popcll(m & ((1ull << voxel) - 1ull)) * 4u;
                    material = (leaf[2 + (bit >> 5)] >> (bit & 31u)) & 0xFu;
                }
                break;
            }
            if (level < LL) {
                const uint32_t* node = item_ptr(d, cIndex);
                cIndex = node[1 + __popc(cChild & ((1u << nextChild) - 1u))];
                cChild = item_ptr(d, cIndex)[0] & 0xFFu;
                cVisit = cChild & intersection_mask(false, level, px, py, pz, levels, r);
            } else {
                uint32_t childMask;
                if (level == LL) {
                    const uint32_t* node = item_ptr(d, cIndex);
                    addr = node[1 + __popc(cChild & ((1u << nextChild) - 1u))];
                    const uint32_t* lp = item_ptr(d, addr);
                    const uint2 lh = make_uint2(lp[0], lp[1]);
                    leafLo = lh.x;
                    leafHi = lh.y;
                    childMask = first_child_mask(leafLo, leafHi);
                } else { // get_second_child_mask, base_dag.h:53-58
                    childMask = (((nextChild & 4u) ? leafHi : leafLo) >> ((nextChild & 3u) * 8u)) & 0xFFu;
                }
                cChild = childMask;
                cVisit = cChild & intersection_mask(false, level, px, py, pz, levels, r);
            }
        }
    }
    if (px == 0 && py == 0 && pz == 0)
        material = 0xFFFFFFFFu; // a miss has no material (Path::is_null, path.h:61-64)

    // createSurfaceInteraction, tracer.cu:353-389.
    const float bx = float(px), by = float(py), bz = float(pz);
    const float t1x = (bx - r.ox) * r.ix, t1y = (by - r.oy) * r.iy, t1z = (bz - r.oz) * r.iz;
    const float t2x = ((bx + 1.0f) - r.ox) * r.ix, t2y = ((by + 1.0f) - r.oy) * r.iy, t2z = ((bz + 1.0f) - r.oz) * r.iz;
    const float dx = cminf(t1x, t2x), dy = cminf(t1y, t2y), dz = cminf(t1z, t2z);
    const int axis = dx > dy ? (dx > dz ? 0 : 2) : (dy > dz ? 1 : 2);
    svdag_hit h;
    h.path[0] = px;
    h.path[1] = py;
    h.path[2] = pz;
    h.material = (uint8_t)material;
    h.pad[0] = h.pad[1] = h.pad[2] = 0;
    for (int a = 0; a < 3; ++a)
        h.normal[a] = h.dpdu[a] = h.dpdv[a] = 0.0f;
    float t;
    if (axis == 0) {
        h.normal[0] = r.dx < 0.0f ? +1.0f : -1.0f;
        h.dpdu[2] = 1.0f;
        h.dpdv[1] = 1.0f;
        t = dx;
    } else if (axis == 1) {
        h.normal[1] = r.dy < 0.0f ? +1.0f : -1.0f;
        h.dpdu[0] = 1.0f;
        h.dpdv[2] = 1.0f;
        t = dy;
    } else {
        h.normal[2] = r.dz < 0.0f ? +1.0f : -1.0f;
        h.dpdu[0] = 1.0f;
        h.dpdv[1] = 1.0f;
        t = dz;
    }
    h.position[0] = r.ox + t * r.dx;
    h.position[1] = r.oy + t * r.dy;
    h.position[2] = r.oz + t * r.dz;
    h.color = 0;
    out[(size_t)(p.height - 1 - y) * p.width + x] = h;
}

__global__ void k_sample(DevDag d, const uint32_t* xyz, uint32_t n, uint32_t* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        uint32_t h = d.ctl->root, result = SVDAG_NO_MATERIAL;
        if (h != kNone) {
            for (uint32_t level = 0; level < d.leafLevel; ++level) {
                const uint32_t s = d.levels - (level + 1);
                const uint32_t child = (((x >> s) & 1u) << 2) | (((y >> s) & 1u) << 1) | ((z >> s) & 1u);
                const uint32_t* node = item_ptr(d, h);
                const uint32_t mask = node[0] & 0xFFu;
                if (!(mask & (1u << child))) {
                    h = kNone;
                    break;
                }
                h = node[1 + __popc(mask & ((1u << child) - 1u))];
            }
            if (h != kNone) {
                const uint32_t v = ((x & 1u) ? 4u : 0u) | ((y & 1u) ? 2u : 0u) | ((z & 1u) ? 1u : 0u) | ((x & 2u) ? 32u : 0u) | ((y & 2u) ? 16u : 0u)
                    | ((z & 2u) ? 8u : 0u);
                const uint32_t* leaf = item_ptr(d, h);
                const unsigned long long m = (unsigned long long)leaf[0] | ((unsigned long long)leaf[1] << 32);
                if ((m >> v) & 1ull) {
                    const uint32_t bit = __popcll(m & ((1ull << v) - 1ull)) * 4u;
                    result = (leaf[2 + (bit >> 5)] >> (bit & 31u)) & 0xFu;
                }
            }
        }
        out[i] = result;
    }
}

} // namespace

svdag_status trace_frame(svdag_ctx* ctx, const svdag_trace_params* p, svdag_hit* out, const uint32_t* root, cudaStream_t s)
{
    const dim3 block(32, 8);
    const dim3 grid((p->width + block.x - 1) / block.x, (p->height + block.y - 1) / block.y);
    k_trace<<<grid, block, 0, s>>>(ctx->dag(), *p, out, root);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

} // namespace svdag

using namespace svdag;

extern "C" {

svdag_status svdag_trace_primary(svdag_ctx* ctx, const svdag_trace_params* p, svdag_hit* out, void* stream)
{
    if (!ctx || !p || !out || p->width == 0 || p->height == 0)
        return SVDAG_ERR_INVALID;
    const dim3 block(32, 8);
    const dim3 grid((p->width + block.x - 1) / block.x, (p->height + block.y - 1) / block.y);
    k_trace<<<grid, block, 0, as_stream(stream)>>>(ctx->dag(), *p, out, nullptr);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

svdag_status svdag_sample_voxels(svdag_ctx* ctx, const uint32_t* xyz, uint32_t count, uint32_t* out, void* stream)
{
    if (!ctx || (count && (!xyz || !out)))
        return SVDAG_ERR_INVALID;
    if (!count)
        return SVDAG_OK;
    k_sample<<<grid_for(ctx, count, 256), 256, 0, as_stream(stream)>>>(ctx->dag(), xyz, count, out);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

} // extern "C"
