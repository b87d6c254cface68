// svdag_trace.cu - primary-ray DAG traversal writing the per-pixel hit buffer, and voxel sampling.
//
// Reference: Tracer::trace_paths / intersect_ray / compute_intersection_mask / createSurfaceInteraction
// (tracer.cu:28-411), ray setup from DAGTracer::resolve_paths (dag_tracer.cu:112-134), voxel queries
// from getVoxelValues_kernel -> DAGUtils::get_value (dag_tracer.cu:361-372, dag_utils.h:146-182).
// Float and double arithmetic follow the reference expression by expression; with -fmad=false nothing
// is contracted, so hits equal the oracle's bit for bit. A child fetch is one load: handles are
// offsets of the items (16-byte units), so the traversal reads the header and the child handle without
// a slab-table decode.
#include <cuda_runtime.h>

#include <cmath>

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
    const RayF& r, float rayTmax = 3.402823466e+38f)
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
    tmax = fminf(tmax, rayTmax); // ray.tmax
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

// Whether the ray meets the box [b0..b2] x [b3..b5] at some t >= 0 (slab test; a NaN from a zero
// direction component on a slab boundary drops that slab's constraint, which only widens the test).
__device__ __forceinline__ bool ray_meets_box(const RayF& r, const float* b)
{
    const float t1x = (b[0] - r.ox) * r.ix, t2x = (b[3] - r.ox) * r.ix;
    const float t1y = (b[1] - r.oy) * r.iy, t2y = (b[4] - r.oy) * r.iy;
    const float t1z = (b[2] - r.oz) * r.iz, t2z = (b[5] - r.oz) * r.iz;
    const float tnear = fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fmaxf(fminf(t1z, t2z), 0.0f));
    const float tfar = fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fmaxf(t1z, t2z));
    return tnear <= tfar;
}

// Primary rays. With INCR the buffer holds the previous frame of the same camera and only pixels
// whose ray meets one of `boxes` (the changed regions since that frame, grown by a margin) are traced
// again. The traversal only ever inspects voxels within the intersection test's tolerance (1e-4) of
// the ray, and which ones it admits depends on the ray alone, so a pixel whose ray meets no changed
// region finds the same voxel as before: its record is already right. That holds while the inverse
// direction stays far from overflow: with an infinite component (a zero or denormal direction
// component) the intersection test computes 0 * inf = NaN on node planes through the origin and can
// admit voxels off the ray, and a component above 1e30 can overflow its products to infinity, so
// such pixels are always traced again.
template <bool INCR>
__global__ void __launch_bounds__(256) k_trace(DevDag d, svdag_trace_params p, svdag_hit* out, const uint32_t* rootPtr,
    const float* boxes, uint32_t nBoxes)
{
    // A block (32 x 8 threads) covers 32 x 8 pixels; each warp takes an 8 x 4 tile of them, whose
    // rays stay closer together through the traversal than a 32-pixel row's (fewer divergent steps).
    const uint32_t tw = (threadIdx.y * 32u + threadIdx.x) >> 5, tl = threadIdx.x & 31u;
    const uint32_t x = blockIdx.x * 32u + (tw & 3u) * 8u + (tl & 7u);
    const uint32_t y = blockIdx.y * 8u + (tw >> 2) * 4u + (tl >> 3);
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
    if constexpr (INCR) {
        bool touched = !(fabsf(r.ix) <= 1e30f && fabsf(r.iy) <= 1e30f && fabsf(r.iz) <= 1e30f);
        for (uint32_t b = 0; b < nBoxes && !touched; ++b)
            touched = ray_meets_box(r, boxes + 6 * b);
        if (!touched)
            return;
    }

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
        // Bit l of `live`: the stack entry of level l still has children to visit. Ascending to the
        // deepest such level below the current one is what the reference's pop loop does one level
        // at a time (entries in between have nothing left); here it is one bit scan.
        uint32_t live = 0;
        for (;;) {
            if (!cVisit) {
                const uint32_t cand = live & ((1u << level) - 1u);
                if (!cand) {
                    px = py = pz = 0;
                    break;
                }
                const uint32_t newLevel = 31u - (uint32_t)__clz(cand);
                cIndex = sIndex[newLevel][tix];
                const uint32_t m = sMasks[newLevel][tix];
                cChild = m & 0xFFu;
                cVisit = m >> 8;
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
            live = cVisit ? (live | (1u << level)) : (live & ~(1u << level));
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
            // The child's mask by level kind, then one intersection test for all lanes together (the
            // branches only fetch; the mask arithmetic runs converged).
            if (level < LL) {
                const uint32_t* node = item_ptr(d, cIndex);
                cIndex = node[1 + __popc(cChild & ((1u << nextChild) - 1u))];
                cChild = item_ptr(d, cIndex)[0] & 0xFFu;
            } else if (level == LL) {
                const uint32_t* node = item_ptr(d, cIndex);
                addr = node[1 + __popc(cChild & ((1u << nextChild) - 1u))];
                const uint32_t* lp = item_ptr(d, addr);
                leafLo = lp[0];
                leafHi = lp[1];
                cChild = first_child_mask(leafLo, leafHi);
            } else { // get_second_child_mask, base_dag.h:53-58
                cChild = (((nextChild & 4u) ? leafHi : leafLo) >> ((nextChild & 3u) * 8u)) & 0xFFu;
            }
            cVisit = cChild & intersection_mask(false, level, px, py, pz, levels, r);
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

// ---------------------------------------------------------------- shading (tracer.cu:413-730)

struct ShadeDev {
    uint32_t palette[SVDAG_NUM_MATERIALS];
    float sun[3];
    float bias, aoLength, sunBrightness, fog;
    uint32_t samples, flags;
    unsigned long long seed;
};

// intersect_ray_node_out_of_order, tracer.cu:275-352: whether any voxel lies on the ray within
// [0, tmax]; children are taken highest index first, whatever the ray's direction.
__device__ bool any_hit(const DevDag& d, uint32_t root, const RayF& r, float tmax, uint32_t (*sIndex)[256], uint32_t (*sMasks)[256],
    uint32_t tix)
{
    if (root == kNone)
        return false;
    const uint32_t levels = d.levels, LL = d.leafLevel;
    uint32_t level = 0, px = 0, py = 0, pz = 0, leafLo = 0, leafHi = 0;
    uint32_t cIndex = root;
    uint32_t cChild = item_ptr(d, root)[0] & 0xFFu;
    uint32_t cVisit = cChild & intersection_mask(true, 0, 0, 0, 0, levels, r, tmax);
    uint32_t live = 0; // as in k_trace: bit l set while stack level l has children left
    for (;;) {
        if (!cVisit) {
            const uint32_t cand = live & ((1u << level) - 1u);
            if (!cand)
                return false;
            const uint32_t newLevel = 31u - (uint32_t)__clz(cand);
            cIndex = sIndex[newLevel][tix];
            const uint32_t m = sMasks[newLevel][tix];
            cChild = m & 0xFFu;
            cVisit = m >> 8;
            const uint32_t up = level - newLevel;
            px >>= up;
            py >>= up;
            pz >>= up;
            level = newLevel;
        }
        const uint32_t nextChild = 31u - (uint32_t)__clz(cVisit);
        cVisit &= ~(1u << nextChild);
        px = (px << 1) | ((nextChild >> 2) & 1u);
        py = (py << 1) | ((nextChild >> 1) & 1u);
        pz = (pz << 1) | (nextChild & 1u);
        sIndex[level][tix] = cIndex;
        sMasks[level][tix] = cChild | (cVisit << 8);
        live = cVisit ? (live | (1u << level)) : (live & ~(1u << level));
        level++;
        if (level == levels)
            return true;
        if (level < LL) {
            const uint32_t* node = item_ptr(d, cIndex);
            cIndex = node[1 + __popc(cChild & ((1u << nextChild) - 1u))];
            cChild = item_ptr(d, cIndex)[0] & 0xFFu;
        } else if (level == LL) {
            const uint32_t* node = item_ptr(d, cIndex);
            const uint32_t* lp = item_ptr(d, node[1 + __popc(cChild & ((1u << nextChild) - 1u))]);
            leafLo = lp[0];
            leafHi = lp[1];
            cChild = first_child_mask(leafLo, leafHi);
        } else {
            cChild = (((nextChild & 4u) ? leafHi : leafLo) >> ((nextChild & 3u) * 8u)) & 0xFFu;
        }
        cVisit = cChild & intersection_mask(false, level, px, py, pz, levels, r, tmax);
    }
}

__device__ __forceinline__ RayF make_rayf(float ox, float oy, float oz, float dx, float dy, float dz) // Ray::create, tracer.cu:32-41
{
    RayF r;
    r.ox = ox;
    r.oy = oy;
    r.oz = oz;
    r.dx = dx;
    r.dy = dy;
    r.dz = dz;
    r.ix = 1.0f / dx;
    r.iy = 1.0f / dy;
    r.iz = 1.0f / dz;
    return r;
}

// Utils::PCG_RNG (utils.h:45-78): PCG-XSH-RR 32 with the stream as increment.
struct Pcg {
    unsigned long long state = 0x853c49e6748fea9bull, inc;
    __device__ explicit Pcg(unsigned long long stream)
        : inc(stream)
    {
        next();
        next();
    }
    __device__ uint32_t next()
    {
        const unsigned long long old = state;
        state = old * 6364136223846793005ull + (inc | 1ull);
        const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((0xFFFFFFFFu - rot + 1u) & 31u));
    }
    __device__ float next_float() { return float(next()) / 4294967296.0f; } // float(UINT32_MAX) is 2^32
};

// sin and cos of x in [0, 2 pi]: reduction by the nearest multiple of pi/2 (in double, exact for
// these arguments to well below float precision) and the Taylor polynomials of sin (degree 9) and
// cos (degree 8) on [-pi/4, pi/4]. The oracle evaluates the same operations in the same order, so
// AO sample directions agree bit for bit.
__device__ __forceinline__ void sincos_quadrant(float x, float& s, float& c)
{
    const float k = rintf(x * 0.63661975f);
    const float r = (float)((double)x - (double)k * 1.5707963267948966);
    const float r2 = r * r;
    const float sp = r + (r * r2) * (-0.16666667f + r2 * (0.008333334f + r2 * (-0.0001984127f + r2 * 2.7557319e-06f)));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (0.041666668f + r2 * (-0.0013888889f + r2 * 2.4801588e-05f)));
    switch ((int)k & 3) {
    case 0:
        s = sp;
        c = cp;
        break;
    case 1:
        s = cp;
        c = -sp;
        break;
    case 2:
        s = -sp;
        c = -cp;
        break;
    default:
        s = -cp;
        c = sp;
        break;
    }
}

__device__ __forceinline__ float srgb_to_linear(float v) // ColorUtils::accurateSRGBToLinear, color_utils.h:233-242
{
    const float lo = v / 12.92f;
    const float hi = powf((v + 0.055f) / 1.055f, 2.4f);
    return (v <= 0.04045f) ? lo : hi;
}
__device__ __forceinline__ float linear_to_srgb(float v) // ColorUtils::accurateLinearToSRGB, :243-252
{
    const float lo = v * 12.92f;
    const float hi = (powf(fabsf(v), 1.0f / 2.4f) * 1.055f) - 0.055f;
    return (v <= 0.0031308f) ? lo : hi;
}
__device__ __forceinline__ uint32_t to_rgb888(float r, float g, float b) // ColorUtils::float3_to_rgb888, :31-37
{
    r = fmaxf(0.f, fminf(r, 1.f));
    g = fmaxf(0.f, fminf(g, 1.f));
    b = fmaxf(0.f, fminf(b, 1.f));
    return (uint32_t(r * 255.0f) << 0) | (uint32_t(g * 255.0f) << 8) | (uint32_t(b * 255.0f) << 16) | 0xff000000u;
}

// One pixel: diffuse colour (trace_colors), sun shadow (trace_shadows), ambient occlusion
// (trace_ambient_occlusion) and lighting (trace_lighting), each step in the reference's order.
__global__ void __launch_bounds__(256) k_shade(DevDag d, svdag_trace_params tp, ShadeDev sp, svdag_hit* hits, uint32_t* rgba, float* sunOut,
    float* aoOut)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    __shared__ uint32_t sIndex[kMaxLevels][256];
    __shared__ uint32_t sMasks[kMaxLevels][256];
    if (x >= tp.width || y >= tp.height)
        return;
    const uint32_t tix = threadIdx.y * blockDim.x + threadIdx.x;
    const size_t i = (size_t)y * tp.width + x;
    svdag_hit& si = hits[i];
    const bool hit = si.path[0] != 0 || si.path[1] != 0 || si.path[2] != 0;
    const uint32_t root = d.ctl->root;
    // computeColorAtSurface (tracer.cu:413-445): black for a miss, a checker for an unknown material
    uint32_t diffuse;
    if (!hit) {
        diffuse = to_rgb888(0.f, 0.f, 0.f);
    } else if (si.material < SVDAG_NUM_MATERIALS) {
        diffuse = sp.palette[si.material] | 0xff000000u;
    } else {
        const float b = float((si.path[0] ^ si.path[1] ^ si.path[2]) & 1u);
        diffuse = to_rgb888(1.f, b, 1.f - b);
    }
    si.color = diffuse;
    const float px = si.position[0], py = si.position[1], pz = si.position[2];
    const float nx = si.normal[0], ny = si.normal[1], nz = si.normal[2];
    float sun = 0.f, ao = 0.f;
    if (hit && (sp.flags & SVDAG_SHADE_SHADOWS)) {
        const RayF r = make_rayf(px + sp.bias * sp.sun[0], py + sp.bias * sp.sun[1], pz + sp.bias * sp.sun[2], sp.sun[0], sp.sun[1], sp.sun[2]);
        const bool occluded = any_hit(d, root, r, 3.402823466e+38f, sIndex, sMasks, tix);
        const float ndotl = fmaxf((nx * r.dx + ny * r.dy) + nz * r.dz, 0.0f);
        sun = occluded ? 0.0f : ndotl;
    }
    if (hit && (sp.flags & SVDAG_SHADE_AO) && sp.samples) {
        const unsigned long long seed = (unsigned long long)(y * tp.width + x) * (sp.seed > 1ull ? sp.seed : 1ull);
        Pcg rng(seed);
        uint32_t samples = 0, open = 0;
        const float ox = px + nx * sp.bias, oy = py + ny * sp.bias, oz = pz + nz * sp.bias;
        for (uint32_t k = 0; k < sp.samples; ++k) {
            const float ux = rng.next_float();
            const float uy = rng.next_float();
            // cosineSampleHemisphere (tracer.cu:643-655)
            const float rr = sqrtf(ux);
            const float theta = 6.2831855f * uy;
            float sn, cs;
            sincos_quadrant(theta, sn, cs);
            const float lx = rr * cs, ly = rr * sn, lz = sqrtf(fmaxf(0.0f, 1 - ux));
            // SurfaceInteraction::transformDirectionToWorld (tracer.h:106-109)
            const float wx = (lx * si.dpdu[0] + ly * si.dpdv[0]) + lz * nx;
            const float wy = (lx * si.dpdu[1] + ly * si.dpdv[1]) + lz * ny;
            const float wz = (lx * si.dpdu[2] + ly * si.dpdv[2]) + lz * nz;
            const RayF r = make_rayf(ox, oy, oz, wx, wy, wz);
            if (!any_hit(d, root, r, sp.aoLength, sIndex, sMasks, tix))
                open += 1;
            samples += 1;
        }
        ao = (float)open / (float)samples;
    }
    if (sunOut)
        sunOut[i] = sun;
    if (aoOut)
        aoOut[i] = ao;
    // trace_lighting (tracer.cu:701-730)
    const float skyR = 187.f / 255.f, skyG = 242.f / 255.f, skyB = 250.f / 255.f;
    float sr, sg, sb;
    if (!hit) {
        sr = skyR;
        sg = skyG;
        sb = skyB;
    } else {
        const float kr = srgb_to_linear(float((diffuse >> 0) & 0xFFu) / 255.0f);
        const float kg = srgb_to_linear(float((diffuse >> 8) & 0xFFu) / 255.0f);
        const float kb = srgb_to_linear(float((diffuse >> 16) & 0xFFu) / 255.0f);
        const float occl = (sp.flags & SVDAG_SHADE_AO) && sp.samples ? ao : 1.0f;
        const float vis = (sp.flags & SVDAG_SHADE_SHADOWS) ? sun : 1.0f;
        const float a = occl * 0.5f;
        sr = ((a * skyR) + ((vis * 0.95f) * sp.sunBrightness)) * kr;
        sg = ((a * skyG) + ((vis * 0.94f) * sp.sunBrightness)) * kg;
        sb = ((a * skyB) + ((vis * 0.47f) * sp.sunBrightness)) * kb;
        if (sp.fog > 0.0f) { // applyFog, tracer.cu:685-699, with the camera ray of this pixel
            const double vx = ((tp.ray_min[0] + (double)x * tp.ray_ddx[0]) + (double)y * tp.ray_ddy[0]) - tp.camera[0];
            const double vy = ((tp.ray_min[1] + (double)x * tp.ray_ddx[1]) + (double)y * tp.ray_ddy[1]) - tp.camera[1];
            const double vz = ((tp.ray_min[2] + (double)x * tp.ray_ddx[2]) + (double)y * tp.ray_ddy[2]) - tp.camera[2];
            const double inv = 1.0 / sqrt(vx * vx + vy * vy + vz * vz);
            const float dx = (float)(vx * inv), dy = (float)(vy * inv), dz = (float)(vz * inv);
            const float ex = (float)tp.camera[0] - px, ey = (float)tp.camera[1] - py, ez = (float)tp.camera[2] - pz;
            const float density = sp.fog * 0.00001f;
            const float amount = 1.0f - expf(-sqrtf((ex * ex + ey * ey) + ez * ez) * density);
            const float sunAmount = 1.01f * fmaxf((dx * sp.sun[0] + dy * sp.sun[1]) + dz * sp.sun[2], 0.0f);
            const float t = powf(sunAmount, 30.0f);
            const float fr = skyR + t * (1.0f - skyR), fg = skyG + t * (1.0f - skyG), fb = skyB + t * (1.0f - skyB);
            const float f = fmaxf(0.0f, fminf(amount, 1.0f));
            sr = sr + f * (fr - sr);
            sg = sg + f * (fg - sg);
            sb = sb + f * (fb - sb);
        }
    }
    rgba[i] = to_rgb888(linear_to_srgb(sr), linear_to_srgb(sg), linear_to_srgb(sb));
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
    k_trace<false><<<grid, block, 0, s>>>(ctx->dag(), *p, out, root, nullptr, 0);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

svdag_status trace_frame_incremental(svdag_ctx* ctx, const svdag_trace_params* p, svdag_hit* out, const uint32_t* root, const float* boxes,
    uint32_t nBoxes, cudaStream_t s)
{
    const dim3 block(32, 8);
    const dim3 grid((p->width + block.x - 1) / block.x, (p->height + block.y - 1) / block.y);
    k_trace<true><<<grid, block, 0, s>>>(ctx->dag(), *p, out, root, boxes, nBoxes);
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
    k_trace<false><<<grid, block, 0, as_stream(stream)>>>(ctx->dag(), *p, out, nullptr, nullptr, 0);
    SVDAG_CUDA(cudaGetLastError());
    return SVDAG_OK;
}

svdag_status svdag_shade(svdag_ctx* ctx, const svdag_trace_params* tp, const svdag_shade_params* sp, svdag_hit* hits, uint32_t* rgba,
    float* sun, float* ao, void* stream)
{
    if (!ctx || !tp || !sp || !hits || !rgba || tp->width == 0 || tp->height == 0 || (sp->flags & ~(SVDAG_SHADE_SHADOWS | SVDAG_SHADE_AO)))
        return SVDAG_ERR_INVALID;
    if (!(sp->ao_ray_length >= 0.0f) || !std::isfinite(sp->shadow_bias) || !std::isfinite(sp->sun_brightness) || !(sp->fog_density >= 0.0f))
        return SVDAG_ERR_INVALID;
    ShadeDev d {};
    for (uint32_t m = 0; m < SVDAG_NUM_MATERIALS; ++m)
        d.palette[m] = sp->material_srgb8[m] & 0x00FFFFFFu;
    for (int a = 0; a < 3; ++a)
        d.sun[a] = sp->sun_direction[a];
    d.bias = sp->shadow_bias;
    d.aoLength = sp->ao_ray_length;
    d.sunBrightness = sp->sun_brightness;
    d.fog = sp->fog_density;
    d.samples = sp->ao_samples;
    d.flags = sp->flags;
    d.seed = sp->random_seed;
    const dim3 block(32, 8);
    const dim3 grid((tp->width + block.x - 1) / block.x, (tp->height + block.y - 1) / block.y);
    k_shade<<<grid, block, 0, as_stream(stream)>>>(ctx->dag(), *tp, d, hits, rgba, sun, ao);
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
