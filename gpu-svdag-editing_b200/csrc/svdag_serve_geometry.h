// svdag_serve_geometry.h - host-side geometry of the serving loop: an edit's admission estimate (the
// item-region bytes it can add), the boxes holding every voxel it can change, and the hit-buffer
// rectangle whose rays can meet such a box. Plain C++ (no CUDA), so the tests compile the same
// functions for the host.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "../../include/svdag.h"

namespace svdag {
namespace serve {

// Upper estimate of the item-region bytes an edit can add: its intermediate SVO bounds the new items.
// Leaves: the footprint's bounding volume in 4^3 bricks, or for spheres and boxes whose volume is
// large, a shell of three bricks' thickness around the surface (interior nodes are filled or emptied
// whole). Nodes above the leaves add at most a seventh; each item takes at most 50 bytes with its
// share of the slab header.
inline unsigned long long edit_reserve_bytes(const svdag_edit& e, uint32_t levels)
{
    const double r = std::max(1.0, (double)e.radius);
    const double side = 2.0 * r / 4.0 + 2.0; // bricks per axis
    const double volume = side * side * side;
    double leaves = volume;
    switch (e.tool) {
    case SVDAG_TOOL_SPHERE_ADD:
    case SVDAG_TOOL_SPHERE_REMOVE:
    case SVDAG_TOOL_SPHERE_PAINT:
        leaves = std::min(volume, 3.0 * 4.0 * M_PI * (r / 4.0 + 1.0) * (r / 4.0 + 1.0));
        break;
    case SVDAG_TOOL_BOX_ADD:
    case SVDAG_TOOL_BOX_REMOVE:
        leaves = std::min(volume, 3.0 * 6.0 * side * side);
        break;
    case SVDAG_TOOL_MOVE:
        leaves = 2.0 * volume;
        break;
    default:
        break;
    }
    const double items = leaves * 8.0 / 7.0 + 8.0 * levels;
    return (unsigned long long)(items * 50.0); // a 48-byte slot (10 words at a 16-byte stride) and 1/24 of a 32-byte header
}

// Hit-buffer rows [row0, row1] and columns [col0, col1] that rays meeting `box` can come from. Pixel (x, y) looks along
// ray_min + x * ddx + y * ddy - camera, so a point P is seen at the (x, y) solving
// P - camera = s * (ray_min - camera) + (s x) * ddx + (s y) * ddy; the rays meeting a box in front of
// the camera pass inside the projection of its corners. False when a corner is not in front.
inline bool box_rows(const svdag_trace_params& p, const float* box, int64_t& row0, int64_t& row1, int64_t& col0, int64_t& col1)
{
    const double a[3] = { p.ray_min[0] - p.camera[0], p.ray_min[1] - p.camera[1], p.ray_min[2] - p.camera[2] };
    const double* u = p.ray_ddx;
    const double* v = p.ray_ddy;
    auto det = [](const double* c0, const double* c1, const double* c2) {
        return c0[0] * (c1[1] * c2[2] - c1[2] * c2[1]) - c1[0] * (c0[1] * c2[2] - c0[2] * c2[1]) + c2[0] * (c0[1] * c1[2] - c0[2] * c1[1]);
    };
    const double D = det(a, u, v);
    if (!(std::fabs(D) > 0.0))
        return false;
    double ymin = 1e300, ymax = -1e300, xmin = 1e300, xmax = -1e300;
    for (int k = 0; k < 8; ++k) {
        const double q[3] = { (k & 1 ? box[3] : box[0]) - p.camera[0], (k & 2 ? box[4] : box[1]) - p.camera[1],
            (k & 4 ? box[5] : box[2]) - p.camera[2] };
        const double s = det(q, u, v) / D; // Cramer's rule for (s, s x, s y)
        if (!(s > 1e-9))
            return false;
        const double y = (det(a, u, q) / D) / s;
        const double x = (det(a, q, v) / D) / s;
        ymin = std::min(ymin, y);
        ymax = std::max(ymax, y);
        xmin = std::min(xmin, x);
        xmax = std::max(xmax, x);
    }
    col0 = std::max<int64_t>((int64_t)std::floor(std::max(xmin, -4.0)) - 2, 0);
    col1 = std::min<int64_t>((int64_t)std::ceil(std::min(xmax, (double)p.width + 4.0)) + 2, (int64_t)p.width - 1);
    const int64_t y0 = (int64_t)std::floor(std::max(ymin, -4.0)) - 2, y1 = (int64_t)std::ceil(std::min(ymax, (double)p.height + 4.0)) + 2;
    row0 = (int64_t)p.height - 1 - y1;
    row1 = (int64_t)p.height - 1 - y0;
    row0 = std::max<int64_t>(row0, 0);
    row1 = std::min<int64_t>(row1, (int64_t)p.height - 1);
    return true;
}

// Boxes (min xyz, max xyz) holding every voxel an edit can change, grown by two voxels (the tracer
// admits voxels within 1e-4 of a ray; the margin also covers float rounding of the box test).
// Returns how many it wrote (a move changes its source and its destination).
inline uint32_t edit_boxes(const svdag_edit& e, float* out)
{
    auto put = [&](float* b, float cx, float cy, float cz, float r) {
        const float lo = r + 2.0f, hi = r + 3.0f; // the sphere centre is offset by +0.5, a box of radius 0 is one voxel
        b[0] = cx - lo;
        b[1] = cy - lo;
        b[2] = cz - lo;
        b[3] = cx + hi;
        b[4] = cy + hi;
        b[5] = cz + hi;
    };
    const float r = std::max(e.radius, 0.1f);
    const float dx = e.dst[0] + (e.center[0] - e.src[0]), dy = e.dst[1] + (e.center[1] - e.src[1]), dz = e.dst[2] + (e.center[2] - e.src[2]);
    switch (e.tool) {
    case SVDAG_TOOL_COPY:
        put(out, dx, dy, dz, r);
        return 1;
    case SVDAG_TOOL_MOVE:
        put(out, e.center[0], e.center[1], e.center[2], r);
        put(out + 6, dx, dy, dz, r);
        return 2;
    default:
        put(out, e.center[0], e.center[1], e.center[2], r);
        return 1;
    }
}

} // namespace serve
} // namespace svdag
