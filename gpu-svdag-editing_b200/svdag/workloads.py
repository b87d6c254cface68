"""Synthetic workloads: the scenes, edit sets and request streams the benchmark and the tests run.

The reference measures on scene files and recorded edit replays that are not available here; these
seeded procedural stand-ins have the stated depths, sizes and edit mixes. Edits are placed on the
terrain surface with the library's own height function (svdag_scene_height, host code) unless the
caller passes another `height(levels, x, z, terrain)` with the same values (the CPU baseline passes
the oracle's, so that it runs without the CUDA library).
"""
import math

import numpy as np

from . import (TOOL_BOX_ADD, TOOL_BOX_PAINT_NOISE, TOOL_BOX_REMOVE, TOOL_COPY, TOOL_SPHERE_ADD, TOOL_SPHERE_PAINT,
               TOOL_SPHERE_REMOVE, Edit, scene_height)

# Depth-10 terrain, 5 fBm octaves, surface at 40-70 % of the height, 8 height-band materials.
C0_LEVELS = 10
C0_TERRAIN = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70)
C0_EDIT_SEED = 2024

# Depth-17 terrain, 8 octaves, 4096 boxes (side 16-512) and spheres (radius 8-256) on the surface.
C2_LEVELS = 17
C2_TERRAIN = dict(seed=0, octaves=8, num_materials=8, min_height_pct=40, max_height_pct=70, num_structures=4096,
                  structure_seed=11)


def make_edit(tool, material=0, center=(0.0, 0.0, 0.0), radius=1.0, src=None, dst=None, noise_seed=0,
              noise_cell_log2=0) -> Edit:
    e = Edit(tool=tool, material=material, radius=float(radius), noise_seed=noise_seed,
             noise_cell_log2=noise_cell_log2)
    e.center[:] = [float(v) for v in center]
    if src is not None:
        e.src[:] = [float(v) for v in src]
    if dst is not None:
        e.dst[:] = [float(v) for v in dst]
    return e


def c0_edits(n=64, seed=C0_EDIT_SEED, levels=C0_LEVELS, terrain=C0_TERRAIN):
    """Sphere edits: centre within +-32 voxels of the surface, integer radius U{4..64}, 50 % add /
    50 % remove, add material U[0, 8). Returns (tool, material, centre, radius) tuples."""
    rng = np.random.default_rng(seed)
    g = 1 << levels
    out = []
    for _ in range(n):
        x, z = (int(v) for v in rng.integers(0, g, 2))
        h = scene_height(levels, x, z, **terrain)
        c = (float(x + rng.integers(-32, 33)), float(h + rng.integers(-32, 33)), float(z + rng.integers(-32, 33)))
        r = float(rng.integers(4, 65))
        add = bool(rng.integers(0, 2))
        out.append((TOOL_SPHERE_ADD if add else TOOL_SPHERE_REMOVE, int(rng.integers(0, 8)), c, r))
    return out


def surface_point(levels, x, z, terrain):
    return (float(x), float(scene_height(levels, x, z, **terrain)), float(z))


def c2_edits(levels=C2_LEVELS, terrain=C2_TERRAIN):
    """The at-scale sequence: a sphere carve of radius 2048, a 512^3 box copy-paste moved by
    (1024, 0, 0), a 1024^3 box paint with materials from 3D value noise. Sizes scale with the grid
    below depth 17 (so the same sequence runs on smaller test scenes)."""
    g = 1 << levels
    k = g / 131072.0
    carve = make_edit(TOOL_SPHERE_REMOVE, 0, surface_point(levels, int(0.30 * g), int(0.30 * g), terrain), 2048 * k)
    # The copy keeps destination voxels where the source is empty, so a source box on higher ground
    # than its destination shows the copy best: take the largest surface drop over a 1024-step
    # move among candidate columns of one band of the grid.
    step = int(1024 * k)
    best = None
    for i in range(64):
        x = int((0.50 + 0.2 * i / 64) * g)
        z = int(0.45 * g)
        drop = scene_height(levels, x, z, **terrain) - scene_height(levels, x + step, z, **terrain)
        if best is None or drop > best[0]:
            best = (drop, x, z)
    src = surface_point(levels, best[1], best[2], terrain)
    dst = (src[0] + step, src[1], src[2])
    copy = make_edit(TOOL_COPY, 0, src, 256 * k, src=src, dst=dst)
    paint = make_edit(TOOL_BOX_PAINT_NOISE, 0, surface_point(levels, int(0.45 * g), int(0.70 * g), terrain), 512 * k,
                      noise_seed=17, noise_cell_log2=max(6 - (C2_LEVELS - levels), 0))
    return [carve, copy, paint]


def _library_height(levels, x, z, terrain):
    return scene_height(levels, x, z, **terrain)


def _log_uniform(rng, lo, hi):
    return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))


def c3_edits(n=256, seed=3, levels=C2_LEVELS, terrain=C2_TERRAIN, rmax=4096.0):
    """Edits of uneven footprint: sphere/box 50/50, radius or half-side log-uniform in [4, rmax],
    40 % add / 40 % remove / 20 % paint, centres within +-32 voxels of the surface, materials
    U[0, 16). The reference's paint tool is a sphere (MyGpuSpherePaintEditor), so paints are spheres."""
    rng = np.random.default_rng(seed)
    g = 1 << levels
    out = []
    for _ in range(n):
        x, z = (int(v) for v in rng.integers(0, g, 2))
        h = scene_height(levels, x, z, **terrain)
        c = (float(x + rng.integers(-32, 33)), float(h + rng.integers(-32, 33)), float(z + rng.integers(-32, 33)))
        r = float(int(_log_uniform(rng, 4.0, rmax)))
        sphere = bool(rng.integers(0, 2))
        u = rng.uniform()
        mat = int(rng.integers(0, 16))
        if u < 0.4:
            tool = TOOL_SPHERE_ADD if sphere else TOOL_BOX_ADD
        elif u < 0.8:
            tool = TOOL_SPHERE_REMOVE if sphere else TOOL_BOX_REMOVE
        else:
            tool = TOOL_SPHERE_PAINT
        out.append(make_edit(tool, mat, c, r))
    return out


def c4_stream(rate, duration_s, seed=4, levels=C2_LEVELS, terrain=C2_TERRAIN, rmax=2048.0, frame_hz=60.0,
              copy_offset=1024, height=None):
    """Served request stream: edit arrivals Poisson at `rate` per second, mix add / remove / paint /
    copy 35/35/20/10, radius log-uniform in [2, rmax], centres within +-32 voxels of the surface,
    copies moved by up to +-copy_offset in x and z; frame requests every 1/frame_hz s. Returns
    (edit_times, edits, frame_times), times in seconds."""
    height = height or _library_height
    rng = np.random.default_rng(seed)
    g = 1 << levels
    times, edits = [], []
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration_s:
            break
        x, z = (int(v) for v in rng.integers(0, g, 2))
        h = height(levels, x, z, terrain)
        c = (float(x + rng.integers(-32, 33)), float(h + rng.integers(-32, 33)), float(z + rng.integers(-32, 33)))
        r = float(max(int(_log_uniform(rng, 2.0, rmax)), 2))
        u = rng.uniform()
        mat = int(rng.integers(0, 16))
        if u < 0.35:
            e = make_edit(TOOL_SPHERE_ADD, mat, c, r)
        elif u < 0.70:
            e = make_edit(TOOL_SPHERE_REMOVE, mat, c, r)
        elif u < 0.90:
            e = make_edit(TOOL_SPHERE_PAINT, mat, c, r)
        else:
            off = rng.integers(-copy_offset, copy_offset + 1, 2)
            dst = (c[0] + float(off[0]), c[1], c[2] + float(off[1]))
            e = make_edit(TOOL_COPY, 0, c, min(r, 256.0), src=c, dst=dst)
        times.append(t)
        edits.append(e)
    frames = list(np.arange(0.0, duration_s, 1.0 / frame_hz))
    return times, edits, frames
