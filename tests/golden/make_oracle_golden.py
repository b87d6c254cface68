"""Writes tests/golden/oracle_c0_golden.json: the oracle's results on a fixed edit sequence, so that a
later change to the oracle that alters them is caught (tests/test_golden.py).

The reference ships no golden vectors for the MyGpuDag path (its tests are the known-answer checks
restated in tests/test_oracle_kat.py). This fixture pins the oracle against itself across changes: the
depth-10 C0 terrain, then 24 sphere edits of the C0 stream and two edits of every other tool, each
followed by the DAG's canonical form (distinct items and content digest per level, Merkle root,
voxel count) and the per-edit counters, and at the end one 128 x 128 primary-ray frame (digest of
its hit records). The edits themselves are stored in the fixture.

usage: python tests/golden/make_oracle_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402

LEVELS = 10
TERRAIN = dict(seed=0, octaves=5, num_materials=8, min_height_pct=40, max_height_pct=70)
CAMERA = ((512.0, 900.0, 512.0), (512.0, 512.0, 512.0), 60.0, 128, 128)
OUT = os.path.join(HERE, "oracle_c0_golden.json")


def edit_list(seed=2024):
    """24 C0-stream spheres (centre within +-32 voxels of the surface, radius U{4..64}, add/remove),
    then two edits of each other tool (box add/remove, sphere paint, copy, box noise paint, move,
    erosion) at surface points."""
    L = oracle.lib()
    tp = oracle.TerrainParams(**TERRAIN)
    g = 1 << LEVELS
    rng = np.random.default_rng(seed)

    def surface(x, z):
        return float(L.oracle_terrain_height(tp, LEVELS, x, z))

    out = []
    for _ in range(24):
        x, z = (int(v) for v in rng.integers(0, g, 2))
        c = [float(x + rng.integers(-32, 33)), surface(x, z) + float(rng.integers(-32, 33)), float(z + rng.integers(-32, 33))]
        r = float(rng.integers(4, 65))
        out.append(dict(tool=int(rng.integers(0, 2)), material=int(rng.integers(0, 8)), center=c, radius=r))
    for tool in (2, 3, 4, 5, 6, 7, 8):
        for _ in range(2):
            x, z = (int(v) for v in rng.integers(64, g - 64, 2))
            c = [float(x), surface(x, z), float(z)]
            e = dict(tool=tool, material=int(rng.integers(0, 8)), center=c, radius=float(rng.integers(6, 40)))
            if tool in (5, 7):
                e["src"] = list(c)
                dx, dz = (int(v) for v in rng.integers(-60, 61, 2))
                e["dst"] = [c[0] + dx, surface(min(max(x + dx, 0), g - 1), min(max(z + dz, 0), g - 1)), c[2] + dz]
            if tool == 6:
                e["noise_seed"], e["noise_cell_log2"] = int(rng.integers(1, 1000)), int(rng.integers(0, 4))
            if tool == 8:  # a voxel of a flat surface has 17 filled neighbours: thresholds above erode it
                e["noise_seed"] = int(rng.integers(17, 23))
            out.append(e)
    return out


def to_edit(d):
    e = oracle.Edit(tool=d["tool"], material=d["material"], radius=d["radius"], noise_seed=d.get("noise_seed", 0),
                    noise_cell_log2=d.get("noise_cell_log2", 0))
    e.center[:] = d["center"]
    e.src[:] = d.get("src", [0.0, 0.0, 0.0])
    e.dst[:] = d.get("dst", [0.0, 0.0, 0.0])
    return e


def run(edits):
    """The oracle's results for the edit list, in the fixture's form."""
    dag = oracle.OracleDag(LEVELS)
    dag.build_terrain(oracle.TerrainParams(**TERRAIN))
    result = {"scene": dag.canon(), "edits": []}
    for d in edits:
        st = dag.edit(to_edit(d))
        result["edits"].append({"status": int(st.status), "svo_nodes": [int(st.svo_nodes[i]) for i in range(LEVELS - 1)],
                                "unique_items": int(st.unique_items), "new_items": int(st.new_items),
                                "edited_voxels": int(st.edited_voxels), "canon": dag.canon()})
    hits = dag.trace(oracle.camera_params(*CAMERA))
    result["frame_sha256"] = hashlib.sha256(np.ascontiguousarray(hits).tobytes()).hexdigest()
    return result


def main():
    oracle.build()
    edits = edit_list()
    golden = {"levels": LEVELS, "terrain": TERRAIN, "camera": CAMERA, "edit_list": edits, **run(edits)}
    with open(OUT, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
        f.write("\n")
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
