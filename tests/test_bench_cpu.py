"""The benchmark's CPU legs: the reference arm and the CPU baseline run the oracle on the host and
never map the CUDA library, and the served stream is the same whichever height function places it."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpu_baseline_maps_no_cuda_library():
    code = (
        "import argparse, bench\n"
        "args = argparse.Namespace(rate=400.0, steps=1, window=0.5)\n"
        "r = bench.cpu_sample(args, 10, budget_s=0.5, min_edits=6)\n"
        "t, hits = bench.cpu_trace_c0(reps=1)\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert r['edits'] >= 6 and r['cpu_baseline']['cores'] >= 1, r\n"
        "assert t['rays_s'] > 0 and len(hits) == 256 * 256\n"
        "assert 'libsvdag' not in maps and 'libcudart' not in maps\n"
        "print('ok')\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]
    assert out.stdout.strip().endswith("ok")


def test_stream_heights_from_the_oracle_equal_the_library(svdag_lib, oracle_mod):
    """c4_stream places edits with a height function; the oracle's terrain height (used by the CPU
    legs) and the library's host svdag_scene_height give the same stream."""
    import svdag.workloads as w

    terrain = dict(w.C2_TERRAIN, num_structures=64)
    params = oracle_mod.TerrainParams(**terrain)
    L = oracle_mod.lib()
    h = lambda lv, x, z, t: L.oracle_terrain_height(params, lv, x, z)
    for levels in (10, 13, 17):
        a = w.c4_stream(500.0, 0.4, seed=9, levels=levels, terrain=terrain)
        b = w.c4_stream(500.0, 0.4, seed=9, levels=levels, terrain=terrain, height=h)
        assert a[0] == b[0] and len(a[1]) == len(b[1]) > 100
        for x, y in zip(a[1], b[1]):
            assert bytes(x) == bytes(y)
