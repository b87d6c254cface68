"""Post-hit shading on the GPU against the oracle: diffuse colours, sun visibility (shadow rays) and
ambient occlusion (PCG-sampled cosine hemisphere rays) must match exactly; the final sRGB8 pixels go
through powf/expf, whose last bits may differ between CUDA and the host C library, so each channel
may differ by 1 and at most 0.5 % of the pixels may differ at all."""
import numpy as np
import pytest

from gpu_util import TERRAIN

pytestmark = pytest.mark.gpu

SCENE = dict(TERRAIN, num_structures=24, structure_seed=5)


def oracle_params(oracle_mod, p):
    po = oracle_mod.TraceParams()
    for f in ("camera", "ray_min", "ray_ddx", "ray_ddy"):
        getattr(po, f)[:] = list(getattr(p, f))
    po.width, po.height = p.width, p.height
    return po


def to_oracle_shade(oracle_mod, s):
    o = oracle_mod.ShadeParams()
    C = __import__("ctypes")
    C.memmove(C.addressof(o), C.addressof(s), C.sizeof(o))
    return o


@pytest.mark.parametrize("fog,samples", [(0.0, 8), (4000.0, 3)])
def test_shading_matches_oracle(svdag_lib, oracle_mod, fog, samples):
    import torch

    levels = 10
    g = svdag_lib.MyGPUHashDAG(levels, pool_bytes=1 << 30)
    g.build_terrain(**SCENE)
    o = oracle_mod.OracleDag(levels)
    o.build_terrain(oracle_mod.TerrainParams(**SCENE))
    p = svdag_lib.get_trace_params((-150.0, 900.0, -120.0), (600.0, 520.0, 560.0), 224, 160)
    tracer = svdag_lib.DAGTracer(p.width, p.height)
    tracer.resolve_paths(p, g)
    hits_in = tracer.hits_numpy().copy()
    shade = svdag_lib.shade_params(levels, shadows=True, ao_samples=samples, ao_ray_length=24.0, fog_density=fog,
                                   sun_brightness=1.0, seed=7)
    rgba, sun, ao = tracer.resolve_lighting(p, g, shade, want_surfaces=True)
    torch.cuda.synchronize()
    g.sync()
    rgba = rgba.cpu().numpy().view(np.uint32)
    sun, ao = sun.cpu().numpy(), ao.cpu().numpy()
    hits = tracer.hits_numpy()
    oh, orgba, osun, oao = o.shade(oracle_params(oracle_mod, p), to_oracle_shade(oracle_mod, shade), hits_in)
    hit = np.any(hits_in["path"] != 0, axis=1)
    assert 0.3 < hit.mean() < 0.99
    assert np.array_equal(hits["color"], oh["color"])
    assert np.array_equal(sun, osun) and np.array_equal(ao, oao)
    assert 0.05 < (sun[hit] == 0).mean() < 0.95  # some pixels in shadow, some lit
    assert (ao[hit] < 1).mean() > 0.05
    a = rgba.view(np.uint8).reshape(-1, 4).astype(int)
    b = orgba.view(np.uint8).reshape(-1, 4).astype(int)
    assert np.abs(a - b).max() <= 1
    assert (a != b).any(axis=1).mean() <= 0.005
    assert (a[:, 3] == 255).all()
    g.free()
