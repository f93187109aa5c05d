"""Scenes uploaded as scene SoA v4 blobs (bf200_scene_create_from_soa) render exactly like the same
scenes given as descriptors: closest hits and per-path radiance bit for bit, for the Cornell box
with spheres, for a many-instance (TLAS) scene and for the layered Cornell box (closure mixtures,
every closure kind, punctual lights in the blob's punctual columns)."""
import numpy as np
import pytest

from bf200 import abi, runtime, scenes, soa

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["cornell", "instances", "layered"])
def test_soa_blob_scene_equals_descriptor_scene(kind):
    if kind == "cornell":
        builder = scenes.cornell_box(scenes.SceneBuilder(), with_spheres=True)
        centre, spread = np.array([0.0, 0.0, 1.0]), 0.6
    elif kind == "layered":
        builder = scenes.cornell_layered(scenes.SceneBuilder())
        centre, spread = np.array([0.0, 0.0, 1.0]), 0.6
    else:
        builder = scenes.bvh_stress(scenes.SceneBuilder(environment=(0.5,) * 4), subdivisions=2)
        centre, spread = np.zeros(3), 8.0
    blob = soa.write(builder)
    rng = np.random.default_rng(4)
    n = 4096
    rays = (abi.Ray * n)()
    inputs = (abi.PathInput * n)()
    for k in range(n):
        o = centre + rng.normal(0.0, spread, 3)
        d = rng.normal(0.0, 1.0, 3)
        d /= np.linalg.norm(d)
        for a in range(3):
            rays[k].origin[a], rays[k].direction[a] = float(o[a]), float(d[a])
        rays[k].t_min, rays[k].t_max, rays[k].time, rays[k].mask = 0.0, float("inf"), 0.5, 0xFFFFFFFF
        inputs[k].primary_ray = rays[k]
        inputs[k].sample.pixel_x, inputs[k].sample.pixel_y = k % 64, k // 64
        inputs[k].sample.sample_index, inputs[k].sample.seed = k, 3
    options = abi.default_options(mis="power", max_depth=8)
    with runtime.Context(0, path_capacity=1 << 14) as ctx:
        from_desc = ctx.create_scene(builder)
        from_blob = ctx.create_scene_from_soa(blob, builder)
        hits = [ctx.closest_hits(s, rays) for s in (from_desc, from_blob)]
        paths = [ctx.trace_paths(s, inputs, options)[0] for s in (from_desc, from_blob)]
        from_desc.close()
        from_blob.close()
    a = np.array([[h.t, *h.barycentrics, h.instance_index, h.primitive_index] for h in hits[0]], np.float64)
    b = np.array([[h.t, *h.barycentrics, h.instance_index, h.primitive_index] for h in hits[1]], np.float64)
    assert np.array_equal(a, b) and (a[:, 4] != 0xFFFFFFFF).sum() > 500
    ra = np.array([list(r.radiance) for r in paths[0]], np.float32)
    rb = np.array([list(r.radiance) for r in paths[1]], np.float32)
    assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32))
