"""Transform-only refit (bf200_scene_refit, AccelBackend::refit). A scene refitted to new instance
transforms must answer exactly like a scene created from those transforms: closest hits (t,
barycentrics, instance, primitive) and occlusion bit for bit, and per-path radiance bit for bit
(the mesh light moves too). Both the TLAS form (> 32 instances) and the eager form are covered.
Any change besides instance transforms is refused and the scene stays usable."""
import copy

import numpy as np
import pytest

from bf200 import abi, runtime, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with runtime.Context(0, path_capacity=1 << 16) as c:
        yield c


def moved(builder, seed, light_too=True):
    """Copy of the builder with every instance transform replaced: rotated, scaled and moved."""
    rng = np.random.default_rng(seed)
    b = copy.copy(builder)
    b.instances = []
    for k, (mesh, material, matrix, mask) in enumerate(builder.instances):
        m = np.array(matrix, np.float32)
        emissive = any(x != 0.0 for x in builder.materials[material][1])
        if emissive and not light_too:
            b.instances.append((mesh, material, m, mask))
            continue
        r = scenes.random_rotation(rng) if not emissive else np.eye(3)  # lights stay facing down
        m[:3, :3] = (r @ m[:3, :3].astype(np.float64) * rng.uniform(0.8, 1.2)).astype(np.float32)
        m[:3, 3] = (m[:3, 3] + rng.uniform(-1.0, 1.0, 3)).astype(np.float32)
        if k == 0:
            m[:3, 0] = -m[:3, 0]  # a mirrored instance: its orientation flag flips
        b.instances.append((mesh, material, m, mask))
    return b


def random_rays(rng, n, centre, spread):
    rays = (abi.Ray * n)()
    for k in range(n):
        o = np.asarray(centre) + rng.normal(0.0, spread, 3)
        d = rng.normal(0.0, 1.0, 3)
        d /= np.linalg.norm(d)
        for a in range(3):
            rays[k].origin[a], rays[k].direction[a] = float(o[a]), float(d[a])
        rays[k].t_min, rays[k].t_max, rays[k].time, rays[k].mask = 0.0, float("inf"), 0.5, 0xFFFFFFFF
    return rays


def hits_array(hits):
    return np.array([[h.t, *h.barycentrics] for h in hits], np.float32), \
        np.array([[h.instance_index, h.primitive_index] for h in hits], np.uint32)


@pytest.mark.parametrize("kind", ["tlas", "eager"])
def test_refit_equals_a_fresh_scene(ctx, kind):
    if kind == "tlas":
        builder = scenes.bvh_stress(scenes.SceneBuilder(environment=(0.5,) * 4), subdivisions=3)
        centre, spread = (0.0, 0.0, 0.0), 8.0
        options = abi.default_options(mis="power", max_depth=8)
    else:
        builder = scenes.cornell_box(scenes.SceneBuilder(), with_spheres=True)
        centre, spread = (0.0, 0.0, 1.0), 0.6
        options = abi.default_options(mis="power", max_depth=8)
    target = moved(builder, 5)
    refitted = ctx.create_scene(builder)
    refitted.refit(target)
    fresh = ctx.create_scene(target)
    rng = np.random.default_rng(9)
    rays = random_rays(rng, 20000, centre, spread)
    a_f, a_i = hits_array(ctx.closest_hits(refitted, rays))
    b_f, b_i = hits_array(ctx.closest_hits(fresh, rays))
    assert np.array_equal(a_i, b_i) and np.array_equal(a_f.view(np.uint32), b_f.view(np.uint32))
    assert (a_i[:, 0] != 0xFFFFFFFF).sum() > 2000
    assert np.array_equal(ctx.occlusions(refitted, rays), ctx.occlusions(fresh, rays))
    # whole paths: the moved light, world normals and orientation flags all enter the radiance
    n = 2048
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray = rays[k]
        inputs[k].sample.pixel_x, inputs[k].sample.pixel_y = k % 64, k // 64
        inputs[k].sample.sample_index, inputs[k].sample.seed = k, 7
    ra, _ = ctx.trace_paths(refitted, inputs, options)
    rb, _ = ctx.trace_paths(fresh, inputs, options)
    la = np.array([list(r.radiance) for r in ra], np.float32)
    lb = np.array([list(r.radiance) for r in rb], np.float32)
    assert np.array_equal(la.view(np.uint32), lb.view(np.uint32))
    refitted.close()
    fresh.close()


def test_refit_refuses_other_changes(ctx):
    builder = scenes.cornell_box(scenes.SceneBuilder(), with_spheres=False)
    scene = ctx.create_scene(builder)
    recoloured = copy.copy(builder)
    recoloured.materials = list(builder.materials)
    recoloured.materials[0] = (scenes.lambertian([0.5] * 4), builder.materials[0][1], 0)
    with pytest.raises(runtime.Bf200Error) as info:
        scene.refit(recoloured)
    assert info.value.status == 4  # INVALID_STATE: no rebuild fallback
    reshaped = copy.copy(builder)
    reshaped.meshes = list(builder.meshes)
    reshaped.meshes[0] = scenes.quad([(-1, -1, 0), (-1, -1, 3), (1, -1, 3), (1, -1, 0)], (0, 1, 0))
    with pytest.raises(runtime.Bf200Error) as info:
        scene.refit(reshaped)
    assert info.value.status == 4
    # still usable, and a legal refit still works after the refusals
    scene.refit(moved(builder, 3, light_too=False))
    hits = ctx.closest_hits(scene, random_rays(np.random.default_rng(1), 256, (0.0, 0.0, 1.0), 0.3))
    assert sum(h.instance_index != 0xFFFFFFFF for h in hits) > 100
    scene.close()
