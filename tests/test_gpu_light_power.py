"""Power-weighted light selection in transport: a Cornell box with three emitters of different
radiance and size, traced with bf200_scene_set_light_powers installed. Per-path radiance is
compared with the oracle under the same powers (tolerances of the other parity tests, helpers) and,
where the compiled reference travelled with the repository (oracle/_ref), with the reference's own
trace_scene_mis using LightSampler::create_power_weighted. Switching back to uniform selection
gives the uniform render again, bit for bit."""
import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import REFERENCE_DIVERGED_FRACTION, arrays, check_paths
from oracle.bindings import Oracle, Reference, reference_available

pytestmark = pytest.mark.gpu


def three_light_box():
    builder = scenes.cornell_box(scenes.SceneBuilder(), with_spheres=True)
    for corners, radiance in [(((-0.9, 0.985, 0.2), (-0.6, 0.985, 0.2), (-0.6, 0.985, 0.5), (-0.9, 0.985, 0.5)),
                               (40.0, 30.0, 20.0, 10.0)),
                              (((0.5, 0.985, 1.5), (0.9, 0.985, 1.5), (0.9, 0.985, 1.9), (0.5, 0.985, 1.9)),
                               (2.0, 3.0, 4.0, 5.0))]:
        light = builder.add_material(scenes.lambertian([0.0] * 4), emission=radiance)
        builder.add_instance(builder.add_mesh(scenes.quad(list(corners), (0, -1, 0))), light)
    return builder


def light_powers(builder):
    """Flux per lane of every emissive instance, in instance order: radiance x area x pi."""
    powers = []
    for mesh_index, material, _, _ in builder.instances:
        emission = builder.materials[material][1]
        if not any(v != 0 for v in emission):
            continue
        mesh = builder.meshes[mesh_index]
        area = 0.0
        for tri in mesh.triangles:
            p = mesh.positions[tri].astype(np.float64)
            area += 0.5 * np.linalg.norm(np.cross(p[1] - p[0], p[2] - p[0]))
        powers.append([float(e) * area * np.pi for e in emission])
    return np.array(powers, np.float32)


def path_inputs(oracle, n, seed):
    width = height = 64
    rng = np.random.default_rng(seed)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(rng.integers(width)), int(rng.integers(height))
        samples[k].sample_index, samples[k].seed = int(rng.integers(1 << 40)), 0x243F6A8885A308D3
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return inputs


def test_power_weighted_paths_match_the_oracle_and_the_reference():
    builder = three_light_box()
    powers = light_powers(builder)
    assert len(powers) == 3 and not np.allclose(powers[0], powers[1])
    options = abi.default_options(mis="power", max_depth=8)
    oracle = Oracle(device_trig=True)
    inputs = path_inputs(oracle, 2048, 21)
    handle = oracle.scene(builder)
    oracle.set_light_powers(handle, powers)
    expected, failures = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    assert failures == 0
    with runtime.Context(0, path_capacity=1 << 14) as ctx:
        scene = ctx.create_scene(builder)
        uniform, _ = ctx.trace_paths(scene, inputs, options)
        scene.set_light_powers(powers)
        got, report = ctx.trace_paths(scene, inputs, options)
        scene.set_light_powers(None)
        again, _ = ctx.trace_paths(scene, inputs, options)
        scene.close()
    assert report.failed_lanes == 0
    check_paths(arrays(got), arrays(expected), "power-weighted three-light box (oracle)")
    u, a = arrays(uniform)["radiance"], arrays(again)["radiance"]
    assert np.array_equal(u.view(np.uint32), a.view(np.uint32))
    assert not np.array_equal(u.view(np.uint32), arrays(got)["radiance"].view(np.uint32))
    if reference_available():
        ref = Reference()
        handle = ref.scene(builder)
        ref.set_light_powers(handle, powers)
        reference, ref_failures = ref.trace(handle, inputs, options)
        ref.destroy(handle)
        assert ref_failures == 0
        exact, _ = check_paths(arrays(got), arrays(reference), "power-weighted three-light box (reference)",
                               diverged=REFERENCE_DIVERGED_FRACTION)
        assert exact >= 0.95
