"""A scene written in the native JSON schema ("blackframe.scene" v1), parsed by
bf200_scene_json_parse and committed by bf200_scene_json_frame, rendered on the device with the
document's own camera, film request and transport options, against the oracle's transport of the
same committed scene.

The document is a Cornell box with an emissive ceiling patch, a two-level instance hierarchy
(a block placed under a rotated parent), a two-closure mixture, a point light and the
environment light whose packet the render uses. Pixels must agree within the parity tolerance
(tests/helpers.py), every pixel must hold the document's samples per pixel, and the film must
equal a second render of the same frame bit for bit.
"""
import json
import os

import numpy as np
import pytest

from bf200 import abi, runtime, scene_json
from helpers import DIVERGED_FRACTION, RELATIVE_TOLERANCE, arrays, relative_error, sensor_from_golden
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu

PACKET = {"nanometers": [471.2129, 588.7129, 706.2129, 823.7129], "pdf": [0.0021276595] * 4}


def quad(p0, p1, p2, p3, normal):
    return {"positions": [p0, p1, p2, p3], "normals": [normal] * 4,
            "texture_coordinates": [[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]],
            "triangles": [[0, 1, 2], [0, 2, 3]]}


def block():
    corners = [[x, y, z] for x in (-0.3, 0.3) for y in (-0.3, 0.3) for z in (-0.3, 0.3)]
    faces = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    positions, normals, uvs, tris = [], [], [], []
    for f in faces:
        a, b, c, d = (np.array(corners[i]) for i in f)
        n = np.cross(b - a, d - a)
        n = [float(np.float32(v)) for v in n / np.linalg.norm(n)]
        base = len(positions)
        positions += [corners[i] for i in f]
        normals += [n] * 4
        uvs += [[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]]
        tris += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
    return {"positions": positions, "normals": normals, "texture_coordinates": uvs, "triangles": tris}


def lambert(ident, reflectance, emission=(0.0, 0.0, 0.0, 0.0)):
    return {"id": ident, "spectral": {
        "wavelengths": PACKET, "emission": list(emission), "normal_map": None, "bump_map": None,
        "closures": {"frame_mode": "shading_normal", "tangent_rotation_radians": 0.0,
                     "components": [{"probability": 1.0, "type": "lambertian_reflection",
                                     "weight": list(reflectance)}]}}}


def document(width=64, height=64, spp=4):
    ident = [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]
    c, s = float(np.float32(np.cos(0.4))), float(np.float32(np.sin(0.4)))
    parent = [c, 0.0, s, 0.2, 0.0, 1.0, 0.0, -0.7, -s, 0.0, c, 1.0, 0.0, 0.0, 0.0, 1.0]
    child = [1.0, 0.0, 0.0, 0.0, 0.0, 1.5, 0.0, 0.15, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]
    walls = [
        quad([-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0], [0, 0, 1]),      # back
        quad([-1, -1, 0], [-1, -1, 2], [1, -1, 2], [1, -1, 0], [0, 1, 0]),    # floor
        quad([-1, 1, 0], [1, 1, 0], [1, 1, 2], [-1, 1, 2], [0, -1, 0]),       # ceiling
        quad([-1, -1, 0], [-1, 1, 0], [-1, 1, 2], [-1, -1, 2], [1, 0, 0]),    # left
        quad([1, -1, 0], [1, -1, 2], [1, 1, 2], [1, 1, 0], [-1, 0, 0]),       # right
        quad([-0.3, 0.99, 0.7], [0.3, 0.99, 0.7], [0.3, 0.99, 1.3], [-0.3, 0.99, 1.3], [0, -1, 0]),  # lamp
    ]
    geometries = [{"id": 10 + k, "mesh": m} for k, m in enumerate(walls)] + [{"id": 30, "mesh": block()}]
    mixture = {"id": 24, "spectral": {
        "wavelengths": PACKET, "emission": [0.0] * 4, "normal_map": None, "bump_map": None,
        "closures": {"frame_mode": "shading_normal", "tangent_rotation_radians": 0.0, "components": [
            {"probability": 0.6, "type": "lambertian_reflection", "weight": [0.6, 0.5, 0.4, 0.3]},
            {"probability": 0.4, "type": "rough_conductor_reflection", "weight": [0.9] * 4,
             "eta": [0.2, 0.4, 0.9, 1.3], "k": [3.1, 2.6, 2.2, 1.9], "alpha_x": 0.25, "alpha_y": 0.12}]}}}
    materials = [lambert(20, [0.75] * 4), lambert(21, [0.75, 0.25, 0.25, 0.2]), lambert(22, [0.2, 0.75, 0.25, 0.2]),
                 lambert(23, [0.0] * 4, emission=(8.0, 6.0, 4.0, 2.0)), mixture]
    wall_materials = [20, 20, 20, 21, 22, 23]
    instances = [{"id": 100 + k, "parent": None, "object": 1, "geometry": 10 + k, "material": m,
                  "local_to_parent": ident, "visibility_mask": 4294967295} for k, m in enumerate(wall_materials)]
    instances += [{"id": 200, "parent": None, "object": 1, "geometry": 30, "material": 20,
                   "local_to_parent": parent, "visibility_mask": 4294967295},
                  {"id": 150, "parent": 200, "object": 1, "geometry": 30, "material": 24,
                   "local_to_parent": child, "visibility_mask": 4294967295}]
    return {
        "schema": "blackframe.scene", "schema_version": 1,
        "active": {"film": 1, "camera": 1, "render_options": 1},
        "films": [{"id": 1, "extent": [width, height], "crop": [0, 0, width, height], "accumulation": "float32"}],
        "cameras": [{"id": 1, "film": 1, "model": {
            "type": "pinhole", "origin": [0.0, 0.0, 3.0], "normal": [0.0, 0.0, 1.0], "tangent": [1.0, 0.0, 0.0],
            "bitangent": [0.0, 1.0, 0.0], "vertical_fov_radians": 1.5707963705062866, "t_min": 0.0,
            "t_max": 1e30, "visibility_mask": 4294967295, "current_medium": 0}}],
        "render_options": [{"id": 1, "film": 1, "samples_per_pixel": spp, "maximum_path_depth": 6,
                            "tile_edge_length": 16, "seed": 0, "pixel_jitter": "uniform", "mis_heuristic": "power",
                            "light_sampling_strategy": "uniform",
                            "depth_limits": {"diffuse": 5, "glossy": 5, "specular": 5, "transmission": 5,
                                             "volume": 0},
                            "russian_roulette": {"mode": "disabled"}}],
        "constant_textures": [], "host_image_textures": [], "objects": [{"id": 1}],
        "geometries": geometries, "materials": materials, "instances": instances,
        "lights": [{"id": 1, "type": "environment", "wavelengths": PACKET, "radiance": [0.05, 0.04, 0.03, 0.02]},
                   {"id": 2, "type": "point", "position": [0.4, 0.6, 1.2], "absolute_position_error": [0.0, 0.0, 0.0],
                    "spectral_radiant_intensity": [0.8, 0.8, 0.6, 0.5]}]}


def test_json_scene_renders_like_the_oracle():
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_plain_64.npz"))
    sensor = sensor_from_golden(g)
    with scene_json.SceneJson(json.dumps(document())) as doc:
        frame = doc.frame()
        width, height, spp = frame.width, frame.height, frame.samples_per_pixel
        with runtime.Context(0, path_capacity=1 << 16) as ctx:
            scene = ctx.create_scene(None, desc=frame.scene)
            sums, counts, report = ctx.render_film(scene, frame.camera, sensor, frame.options, spp, seed=frame.seed,
                                                   precision=frame.precision)
            again, _, _ = ctx.render_film(scene, frame.camera, sensor, frame.options, spp, seed=frame.seed,
                                          precision=frame.precision)
            scene.close()
        assert (counts == spp).all() and report.path_count == width * height * spp
        assert (sums.view(np.uint32) == again.view(np.uint32)).all()
        px, py, s = np.meshgrid(np.arange(width), np.arange(height), np.arange(spp), indexing="ij")
        order = np.lexsort((px.ravel(), py.ravel(), s.ravel()))
        px, py, s = px.ravel()[order], py.ravel()[order], s.ravel()[order]
        samples = (abi.SampleIndex * len(px))()
        for k in range(len(px)):
            samples[k].pixel_x, samples[k].pixel_y = int(px[k]), int(py[k])
            samples[k].sample_index, samples[k].seed = int(s[k]), int(frame.seed)
        oracle = Oracle(device_trig=True)
        rays = oracle.camera_rays(frame.camera, samples)
        inputs = (abi.PathInput * len(px))()
        for k in range(len(px)):
            inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
        handle = oracle.scene(None, desc=frame.scene)
        results, failures = oracle.trace(handle, inputs, frame.options)
        oracle.destroy(handle)
    assert failures == 0
    expected, _ = oracle.film(arrays(results)["radiance"], samples, sensor, width, height, 0)
    err = relative_error(sums.astype(np.float64), expected)
    assert (err <= RELATIVE_TOLERANCE).mean() >= 1.0 - DIVERGED_FRACTION
    assert sums[..., :3].sum() > 0.0
