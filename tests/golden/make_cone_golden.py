"""Writes tests/golden/cones.npz: the reference's own ray-cone functions (RayCone.hpp and
PinholeCamera.hpp, compiled into oracle/_ref/libbfref.so by `make -C oracle ref`) on seeded cases.

* scatter_*: renderer::propagate_ray_cone_scattering for closures of every kind, valid and invalid
  event lobes, local directions in either hemisphere (unit to float rounding, plus a set that is
  clearly not unit), and cones from zero to the edges of float range.
* advance_*: renderer::advance_ray_cone(cone, distance), with distances that underflow the growth,
  leave a wide cone's width unchanged, or overflow it.
* camera_*: PinholeCamera::generate_primary_ray_cone of the 256 x 256 Cornell camera for seeded
  (pixel, sample) indices: the primary cones of the device's cone-carrying trace tests.

The wavefront restatement tests directions to 128 ulp of unit length where RayCone.hpp allows 256,
and measures a ray direction as max|d| * |d / max|d|| where RayCone.hpp calls std::hypot; the cases
stay clear of both differences (unit directions come from float64 normalisation; the advance cases
take the distance directly).

Run from the repository root: python tests/golden/make_cone_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from bf200 import abi, scenes  # noqa: E402
from oracle.bindings import Reference  # noqa: E402

DIFFUSE, GLOSSY, SPECULAR, REFLECTION, TRANSMISSION, VOLUME = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20


def unit_vectors(rng, n, positive):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[:, 2] = np.abs(v[:, 2]) * np.where(positive, 1.0, -1.0)
    v[np.abs(v[:, 2]) < 1e-3, 2] = np.where(positive, 1e-3, -1e-3)[np.abs(v[:, 2]) < 1e-3]
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v.astype(np.float32)


def cone_values(rng, n):
    pick = rng.integers(0, 8, n)
    value = np.exp(rng.uniform(np.log(1e-6), np.log(1e3), n))
    value = np.where(pick == 0, 0.0, value)
    value = np.where(pick == 1, 3e38, value)       # near the top of float range
    value = np.where(pick == 2, 1e-44, value)      # subnormal
    return value.astype(np.float32)


def scatter_cases(rng, n):
    kinds = rng.choice([1, 1, 2, 3, 3, 4, 4, 4, 5, 6, 0, 7], n).astype(np.uint32)
    events = np.zeros(n, np.uint32)
    transmit = rng.random(n) < 0.5
    for k in range(n):
        kind = int(kinds[k])
        if rng.random() < 0.12:
            events[k] = rng.choice([0, VOLUME | REFLECTION | DIFFUSE, DIFFUSE | GLOSSY | REFLECTION,
                                    DIFFUSE | REFLECTION | TRANSMISSION, GLOSSY, 0x40 | GLOSSY | REFLECTION,
                                    GLOSSY | TRANSMISSION, SPECULAR | REFLECTION, DIFFUSE | REFLECTION])
            continue
        family = {1: DIFFUSE, 2: DIFFUSE, 3: GLOSSY, 4: GLOSSY, 5: SPECULAR, 6: SPECULAR}.get(kind, GLOSSY)
        direction = REFLECTION
        if kind == 4 and transmit[k]:
            direction = TRANSMISSION
        if kind == 6:
            direction = TRANSMISSION
        events[k] = family | direction
    parameters = np.zeros((n, 10), np.float32)
    parameters[:, 0] = rng.uniform(1.0, 1.8, n)
    parameters[:, 1] = rng.uniform(1.0, 2.5, n)
    parameters[:, 2:4] = rng.uniform(0.0, 1.0, (n, 2))
    parameters[:, 8:10] = rng.uniform(0.0, 1.0, (n, 2))
    odd = rng.random(n)
    parameters[odd < 0.03, 8] = -0.25                  # a negative roughness
    parameters[(odd >= 0.03) & (odd < 0.06), 3] = np.inf
    parameters[(odd >= 0.06) & (odd < 0.09), 0] = 0.0   # a zero eta
    parameters[(odd >= 0.09) & (odd < 0.1), 1] = 1e-38  # an eta ratio that overflows
    wo_up = rng.random(n) < 0.8
    wo = unit_vectors(rng, n, wo_up)
    # incoming on the side the event asks for, with a few on the wrong side
    wi_up = np.where((events & TRANSMISSION) != 0, ~wo_up, wo_up)
    flip = rng.random(n) < 0.05
    wi = unit_vectors(rng, n, np.where(flip, ~wi_up, wi_up))
    bad = rng.random(n) < 0.03
    wi[bad] *= np.float32(1.01)                          # clearly not unit
    grazing = rng.random(n) < 0.02
    wi[grazing, 2] = np.float32(0.0)
    cones = np.stack([cone_values(rng, n), cone_values(rng, n)], axis=1)
    neg = rng.random(n) < 0.02
    cones[neg, 0] = -1.0
    return cones, kinds, parameters, events, wo, wi


def advance_cases(rng, n):
    cones = np.stack([cone_values(rng, n), cone_values(rng, n)], axis=1)
    distances = np.exp(rng.uniform(np.log(1e-8), np.log(1e4), n)).astype(np.float32)
    pick = rng.integers(0, 10, n)
    distances = np.where(pick == 0, 0.0, distances)
    distances = np.where(pick == 1, 1e-40, distances)            # growth underflows
    distances = np.where(pick == 2, 3e38, distances)             # overflows
    cones[pick == 3, 0] = np.float32(1e3)                        # width far above the growth
    cones[pick == 3, 1] = np.float32(1e-3)
    distances = np.where(pick == 3, 1e-7, distances)
    distances = np.where(pick == 4, np.inf, distances)
    distances = np.where(pick == 5, -1.0, distances)
    return cones, distances.astype(np.float32)


def camera_cases(rng, n, width, height):
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(rng.integers(width)), int(rng.integers(height))
        samples[k].sample_index, samples[k].seed = int(rng.integers(1 << 40)), 0x243F6A8885A308D3
    table = np.array([[s.pixel_x, s.pixel_y, s.sample_index, s.seed] for s in samples], np.uint64)
    return samples, table


def main():
    ref = Reference()
    rng = np.random.default_rng(20261204)
    cones, kinds, parameters, events, wo, wi = scatter_cases(rng, 4096)
    scattered, scatter_failures = ref.cone_scatter(cones, kinds, parameters, events, wo, wi)
    a_cones, distances = advance_cases(rng, 2048)
    advanced, advance_failures = ref.cone_advance(a_cones, distances)
    width, height = 256, 256
    samples, table = camera_cases(rng, 4096, width, height)
    origin, normal, tangent = scenes.camera_frame_inputs()
    camera = ref.camera_cones(origin, normal, tangent, width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME, samples)
    np.savez_compressed(os.path.join(HERE, "cones.npz"),
                        scatter_cones=cones, scatter_kinds=kinds, scatter_parameters=parameters,
                        scatter_events=events, scatter_wo=wo, scatter_wi=wi, scatter_out=scattered,
                        advance_cones=a_cones, advance_distances=distances, advance_out=advanced,
                        camera_samples=table, camera_cones=camera)
    print(f"scatter: {len(kinds)} cases, {scatter_failures} refused; advance: {len(distances)} cases, "
          f"{advance_failures} refused; camera cones: width {camera[:, 0].min()}..{camera[:, 0].max()}, "
          f"spread {camera[:, 1].min()}..{camera[:, 1].max()}")


if __name__ == "__main__":
    main()
