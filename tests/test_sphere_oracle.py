"""The oracle's analytic sphere intersection (oracle/bfo_oracle.cpp intersect_sphere) against the
reference's own renderer::Sphere results frozen in tests/golden/spheres.npz (made by
tests/golden/make_sphere_golden.py from the compiled reference): status, t, normal and position
bit for bit, including the reference's SphereTest cases."""
import os

import numpy as np

from bf200 import abi
from oracle.bindings import Oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "spheres.npz")


def rays_from(rows):
    rays = (abi.Ray * len(rows))()
    for k, row in enumerate(rows):
        for i in range(3):
            rays[k].origin[i] = float(row[i])
            rays[k].direction[i] = float(row[3 + i])
        rays[k].t_min, rays[k].t_max = float(row[6]), float(row[7])
        rays[k].time, rays[k].mask = 0.5, 0xFFFFFFFF
    return rays


def test_golden_pins_the_reference_sphere_tests():
    g = np.load(GOLDEN)
    out = g["pair_out"]
    assert out[0, 0] == 1 and out[0, 1] == 2.0 and out[1, 1] == 4.0  # near and far roots
    assert out[4, 0] == 0  # both roots excluded by the open-ended bounds
    assert out[5, 1] == 0.5 and out[7, 1] == 2.0  # internal root, double tangent
    assert out[8, 1] == 1.0e5 and tuple(out[8, 5:8]) == (3.0, 4.0, 0.0)  # distant oblique tangent
    assert out[9, 1] == 1.0 and out[10, 0] == 0 and out[11, 0] == 1  # rounding-sensitive tangent
    assert out[int(g["reference_cases"]) - 1, 0] == 2  # arithmetic error, not a miss


def test_oracle_sphere_intersection_matches_the_reference_bit_for_bit():
    g = np.load(GOLDEN)
    oracle = Oracle()
    got = oracle.sphere_intersect(g["pair_spheres"], rays_from(g["pair_rays"]))
    assert np.array_equal(got.view(np.uint32), g["pair_out"].view(np.uint32))
    rays = rays_from(g["scene_rays"])
    for s in range(len(g["scene_spheres"])):
        spheres = np.repeat(g["scene_spheres"][s:s + 1], len(rays), 0)
        got = oracle.sphere_intersect(spheres, rays)
        assert np.array_equal(got.view(np.uint32), g["scene_out"][:, s, :].view(np.uint32)), s
