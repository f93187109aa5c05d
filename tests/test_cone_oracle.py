"""Pins the oracle's ray-cone restatement (the reference wavefront's advance_ray_cone_to_hit and
propagate_ray_cone_scattering) on the reference's own RayCone.hpp: tests/golden/cones.npz, made by
tests/golden/make_cone_golden.py from the compiled reference. Values and refusals bit for bit.
Where the compiled reference is present, fresh seeded cases are checked against it as well.
CPU only."""
import numpy as np
import pytest

from oracle.bindings import Oracle, Reference, CheckerError


def same(a, b):
    """Bitwise equality with NaN (a refusal) matching NaN."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    both_nan = np.isnan(a) & np.isnan(b)
    return np.where(both_nan, True, a.view(np.uint32) == b.view(np.uint32))


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def negative_roughness(kinds, parameters):
    """Rough conductors with one negative roughness parameter: the wavefront refuses them
    (CudaWavefrontStages.cu:3704-3712) where RayCone.hpp:347-352 takes max(alpha_x, alpha_y). No
    traced path meets one (scene upload refuses a negative roughness), so the two agree on every
    scene the backend accepts."""
    p = parameters
    return (kinds == 3) & np.isfinite(p[:, 8]) & np.isfinite(p[:, 9]) & ((p[:, 8] < 0) | (p[:, 9] < 0)) & (
        np.maximum(p[:, 8], p[:, 9]) >= 0)


def test_scattering_matches_the_reference(oracle, golden):
    g = golden("cones")
    out, failures = oracle.cone_scatter(g["scatter_cones"], g["scatter_kinds"], g["scatter_parameters"],
                                        g["scatter_events"], g["scatter_wo"], g["scatter_wi"])
    diverge = negative_roughness(g["scatter_kinds"], g["scatter_parameters"])
    assert diverge.sum() > 10 and np.isnan(out[diverge]).all()
    ok = same(out, g["scatter_out"]).all(axis=1) | diverge
    assert ok.all(), np.nonzero(~ok)[0][:10]
    refused = np.isnan(g["scatter_out"][:, 0])
    assert failures == (refused | diverge).sum()
    # the fixture exercises every policy and both outcomes
    accepted_kinds = set(g["scatter_kinds"][~refused].tolist())
    assert {1, 2, 3, 4, 5, 6} <= accepted_kinds
    assert 500 < refused.sum() < len(refused) - 1500
    transmitted = (g["scatter_events"] & 0x10) != 0
    assert (transmitted & ~refused).sum() > 200


@pytest.mark.parametrize("direction", [(0.0, 0.0, 1.0), (0.0, 0.0, -1.0), (1.0, 0.0, 0.0), (0.0, -1.0, 0.0)])
def test_advance_matches_the_reference(oracle, golden, direction):
    """Unit axis directions: the wavefront's direction length is exactly 1, so the travelled
    distance is the hit parameter and the reference's advance_ray_cone(cone, distance) applies."""
    g = golden("cones")
    n = len(g["advance_distances"])
    directions = np.tile(np.array(direction, np.float32), (n, 1))
    out, failures = oracle.cone_advance(g["advance_cones"], directions, g["advance_distances"])
    ok = same(out, g["advance_out"])
    assert ok.all(), np.nonzero(~ok)[0][:10]
    assert failures == np.isnan(g["advance_out"]).sum()


def test_advance_measures_non_unit_directions(oracle):
    """A direction of length L scales the travelled distance by L: power-of-two lengths are exact,
    and the zero or non-finite direction is refused."""
    cones = np.array([[0.5, 0.25]] * 4, np.float32)
    directions = np.array([[0, 8, 0], [0, 0, 0.125], [0, 0, 0], [np.inf, 0, 0]], np.float32)
    widths, failures = oracle.cone_advance(cones, directions, np.array([1.0, 16.0, 1.0, 1.0], np.float32))
    assert widths[0] == np.float32(0.5 + 0.25 * 8) and widths[1] == np.float32(0.5 + 0.25 * 2)
    assert np.isnan(widths[2:]).all() and failures == 2


def test_fresh_cases_against_the_compiled_reference(oracle):
    try:
        ref = Reference()
    except CheckerError:
        pytest.skip("the compiled reference (oracle/_ref) is not built here")
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "make_cone_golden", os.path.join(os.path.dirname(__file__), "golden", "make_cone_golden.py"))
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    rng = np.random.default_rng(99)
    case = maker.scatter_cases(rng, 20000)
    want, _ = ref.cone_scatter(*case)
    got, _ = oracle.cone_scatter(*case)
    assert (same(got, want).all(axis=1) | negative_roughness(case[1], case[2])).all()
    cones, distances = maker.advance_cases(rng, 20000)
    want, _ = ref.cone_advance(cones, distances)
    got, _ = oracle.cone_advance(cones, np.tile(np.array([0, 1, 0], np.float32), (len(distances), 1)), distances)
    assert same(got, want).all()
