"""The spatial light tree (bf200_light_tree_select / bf200_light_tree_probability) against the
reference's LightSampler::create_spatial_tree: the slot and probability selected for canonical
samples at query points, and the probability of every light, bit for bit, on the seeded light sets
of tests/golden/light_tree.npz (made by tests/golden/make_light_tree_golden.py from the compiled
reference): one light, clustered and spread boxes, point-like and flat boxes, zero-power lights,
unbounded lights beside finite ones and alone, coincident centroids. Fresh seeded sets are checked
against the compiled reference where it is built. Host code only."""
import importlib.util
import os

import numpy as np
import pytest

from bf200 import runtime
from oracle.bindings import CheckerError, Reference


def same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def test_light_tree_matches_the_reference(golden):
    g = golden("light_tree")
    checked = 0
    for k in range(int(g["sets"])):
        lo, hi, p = g[f"lo_{k}"], g[f"hi_{k}"], g[f"powers_{k}"]
        selected, probability = runtime.light_tree_select(lo, hi, p, g[f"positions_{k}"], g[f"samples_{k}"])
        assert np.array_equal(selected, g[f"selected_{k}"]), k
        assert same(probability, g[f"probability_{k}"]), k
        grid = np.repeat(g[f"positions_{k}"][:32], len(p), axis=0)
        indices = np.tile(np.arange(len(p), dtype=np.uint32), 32)
        each = runtime.light_tree_probability(lo, hi, p, grid, indices).reshape(32, len(p))
        assert same(each, g[f"each_{k}"]), k
        # a selection's probability is the probability of the light it selected
        ok = selected != 0xFFFFFFFF
        again = runtime.light_tree_probability(lo, hi, p, g[f"positions_{k}"][ok], selected[ok])
        assert same(again, probability[ok]), k
        checked += int(ok.sum())
    assert checked > 2000


def test_light_tree_refusals():
    lo = np.zeros((2, 3), np.float32)
    hi = np.ones((2, 3), np.float32)
    p = np.ones((2, 4), np.float32)
    with pytest.raises(runtime.Bf200Error) as info:  # unordered bounds
        runtime.light_tree_select(hi, lo, p, np.zeros((1, 3)), [0.5])
    assert info.value.status == 1
    half = np.array([[-np.inf, 0, 0], [0, 0, 0]], np.float32)  # neither finite nor canonically unbounded
    with pytest.raises(runtime.Bf200Error) as info:
        runtime.light_tree_select(half, hi, p, np.zeros((1, 3)), [0.5])
    assert info.value.status == 1
    with pytest.raises(runtime.Bf200Error):  # no power at all
        runtime.light_tree_select(lo, hi, np.zeros((2, 4), np.float32), np.zeros((1, 3)), [0.5])
    # per-query refusals: a sample outside [0, 1), a non-finite point, a slot out of range
    selected, probability = runtime.light_tree_select(lo, hi, p, [[0, 0, 0], [np.nan, 0, 0]], [1.0, 0.5])
    assert list(selected) == [0xFFFFFFFF, 0xFFFFFFFF] and list(probability) == [-1.0, -1.0]
    assert list(runtime.light_tree_probability(lo, hi, p, [[0, 0, 0]], [5])) == [-1.0]


def test_fresh_sets_against_the_compiled_reference():
    try:
        ref = Reference()
    except CheckerError:
        pytest.skip("the compiled reference (oracle/_ref) is not built here")
    spec = importlib.util.spec_from_file_location(
        "make_light_tree_golden", os.path.join(os.path.dirname(__file__), "golden", "make_light_tree_golden.py"))
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    rng = np.random.default_rng(4242)
    for lo, hi, p in maker.light_sets(rng):
        positions, samples = maker.queries(rng, lo, hi, 512)
        want, code = ref.light_tree(lo, hi, p, positions, samples=samples)
        assert code == 0
        selected, probability = runtime.light_tree_select(lo, hi, p, positions, samples)
        assert np.array_equal(selected, want[0]) and same(probability, want[1])


# The known answers of the reference's own LightTreeTest (Tests/Renderer/Light/LightTreeTest.cpp),
# float transport scalar.

def point(*xyz):
    return np.array([xyz], np.float32)


def test_spatial_importance_is_symmetric_and_scale_invariant():
    """LightTreeTest.cpp:125-165: two unit-power point lights at x = -10 and 10."""
    lo = hi = np.concatenate([point(-10, 0, 0), point(10, 0, 0)])
    p = np.ones((2, 4), np.float32)
    q = runtime.light_tree_probability(lo, hi, p, [[-10, 0, 0], [-10, 0, 0], [10, 0, 0], [10, 0, 0]], [0, 1, 0, 1])
    left_from_left, right_from_left, left_from_right, right_from_right = (float(v) for v in q)
    eps = float(np.finfo(np.float32).eps)
    assert abs(left_from_left - 2.0 / 3.0) <= 8 * eps
    assert abs(left_from_left - right_from_right) <= 2 * eps
    assert abs(right_from_left - left_from_right) <= 2 * eps
    assert left_from_left > right_from_left
    scaled = np.concatenate([point(-1000, 20, 30), point(1000, 20, 30)])
    again = runtime.light_tree_probability(scaled, scaled, p, [[-1000, 20, 30]], [0])
    assert again[0] == np.float32(left_from_left)


def test_extreme_finite_distances_keep_relative_probability():
    """LightTreeTest.cpp:208-242: a query at FLT_MAX, and lights at -FLT_MAX and FLT_MAX."""
    big = np.finfo(np.float32).max
    eps = float(np.finfo(np.float32).eps)
    lights = np.concatenate([point(0, 0, 0), point(1, 0, 0)])
    p = np.ones((2, 4), np.float32)
    far = runtime.light_tree_probability(lights, lights, p, [[big, 0, 0], [big, 0, 0]], [0, 1])
    assert all(abs(float(v) - 0.5) <= 8 * eps for v in far)
    wide = np.concatenate([point(-big, 0, 0), point(big, 0, 0)])
    assert list(runtime.light_tree_probability(wide, wide, p, [[0, 0, 0], [0, 0, 0]], [0, 1])) == [0.5, 0.5]


def test_upper_edge_remap_stays_inside_the_canonical_domain():
    """LightTreeTest.cpp:244-272: the largest sample below 1 selects the last light of three
    unbounded lights, with the probability the tree gives that light."""
    small = np.float32(0.00003418326)
    half = (np.float32(1) - small) / np.float32(2)
    lo = np.full((3, 3), -np.inf, np.float32)
    hi = np.full((3, 3), np.inf, np.float32)
    p = np.array([[small] * 4, [half] * 4, [half] * 4], np.float32)
    u = np.nextafter(np.float32(1), np.float32(0))
    selected, probability = runtime.light_tree_select(lo, hi, p, [[0, 0, 0]], [u])
    assert selected[0] == 2
    assert probability[0] == runtime.light_tree_probability(lo, hi, p, [[0, 0, 0]], [2])[0]


def test_large_balanced_distribution_is_exactly_normalized():
    """LightTreeTest.cpp:275-314: 1,024 equal unbounded lights give every light exactly 1/1024 and
    65,536 stratified samples select each light 64 times."""
    n = 1024
    lo = np.full((n, 3), -np.inf, np.float32)
    hi = np.full((n, 3), np.inf, np.float32)
    p = np.ones((n, 4), np.float32)
    where = np.tile(np.array([[17, -3, 9]], np.float32), (n, 1))
    probabilities = runtime.light_tree_probability(lo, hi, p, where, np.arange(n, dtype=np.uint32))
    assert (probabilities == np.float32(1) / np.float32(1024)).all()
    total = np.float32(0)
    for v in probabilities:
        total = np.float32(total + v)
    assert total == np.float32(1)
    samples = ((np.arange(65536, dtype=np.float32) + np.float32(0.5)) / np.float32(65536)).astype(np.float32)
    selected, selection = runtime.light_tree_select(lo, hi, p, np.tile(where[:1], (65536, 1)), samples)
    assert (selection == np.float32(1) / np.float32(1024)).all()
    assert (np.bincount(selected, minlength=n) == 64).all()


def test_oracle_tree_transport_matches_the_reference(golden):
    """The oracle selecting by the tree inside transport (NEE at the shading point, emission MIS at
    the previous vertex, every light's support checked at each shading point) against the
    reference's trace_scene_mis with LightSampler::create_spatial_tree on the three-light box
    (tests/golden/light_tree_transport.npz, `make_light_tree_golden.py transport`)."""
    from bf200 import abi
    from helpers import arrays, bit_equal
    from oracle.bindings import Oracle
    from test_gpu_light_power import path_inputs, three_light_box
    spec = importlib.util.spec_from_file_location(
        "make_light_tree_golden", os.path.join(os.path.dirname(__file__), "golden", "make_light_tree_golden.py"))
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    g = golden("light_tree_transport")
    builder = three_light_box()
    oracle = Oracle()
    inputs = path_inputs(oracle, 512, 23)
    h = oracle.scene(builder)
    oracle.set_light_tree(h, maker.tree_box_inputs(builder))
    results, failures = oracle.trace(h, inputs, abi.default_options(mis="power", max_depth=8))
    plain, _ = oracle.trace(h, inputs, abi.default_options(mis="power", max_depth=8))
    oracle.destroy(h)
    got = arrays(results)
    assert failures == 0 and (g["lane_status"] == 0).all()
    for key in ("radiance", "beta"):
        assert bit_equal(got[key], g[key]).all(), key
    for key in ("depth", "termination"):
        assert np.array_equal(got[key], g[key]), key
    # the tree changes the selection, so the radiance differs from uniform selection on most paths
    uniform = Oracle()
    h = uniform.scene(builder)
    base, _ = uniform.trace(h, inputs, abi.default_options(mis="power", max_depth=8))
    uniform.destroy(h)
    assert (~bit_equal(arrays(base)["radiance"], got["radiance"]).all(axis=1)).mean() > 0.3
    assert bit_equal(arrays(plain)["radiance"], got["radiance"]).all()
