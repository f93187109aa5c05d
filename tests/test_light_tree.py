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
