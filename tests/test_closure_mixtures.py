"""Closure mixtures, the energy-preserving Oren-Nayar and specular closures, and punctual lights:
the oracle restatement against the reference's own trace_scene_mis on the cornell_layered_256
workload (tests/golden/layered.npz, made by tests/golden/make_layered_golden.py from the compiled
reference), bit for bit on every output of every path; and on fresh paths against the live
reference where it is built. CPU only."""
import importlib.util
import os

import numpy as np
import pytest

from bf200 import abi, scenes
from helpers import arrays, bit_equal
from oracle.bindings import Oracle, Reference, reference_available

HERE = os.path.dirname(os.path.abspath(__file__))


def maker():
    spec = importlib.util.spec_from_file_location("make_layered_golden",
                                                  os.path.join(HERE, "golden", "make_layered_golden.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def oracle_inputs(table):
    """The fixture's paths with primary rays of the oracle's camera (bit-exact with the
    reference camera, tests/test_oracle_golden.py)."""
    from bf200 import runtime
    _, _, (width, height, _) = scenes.build_workload("cornell_layered_256")
    n = len(table)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    rays = Oracle().camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return inputs


def compare(results, want, label):
    got = arrays(results)
    assert np.array_equal(got["lane_status"] != 0, want["lane_status"] != 0), label
    keep = want["lane_status"] == 0
    for key in ("radiance", "beta", "eta"):
        same = bit_equal(got[key][keep], want[key][keep])
        same = same.all(axis=1) if same.ndim > 1 else same
        assert same.all(), (label, key, np.nonzero(keep)[0][~same][:10])
    for key in ("depth", "termination"):
        assert np.array_equal(got[key][keep], want[key][keep]), (label, key)
    counters = np.array([list(r.depth_counters) for r in results], np.uint32)
    flags = np.array([r.delta_flags for r in results], np.uint32)
    assert np.array_equal(counters[keep], want["depth_counters"][keep]), label
    assert np.array_equal(flags[keep], want["delta_flags"][keep]), label
    terminal = np.array([list(r.terminal_ray.origin) + list(r.terminal_ray.direction) for r in results], np.float32)
    assert bit_equal(terminal[keep], want["terminal"][keep]).all(), label


def test_oracle_matches_the_reference_fixture(golden):
    g = golden("layered")
    builder, options, _ = scenes.build_workload("cornell_layered_256")
    oracle = Oracle()
    handle = oracle.scene(builder)
    results, failures = oracle.trace(handle, oracle_inputs(g["samples"]), options)
    oracle.destroy(handle)
    assert failures == int((g["lane_status"] != 0).sum())
    compare(results, g, "fixture")
    # the fixture exercises what it is for: specular chains, glossy and diffuse bounces, deep paths
    assert (g["depth_counters"][:, 2] > 0).sum() > 50 and (g["depth_counters"][:, 1] > 0).sum() > 50
    assert ((g["delta_flags"] & 1) != 0).sum() > 10 and (g["radiance"] > 0).any(axis=1).mean() > 0.5


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
def test_oracle_matches_the_reference_on_fresh_paths():
    m = maker()
    builder, options, (width, height, spp) = scenes.build_workload("cornell_layered_256")
    table = m.sample_table(np.random.default_rng(7), 96, width, height, spp)
    reference = Reference()
    inputs = m.inputs_from(reference, table)
    handle = reference.scene(builder)
    expected, _ = reference.trace(handle, inputs, options)
    reference.destroy(handle)
    want = arrays(expected)
    want["depth_counters"] = np.array([list(r.depth_counters) for r in expected], np.uint32)
    want["delta_flags"] = np.array([r.delta_flags for r in expected], np.uint32)
    want["terminal"] = m.terminal(expected)
    oracle = Oracle()
    handle = oracle.scene(builder)
    results, _ = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    compare(results, want, "fresh")
