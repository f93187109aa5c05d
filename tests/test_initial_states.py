"""Paths started from depth-zero PathStates other than PathState::create_initial: the oracle
against the reference's own trace_scene_mis (tests/golden/initial_states.npz, made by
tests/golden/make_state_golden.py from the compiled reference), bit for bit: zero throughput, a
1e30 throughput, seeded throughputs with radiance already accumulated and eta scales other than
1, one dark lane, and the initial state itself. CPU only."""
import importlib.util
import os

import numpy as np
import pytest

from bf200 import abi, scenes
from helpers import arrays, bit_equal
from oracle.bindings import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def maker():
    spec = importlib.util.spec_from_file_location("make_state_golden",
                                                  os.path.join(HERE, "golden", "make_state_golden.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def samples_from(table):
    samples = (abi.SampleIndex * len(table))()
    for k in range(len(table)):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    return samples


def test_oracle_initial_states_match_the_reference(golden):
    g = golden("initial_states")
    m = maker()
    builder, options, (width, height, _) = scenes.build_workload(m.WORKLOAD)
    inputs = m.inputs_for(samples_from(g["samples"]), width, height)
    states = m.states_from(g["beta_in"], g["radiance_in"], g["eta_in"])
    oracle = Oracle()
    handle = oracle.scene(builder)
    cones = np.zeros((len(inputs), 2), np.float32)
    results, _, failures = oracle.trace_cones(handle, inputs, cones, options, states=states)
    plain, _ = oracle.trace(handle, inputs, options)
    oracle.destroy(handle)
    got = arrays(results)
    assert failures == int((g["lane_status"] != 0).sum())
    assert np.array_equal(got["lane_status"], g["lane_status"])
    for key in ("radiance", "beta", "eta"):
        assert bit_equal(got[key], g[key]).all(), (key, np.nonzero(~bit_equal(got[key], g[key]).all(axis=-1)
                                                                     if got[key].ndim > 1 else
                                                                     ~bit_equal(got[key], g[key]))[0][:10])
    for key in ("depth", "termination"):
        assert np.array_equal(got[key], g[key]), key
    # the zero-throughput paths end at their first hit (or escape) without any sampled bounce
    zero = (g["beta_in"] == 0.0).all(axis=1)
    assert zero.sum() > 100 and (got["depth"][zero] == 0).all()
    assert set(got["termination"][zero].tolist()) <= {0, 3}
    # paths that start from the initial state are the plain trace's paths
    initial = (g["beta_in"] == 1.0).all(axis=1) & (g["radiance_in"] == 0.0).all(axis=1) & (g["eta_in"] == 1.0)
    assert initial.sum() > 100
    base = arrays(plain)
    assert bit_equal(got["radiance"][initial], base["radiance"][initial]).all()


def test_invalid_initial_states_fail_the_oracle_lane():
    m = maker()
    builder, options, (width, height, _) = scenes.build_workload(m.WORKLOAD)
    table = np.array([[10, 10, 3, 0], [20, 20, 4, 0], [30, 30, 5, 0]], np.uint64)
    inputs = m.inputs_for(samples_from(table), width, height)
    beta = np.array([[1, 1, 1, 1], [-1, 1, 1, 1], [1, 1, 1, 1]], np.float32)
    radiance = np.zeros((3, 4), np.float32)
    eta = np.array([1.0, 1.0, 0.0], np.float32)
    oracle = Oracle()
    handle = oracle.scene(builder)
    results, _, failures = oracle.trace_cones(handle, inputs, np.zeros((3, 2), np.float32), options,
                                              states=m.states_from(beta, radiance, eta))
    oracle.destroy(handle)
    assert failures == 2 and [r.lane_status for r in results] == [0, 1, 1]
