"""Ray cones and initial path states through the device wavefront (bf200_trace_paths_with_cones*).

* Paths of the Cornell box with its conductor and dielectric spheres, started with the reference
  camera's own primary cones (tests/golden/cones.npz, PinholeCamera::generate_primary_ray_cone):
  every terminal cone matches the oracle's restatement of the reference wavefront's cone
  propagation bit for bit on paths whose radiance is bit-exact, and within the parity tolerance on
  the rest; lane failures match.
* Carrying cones changes no path: results equal bf200_trace_paths bit for bit on every lane the
  cones do not fail.
* Invalid primary cones: refused for the whole host call (INVALID_ARGUMENT), failed per lane in
  the device call.
* Depth-zero initial states other than PathState::create_initial: device paths vs the oracle
  (whose results are pinned on the reference by tests/test_initial_states.py).
"""
import ctypes as C

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import arrays, bit_equal, check_paths, relative_error, RELATIVE_TOLERANCE
from oracle.bindings import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with runtime.Context(0, path_capacity=1 << 16) as c:
        yield c


@pytest.fixture(scope="module")
def workload(golden):
    """The Cornell box with a rough conductor and a rough dielectric sphere, 4096 primary paths of
    the reference camera with the reference camera's cones."""
    g = golden("cones")
    builder, options, (width, height, _) = scenes.build_workload("cornell_spheres_256")
    table = g["camera_samples"]
    n = len(table)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    rays = Oracle(device_trig=True).camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return builder, options, inputs, g["camera_cones"]


def terminal_rays(results):
    return np.array([list(r.terminal_ray.origin) + list(r.terminal_ray.direction) for r in results], np.float32)


def same_paths(results, expected, got, want):
    """Paths with bit-identical radiance, throughput, depth and terminal ray."""
    return (bit_equal(got["radiance"], want["radiance"]).all(axis=1) & bit_equal(got["beta"], want["beta"]).all(
        axis=1) & (got["depth"] == want["depth"]) &
            bit_equal(terminal_rays(results), terminal_rays(expected)).all(axis=1))


def test_terminal_cones_match_the_oracle(ctx, workload):
    builder, options, inputs, cones = workload
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    expected, expected_cones, failures = oracle.trace_cones(handle, inputs, cones, options)
    oracle.destroy(handle)
    scene = ctx.create_scene(builder)
    results, got_cones, report = ctx.trace_paths_with_cones(scene, inputs, cones, options)
    scene.close()
    got, want = arrays(results), arrays(expected)
    failed = want["lane_status"] != 0
    assert (got["lane_status"] != 0).sum() == report.failed_lanes
    assert np.array_equal(got["lane_status"] != 0, failed), np.nonzero((got["lane_status"] != 0) != failed)[0][:10]
    keep = ~failed
    exact, close = check_paths({k: v[keep] for k, v in got.items()}, {k: v[keep] for k, v in want.items()},
                               "cornell_spheres_256 with cones")
    assert exact >= 0.95
    # A path whose radiance, throughput and depth are bit-identical may still have taken a direction
    # one ulp apart at an earlier bounce (the sine/cosine rounding of the parity tolerance): a
    # Lambertian throughput does not depend on it, but the next hit distance, and so the cone, does.
    # Identical paths are therefore those whose terminal rays are identical too.
    same_path = same_paths(results, expected, got, want) & keep
    cone_equal = bit_equal(got_cones, expected_cones).all(axis=1)
    assert same_path.mean() >= 0.99
    assert cone_equal[same_path].all(), np.nonzero(same_path & ~cone_equal)[0][:10]
    near = (relative_error(got_cones, expected_cones) <= RELATIVE_TOLERANCE).all(axis=1)
    assert near[keep].all()
    # the reference's stage counts (CudaWavefrontStageLaneCounts): every extension segment is a
    # camera ray or a continuation, each hit or missed, and every shaded lane drew a closure sample
    # and (with lights and a non-black closure) a light sample
    n = len(inputs)
    assert report.terminated_paths == n - report.failed_lanes
    if report.failed_lanes == 0:
        assert report.extension_segments == n + report.continuation_segments
    assert 0 < report.miss_segments < report.extension_segments
    hits = report.extension_segments - report.miss_segments
    assert report.continuation_segments <= report.closure_samples <= hits
    assert report.shadow_segments <= report.light_samples <= report.closure_samples
    assert report.light_samples > report.shadow_segments > 0
    # the cones grew: every path that scattered left with a spread of at least the smallest policy
    scattered = keep & (got["depth"] > 0)
    assert scattered.sum() > 1000 and (got_cones[scattered, 1] >= 0.05).all()
    assert (got_cones[scattered, 0] > 0.0).all()


def test_cones_change_no_path(ctx, workload):
    builder, options, inputs, cones = workload
    scene = ctx.create_scene(builder)
    plain, _ = ctx.trace_paths(scene, inputs, options)
    coned, _, _ = ctx.trace_paths_with_cones(scene, inputs, cones, options)
    scene.close()
    a, b = arrays(plain), arrays(coned)
    keep = b["lane_status"] == 0
    assert keep.mean() > 0.99
    for key in ("radiance", "beta", "eta"):
        assert bit_equal(a[key][keep], b[key][keep]).all(), key
    for key in ("depth", "termination", "lane_status"):
        assert np.array_equal(a[key][keep], b[key][keep]), key
    for k in np.nonzero(keep)[0][:256]:
        assert bytes(plain[k]) == bytes(coned[k])


def test_invalid_primary_cones(ctx, workload):
    import torch
    builder, options, inputs, cones = workload
    scene = ctx.create_scene(builder)
    n = 64
    sub = (abi.PathInput * n)(*inputs[:n])
    for bad in ((np.nan, 0.001), (0.0, -1.0), (np.inf, 0.0)):
        c = np.array(cones[:n], np.float32)
        c[7] = bad
        with pytest.raises(runtime.Bf200Error) as info:
            ctx.trace_paths_with_cones(scene, sub, c, options)
        assert info.value.status == 1  # INVALID_ARGUMENT, for the whole call
    # device inputs: the lane with the invalid cone fails, the others are traced
    c = np.array(cones[:n], np.float32)
    c[7] = (np.nan, 0.001)
    raw = np.frombuffer(bytes(sub), np.uint8)
    d_in = torch.from_numpy(raw.copy()).cuda()
    d_cones = torch.from_numpy(c.reshape(-1)).cuda()
    d_out = torch.zeros(n * C.sizeof(abi.PathResult), dtype=torch.uint8, device="cuda")
    d_terminal = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
    report = ctx.trace_paths_with_cones_device(scene, d_in.data_ptr(), d_cones.data_ptr(), n, options,
                                               d_out.data_ptr(), d_terminal.data_ptr())
    torch.cuda.synchronize()
    results = (abi.PathResult * n).from_buffer_copy(d_out.cpu().numpy().tobytes())
    host, host_cones, _ = ctx.trace_paths_with_cones(scene, sub, np.where(np.isnan(c), 0.0, c), options)
    scene.close()
    status = np.array([r.lane_status for r in results])
    assert status[7] == 1 and report.failed_lanes == 1  # BF200_LANE_NUMERICAL_FAILURE
    others = np.arange(n) != 7
    assert (status[others] == 0).all()
    for k in np.nonzero(others)[0]:
        assert bytes(results[k]) == bytes(host[k])
    assert np.array_equal(d_terminal.cpu().numpy().reshape(n, 2)[others].view(np.uint32),
                          host_cones[others].view(np.uint32))


def test_initial_states_match_the_oracle(ctx, golden):
    """Depth-zero initial states other than PathState::create_initial (zero and 1e30 throughput,
    accumulated radiance, eta scales other than 1; tests/golden/initial_states.npz, whose oracle
    results are pinned on the reference by tests/test_initial_states.py): device paths against the
    oracle, with the parity tolerances, and the same lane failures."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "make_state_golden", os.path.join(os.path.dirname(__file__), "golden", "make_state_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    g = golden("initial_states")
    builder, options, (width, height, _) = scenes.build_workload(m.WORKLOAD)
    table = g["samples"]
    samples = (abi.SampleIndex * len(table))()
    for k in range(len(table)):
        samples[k].pixel_x, samples[k].pixel_y = int(table[k, 0]), int(table[k, 1])
        samples[k].sample_index, samples[k].seed = int(table[k, 2]), int(table[k, 3])
    inputs = m.inputs_for(samples, width, height)
    states = m.states_from(g["beta_in"], g["radiance_in"], g["eta_in"])
    cones = np.tile(np.array([0.0, 0.0025], np.float32), (len(table), 1))
    oracle = Oracle(device_trig=True)
    handle = oracle.scene(builder)
    expected, expected_cones, _ = oracle.trace_cones(handle, inputs, cones, options, states=states)
    oracle.destroy(handle)
    scene = ctx.create_scene(builder)
    results, got_cones, report = ctx.trace_paths_with_cones(scene, inputs, cones, options, states=states)
    scene.close()
    got, want = arrays(results), arrays(expected)
    assert np.array_equal(got["lane_status"] != 0, want["lane_status"] != 0)
    keep = want["lane_status"] == 0
    exact, close = check_paths({k: v[keep] for k, v in got.items()}, {k: v[keep] for k, v in want.items()},
                               "initial states")
    assert exact >= 0.95
    zero = (g["beta_in"] == 0.0).all(axis=1)
    assert (got["depth"][zero] == 0).all() and set(got["termination"][zero].tolist()) <= {0, 3}
    same_path = same_paths(results, expected, got, want) & keep
    assert bit_equal(got_cones, expected_cones).all(axis=1)[same_path].mean() >= 0.999
    assert (relative_error(got_cones, expected_cones) <= RELATIVE_TOLERANCE).all(axis=1)[same_path].all()
    # invalid states: refused for the whole host call
    bad = m.states_from(g["beta_in"][:4], g["radiance_in"][:4], g["eta_in"][:4])
    bad[2].eta_scale = 0.0
    scene = ctx.create_scene(builder)
    sub = (abi.PathInput * 4)(*inputs[:4])
    with pytest.raises(runtime.Bf200Error) as info:
        ctx.trace_paths_with_cones(scene, sub, cones[:4], options, states=bad)
    scene.close()
    assert info.value.status == 1
