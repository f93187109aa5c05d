"""The spatial light tree traversed on the device (bf200_light_tree_select_device) against the
reference's LightSampler::create_spatial_tree selections (tests/golden/light_tree.npz, made by
tests/golden/make_light_tree_golden.py from the compiled reference). The device rounds double
logarithms and exponentials to float where the reference calls the C library's float functions,
so probabilities agree to a relative 1e-5 and selections agree except where a sample lies within
that difference of a branch boundary."""
import numpy as np
import pytest

from bf200 import runtime

pytestmark = pytest.mark.gpu


def test_device_light_tree_matches_the_reference(golden):
    import torch
    g = golden("light_tree")
    total = agree = exact = 0
    for k in range(int(g["sets"])):
        lo, hi, p = g[f"lo_{k}"], g[f"hi_{k}"], g[f"powers_{k}"]
        positions = np.ascontiguousarray(g[f"positions_{k}"], np.float32)
        samples = np.ascontiguousarray(g[f"samples_{k}"], np.float32)
        n = len(samples)
        d_positions = torch.from_numpy(positions.reshape(-1)).cuda()
        d_samples = torch.from_numpy(samples).cuda()
        d_lights = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_probabilities = torch.zeros(n, dtype=torch.float32, device="cuda")
        runtime.light_tree_select_device(lo, hi, p, d_positions.data_ptr(), d_samples.data_ptr(), n,
                                         d_lights.data_ptr(), d_probabilities.data_ptr())
        torch.cuda.synchronize()
        lights = d_lights.cpu().numpy().view(np.uint32)
        probabilities = d_probabilities.cpu().numpy()
        want_lights, want_probabilities = g[f"selected_{k}"], g[f"probability_{k}"]
        same = lights == want_lights
        valid = same & (want_lights != 0xFFFFFFFF)
        relative = np.abs(probabilities.astype(np.float64) - want_probabilities) / np.maximum(
            np.abs(want_probabilities.astype(np.float64)), 1e-30)
        assert (relative[valid] <= 1e-5).all(), (k, float(relative[valid].max()))
        total += n
        agree += int(same.sum())
        exact += int((valid & (probabilities.view(np.uint32) == want_probabilities.view(np.uint32))).sum())
    assert agree >= 0.99 * total, (agree, total)
    print(f"light tree on the device: {agree}/{total} selections agree, {exact} probabilities bit-exact")


def test_tree_selected_paths_match_the_oracle():
    """Transport selecting lights by the tree (bf200_scene_set_light_tree) on the three-light box:
    per-path radiance against the oracle's tree transport, whose results are bit-exact against the
    reference's trace_scene_mis with the tree (tests/test_light_tree.py), with the tolerances of the
    other parity tests. Clearing the tree gives the uniform-selection render again, bit for bit."""
    import importlib.util
    import os
    from bf200 import abi
    from helpers import arrays, bit_equal, check_paths
    from oracle.bindings import Oracle
    from test_gpu_light_power import path_inputs, three_light_box
    spec = importlib.util.spec_from_file_location(
        "make_light_tree_golden", os.path.join(os.path.dirname(__file__), "golden", "make_light_tree_golden.py"))
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    builder = three_light_box()
    lights = maker.tree_box_inputs(builder)
    oracle = Oracle(device_trig=True)
    inputs = path_inputs(oracle, 4096, 31)
    options = abi.default_options(mis="power", max_depth=8)
    h = oracle.scene(builder)
    oracle.set_light_tree(h, lights)
    expected, failures = oracle.trace(h, inputs, options)
    oracle.destroy(h)
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        scene = ctx.create_scene(builder)
        uniform, _ = ctx.trace_paths(scene, inputs, options)
        scene.set_light_tree(lights)
        results, report = ctx.trace_paths(scene, inputs, options)
        scene.set_light_tree(None)
        again, _ = ctx.trace_paths(scene, inputs, options)
        scene.close()
    got, want = arrays(results), arrays(expected)
    assert failures == 0 and report.failed_lanes == 0
    # the device's rounded double logarithms and exponentials leave about 1 % of tree probabilities
    # an ulp from the C library's; a path evaluates several, so fewer paths are bit-exact than in the
    # CDF-selection tests, while all stay within the relative 1e-5 gate
    exact, close = check_paths(got, want, "light-tree selection")
    assert exact >= 0.8
    assert (~bit_equal(arrays(uniform)["radiance"], got["radiance"]).all(axis=1)).mean() > 0.3
    assert bit_equal(arrays(again)["radiance"], arrays(uniform)["radiance"]).all()


def test_repeated_tree_updates_keep_device_memory_flat():
    """A caller sets the tree again after every refit and may clear it in between: the scene reuses
    its tree buffers (or frees them when the tree is cleared), so free device memory after 50 such
    rounds is where the first tree left it."""
    import importlib.util
    import os
    import torch
    from test_gpu_light_power import three_light_box
    spec = importlib.util.spec_from_file_location(
        "make_light_tree_golden", os.path.join(os.path.dirname(__file__), "golden", "make_light_tree_golden.py"))
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    builder = three_light_box()
    lights = maker.tree_box_inputs(builder)
    with runtime.Context(0, path_capacity=1 << 12) as ctx:
        scene = ctx.create_scene(builder)
        scene.set_light_tree(lights)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        for _ in range(50):
            scene.set_light_tree(lights)
            scene.set_light_tree(None)
            scene.set_light_tree(lights)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        scene.close()
    assert free_after >= free_before - (2 << 20), f"{(free_before - free_after) >> 20} MiB lost"


def _tree_box():
    import importlib.util
    import os
    from test_gpu_light_power import three_light_box
    spec = importlib.util.spec_from_file_location(
        "make_light_tree_golden", os.path.join(os.path.dirname(__file__), "golden", "make_light_tree_golden.py"))
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    builder = three_light_box()
    return builder, maker.tree_box_inputs(builder)


def test_tree_selection_on_the_cone_path_and_after_a_refit():
    """With the tree set, the cone-carrying trace (its own shading instantiation) gives the plain
    trace's radiance on every lane both complete, and a refit followed by setting the tree again
    gives the plain trace's results bit for bit."""
    import numpy as np
    from bf200 import abi
    from helpers import arrays, bit_equal
    from oracle.bindings import Oracle
    from test_gpu_light_power import path_inputs
    builder, lights = _tree_box()
    inputs = path_inputs(Oracle(device_trig=True), 4096, 37)
    options = abi.default_options(mis="power", max_depth=8)
    cones = np.tile(np.array([[0.0, 1e-3]], np.float32), (len(inputs), 1))
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        scene = ctx.create_scene(builder)
        scene.set_light_tree(lights)
        plain, _ = ctx.trace_paths(scene, inputs, options)
        coned, _, report = ctx.trace_paths_with_cones(scene, inputs, cones, options)
        scene.refit(builder)
        scene.set_light_tree(lights)
        again, _ = ctx.trace_paths(scene, inputs, options)
        scene.close()
    p, c, a = arrays(plain), arrays(coned), arrays(again)
    both = (p["lane_status"] == 0) & (c["lane_status"] == 0)
    assert both.mean() > 0.99 and report.closure_samples > 0
    assert bit_equal(p["radiance"][both], c["radiance"][both]).all()
    assert bit_equal(p["radiance"], a["radiance"]).all() and (p["termination"] == a["termination"]).all()


def test_tree_film_equals_the_tree_trace():
    """A film rendered with the tree set equals, pixel for pixel within the parity tolerance, the
    film accumulated from the tree-selecting trace of the same (pixel, sample) paths (that trace is
    checked against the oracle's tree transport above)."""
    import os
    import numpy as np
    from bf200 import abi, scenes
    from helpers import DIVERGED_FRACTION, RELATIVE_TOLERANCE, arrays, relative_error, sensor_from_golden
    from oracle.bindings import Oracle
    builder, lights = _tree_box()
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell_spheres_256.npz"))
    sensor = sensor_from_golden(g)
    width, height, spp = 32, 32, 2
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    options = abi.default_options(mis="power", max_depth=8)
    px, py, s = np.meshgrid(np.arange(width), np.arange(height), np.arange(spp), indexing="ij")
    order = np.lexsort((px.ravel(), py.ravel(), s.ravel()))
    px, py, s = px.ravel()[order], py.ravel()[order], s.ravel()[order]
    samples = (abi.SampleIndex * len(px))()
    for k in range(len(px)):
        samples[k].pixel_x, samples[k].pixel_y, samples[k].sample_index = int(px[k]), int(py[k]), int(s[k])
    oracle = Oracle(device_trig=True)
    rays = oracle.camera_rays(cam, samples)
    inputs = (abi.PathInput * len(px))()
    for k in range(len(px)):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        scene = ctx.create_scene(builder)
        scene.set_light_tree(lights)
        sums, counts, _ = ctx.render_film(scene, cam, sensor, options, spp, seed=0)
        results, _ = ctx.trace_paths(scene, inputs, options)
        scene.close()
    expected, _ = oracle.film(arrays(results)["radiance"], samples, sensor, width, height, 0)
    assert (counts == spp).all()
    err = relative_error(sums.astype(np.float64), expected)
    assert (err <= RELATIVE_TOLERANCE).mean() >= 1.0 - DIVERGED_FRACTION
