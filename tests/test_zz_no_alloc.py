"""The allocation-free entry point, bf200_trace_paths_device_noalloc, against the ordinary device
entry point, bf200_trace_paths_device.

Both trace the same device inputs. Two allocation-free calls in a row must each return result
records byte-identical to the ordinary call's. The output buffers are poisoned before every call,
so a record the call failed to write shows up as a difference. The file name makes pytest collect
it last. It passes run alone and after every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from bf200 import abi, runtime, scenes

pytestmark = pytest.mark.gpu

RESULT_BYTES = C.sizeof(abi.PathResult)


def _inputs(name, n, seed):
    from oracle.bindings import Oracle

    _, _, (width, height, spp) = scenes.build_workload(name)
    rng = np.random.default_rng(seed)
    cam = runtime.camera_create(*scenes.camera_frame_inputs(), width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    samples = (abi.SampleIndex * n)()
    for k in range(n):
        samples[k].pixel_x, samples[k].pixel_y = int(rng.integers(width)), int(rng.integers(height))
        samples[k].sample_index, samples[k].seed = int(rng.integers(spp)), 0
    rays = Oracle(device_trig=True).camera_rays(cam, samples)
    inputs = (abi.PathInput * n)()
    for k in range(n):
        inputs[k].primary_ray, inputs[k].sample = rays[k], samples[k]
    return inputs


@pytest.mark.parametrize("name,capacity", [("cornell_spheres_256", 4096), ("cornell_plain_64", 0)])
def test_noalloc_matches_device_entry_point_on_two_calls(name, capacity):
    import torch

    builder, options, _ = scenes.build_workload(name)
    n = 20000
    host_inputs = np.frombuffer(_inputs(name, n, seed=91), np.uint8).copy()
    with runtime.Context(0, path_capacity=1 << 16) as ctx:
        scene = ctx.create_scene(builder)
        d_in = torch.from_numpy(host_inputs).cuda()
        reference = torch.full((n * RESULT_BYTES,), 0xAB, dtype=torch.uint8, device="cuda")
        ref_report = ctx.trace_paths_device(scene, d_in.data_ptr(), n, options, reference.data_ptr())
        torch.cuda.synchronize()
        expected = reference.cpu().numpy()
        assert ref_report.failed_lanes == 0
        for call in range(2):
            out = torch.full((n * RESULT_BYTES,), 0x5C + call, dtype=torch.uint8, device="cuda")
            report = ctx.trace_paths_device_noalloc(scene, d_in.data_ptr(), n, options, out.data_ptr(),
                                                   path_capacity=capacity)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert report.path_count == n and report.failed_lanes == 0
            assert report.extension_segments == ref_report.extension_segments
            assert report.shadow_segments == ref_report.shadow_segments
            differing = np.nonzero((got != expected).reshape(n, RESULT_BYTES).any(axis=1))[0]
            assert differing.size == 0, f"call {call}: {differing.size} records differ, first {differing[:8]}"
        scene.close()


def test_noalloc_rejects_capacity_above_the_scratch_limit():
    import torch

    builder, options, _ = scenes.build_workload("cornell_plain_64")
    host_inputs = np.frombuffer(_inputs("cornell_plain_64", 16, seed=3), np.uint8).copy()
    with runtime.Context(0, path_capacity=1 << 12) as ctx:
        scene = ctx.create_scene(builder)
        d_in = torch.from_numpy(host_inputs).cuda()
        out = torch.zeros(16 * RESULT_BYTES, dtype=torch.uint8, device="cuda")
        with pytest.raises(runtime.Bf200Error) as info:
            ctx.trace_paths_device_noalloc(scene, d_in.data_ptr(), 16, options, out.data_ptr(),
                                           path_capacity=65537)
        assert info.value.status == 5  # OUT_OF_RANGE
        assert "65536 slots" in str(info.value)
        scene.close()
