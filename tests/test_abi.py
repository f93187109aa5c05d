"""The C-ABI boundary on the CPU: the library loads, exports what include/bf200.h declares,
answers the Blackframe extension / XPU queries like a plugin must, and its records have the
header's layouts. No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from bf200 import abi, runtime, scenes
from helpers import bit_equal


def declared_symbols(repo_root):
    text = open(os.path.join(repo_root, "include", "bf200.h")).read()
    names = set(re.findall(r"BF200_EXPORT\s+[\w\s\*]+?\b((?:bf200|blackframe)_\w+)\s*\(", text))
    names |= set(re.findall(r"BF200_EXPORT blackframe_status\s*\n\s*(blackframe_\w+)\(", text))
    return names


def test_library_exports_every_declared_symbol(repo_root):
    lib = runtime.library()
    declared = declared_symbols(repo_root)
    assert "blackframe_query_extension" in declared and "bf200_trace_paths" in declared
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/bf200.h but not exported"
    assert set(runtime.EXPORTED_SYMBOLS) <= declared


def test_record_layouts_match_the_header(repo_root, tmp_path):
    abi.check_layouts()
    probe = tmp_path / "layout.c"
    names = ["bf200_closure_v1", "bf200_material_v1", "bf200_geometry_v1", "bf200_instance_v1",
             "bf200_ray_v1", "bf200_sample_index_v1", "bf200_path_input_v1", "bf200_path_result_v1",
             "bf200_transport_options_v1", "bf200_camera_v1", "bf200_sensor_v1",
             "bf200_film_request_v1", "bf200_report_v1", "bf200_hit_v1", "blackframe_extension_api_v1",
             "blackframe_xpu_device_descriptor_v1", "bf200_scene_desc_v1", "bf200_film_v1", "bf200_ray_cone_v1", "bf200_path_state_v1",
             "bf200_light_tree_input_v1", "bf200_scene_json_limits_v1", "bf200_scene_json_frame_v1",
             "bf200_scene_stats_v1"]
    body = "".join(f'printf("%zu\\n", sizeof({n}));' for n in names)
    probe.write_text(f'#include "bf200.h"\n#include <stdio.h>\nint main(void){{{body}return 0;}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(repo_root, "include"), str(probe), "-o", str(exe)],
                   check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    records = [abi.Closure, abi.Material, abi.Geometry, abi.Instance, abi.Ray, abi.SampleIndex, abi.PathInput,
               abi.PathResult, abi.TransportOptions, abi.Camera, abi.Sensor, abi.FilmRequest, abi.Report, abi.Hit,
               abi.ExtensionApi, abi.XpuDeviceDescriptor, abi.SceneDesc, abi.Film, abi.RayCone, abi.PathState, abi.LightTreeInput,
               abi.SceneJsonLimits, abi.SceneJsonFrame, abi.SceneStats]
    assert sizes == [C.sizeof(r) for r in records]


def test_extension_query_and_interfaces():
    lib = runtime.library()
    status, api = runtime.query_extension()
    assert status == 0 and api.abi_major == 1 and api.reserved == 0
    assert api.struct_size == C.sizeof(abi.ExtensionApi)
    # XPU v1 (XpuBackend.cpp:57-100)
    xpu = abi.XpuBackendApi()
    xpu.struct_size = C.sizeof(abi.XpuBackendApi)
    xpu_id = abi.InterfaceId(0x96C6E70DD06B4B93, 0xA9514AB777F49D37)
    assert api.get_interface(None, xpu_id, 1, 0, C.cast(C.byref(xpu), C.c_void_p), C.sizeof(xpu)) == 0
    assert xpu.abi_major == 1 and xpu.reserved == 0 and xpu.backend_name.size > 0
    count = abi.u32(99)
    assert xpu.get_device_count(None, C.byref(count)) == 0
    descriptor = abi.XpuDeviceDescriptor()
    descriptor.struct_size = C.sizeof(descriptor)
    assert xpu.get_device_descriptor(None, count.value, C.byref(descriptor)) == 5  # OUT_OF_RANGE
    # render interface
    render = (C.c_uint8 * 256)()
    render_id = abi.InterfaceId(0x6266323030726E64, 0x7761766566726E31)
    assert api.get_interface(None, render_id, 1, 0, C.cast(render, C.c_void_p), 256) == 0
    header = np.frombuffer(bytes(render[:16]), np.uint32)
    assert header[0] == 120 and header[1] == 1 and header[2] == 1
    # nine v1.0 entry points, the two of minor 1 (SoA scenes, cones and initial states), two zeros
    slots = np.frombuffer(bytes(render[16:120]), np.uint64)
    assert (slots[:11] != 0).all() and (slots[11:] == 0).all()
    # errors: unknown id, wrong major, short output
    assert api.get_interface(None, abi.InterfaceId(1, 2), 1, 0, C.cast(render, C.c_void_p), 256) == 3
    assert api.get_interface(None, render_id, 2, 0, C.cast(render, C.c_void_p), 256) == 2
    assert api.get_interface(None, xpu_id, 1, 0, C.cast(render, C.c_void_p), 8) == 1
    bad = abi.ExtensionQuery(C.sizeof(abi.ExtensionQuery), 2, 0, 0)
    out = abi.ExtensionApi()
    out.struct_size = C.sizeof(out)
    assert lib.blackframe_query_extension(C.byref(bad), C.byref(out)) == 2


@pytest.mark.parametrize("name", ["cornell_plain_64", "cornell_spheres_256"])
def test_camera_create_matches_reference_camera(golden, name):
    g = golden(name)
    _, _, (width, height, _) = scenes.build_workload(name)
    origin, normal, tangent = scenes.camera_frame_inputs()
    cam = runtime.camera_create(origin, normal, tangent, width, height, scenes.CAMERA_VFOV, scenes.PATH_TIME)
    mine = np.array(list(cam.origin) + list(cam.tangent) + list(cam.bitangent) + list(cam.normal) +
                    [cam.half_width, cam.half_height], np.float32)
    assert bit_equal(mine, g["camera"]).all()


def test_invalid_arguments_are_rejected_without_a_device():
    lib = runtime.library()
    handle = C.c_void_p()
    assert lib.bf200_context_create(-1, 0, C.byref(handle)) == 5
    assert lib.bf200_trace_paths(None, None, None, 1, None, None, None) == 1
    assert lib.bf200_context_destroy(None) == 1
    # the cone and initial-state entry points: null arrays are refused before any device work
    assert lib.bf200_trace_paths_with_cones(None, None, None, None, None, 1, None, None, None, None) == 1
    assert lib.bf200_trace_paths_with_cones_device(None, None, None, None, None, 1, None, None, None, None) == 1
