"""The C++ adapter (blackframe-renderer_b200/adapter/WavefrontTransport.cpp) against the reference's
own headers and CPU libraries:
* it compiles, defining the CudaWavefrontTransportWorkspace members and both
  trace_cuda_wavefront_transport overloads that WavefrontTransport.hpp declares, so a Blackframe
  build can link it in place of its CUDA WavefrontTransport.cpp;
* its own logic (tests/adapter_probe.cpp, linked with the compiled reference libraries): the
  reference's preflight codes and messages, the light-sampler checks, the status and termination
  mappings, and workspace creation.
Needs the reference tree (the BLACKFRAME_REFERENCE environment variable, or the checkout path of
the build machine below), g++ with C++23 and, for the probe, oracle/_ref/libbfref.so; skipped where
they are absent. No GPU work is done."""
import os
import re
import shutil
import subprocess

import pytest

from bf200.build import reference_root

REFERENCE = reference_root() or ""
ROOTS = ["Core/Include", "Renderer/Include", "Engine/Include", "XPU/CUDA/Host/Include", "XPU/Shared/Include",
         "XPU/CUDA/Include", "Backends/GPU/CUDA/Include"]


def compile_adapter(repo_root, tmp_path):
    blackframe = os.path.join(REFERENCE, "Blackframe")
    if not os.path.isdir(blackframe) or shutil.which("g++") is None:
        pytest.skip("the reference tree or g++ is not available")
    cuda_include = "/usr/local/cuda/include"
    if not os.path.exists(os.path.join(cuda_include, "cuda_runtime_api.h")):
        pytest.skip("the CUDA headers are not available")
    source = os.path.join(repo_root, "blackframe-renderer_b200", "adapter", "WavefrontTransport.cpp")
    obj = tmp_path / "WavefrontTransport.o"
    cmd = (["g++", "-std=c++23", "-O1", "-Wall", "-Wextra", "-Werror", "-c", source, "-o", str(obj)] +
           [f"-I{os.path.join(blackframe, root)}" for root in ROOTS] +
           [f"-I{cuda_include}", f"-I{os.path.join(repo_root, 'include')}"])
    done = subprocess.run(cmd, capture_output=True, text=True)
    assert done.returncode == 0, done.stderr[-4000:]
    return obj


def test_adapter_compiles_against_the_reference_headers(repo_root, tmp_path):
    obj = compile_adapter(repo_root, tmp_path)
    symbols = subprocess.run(["nm", "-C", "--defined-only", str(obj)], capture_output=True, text=True,
                             check=True).stdout
    # every member of the reference interface is defined here
    for name in ["blackframe::engine::trace_cuda_wavefront_transport(blackframe::engine::CudaWavefrontTransportWorkspace&",
                 "blackframe::engine::trace_cuda_wavefront_transport(blackframe::engine::CudaSceneSoA const&",
                 "blackframe::engine::CudaWavefrontTransportWorkspace::create(",
                 "blackframe::engine::CudaWavefrontTransportWorkspace::close()",
                 "blackframe::engine::CudaWavefrontTransportWorkspace::capacity() const",
                 "blackframe::engine::CudaWavefrontTransportWorkspace::device_ordinal() const",
                 "blackframe::engine::CudaWavefrontTransportWorkspace::~CudaWavefrontTransportWorkspace()",
                 "blackframe::engine::CudaWavefrontTransportWorkspace::CudaWavefrontTransportWorkspace("]:
        assert name in symbols, name
    # and it calls through the C ABI only
    undefined = subprocess.run(["nm", "-u", str(obj)], capture_output=True, text=True, check=True).stdout
    called = set(re.findall(r"\b(bf200_\w+)", undefined))
    assert {"bf200_context_create", "bf200_context_destroy", "bf200_scene_create_from_soa", "bf200_scene_destroy",
            "bf200_trace_paths_with_cones"} <= called


def test_adapter_logic_against_the_reference_libraries(repo_root, tmp_path):
    blackframe = os.path.join(REFERENCE, "Blackframe")
    ref_lib = os.path.join(repo_root, "oracle", "_ref")
    bf_lib = os.path.join(repo_root, "blackframe-renderer_b200", "bf200")
    cuda_lib = "/usr/local/cuda/lib64"
    if (not os.path.isdir(blackframe) or shutil.which("g++") is None or
            not os.path.exists(os.path.join(ref_lib, "libbfref.so")) or
            not os.path.exists(os.path.join(cuda_lib, "libcudart.so"))):
        pytest.skip("the reference tree, its compiled libraries or the CUDA runtime is not available")
    exe = tmp_path / "adapter_probe"
    cmd = (["g++", "-std=c++23", "-O1", "-Wall", "-Wextra", os.path.join(repo_root, "tests", "adapter_probe.cpp"),
            "-o", str(exe)] + [f"-I{os.path.join(blackframe, root)}" for root in ROOTS] +
           ["-I/usr/local/cuda/include", f"-I{os.path.join(repo_root, 'include')}", f"-L{ref_lib}", "-lbfref",
            f"-L{bf_lib}", "-lbf200", f"-L{cuda_lib}", "-lcudart", f"-Wl,-rpath,{ref_lib}:{bf_lib}:{cuda_lib}"])
    built = subprocess.run(cmd, capture_output=True, text=True)
    assert built.returncode == 0, built.stderr[-4000:]
    ran = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert ran.returncode == 0, ran.stdout + ran.stderr
    assert ran.stdout.count("ok ") >= 16 and "FAIL" not in ran.stdout
