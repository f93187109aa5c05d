"""The C++ adapter (blackframe-renderer_b200/adapter/WavefrontTransport.cpp) compiles against the
reference's own headers: it defines the CudaWavefrontTransportWorkspace members and both
trace_cuda_wavefront_transport overloads that WavefrontTransport.hpp declares, so a Blackframe
build can link it in place of its CUDA WavefrontTransport.cpp. Needs the reference tree (the
BLACKFRAME_REFERENCE environment variable, default /root/reference) and g++ with C++23; skipped
where either is absent. CPU only: nothing is run."""
import os
import re
import shutil
import subprocess

import pytest

REFERENCE = os.environ.get("BLACKFRAME_REFERENCE", "/root/reference")
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
