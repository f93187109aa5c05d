"""Builds the in-tree shared libraries.

* bf200/libbf200.so : the product — host runtime + sm_100a kernels (nvcc, -gencode
  arch=compute_100a,code=sm_100a, no FMA contraction so float arithmetic keeps the reference's
  operation order).
* oracle/liboracle.so, oracle/_ref/libbfref.so : the CPU checkers (oracle/Makefile); the second
  only when the reference tree is available to compile from.
"""
import os
import shutil
import subprocess
import sys

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(PACKAGE_DIR), "csrc")
REPO = os.path.dirname(os.path.dirname(PACKAGE_DIR))
INCLUDE = os.path.join(REPO, "include")
LIBRARY = os.path.join(PACKAGE_DIR, "libbf200.so")
SOURCES = ["bf200_kernels.cu", "bf200_shade_plain.cu", "bf200_shade_cone.cu", "bf200_shade_tree.cu",
           "bf200_shade_cone_tree.cu", "bf200_shade_adjoint.cu", "bf200_compact.cu", "bf200_sobol.cu", "bf200_host.cu", "bf200_import.cpp", "bf200_soa.cpp", "bf200_light_tree.cpp", "bf200_light_tree.cu",
           "bf200_envmap.cpp", "bf200_envmap.cu", "bf200_records.cpp", "bf200_scene_json.cpp", "bf200_lbvh.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-std=c++17", "-O3", "-lineinfo", "-fmad=false",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
    "-shared",
]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build bf200")
    return path


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    mtime = os.path.getmtime(target)
    return any(os.path.getmtime(p) > mtime for p in inputs)


def build_library(force=False, verbose=False):
    """Compiles every translation unit to an object under _build/ (in parallel, one nvcc per
    source; the units share no device symbols, so this is the same program as one nvcc call over
    all of them) and links the shared library."""
    from concurrent.futures import ThreadPoolExecutor

    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "bf200.h")]
    if not force and not _stale(LIBRARY, deps):
        return LIBRARY
    objdir = os.path.join(REPO, "_build", "bf200")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    headers = [p for p in deps if not p.endswith((".cu", ".cpp"))]

    def compile_one(source):
        src = os.path.join(CSRC, source)
        obj = os.path.join(objdir, source + ".o")
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc()] + compile_flags + ["-I" + INCLUDE, "-I" + CSRC, "-c", "-o", obj, src]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objects = list(pool.map(compile_one, SOURCES))
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIBRARY] + objects
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIBRARY


# Where this build script reads the reference sources for the checkers (oracle/_ref) when they are
# present: BF200_REFERENCE, else the reference checkout of the build machine.
REFERENCE_CHECKOUT = "/root/reference"


def reference_root():
    """The reference source tree the checkers are built from, or None where it is absent."""
    root = os.environ.get("BF200_REFERENCE", REFERENCE_CHECKOUT)
    return root if os.path.isdir(os.path.join(root, "Blackframe")) else None


def build_oracle(reference=None, verbose=False):
    oracle_dir = os.path.join(REPO, "oracle")
    subprocess.run(["make", "-s", "-C", oracle_dir, "oracle"], check=True)
    reference = reference or reference_root()
    if reference is not None:
        subprocess.run(["make", "-s", "-j8", "-C", oracle_dir, "ref", "refcuda", "REF=" + reference], check=True)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_oracle(verbose=True)
