"""Scene SoA v4 blobs (bf200_scene_create_from_soa): header validation as
validate_scene_soa_header does it, the content hash, and the refusals, on the CPU (no context: a
valid blob gets as far as "null context"). The GPU half (tests/test_gpu_scene_soa.py) renders
scenes created from blobs."""
import ctypes as C
import struct

import pytest

from bf200 import runtime, scenes, soa


def load(blob):
    lib = runtime.library()
    handle = C.c_void_p()
    message = C.create_string_buffer(256)
    data = C.create_string_buffer(bytes(blob), len(blob))
    status = lib.bf200_scene_create_from_soa(None, data, len(blob), C.byref(handle), message, len(message))
    return status, message.value.decode()


def rehash(blob):
    blob = bytearray(blob)
    struct.pack_into("<Q", blob, 32, soa._fnv1a(blob))
    return bytes(blob)


@pytest.fixture(scope="module")
def blob():
    return soa.write(scenes.cornell_box(scenes.SceneBuilder(), with_spheres=False))


def test_a_valid_blob_passes_every_check(blob):
    assert load(blob) == (1, "null context")


def test_header_and_hash_checks(blob):
    bad = bytearray(blob)
    struct.pack_into("<Q", bad, 0, 0)  # magic
    assert load(rehash(bad))[1] == "scene SoA header: bad magic"
    bad = bytearray(blob)
    struct.pack_into("<H", bad, 8, 3)  # major version
    assert load(rehash(bad))[1] == "scene SoA header: incompatible version"
    bad = bytearray(blob)
    bad[-1] ^= 1  # content changed, hash not updated
    assert load(bytes(bad))[1] == "scene SoA content hash mismatch"
    assert load(blob[:-16])[0] == 1  # truncated
    bad = bytearray(blob)
    struct.pack_into("<Q", bad, 152 + 24 * 6, struct.unpack_from("<Q", bad, 152 + 24 * 6)[0] + 16)  # a column offset
    assert load(rehash(bad))[1] == "scene SoA header: invalid column descriptor"


def test_unsupported_content_is_refused(blob):
    bad = bytearray(blob)
    struct.pack_into("<Q", bad, 96, 1)  # one punctual light: its columns no longer match
    assert load(rehash(bad))[1].startswith("scene SoA header")
