"""Freezes the reference codec's decisions on a seeded scene JSON corpus into
tests/golden/scene_json.npz, for tests/test_scene_json.py.

Each case is a document (tests/scene_json_corpus.py: valid descriptions, one-rule mutations of
them, byte-level syntax breaks, and budget limits just below and at what a document needs) with
the status code the reference's deserialize_scene_description_json returns and, when it accepts,
the bytes serialize_scene_description_json writes. For the accepted valid documents the fixture
also holds the FrameScene::create commit: instance identifiers with their world transforms and
inverses, and the instance identifiers of the mesh area lights.

Run from the repository root after `make -C oracle ref REF=<reference tree>`:
    python tests/golden/make_scene_json_golden.py
"""
import ctypes as C
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import scene_json_corpus as corpus  # noqa: E402

SEED, COUNT = 20261204, 3
FRAME_SEED, FRAME_COUNT = 4051, 12  # extra valid documents for the frame commit


def frame_of(lib, text):
    ids = (C.c_uint32 * 4096)()
    world = (C.c_float * (16 * 4096))()
    inverse = (C.c_float * (16 * 4096))()
    lights = (C.c_uint32 * 4096)()
    count, light_count = C.c_uint64(), C.c_uint64()
    message = C.create_string_buffer(1024)
    rc = lib.bfref_scene_json_frame(text, len(text), ids, world, inverse, 4096, C.byref(count), lights, 4096,
                                    C.byref(light_count), message, len(message))
    if rc != 0:
        return None
    n, m = count.value, light_count.value
    return (np.array(ids[:n], np.uint32), np.array(world[:16 * n], np.float32).reshape(n, 16),
            np.array(inverse[:16 * n], np.float32).reshape(n, 16), np.array(lights[:m], np.uint32))


def main():
    lib = corpus.reference_library()
    if lib is None:
        raise SystemExit("oracle/_ref/libbfref.so is not built")
    lib.bfref_scene_json_frame.restype = C.c_int
    cases = corpus.corpus(SEED, COUNT)
    rng = np.random.default_rng(FRAME_SEED)
    cases += [(f"valid frame {i}", corpus.dumps(corpus.valid_document(rng), rng).encode(), None)
              for i in range(FRAME_COUNT)]
    labels, texts, limits, codes, canonical = [], [], [], [], []
    frames = {}
    for label, text, lim in cases:
        code, canon, _ = corpus.reference_outcome(lib, text, lim)
        labels.append(label)
        texts.append(text)
        limits.append(corpus.limit_vector(lim) if lim is not None else [0] * 9)
        codes.append(code)
        canonical.append(canon)
        if label.startswith("valid") and code == 0:
            frame = frame_of(lib, text)
            if frame is not None:
                frames[len(labels) - 1] = frame
    blob = zlib.compress(b"".join(texts), 9)
    canon_blob = zlib.compress(b"".join(canonical), 9)
    out = {
        "labels": np.array(labels),
        "texts": np.frombuffer(blob, np.uint8),
        "text_sizes": np.array([len(t) for t in texts], np.uint64),
        "limits": np.array(limits, np.uint64),
        "codes": np.array(codes, np.uint32),
        "canonical": np.frombuffer(canon_blob, np.uint8),
        "canonical_sizes": np.array([len(c) for c in canonical], np.uint64),
        "frame_cases": np.array(sorted(frames), np.uint32),
    }
    for k, (ids, world, inverse, lights) in frames.items():
        out[f"frame{k}/ids"] = ids
        out[f"frame{k}/world"] = world
        out[f"frame{k}/inverse"] = inverse
        out[f"frame{k}/lights"] = lights
    sizes = (C.c_uint64 * 14)()
    lib.bfref_scene_json_record_sizes(sizes)
    out["record_sizes"] = np.array(sizes[:], np.uint64)
    path = os.path.join(HERE, "scene_json.npz")
    np.savez_compressed(path, **out)
    print(f"{len(cases)} cases ({sum(c == 0 for c in codes)} accepted, {len(frames)} frames) -> {path} "
          f"({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
