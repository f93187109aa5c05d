"""The native scene JSON codec (bf200_scene_json_*) against the reference's own codec.

* tests/golden/scene_json.npz (tests/golden/make_scene_json_golden.py) holds the compiled
  reference's decisions on a seeded corpus: valid descriptions of every record kind, one-rule
  mutations of them, byte-level syntax breaks and budget limits. The codec must return the same
  status code for every document and, for every accepted one, the same canonical bytes as the
  reference's serializer. Two deliberate differences: host-image textures and normal/bump maps
  are refused as unavailable (this backend has no image textures), so a document whose texture
  record the reference refuses for its contents is refused as unavailable here.
* For accepted documents the committed frame (bf200_scene_json_frame) carries the instance world
  transforms and inverses of FrameScene::create, bit for bit, and the mesh lights it derives.
* With the compiled reference present, fresh seeds are fuzzed against it live.
"""
import ctypes as C
import os
import zlib

import numpy as np
import pytest

import scene_json_corpus as corpus
from bf200 import abi, runtime, scene_json

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "scene_json.npz")
DIVERGENT = ("host image", "normal map")


def unpack(blob, sizes):
    data = zlib.decompress(blob.tobytes())
    out, at = [], 0
    for n in sizes:
        out.append(data[at:at + int(n)])
        at += int(n)
    return out


@pytest.fixture(scope="module")
def golden():
    g = dict(np.load(GOLDEN))
    g["texts"] = unpack(g["texts"], g["text_sizes"])
    g["canonical"] = unpack(g["canonical"], g["canonical_sizes"])
    return g


def overrides_of(row):
    if not any(row):
        return None
    return dict(zip(corpus.LIMIT_ORDER, (int(v) for v in row)))


def check_case(label, text, lim, code, canonical, got):
    got_code, got_canonical, message = got
    if label.startswith(DIVERGENT) and code != 0:
        assert got_code in (code, 2), (label, code, got_code, message)
        return
    assert got_code == code, f"{label}: reference {code}, codec {got_code} ({message})"
    if code == 0:
        assert got_canonical == canonical, f"{label}: canonical bytes differ"


def test_codec_matches_the_reference_fixture(golden):
    accepted = 0
    for k, label in enumerate(golden["labels"]):
        label = str(label)
        lim = overrides_of(golden["limits"][k])
        code, canonical = int(golden["codes"][k]), golden["canonical"][k]
        got = corpus.product_outcome(golden["texts"][k], lim)
        check_case(label, golden["texts"][k], lim, code, canonical, got)
        accepted += code == 0
    assert accepted >= 20 and len(golden["labels"]) >= 400


def test_every_status_code_the_corpus_reaches(golden):
    # invalid_argument, incompatible and resource_exhausted all occur, besides acceptance
    assert {0, 1, 4, 5} <= set(int(c) for c in golden["codes"])


def test_canonical_bytes_are_a_fixed_point(golden):
    """Parsing the canonical bytes gives them back, except for the largest float: its 9-digit
    form (3.40282347e+38) is above FLT_MAX as a double, so to_transport_scalar refuses it, in the
    reference as here."""
    checked = 0
    for k in np.flatnonzero(golden["codes"] == 0):
        once = corpus.product_outcome(golden["texts"][k], None)[1]
        code, twice, _ = corpus.product_outcome(once, None)
        if str(golden["labels"][k]).startswith("t_max largest"):
            assert code == 1 and b"3.40282347e+38" in once
            continue
        assert code == 0 and once == twice
        checked += 1
    assert checked >= 20


def test_frame_commit_matches_frame_scene(golden):
    for k in golden["frame_cases"]:
        text = golden["texts"][int(k)]
        ids, world = golden[f"frame{k}/ids"], golden[f"frame{k}/world"]
        inverse, lights = golden[f"frame{k}/inverse"], golden[f"frame{k}/lights"]
        with scene_json.SceneJson(text) as doc:
            frame = doc.frame()
            s = frame.scene
            n = s.instance_count
            assert n == len(ids)
            got_ids = np.array([s.instances[i].instance_id for i in range(n)], np.uint32)
            got_world = np.array([list(s.instances[i].object_to_world) for i in range(n)], np.float32)
            got_inverse = np.array([list(s.instances[i].world_to_object) for i in range(n)], np.float32)
            assert (got_ids == ids).all()
            assert (got_world.view(np.uint32) == world.view(np.uint32)).all()
            assert (got_inverse.view(np.uint32) == inverse.view(np.uint32)).all()
            # mesh area lights: one per instance whose material emits, in instance order
            emits = [any(v != 0.0 for v in s.materials[s.instances[i].material_index].emitted_radiance)
                     for i in range(n)]
            assert [int(i) for i, e in zip(got_ids, emits) if e] == [int(v) for v in lights]


def test_frame_carries_the_active_selection():
    rng = np.random.default_rng(3)
    doc = corpus.valid_document(rng)
    with scene_json.SceneJson(corpus.dumps(doc)) as parsed:
        f = parsed.frame()
    film, cam, opt = doc["films"][0], doc["cameras"][0]["model"], doc["render_options"][0]
    assert (f.width, f.height) == tuple(film["extent"]) and list(f.crop) == film["crop"]
    assert f.precision == ["float32", "float64"].index(film["accumulation"])
    assert f.samples_per_pixel == opt["samples_per_pixel"] and f.seed == opt["seed"]
    assert f.camera.jitter_mode == ["center", "uniform"].index(opt["pixel_jitter"])
    assert f.options.mis_heuristic == ["balance", "power"].index(opt["mis_heuristic"])
    assert list(f.options.depth_limits) == [opt["depth_limits"][k] for k in
                                            ("diffuse", "glossy", "specular", "transmission", "volume")]
    assert list(f.camera.normal) == cam["normal"] and f.camera.t_max == np.float32(cam["t_max"])
    # the projection constants are PinholeCamera::create's, as bf200_camera_create derives them
    ref = runtime.camera_create(cam["origin"], cam["normal"], cam["tangent"], f.width, f.height,
                                cam["vertical_fov_radians"])
    assert (f.camera.half_width, f.camera.half_height) == (ref.half_width, ref.half_height)
    env = [l for l in doc["lights"] if l["type"] == "environment"][0]
    assert list(f.scene.wavelength_nanometers) == [np.float32(v) for v in env["wavelengths"]["nanometers"]]
    assert f.scene.punctual_light_count == len(doc["lights"]) - 1


def test_unsupported_records_and_frames_are_refused():
    rng = np.random.default_rng(4)
    doc = corpus.valid_document(rng)
    doc["host_image_textures"] = [{"id": 900, "image": {"source_path": "a.exr"}}]
    assert scene_json.parse_status(corpus.dumps(doc))[0] == 2
    doc = corpus.valid_document(rng)
    doc["materials"][0]["spectral"]["bump_map"] = {"texture": 1}
    assert scene_json.parse_status(corpus.dumps(doc))[0] == 2
    doc = corpus.valid_document(rng)
    doc["instances"] = []
    with scene_json.SceneJson(corpus.dumps(doc)) as parsed:
        with pytest.raises(scene_json.SceneJsonError) as info:
            parsed.frame()
        assert info.value.code == 2
    doc = corpus.valid_document(rng)
    for m in doc["materials"]:
        m["spectral"] = None
    doc["lights"] = []
    with scene_json.SceneJson(corpus.dumps(doc)) as parsed:  # valid without a packet, not renderable
        with pytest.raises(scene_json.SceneJsonError) as info:
            parsed.frame()
        assert info.value.code == 2


def test_record_budget_sizes_are_the_references(golden):
    # the decoded-byte budget charges the reference's record sizes (bf200_scene_json.cpp constants)
    assert list(golden["record_sizes"]) == [32, 80, 72, 24, 24, 4, 24, 712, 92, 72, 12, 12, 8, 12]


@pytest.mark.skipif(corpus.reference_library() is None, reason="the compiled reference is not built here")
@pytest.mark.parametrize("seed", [11, 12])
def test_codec_against_the_live_reference(seed):
    lib = corpus.reference_library()
    for label, text, lim in corpus.corpus(seed, 2):
        code, canonical, _ = corpus.reference_outcome(lib, text, lim)
        check_case(label, text, lim, code, canonical, corpus.product_outcome(text, lim))


@pytest.mark.skipif(corpus.reference_library() is None, reason="the compiled reference is not built here")
def test_record_sizes_against_the_live_reference():
    lib = corpus.reference_library()
    sizes = (C.c_uint64 * 14)()
    lib.bfref_scene_json_record_sizes(sizes)
    assert list(sizes) == [32, 80, 72, 24, 24, 4, 24, 712, 92, 72, 12, 12, 8, 12]
