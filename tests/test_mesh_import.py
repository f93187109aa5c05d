"""OBJ / ASCII PLY import (bf200_mesh_load) against the reference's own loader
(engine::load_obj_triangle_mesh / load_ply_triangle_mesh). tests/golden/meshes.npz holds what the
compiled reference returned for every file of tests/golden/meshes/ (made by
tests/golden/make_mesh_golden.py): an accepted file must give bit-identical aligned arrays, and a
refused file must be refused, in the same status class. Host code only; no GPU."""
import os

import numpy as np
import pytest

from bf200 import runtime

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "meshes.npz"))
NAMES = [str(n) for n in GOLDEN["names"]]
# reference StatusCode -> bf200 status: invalid_argument -> INVALID_ARGUMENT, incompatible ->
# INVALID_STATE (no substitution), resource_exhausted -> OUT_OF_RANGE
STATUS_OF_REFERENCE = {1: 1, 4: 4, 5: 5}


@pytest.mark.parametrize("name", NAMES)
def test_mesh_import_matches_the_reference_loader(name):
    key = name.replace(".", "_")
    path = os.path.join(HERE, "golden", "meshes", name)
    code = int(GOLDEN[key + "_code"])
    if code != 0:
        with pytest.raises(runtime.Bf200Error) as info:
            runtime.load_mesh(path)
        assert info.value.status == STATUS_OF_REFERENCE[code], (name, str(info.value))
        return
    mesh = runtime.load_mesh(path)
    for part, got in zip(("positions", "normals", "uvs", "triangles"), mesh):
        want = GOLDEN[f"{key}_{part}"]
        assert got.shape == want.shape, (name, part)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, part)


def test_mesh_paths_must_be_absolute_with_a_known_extension(tmp_path):
    with pytest.raises(runtime.Bf200Error):
        runtime.load_mesh("tests/golden/meshes/quad.obj")
    with pytest.raises(runtime.Bf200Error):
        runtime.load_mesh(str(tmp_path / "missing.obj"))
    other = tmp_path / "quad.OBJ"
    other.write_text(open(os.path.join(HERE, "golden", "meshes", "seams.obj")).read())
    with pytest.raises(runtime.Bf200Error):
        runtime.load_mesh(str(other))


def test_imported_mesh_builds_a_scene_description():
    from bf200 import scenes
    positions, normals, uvs, triangles = runtime.load_mesh(os.path.join(HERE, "golden", "meshes", "sphere9.obj"))
    mesh = scenes.Mesh(positions, normals, uvs, triangles)
    builder = scenes.SceneBuilder()
    builder.add_instance(builder.add_mesh(mesh), builder.add_material(scenes.lambertian([0.5] * 4)))
    desc = builder.desc()
    assert desc.triangle_count == len(triangles) and desc.vertex_count == len(positions)


def test_random_meshes_match_the_compiled_reference(tmp_path):
    """Seeded random OBJ and PLY files with varied number spellings (signs, exponents, 1 to 17
    digits, negative zero, relative indices), loaded by both importers. Runs where the reference
    was compiled (oracle/_ref); elsewhere the frozen fixtures above cover the same rules."""
    from oracle.bindings import Reference, reference_available
    if not reference_available():
        pytest.skip("oracle/_ref not built here")
    ref = Reference()
    rng = np.random.default_rng(31)

    def spell(x):
        digits = int(rng.integers(1, 18))
        text = f"{x:.{digits}g}"
        if rng.random() < 0.2 and not text.startswith("-"):
            text = "+" + text
        if rng.random() < 0.1:
            text = f"{x:.{digits}e}".replace("e", "E")
        return text

    for k in range(24):
        n_v = int(rng.integers(3, 40))
        p = rng.normal(0.0, 10.0 ** rng.integers(-3, 4), (n_v, 3))
        p[rng.random((n_v, 3)) < 0.05] = -0.0
        uv = rng.uniform(-2, 2, (n_v, 2))
        nrm = rng.normal(size=(n_v, 3))
        nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
        tris = np.array([rng.choice(n_v, 3, replace=False) for _ in range(int(rng.integers(1, 30)))])
        if k % 2 == 0:
            lines = ["v " + " ".join(spell(x) for x in row) for row in p]
            lines += ["vt " + " ".join(spell(x) for x in row) for row in uv]
            lines += ["vn " + " ".join(f"{float(x):.9g}" for x in row) for row in nrm]
            for tri in tris:
                corners = []
                for i in tri:
                    rel = rng.random() < 0.3
                    idx = (i - n_v) if rel else i + 1
                    corners.append(f"{idx}/{idx}/{idx}")
                lines.append("f " + " ".join(corners))
            path = tmp_path / f"r{k}.obj"
        else:
            lines = ["ply", "format ascii 1.0", f"element vertex {n_v}", "property double x", "property float y",
                     "property double z", "property float nx", "property float ny", "property float nz",
                     "property double u", "property float v", f"element face {len(tris)}",
                     "property list uchar int vertex_indices", "end_header"]
            lines += [" ".join([spell(x) for x in p[i]] + [f"{float(x):.9g}" for x in nrm[i]] +
                               [spell(x) for x in uv[i]]) for i in range(n_v)]
            lines += ["3 " + " ".join(str(i) for i in tri) for tri in tris]
            path = tmp_path / f"r{k}.ply"
        path.write_text("\n".join(lines) + "\n")
        want, code, message = ref.load_mesh(str(path))
        if want is None:
            with pytest.raises(runtime.Bf200Error):
                runtime.load_mesh(str(path))
            continue
        got = runtime.load_mesh(str(path))
        for g, w in zip(got, want):
            assert np.array_equal(np.asarray(g).view(np.uint32), np.asarray(w).view(np.uint32)), path.name
