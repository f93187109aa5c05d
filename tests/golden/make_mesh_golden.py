"""Writes the mesh-import fixtures: tests/golden/meshes/*.obj|*.ply, and tests/golden/meshes.npz with
what the reference's own loader (engine::load_obj_triangle_mesh / load_ply_triangle_mesh, compiled
into oracle/_ref/libbfref.so by `make -C oracle ref`) returns for each: the aligned arrays of an
accepted file, or the reference StatusCode of a refused one.

The files cover the format rules of the reference importer and of its tests
(Tests/Engine/TriangleMeshImportTest.cpp): shared corners, bit-distinct seams, negative relative
indices, metadata records, comments, CRLF lines, PLY property orders, aliases and scalar types,
plus one file per refusal (faces that are not triangles, incomplete corners, index zero or out of
range, unsupported records and encodings, non-unit normals, non-finite, hexadecimal, overflowing
and underflowing scalars, degenerate triangles, duplicated or missing PLY properties, list and
index types out of range, truncated headers, trailing data). Two larger seeded meshes are written
with 9- and 17-digit decimals, so float rounding through double is exercised.

Run from the repository root: python tests/golden/make_mesh_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
MESHES = os.path.join(HERE, "meshes")
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "blackframe-renderer_b200"))

from bf200 import scenes  # noqa: E402
from oracle.bindings import Reference  # noqa: E402

QUAD_OBJ = """# a unit quad: shared corners, metadata and comments
mtllib quad.mtl
o quad
g front
usemtl white
s off
v -1 -1 0
v +1 -1 0  # trailing comment
v 1.0e0 1 0
v -1 1.0E+00 0
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
f 1/1/1 2/2/1 3/3/1
f -4/-4/-1 -2/-2/-1 -1/-1/-1
"""

SEAM_OBJ = """v 0 0 0
v 1 0 0
v 0 1 0
v 5 5 5
vt 0 0
vt 1 0
vt 0 1
vt 0.5 0.5
vn 0 0 1
vn 0 0 -1
f 1/1/1 2/2/1 3/3/1
f 1/4/2 3/3/2 2/2/2
"""

QUAD_PLY = """ply
format ascii 1.0
comment a unit quad
element vertex 4
property float x
property float y
property float z
property float nx
property float ny
property float nz
property float u
property float v
element face 2
property list uchar int vertex_indices
end_header
-1 -1 0 0 0 1 0 0
1 -1 0 0 0 1 1 0
1 1 0 0 0 1 1 1
-1 1 0 0 0 1 0 1
3 0 1 2
3 0 2 3
"""

ORDER_PLY = """ply
format ascii 1.0
obj_info permuted properties, aliases and scalar types
element vertex 3
property double nz
property short x
property float s
property int y
property float ny
property double t
property char z
property float nx
element face 1
property list uint8 uint32 vertex_index
end_header
1 0 0.25 0 0 0.75 0 0
1 2 +1 0 0 0 0 0
1 0 0 3 0 1e-1 -1 0
3 0 1 2

"""


def bad(name, text):
    return name, text


def refused_cases():
    v3 = "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\n"
    ply_head = ("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
                "property float nx\nproperty float ny\nproperty float nz\nproperty float u\nproperty float v\n"
                "element face 1\nproperty list uchar int vertex_indices\nend_header\n")
    ply_verts = "0 0 0 0 0 1 0 0\n1 0 0 0 0 1 0 0\n0 1 0 0 0 1 0 0\n"
    return [
        bad("bad_quad_face.obj", v3 + "v 1 1 0\nf 1/1/1 2/1/1 4/1/1 3/1/1\n"),
        bad("bad_corner.obj", v3 + "f 1//1 2//1 3//1\n"),
        bad("bad_index_zero.obj", v3 + "f 0/1/1 2/1/1 3/1/1\n"),
        bad("bad_index_range.obj", v3 + "f 1/1/1 2/1/1 4/1/1\n"),
        bad("bad_record.obj", v3 + "l 1 2\nf 1/1/1 2/1/1 3/1/1\n"),
        bad("bad_position.obj", "v 0 0\n"),
        bad("bad_normal.obj", "vn 0 0 2\n"),
        bad("bad_hex.obj", "v 0x1p0 0 0\n"),
        bad("bad_infinite.obj", "v inf 0 0\n"),
        bad("bad_overflow.obj", "v 1e39 0 0\n"),
        bad("bad_underflow.obj", "v 1e-50 0 0\n"),
        bad("bad_degenerate.obj", "v 0 0 0\nv 1 1 1\nv 2 2 2\nvt 0 0\nvn 0 0 1\nf 1/1/1 2/1/1 3/1/1\n"),
        bad("bad_group.obj", v3 + "g a b\nf 1/1/1 2/1/1 3/1/1\n"),
        bad("bad_empty.obj", "# nothing\n"),
        bad("bad_binary.ply", ply_head.replace("ascii 1.0", "binary_little_endian 1.0") + ply_verts + "3 0 1 2\n"),
        bad("bad_missing_uv.ply", ply_head.replace("property float u\nproperty float v\n", "") +
            "0 0 0 0 0 1\n1 0 0 0 0 1\n0 1 0 0 0 1\n3 0 1 2\n"),
        bad("bad_alias.ply", ply_head.replace("property float v\n", "property float s\n") + ply_verts + "3 0 1 2\n"),
        bad("bad_quad.ply", ply_head + ply_verts + "4 0 1 2 0\n"),
        bad("bad_face_index.ply", ply_head + ply_verts + "3 0 1 3\n"),
        bad("bad_trailing.ply", ply_head + ply_verts + "3 0 1 2\n7\n"),
        bad("bad_negative.ply", ply_head + ply_verts + "3 0 -1 2\n"),
        bad("bad_list_type.ply", ply_head + ply_verts + "256 0 1 2\n"),
        bad("bad_truncated.ply", "ply\nformat ascii 1.0\nelement vertex 3\n"),
        bad("bad_vertex_fields.ply", ply_head + "0 0 0 0 0 1 0\n1 0 0 0 0 1 0 0\n0 1 0 0 0 1 0 0\n3 0 1 2\n"),
    ]


def big_mesh(digits, subdivisions, seed):
    """A seeded displaced icosphere with smooth unit normals, written with `digits` significant digits."""
    v, f = scenes.icosphere(subdivisions)
    rng = np.random.default_rng(seed)
    p = v * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, len(v)))[:, None]
    n = v / np.linalg.norm(v, axis=1, keepdims=True)
    uv = rng.uniform(0.0, 1.0, (len(v), 2))
    fmt = "{:.%dg}" % digits
    obj = ["# seeded icosphere"]
    obj += ["v " + " ".join(fmt.format(x) for x in row) for row in p]
    obj += ["vt " + " ".join(fmt.format(x) for x in row) for row in uv]
    # normals normalised in float32 first, so they pass the unit-length check after parsing
    n32 = n.astype(np.float32)
    obj += ["vn " + " ".join("{:.9g}".format(float(x)) for x in row) for row in n32]
    obj += ["f " + " ".join(f"{i + 1}/{i + 1}/{i + 1}" for i in tri) for tri in f]
    ply = ["ply", "format ascii 1.0", f"element vertex {len(v)}", "property double x", "property double y",
           "property double z", "property float nx", "property float ny", "property float nz", "property float u",
           "property float v", f"element face {len(f)}", "property list uchar uint vertex_indices", "end_header"]
    ply += [" ".join([fmt.format(x) for x in p[k]] + ["{:.9g}".format(float(x)) for x in n32[k]] +
                     [fmt.format(x) for x in uv[k]]) for k in range(len(v))]
    ply += ["3 " + " ".join(str(i) for i in tri) for tri in f]
    return "\n".join(obj) + "\n", "\n".join(ply) + "\n"


def main():
    os.makedirs(MESHES, exist_ok=True)
    files = [("quad.obj", QUAD_OBJ.replace("\n", "\r\n")), ("seams.obj", SEAM_OBJ), ("quad.ply", QUAD_PLY),
             ("order.ply", ORDER_PLY)]
    obj9, ply9 = big_mesh(9, 3, 11)
    obj17, ply17 = big_mesh(17, 3, 12)
    files += [("sphere9.obj", obj9), ("sphere9.ply", ply9), ("sphere17.obj", obj17), ("sphere17.ply", ply17)]
    files += refused_cases()
    ref = Reference()
    out = {}
    for name, text in files:
        path = os.path.join(MESHES, name)
        with open(path, "w", newline="") as handle:
            handle.write(text)
        mesh, code, message = ref.load_mesh(path)
        key = name.replace(".", "_")
        out[key + "_code"] = np.int64(code)
        if mesh is not None:
            for part, array in zip(("positions", "normals", "uvs", "triangles"), mesh):
                out[f"{key}_{part}"] = array
        print(f"{name}: {'accepted' if mesh is not None else f'refused ({code}) {message}'}")
    out["names"] = np.array([name for name, _ in files])
    np.savez_compressed(os.path.join(HERE, "meshes.npz"), **out)


if __name__ == "__main__":
    main()
