"""Scene SoA blob writer, ABI v4: a SceneBuilder's scene as the column blob a Blackframe host
serialises a FrameScene into (SceneSoaHeader + 194 columns, 16-byte aligned, FNV-1a 64 content
hash over the blob with the hash field read as zero; layout of
Blackframe/XPU/Shared/Include/Blackframe/XPU/Shared/SceneSoaAbi.hpp). bf200_scene_create_from_soa
reads such blobs. Every material is written as spectral at the builder's packet; instances have no
parents; punctual lights are written as SceneSoA serialises them (kind 0 point, 1 directional,
2 spot; SceneSoA.cpp:241-300); there are no textures."""
import struct

import numpy as np

MAGIC = 0x34414F53464B4C42
HEADER_BYTES = 4848
COLUMNS = 194


def _element_size(c):
    if (2 <= c <= 5) or c in (31, 32, 185, 186, 191, 192):
        return 8
    if c == 18 or 27 <= c <= 30 or c in (33, 57, 166, 176) or 152 <= c <= 155:
        return 1
    return 4


def _fnv1a(data):
    h = 14695981039346656037
    for i, b in enumerate(data):
        if 32 <= i < 40:
            b = 0
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def write(builder):
    """The builder's scene as a v4 blob (bytes)."""
    desc = builder.desc()  # resolves the arrays exactly as the descriptor path sees them
    geometries = [desc.geometries[g] for g in range(desc.geometry_count)]
    materials = [desc.materials[m] for m in range(desc.material_count)]
    closures = [desc.closures[k] for k in range(desc.closure_count)]
    instances = [desc.instances[i] for i in range(desc.instance_count)]
    positions, normals, uvs, triangles = builder._positions, builder._normals, builder._uvs, builder._triangles
    emissive = [inst.instance_id for inst in instances
                if any(materials[inst.material_index].emitted_radiance[l] != 0 for l in range(4))]
    counts = {
        "object": len(instances), "geometry": len(geometries), "vertex": len(positions), "triangle": len(triangles),
        "material": len(materials), "closure": len(closures), "instance": len(instances),
        "punctual": len(builder.punctual),
        "mesh_light": len(emissive), "environment": 1, "texture": 0, "image_texture": 0, "image_mip": 0,
        "image_texel": 0}
    nm = [desc.wavelength_nanometers[l] for l in range(4)]
    pdf = [desc.wavelength_pdf[l] for l in range(4)]
    env = [desc.environment_radiance[l] for l in range(4)]
    cols = {}

    def col(c, fmt, values):
        cols[c] = (fmt, list(values))

    col(0, "I", [inst.object_id for inst in instances])
    col(1, "I", [g.geometry_id for g in geometries])
    col(2, "Q", [g.vertex_offset for g in geometries])
    col(3, "Q", [g.vertex_count for g in geometries])
    col(4, "Q", [g.triangle_offset for g in geometries])
    col(5, "Q", [g.triangle_count for g in geometries])
    for a in range(3):
        col(6 + a, "f", positions[:, a])
        col(9 + a, "f", normals[:, a])
        col(14 + a, "I", triangles[:, a])
    for a in range(2):
        col(12 + a, "f", uvs[:, a])
    col(17, "I", [m.material_id for m in materials])
    col(18, "B", [1] * len(materials))
    for l in range(4):
        col(19 + l, "f", [nm[l]] * len(materials))
        col(23 + l, "f", [pdf[l]] * len(materials))
        col(27 + l, "B", [1] * len(materials))
        col(35 + l, "f", [m.emitted_radiance[l] for m in materials])
    col(31, "Q", [m.closure_offset for m in materials])
    col(32, "Q", [m.closure_count for m in materials])
    col(33, "B", [m.frame_mode for m in materials])
    col(34, "f", [m.tangent_rotation_radians for m in materials])
    probability = [0.0] * len(closures)
    for m in materials:
        for k in range(m.closure_count):
            probability[m.closure_offset + k] = m.component_probabilities[k]
    col(39, "I", [c.kind for c in closures])
    col(40, "I", [c.lobes for c in closures])
    for l in range(4):
        col(41 + l, "f", [c.weight[l] for c in closures])
    for p in range(10):
        col(45 + p, "f", [c.parameters[p] for c in closures])
    col(55, "f", probability)
    ids = {g: geometries[g].geometry_id for g in range(len(geometries))}
    mids = {m: materials[m].material_id for m in range(len(materials))}
    col(56, "I", [inst.instance_id for inst in instances])
    col(57, "B", [0] * len(instances))
    col(58, "I", [0] * len(instances))
    col(59, "I", [inst.object_id for inst in instances])
    col(60, "I", [ids[inst.geometry_index] for inst in instances])
    col(61, "I", [mids[inst.material_index] for inst in instances])
    col(62, "I", [inst.visibility_mask for inst in instances])
    for e in range(16):
        col(63 + e, "f", [inst.object_to_world[e] for inst in instances])   # local to parent (no parents)
        col(79 + e, "f", [inst.world_to_object[e] for inst in instances])
        col(95 + e, "f", [inst.object_to_world[e] for inst in instances])
        col(111 + e, "f", [inst.world_to_object[e] for inst in instances])
    lights = builder.punctual
    col(127, "I", [{1: 0, 2: 1, 3: 2}[light.kind] for light in lights])
    for a in range(3):
        col(128 + a, "f", [light.position[a] for light in lights])
        col(131 + a, "f", [light.position_error[a] for light in lights])
        col(134 + a, "f", [light.direction[a] for light in lights])
    col(137, "f", [light.inner_half_angle for light in lights])
    col(138, "f", [light.outer_half_angle for light in lights])
    for l in range(4):
        col(139 + l, "f", [light.spectrum[l] for light in lights])
    col(143, "I", emissive)
    for l in range(4):
        col(144 + l, "f", [nm[l]])
        col(148 + l, "f", [pdf[l]])
        col(152 + l, "B", [1])
        col(156 + l, "f", [env[l]])
    col(166, "B", [0] * len(materials))
    col(176, "B", [0] * len(materials))
    for c in list(range(167, 176)) + list(range(177, 184)):
        col(c, "f" if c == 179 else "I", [0] * len(materials))
    # column descriptors, 16-byte aligned after the header
    descriptors, body, cursor = [], bytearray(), HEADER_BYTES
    for c in range(COLUMNS):
        fmt, values = cols.get(c, ("I", []))
        size = _element_size(c)
        if not values:
            descriptors.append((0, 0, size))
            continue
        pad = (-cursor) % 16
        body += b"\0" * pad
        cursor += pad
        data = np.asarray(values, {"I": np.uint32, "Q": np.uint64, "f": np.float32, "B": np.uint8}[fmt]).tobytes()
        assert len(data) == size * len(values)
        descriptors.append((cursor, len(values), size))
        body += data
        cursor += len(data)
    header = struct.pack("<QHHIIIQQ", MAGIC, 4, 0, HEADER_BYTES, COLUMNS, 1, cursor, 0)
    header += struct.pack("<14Q", counts["object"], counts["geometry"], counts["vertex"], counts["triangle"],
                          counts["material"], counts["closure"], counts["instance"], counts["punctual"],
                          counts["mesh_light"], counts["environment"], counts["texture"], counts["image_texture"],
                          counts["image_mip"], counts["image_texel"])
    for offset, count, size in descriptors:
        header += struct.pack("<QQII", offset, count, size, 0)
    header += b"\0" * 40
    assert len(header) == HEADER_BYTES
    blob = bytearray(header + bytes(body))
    struct.pack_into("<Q", blob, 32, _fnv1a(blob))
    return bytes(blob)
