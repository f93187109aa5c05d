"""Seeded documents of the native scene JSON schema ("blackframe.scene" v1) for the codec's parity
tests: valid descriptions that exercise every record kind, and mutations of them that break one
rule each (syntax, schema, value domains, references, hierarchy, spectral consistency, budgets).

The expected outcome of each document is whatever the reference's own codec decides
(oracle/_ref/libbfref.so, bfref_scene_json_canonical): tests/golden/make_scene_json_golden.py
freezes those decisions, and tests/test_scene_json.py replays them and fuzzes fresh documents
against the compiled reference when it is present.
"""
import copy
import json
import math

import numpy as np

PACKET = {"nanometers": [471.2129, 588.7129, 706.2129, 823.7129], "pdf": [0.0021276595, 0.0021276595,
                                                                         0.0021276595, 0.0021276595]}


def f32(x):
    return float(np.float32(x))


def f32s(values):
    return [f32(v) for v in values]


def unit(rng, n=3):
    v = rng.normal(size=n)
    v = v / np.linalg.norm(v)
    return f32s(v)


def rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def camera_model(rng, exact=False):
    if exact:
        t, b, n = [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]
    else:
        r = rotation(rng)
        t, b, n = f32s(r[:, 0]), f32s(r[:, 1]), f32s(r[:, 2])
    return {"type": "pinhole", "origin": f32s(rng.uniform(-5, 5, 3)), "normal": n, "tangent": t, "bitangent": b,
            "vertical_fov_radians": f32(rng.uniform(0.2, 2.5)), "t_min": f32(rng.choice([0.0, 1e-4])),
            "t_max": f32(rng.choice([1e30, 100.0, 3.4e38])), "visibility_mask": int(rng.integers(0, 2**32)),
            "current_medium": 0}


def mesh(rng, vertices=None, triangles=None):
    v = int(vertices or rng.integers(3, 12))
    t = int(triangles or rng.integers(1, 10))
    positions = [f32s(rng.uniform(-2, 2, 3)) for _ in range(v)]
    normals = [unit(rng) for _ in range(v)]
    uvs = [f32s(rng.uniform(0, 1, 2)) for _ in range(v)]
    tris = []
    while len(tris) < t:
        a, b, c = (int(i) for i in rng.choice(v, 3, replace=False))
        tris.append([a, b, c])
    return {"positions": positions, "normals": normals, "texture_coordinates": uvs, "triangles": tris}


def closure(rng, kind, probability):
    w = f32s(rng.uniform(0, 1, 4))
    c = {"probability": probability, "type": kind, "weight": w}
    if kind == "rough_diffuse_reflection":
        c["roughness"] = f32(rng.uniform(0, 1))
    elif kind == "rough_conductor_reflection":
        c["eta"] = f32s(rng.uniform(0.1, 3, 4))
        c["k"] = f32s(rng.uniform(0, 5, 4))
        c["alpha_x"], c["alpha_y"] = f32(rng.uniform(0.02, 1)), f32(rng.uniform(0.02, 1))
    elif kind == "rough_dielectric":
        c["exterior_eta"], c["interior_eta"] = 1.0, f32(rng.uniform(1.1, 2.4))
        c["alpha_x"], c["alpha_y"] = f32(rng.uniform(0.02, 1)), f32(rng.uniform(0.02, 1))
    elif kind == "specular_transmission":
        c["exterior_eta"], c["interior_eta"] = 1.0, f32(rng.uniform(1.1, 2.4))
    return c


KINDS = ["lambertian_reflection", "rough_diffuse_reflection", "rough_conductor_reflection", "rough_dielectric",
         "specular_reflection", "specular_transmission"]


def probabilities(rng, n):
    if n == 1:
        return [1.0]
    choice = rng.integers(4)
    if choice == 0:
        return [1.0 / n] * n if n in (2, 4, 8) else f32s(np.full(n, 1.0 / n))
    if choice == 1 and n == 2:
        return [0.3, 0.7]
    p = rng.dirichlet(np.ones(n))
    return f32s(p)


def material(rng, ident, emissive=False):
    n = int(rng.integers(0, 4)) if rng.random() < 0.9 else int(rng.integers(4, 9))
    kinds = [KINDS[int(k)] for k in rng.integers(0, len(KINDS), n)]
    p = probabilities(rng, n) if n else []
    emission = f32s(rng.uniform(0, 5, 4)) if emissive else [0.0, 0.0, 0.0, 0.0]
    return {"id": ident, "spectral": {
        "wavelengths": copy.deepcopy(PACKET),
        "closures": {"frame_mode": "shading_normal" if rng.random() < 0.9 else "surface_tangent",
                     "tangent_rotation_radians": f32(rng.uniform(-3.1, 3.1)) if rng.random() < 0.3 else 0.0,
                     "components": [closure(rng, k, p[i]) for i, k in enumerate(kinds)]},
        "emission": emission, "normal_map": None, "bump_map": None}}


def affine(rng):
    m = rotation(rng) * rng.uniform(0.3, 2.0)
    out = np.eye(4)
    out[:3, :3] = m
    out[:3, 3] = rng.uniform(-4, 4, 3)
    return f32s(out.ravel())


def identity():
    return [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]


def light(rng, ident, kind):
    if kind == "point":
        return {"id": ident, "type": "point", "position": f32s(rng.uniform(-3, 3, 3)),
                "absolute_position_error": f32s(rng.uniform(0, 1e-3, 3)),
                "spectral_radiant_intensity": f32s(rng.uniform(0, 10, 4))}
    if kind == "directional":
        return {"id": ident, "type": "directional", "propagation_direction": unit(rng),
                "spectral_irradiance": f32s(rng.uniform(0, 3, 4))}
    if kind == "spot":
        outer = f32(rng.uniform(0.1, 1.5))
        inner = f32(rng.choice([0.0, outer, outer * rng.uniform(0.2, 0.9)]))
        return {"id": ident, "type": "spot", "position": f32s(rng.uniform(-3, 3, 3)),
                "absolute_position_error": [0.0, 0.0, 0.0], "emission_direction": unit(rng),
                "inner_half_angle_radians": inner, "outer_half_angle_radians": outer,
                "on_axis_spectral_radiant_intensity": f32s(rng.uniform(0, 10, 4))}
    return {"id": ident, "type": "environment", "wavelengths": copy.deepcopy(PACKET),
            "radiance": f32s(rng.uniform(0, 1, 4))}


def valid_document(rng, size="small"):
    """A description that every rule accepts (ids shuffled, so the codec sorts them)."""
    width, height = int(rng.integers(1, 300)), int(rng.integers(1, 300))
    films = [{"id": 7, "extent": [width, height], "crop": [0, 0, width, height],
              "accumulation": str(rng.choice(["float32", "float64"]))}]
    if rng.random() < 0.5:
        w2, h2 = int(rng.integers(2, 64)), int(rng.integers(2, 64))
        films.append({"id": 3, "extent": [w2, h2], "crop": [1, 1, w2, h2], "accumulation": "float32"})
    cameras = [{"id": 11, "film": 7, "model": camera_model(rng, exact=rng.random() < 0.3)}]
    if len(films) > 1:
        cameras.append({"id": 2, "film": 3, "model": camera_model(rng)})
    depth = int(rng.integers(1, 12))
    roulette = ({"mode": "disabled"} if rng.random() < 0.5 else
                {"mode": "enabled", "first_eligible_depth": int(rng.integers(1, 5)),
                 "minimum_survival_probability": 0.05, "maximum_survival_probability": f32(rng.uniform(0.05, 1))})
    options = [{"id": 5, "film": 7, "samples_per_pixel": int(rng.integers(1, 64)), "maximum_path_depth": depth,
                "tile_edge_length": int(rng.integers(1, 64)), "seed": int(rng.integers(0, 2**63)),
                "pixel_jitter": str(rng.choice(["center", "uniform"])),
                "mis_heuristic": str(rng.choice(["balance", "power"])),
                "light_sampling_strategy": str(rng.choice(["uniform", "power_weighted", "spatial_tree"])),
                "depth_limits": {k: int(rng.integers(0, depth + 1)) for k in
                                 ("diffuse", "glossy", "specular", "transmission", "volume")},
                "russian_roulette": roulette}]
    constant_textures = []
    for k in range(int(rng.integers(0, 4))):
        kind = ["float", "color", "spectrum"][k % 3]
        value = f32(rng.normal()) if kind == "float" else f32s(rng.normal(size=3 if kind == "color" else 4))
        constant_textures.append({"id": 40 + k, "type": kind, "value": value})
    geometry_count = int(rng.integers(1, 4)) if size == "small" else 2
    geometries = [{"id": 100 + 3 * g, "mesh": mesh(rng) if size == "small" else mesh(rng, 400, 600)}
                  for g in range(geometry_count)]
    objects = [{"id": o} for o in (9, 1, 4)]
    materials = [material(rng, 200 + m, emissive=(m == 0)) for m in range(int(rng.integers(1, 4)))]
    instances = []
    ids = list(rng.permutation(np.arange(300, 300 + int(rng.integers(1, 7)))))
    for k, ident in enumerate(ids):
        parent = int(ids[int(rng.integers(0, k))]) if k > 0 and rng.random() < 0.5 else None
        instances.append({"id": int(ident), "parent": parent, "object": int(rng.choice([9, 1, 4])),
                          "geometry": geometries[int(rng.integers(len(geometries)))]["id"],
                          "material": materials[int(rng.integers(len(materials)))]["id"],
                          "local_to_parent": affine(rng) if rng.random() < 0.8 else identity(),
                          "visibility_mask": int(rng.integers(0, 2**32))})
    lights = [light(rng, 500, "environment")]
    for k, kind in enumerate(rng.choice(["point", "directional", "spot"], int(rng.integers(0, 4)))):
        lights.append(light(rng, 510 - k, str(kind)))
    doc = {"schema": "blackframe.scene", "schema_version": 1,
           "active": {"film": 7, "camera": 11, "render_options": 5},
           "films": films, "cameras": cameras, "render_options": options,
           "constant_textures": constant_textures, "host_image_textures": [], "objects": objects,
           "geometries": geometries, "materials": materials, "instances": instances, "lights": lights}
    return doc


def dumps(doc, rng=None):
    """Compact or spaced JSON text of a document."""
    if rng is not None and rng.random() < 0.3:
        return json.dumps(doc, indent=1)
    return json.dumps(doc, separators=(",", ":"))


def _set(doc, path, value):
    node = doc
    for key in path[:-1]:
        node = node[key]
    node[path[-1]] = value


def _delete(doc, path):
    node = doc
    for key in path[:-1]:
        node = node[key]
    del node[path[-1]]


def structural_mutations(doc, rng):
    """(label, document) pairs, each breaking one rule of the schema or of SceneDescription::create."""
    out = []

    def mutate(label, fn):
        d = copy.deepcopy(doc)
        fn(d)
        out.append((label, d))

    mat0 = ["materials", 0, "spectral"]
    mutate("missing root key", lambda d: _delete(d, ["lights"]))
    mutate("unknown root key", lambda d: _set(d, ["extra"], 1))
    mutate("schema name", lambda d: _set(d, ["schema"], "blackframe.scenes"))
    mutate("schema version", lambda d: _set(d, ["schema_version"], 2))
    mutate("identifier domain", lambda d: _set(d, ["films", 0, "id"], 2**32))
    mutate("negative identifier", lambda d: _set(d, ["objects", 0, "id"], -1))
    mutate("float identifier", lambda d: _set(d, ["objects", 0, "id"], 1.0))
    mutate("unknown film", lambda d: _set(d, ["active", "film"], 8))
    mutate("unknown camera", lambda d: _set(d, ["active", "camera"], 12))
    mutate("unknown options", lambda d: _set(d, ["active", "render_options"], 6))
    mutate("crop outside", lambda d: _set(d, ["films", 0, "crop", 2], d["films"][0]["extent"][0] + 1))
    mutate("empty crop", lambda d: _set(d, ["films", 0, "crop", 0], d["films"][0]["crop"][2]))
    mutate("zero extent", lambda d: _set(d, ["films", 0, "extent"], [0, 4]))
    mutate("huge extent", lambda d: _set(d, ["films", 0, "extent"], [2**21, 4]))
    mutate("too many pixels", lambda d: (_set(d, ["films", 0, "extent"], [2**20, 2**20]),
                                         _set(d, ["films", 0, "crop"], [0, 0, 2**20, 2**20])))
    mutate("accumulation enum", lambda d: _set(d, ["films", 0, "accumulation"], "float16"))
    mutate("extent arity", lambda d: _set(d, ["films", 0, "extent"], [4, 4, 4]))
    mutate("camera type", lambda d: _set(d, ["cameras", 0, "model", "type"], "orthographic"))
    mutate("camera frame", lambda d: _set(d, ["cameras", 0, "model", "normal"], [0.0, 0.0, 1.01]))
    mutate("camera left-handed", lambda d: _set(d, ["cameras", 0, "model", "normal"],
                                                [-v for v in d["cameras"][0]["model"]["normal"]]))
    mutate("camera fov", lambda d: _set(d, ["cameras", 0, "model", "vertical_fov_radians"], 3.2))
    mutate("camera bounds", lambda d: _set(d, ["cameras", 0, "model", "t_max"], -1.0))
    mutate("camera medium", lambda d: _set(d, ["cameras", 0, "model", "current_medium"], 1))
    mutate("camera film", lambda d: _set(d, ["cameras", 0, "film"], 99))
    mutate("active camera film", lambda d: d["films"].append(
        {"id": 8, "extent": [4, 4], "crop": [0, 0, 4, 4], "accumulation": "float32"}) or
        _set(d, ["cameras", 0, "film"], 8))
    mutate("camera missing key", lambda d: _delete(d, ["cameras", 0, "model", "t_min"]))
    mutate("spp zero", lambda d: _set(d, ["render_options", 0, "samples_per_pixel"], 0))
    mutate("spp huge", lambda d: _set(d, ["render_options", 0, "samples_per_pixel"], 2**24 + 1))
    mutate("depth zero", lambda d: (_set(d, ["render_options", 0, "maximum_path_depth"], 0)))
    mutate("depth huge", lambda d: _set(d, ["render_options", 0, "maximum_path_depth"], 5000))
    mutate("tile huge", lambda d: _set(d, ["render_options", 0, "tile_edge_length"], 4097))
    mutate("category depth", lambda d: _set(d, ["render_options", 0, "depth_limits", "glossy"],
                                            d["render_options"][0]["maximum_path_depth"] + 1))
    mutate("jitter enum", lambda d: _set(d, ["render_options", 0, "pixel_jitter"], "gaussian"))
    mutate("seed range", lambda d: _set(d, ["render_options", 0, "seed"], 2**64))
    mutate("roulette no mode", lambda d: _set(d, ["render_options", 0, "russian_roulette"], {}))
    mutate("roulette disabled params", lambda d: _set(d, ["render_options", 0, "russian_roulette"],
                                                      {"mode": "disabled", "first_eligible_depth": 1}))
    mutate("roulette bounds", lambda d: _set(d, ["render_options", 0, "russian_roulette"],
                                             {"mode": "enabled", "first_eligible_depth": 2,
                                              "minimum_survival_probability": 0.5,
                                              "maximum_survival_probability": 0.25}))
    mutate("roulette depth", lambda d: _set(d, ["render_options", 0, "russian_roulette"],
                                            {"mode": "enabled", "first_eligible_depth": 0,
                                             "minimum_survival_probability": 0.5,
                                             "maximum_survival_probability": 1.0}))
    mutate("roulette partial", lambda d: _set(d, ["render_options", 0, "russian_roulette"],
                                              {"mode": "enabled", "first_eligible_depth": 2}))
    mutate("roulette mode", lambda d: _set(d, ["render_options", 0, "russian_roulette"], {"mode": "sometimes"}))
    mutate("texture shape", lambda d: d["constant_textures"].append({"id": 60, "type": "color", "value": [1.0, 2.0]}))
    mutate("texture type", lambda d: d["constant_textures"].append({"id": 61, "type": "spectrum", "value": 1.0}))
    mutate("duplicate texture", lambda d: d["constant_textures"].extend(
        [{"id": 62, "type": "float", "value": 1.0}, {"id": 62, "type": "float", "value": 2.0}]))
    mutate("host image", lambda d: _set(d, ["host_image_textures"], [{"id": 70, "image": {}}]))
    mutate("duplicate object", lambda d: d["objects"].append({"id": 9}))
    mutate("object key", lambda d: _set(d, ["objects", 0], {"ident": 9}))
    mutate("empty mesh", lambda d: _set(d, ["geometries", 0, "mesh", "triangles"], []))
    mutate("mesh index", lambda d: _set(d, ["geometries", 0, "mesh", "triangles", 0, 0],
                                        len(d["geometries"][0]["mesh"]["positions"])))
    mutate("mesh normal", lambda d: _set(d, ["geometries", 0, "mesh", "normals", 0], [0.0, 0.0, 0.5]))
    mutate("mesh misaligned", lambda d: d["geometries"][0]["mesh"]["texture_coordinates"].pop())
    mutate("mesh extra normal", lambda d: d["geometries"][0]["mesh"]["normals"].append([0.0, 0.0, 1.0]))
    mutate("mesh degenerate", lambda d: _set(d, ["geometries", 0, "mesh", "triangles", 0],
                                             [d["geometries"][0]["mesh"]["triangles"][0][0]] * 2 +
                                             [d["geometries"][0]["mesh"]["triangles"][0][2]]))

    def collinear(d):
        m = d["geometries"][0]["mesh"]
        a, b, c = m["triangles"][0]
        pa, pb = m["positions"][a], m["positions"][b]
        m["positions"][c] = [pa[i] + 2.0 * (pb[i] - pa[i]) for i in range(3)] if all(
            float(np.float32(pa[i] + 2.0 * (pb[i] - pa[i]))) == pa[i] + 2.0 * (pb[i] - pa[i]) for i in range(3)) else pa
    mutate("mesh collinear", collinear)
    mutate("duplicate geometry", lambda d: d["geometries"].append(copy.deepcopy(d["geometries"][0])))
    mutate("closure weight", lambda d: d["materials"][0]["spectral"]["closures"]["components"].append(
        {"probability": 1.0, "type": "lambertian_reflection", "weight": [1.5, 0.5, 0.5, 0.5]}))
    mutate("closure type", lambda d: _set(d, mat0 + ["closures", "components"],
                                          [{"probability": 1.0, "type": "phong", "weight": [0.5] * 4}]))
    mutate("closure extra param", lambda d: _set(d, mat0 + ["closures", "components"],
                                                 [{"probability": 1.0, "type": "lambertian_reflection",
                                                   "weight": [0.5] * 4, "roughness": 0.5}]))
    mutate("closure missing param", lambda d: _set(d, mat0 + ["closures", "components"],
                                                   [{"probability": 1.0, "type": "rough_diffuse_reflection",
                                                     "weight": [0.5] * 4}]))
    mutate("dielectric same eta", lambda d: _set(d, mat0 + ["closures", "components"],
                                                 [{"probability": 1.0, "type": "rough_dielectric",
                                                   "weight": [0.5] * 4, "exterior_eta": 1.5, "interior_eta": 1.5,
                                                   "alpha_x": 0.3, "alpha_y": 0.3}]))
    mutate("conductor alpha", lambda d: _set(d, mat0 + ["closures", "components"],
                                             [{"probability": 1.0, "type": "rough_conductor_reflection",
                                               "weight": [0.5] * 4, "eta": [1.0] * 4, "k": [0.0] * 4,
                                               "alpha_x": 0.0, "alpha_y": 0.3}]))
    mutate("probabilities", lambda d: _set(d, mat0 + ["closures", "components"],
                                           [closure(rng, "lambertian_reflection", 0.6),
                                            closure(rng, "specular_reflection", 0.6)]))
    mutate("single probability", lambda d: _set(d, mat0 + ["closures", "components"],
                                                 [closure(rng, "lambertian_reflection", 0.5)]))
    mutate("too many closures", lambda d: _set(d, mat0 + ["closures", "components"],
                                               [closure(rng, "lambertian_reflection", 0.125)] * 9))
    mutate("rotation range", lambda d: _set(d, mat0 + ["closures", "tangent_rotation_radians"], 3.2))
    mutate("frame mode", lambda d: _set(d, mat0 + ["closures", "frame_mode"], "world"))
    mutate("normal map", lambda d: _set(d, mat0 + ["normal_map"], {"texture": 70}))
    mutate("emission negative", lambda d: _set(d, mat0 + ["emission"], [1.0, -1.0, 0.0, 0.0]))
    mutate("packet mismatch", lambda d: _set(d, mat0 + ["wavelengths", "nanometers", 0], 480.0))
    mutate("packet range", lambda d: (_set(d, mat0 + ["wavelengths", "nanometers", 0], 300.0),
                                      _set(d, ["lights", 0, "wavelengths", "nanometers", 0], 300.0)))
    mutate("packet pdf", lambda d: (_set(d, mat0 + ["wavelengths", "pdf", 1], 0.0),
                                    _set(d, ["lights", 0, "wavelengths", "pdf", 1], 0.0)))
    mutate("null material", lambda d: _set(d, ["materials", 0, "spectral"], None))
    mutate("duplicate material", lambda d: d["materials"].append(copy.deepcopy(d["materials"][0])))
    mutate("instance object", lambda d: _set(d, ["instances", 0, "object"], 77))
    mutate("instance geometry", lambda d: _set(d, ["instances", 0, "geometry"], 77))
    mutate("instance material", lambda d: _set(d, ["instances", 0, "material"], 77))
    mutate("instance parent", lambda d: _set(d, ["instances", 0, "parent"], 77))
    mutate("self parent", lambda d: _set(d, ["instances", 0, "parent"], d["instances"][0]["id"]))

    def cycle(d):
        d["instances"].append({**copy.deepcopy(d["instances"][0]), "id": 990, "parent": 991})
        d["instances"].append({**copy.deepcopy(d["instances"][0]), "id": 991, "parent": 990})
    mutate("parent cycle", cycle)
    mutate("singular matrix", lambda d: _set(d, ["instances", 0, "local_to_parent"], [0.0] * 15 + [1.0]))
    mutate("projective matrix", lambda d: _set(d, ["instances", 0, "local_to_parent", 12], 0.5))
    mutate("matrix arity", lambda d: _set(d, ["instances", 0, "local_to_parent"], identity()[:15]))
    mutate("two environments", lambda d: d["lights"].append(light(rng, 600, "environment")))
    mutate("no environment", lambda d: _set(d, ["lights"], [l for l in d["lights"] if l["type"] != "environment"]))
    mutate("environment radiance", lambda d: _set(d, ["lights", 0, "radiance", 0], -0.5))
    mutate("light type", lambda d: d["lights"].append({"id": 601, "type": "area"}))
    mutate("light params", lambda d: d["lights"].append({**light(rng, 602, "point"), "radiance": [1.0] * 4}))
    mutate("directional length", lambda d: d["lights"].append(
        {**light(rng, 603, "directional"), "propagation_direction": [0.0, 0.0, 2.0]}))
    mutate("spot cone", lambda d: d["lights"].append(
        {**light(rng, 604, "spot"), "inner_half_angle_radians": 1.0, "outer_half_angle_radians": 0.5}))
    mutate("point error", lambda d: d["lights"].append(
        {**light(rng, 605, "point"), "absolute_position_error": [0.0, -1.0, 0.0]}))
    mutate("duplicate light", lambda d: d["lights"].append(copy.deepcopy(d["lights"][0])))
    mutate("float overflow", lambda d: _set(d, ["cameras", 0, "model", "origin", 0], 1e39))
    mutate("float underflow", lambda d: _set(d, ["cameras", 0, "model", "origin", 0], 1e-50))
    mutate("float denormal", lambda d: _set(d, ["cameras", 0, "model", "origin", 0], 1e-40))
    mutate("t_max largest", lambda d: _set(d, ["cameras", 0, "model", "t_max"], 3.4028234663852886e38))
    mutate("string for number", lambda d: _set(d, ["render_options", 0, "seed"], "7"))
    mutate("empty scene", lambda d: (_set(d, ["instances"], []), _set(d, ["materials"], []),
                                     _set(d, ["geometries"], []), _set(d, ["lights"], [])))
    return out


def text_mutations(text, rng):
    """(label, text) pairs that break the JSON syntax or its closed-object rules at the byte level."""
    out = []
    k = text.index('"films"')
    out.append(("duplicate key", text[:k] + '"films":[],' + text[k:]))
    out.append(("trailing data", text + " x"))
    out.append(("trailing whitespace", text + " \n\t\r"))
    out.append(("two roots", text + " {}"))
    out.append(("truncated", text[: len(text) // 2]))
    out.append(("empty", ""))
    out.append(("leading zero", text.replace('"schema_version":1', '"schema_version":01', 1)))
    out.append(("plus sign", text.replace('"schema_version":1', '"schema_version":+1', 1)))
    out.append(("exponent integer", text.replace('"schema_version":1', '"schema_version":1e0', 1)))
    out.append(("bad escape", text.replace('"blackframe.scene"', '"blackframe\\q.scene"', 1)))
    out.append(("unicode escape", text.replace('"blackframe.scene"', '"blackframe\\u002escene"', 1)))
    out.append(("escaped key", text.replace('"schema_version"', '"schema\\u005fversion"', 1)))
    out.append(("lone surrogate", text.replace('"blackframe.scene"', '"\\ud800x"', 1)))
    out.append(("surrogate pair", text.replace('"float32"', '"\\ud83d\\ude00"', 1)))
    out.append(("control byte", text.replace('"blackframe.scene"', '"black\x01frame"', 1)))
    out.append(("invalid utf8", text.replace('"float32"', '"\xc3\x28"', 1)))
    out.append(("single quote", text.replace('"schema"', "'schema'", 1)))
    out.append(("comment", "/* c */" + text))
    out.append(("bom", "﻿" + text))
    out.append(("number suffix", text.replace('"schema_version":1', '"schema_version":1x', 1)))
    out.append(("fraction digit", text.replace('"schema_version":1', '"schema_version":1.', 1)))
    out.append(("literal", text.replace('"normal_map":null', '"normal_map":nul', 1)))
    out.append(("true literal", text.replace('"normal_map":null', '"normal_map":true', 1)))
    out.append(("trailing comma", text.replace('"host_image_textures":[]', '"host_image_textures":[],', 1)
                .replace('"objects"', '"objects"', 1)[:-1] + ",}"))
    return out


def limit_cases(doc_text):
    """(label, limits dict) pairs over a valid document: each budget just below and at its need."""
    out = [("defaults", None)]
    n = len(doc_text.encode())
    out.append(("encoded exact", {"maximum_encoded_bytes": n}))
    out.append(("encoded short", {"maximum_encoded_bytes": n - 1}))
    out.append(("depth 5", {"maximum_nesting_depth": 5}))
    out.append(("depth 6", {"maximum_nesting_depth": 6}))
    out.append(("values 100", {"maximum_total_values": 100}))
    out.append(("strings 64", {"maximum_total_string_bytes": 64}))
    out.append(("records 1", {"maximum_records_per_registry": 1}))
    out.append(("records 2", {"maximum_records_per_registry": 2}))
    out.append(("vertices 5", {"maximum_mesh_vertices": 5}))
    out.append(("triangles 3", {"maximum_mesh_triangles": 3}))
    out.append(("decoded 1000", {"maximum_decoded_bytes": 1000}))
    out.append(("decoded 3000", {"maximum_decoded_bytes": 3000}))
    out.append(("zero limit", {"maximum_total_values": 0}))
    out.append(("above maximum", {"maximum_nesting_depth": 129}))
    return out


LIMIT_ORDER = ["maximum_encoded_bytes", "maximum_nesting_depth", "maximum_total_values",
               "maximum_total_string_bytes", "maximum_records_per_registry", "maximum_mesh_vertices",
               "maximum_mesh_triangles", "maximum_image_scalar_values", "maximum_decoded_bytes"]
DEFAULTS = {"maximum_encoded_bytes": 64 << 20, "maximum_nesting_depth": 64, "maximum_total_values": 64_000_000,
            "maximum_total_string_bytes": 16 << 20, "maximum_records_per_registry": 1_000_000,
            "maximum_mesh_vertices": 4_000_000, "maximum_mesh_triangles": 4_000_000,
            "maximum_image_scalar_values": 16_000_000, "maximum_decoded_bytes": 512 << 20}


def limit_vector(overrides):
    """The nine limits in the reference harness's order (None: defaults)."""
    if overrides is None:
        return None
    values = dict(DEFAULTS, **overrides)
    return [values[k] for k in LIMIT_ORDER]


def corpus(seed, count):
    """(label, text bytes, limits overrides or None) triples: `count` valid documents and their mutations."""
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        doc = valid_document(rng)
        text = dumps(doc, rng)
        cases.append((f"valid {i}", text.encode("utf-8", "surrogatepass"), None))
        for label, mutated in structural_mutations(doc, rng):
            cases.append((f"{label} {i}", dumps(mutated, rng).encode(), None))
        for label, mutated in text_mutations(dumps(doc), rng):
            cases.append((f"{label} {i}", mutated.encode("latin-1") if label == "invalid utf8"
                           else mutated.encode("utf-8", "surrogatepass"), None))
        if i < 3:
            for label, lim in limit_cases(text):
                cases.append((f"{label} {i}", text.encode(), lim))
    return cases


def reference_outcome(lib, text, overrides):
    """(code, canonical bytes or b'', message) of the compiled reference for one case."""
    import ctypes as C
    lim = limit_vector(overrides)
    lim_arg = (C.c_uint64 * 9)(*lim) if lim is not None else None
    size = C.c_uint64()
    message = C.create_string_buffer(1024)
    cap = max(1 << 16, 4 * len(text) + 4096)
    out = C.create_string_buffer(cap)
    code = lib.bfref_scene_json_canonical(text, C.c_uint64(len(text)), lim_arg, out, C.c_uint64(cap), C.byref(size),
                                          message, C.c_uint64(len(message)))
    canonical = out.raw[:size.value] if code == 0 else b""
    return code, canonical, message.value.decode(errors="replace")


def product_outcome(text, overrides):
    """(code, canonical bytes or b'', message) of this library's codec for one case."""
    from bf200 import scene_json
    lim = scene_json.limits(**overrides) if overrides is not None else None
    try:
        with scene_json.SceneJson(text, lim) as doc:
            return 0, doc.canonical(lim), ""
    except scene_json.SceneJsonError as e:
        return e.code, b"", e.message


def reference_library():
    import ctypes as C
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libbfref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.bfref_scene_json_canonical.restype = C.c_int
    lib.bfref_scene_json_canonical.argtypes = [C.c_char_p, C.c_uint64, C.c_void_p, C.c_char_p, C.c_uint64,
                                               C.POINTER(C.c_uint64), C.c_char_p, C.c_uint64]
    return lib


def is_finite_number(x):
    return isinstance(x, float) and math.isfinite(x)
