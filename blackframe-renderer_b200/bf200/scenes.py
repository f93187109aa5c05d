"""Seeded synthetic scenes for the Cornell-box workloads, flattened to bf200 scene records.

A scene here is what a Blackframe caller hands the backend after FrameScene::create: triangle
meshes, one spectral material per closure mixture (resolved at the frame's single four-lane
wavelength packet), root instances in identifier order with their object_to_world matrix and
its inverse, and a constant environment. The inverse is computed with the same Gauss-Jordan
elimination, in float32, that FrameScene uses (Blackframe/Renderer/Include/Blackframe/
Renderer/MatrixOperations.hpp:30-94), so the records are bit-identical to the committed scene.

Workloads (scene geometry and transport settings):
  cornell_plain   : unit box, 5 Lambert walls, two rotated Lambert cuboids, 0.25 x 0.25 emitter
                    with radiance 17, balance MIS, depth 8, Russian roulette from depth 3.
  cornell_spheres : the same box plus a GGX conductor sphere (gold-like eta/k, alpha 0.2) and a
                    GGX rough dielectric sphere (eta 1.5, alpha 0.05), both 64 x 32 UV spheres;
                    power MIS, depth 16.
"""
import ctypes as C
import math
import struct
from fractions import Fraction

import numpy as np

from . import abi

F32 = np.float32


# ------------------------------------------------------------------------------------------------
# float32 helpers with the reference's rounding
# ------------------------------------------------------------------------------------------------

def f32_round(value):
    """Round an exact rational (or float) to the nearest float32, ties to even."""
    if isinstance(value, float):
        value = Fraction(value)
    if value == 0:
        return F32(0.0)
    # Python's float() of a Fraction is correctly rounded to double; then widen the check.
    candidate = F32(float(value))
    exact_candidate = Fraction(float(candidate))
    if exact_candidate == value:
        return candidate
    below = candidate if exact_candidate < value else np.nextafter(candidate, F32(-np.inf))
    above = np.nextafter(below, F32(np.inf))
    distance_below = value - Fraction(float(below))
    distance_above = Fraction(float(above)) - value
    if distance_below < distance_above:
        return F32(below)
    if distance_above < distance_below:
        return F32(above)
    bits = struct.unpack("<I", struct.pack("<f", float(below)))[0]
    return F32(below) if bits % 2 == 0 else F32(above)


def f32_fma(a, b, c):
    """std::fma on float32 operands: one rounding of a*b + c."""
    return f32_round(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


def sample_uniform_visible_wavelengths(unit_sample):
    """WavelengthSampling.hpp:61-88: four circularly stratified lanes over 360-830 nm."""
    u = F32(unit_sample)
    nanometers, pdfs = [], []
    pdf = F32(1.0) / F32(470.0)
    for lane in range(4):
        offset = F32(lane) / F32(4.0)
        wrap_threshold = F32(1.0) - offset
        if lane != 0 and u >= wrap_threshold:
            shifted = F32(u - wrap_threshold)
        else:
            shifted = F32(u + offset)
        nanometers.append(f32_fma(F32(470.0), shifted, F32(360.0)))
        pdfs.append(pdf)
    return nanometers, pdfs


def tabulated_spectrum(table, nanometers):
    """Resolve a piecewise-linear reflectance table [(nm, value), ...] at the packet lanes."""
    xs = [p[0] for p in table]
    ys = [p[1] for p in table]
    return [F32(np.interp(float(nm), xs, ys)) for nm in nanometers]


# ------------------------------------------------------------------------------------------------
# affine transforms in float32
# ------------------------------------------------------------------------------------------------

def identity():
    return np.eye(4, dtype=F32)


def affine_inverse(matrix):
    """MatrixOperations.hpp:30-94: partial-pivot Gauss-Jordan on [M | I] in float32."""
    augmented = np.zeros((4, 8), dtype=F32)
    augmented[:, :4] = matrix
    augmented[:, 4:] = np.eye(4, dtype=F32)
    for pivot_column in range(4):
        pivot_row = pivot_column
        pivot_magnitude = abs(augmented[pivot_row, pivot_column])
        for candidate in range(pivot_column + 1, 4):
            magnitude = abs(augmented[candidate, pivot_column])
            if magnitude > pivot_magnitude:
                pivot_magnitude = magnitude
                pivot_row = candidate
        if pivot_magnitude == 0:
            raise ValueError("A singular matrix has no inverse.")
        if pivot_row != pivot_column:
            augmented[[pivot_column, pivot_row]] = augmented[[pivot_row, pivot_column]]
        pivot = F32(augmented[pivot_column, pivot_column])
        for column in range(8):
            augmented[pivot_column, column] = F32(augmented[pivot_column, column] / pivot)
        for row in range(4):
            if row == pivot_column:
                continue
            factor = F32(augmented[row, pivot_column])
            for column in range(8):
                product = F32(factor * augmented[pivot_column, column])
                augmented[row, column] = F32(augmented[row, column] - product)
    result = augmented[:, 4:].copy()
    if not np.all(np.isfinite(result)):
        raise ValueError("Matrix inversion produced a non-finite result.")
    return result


def rotation_y_scale_translate(angle_degrees, scale, translation):
    """object_to_world = T * R_y * S, entries rounded to float32 once each."""
    angle = math.radians(angle_degrees)
    c, s = math.cos(angle), math.sin(angle)
    sx, sy, sz = scale
    m = np.zeros((4, 4), dtype=np.float64)
    m[0, 0], m[0, 1], m[0, 2] = c * sx, 0.0, s * sz
    m[1, 0], m[1, 1], m[1, 2] = 0.0, sy, 0.0
    m[2, 0], m[2, 1], m[2, 2] = -s * sx, 0.0, c * sz
    m[0, 3], m[1, 3], m[2, 3] = translation
    m[3, 3] = 1.0
    return m.astype(F32)


def uniform_scale_translate(radius, center):
    m = identity()
    m[0, 0] = m[1, 1] = m[2, 2] = F32(radius)
    m[0, 3], m[1, 3], m[2, 3] = (F32(v) for v in center)
    return m


# ------------------------------------------------------------------------------------------------
# meshes
# ------------------------------------------------------------------------------------------------

class Sphere:
    """An analytic sphere geometry: centre and radius in object space."""

    def __init__(self, centre, radius):
        self.centre = np.asarray(centre, F32).reshape(3)
        self.radius = F32(radius)
        self.positions = self.centre.reshape(1, 3)
        self.normals = np.zeros((1, 3), F32)
        self.uvs = np.zeros((1, 2), F32)
        self.triangles = np.zeros((0, 3), np.uint32)


class Mesh:
    def __init__(self, positions, normals, uvs, triangles):
        self.positions = np.asarray(positions, dtype=F32).reshape(-1, 3)
        self.normals = np.asarray(normals, dtype=F32).reshape(-1, 3)
        self.uvs = np.asarray(uvs, dtype=F32).reshape(-1, 2)
        self.triangles = np.asarray(triangles, dtype=np.uint32).reshape(-1, 3)


def quad(corners, normal):
    """Two triangles (0,1,2), (0,2,3) with one normal and unit-square UVs."""
    return Mesh(corners, [normal] * 4, [(0, 0), (1, 0), (1, 1), (0, 1)], [(0, 1, 2), (0, 2, 3)])


def unit_box():
    """Axis-aligned cube [-0.5, 0.5]^3: 6 faces x 4 vertices, flat normals, 12 triangles."""
    faces = [
        ((1, 0, 0), [(0.5, -0.5, -0.5), (0.5, 0.5, -0.5), (0.5, 0.5, 0.5), (0.5, -0.5, 0.5)]),
        ((-1, 0, 0), [(-0.5, -0.5, -0.5), (-0.5, -0.5, 0.5), (-0.5, 0.5, 0.5), (-0.5, 0.5, -0.5)]),
        ((0, 1, 0), [(-0.5, 0.5, -0.5), (-0.5, 0.5, 0.5), (0.5, 0.5, 0.5), (0.5, 0.5, -0.5)]),
        ((0, -1, 0), [(-0.5, -0.5, -0.5), (0.5, -0.5, -0.5), (0.5, -0.5, 0.5), (-0.5, -0.5, 0.5)]),
        ((0, 0, 1), [(-0.5, -0.5, 0.5), (0.5, -0.5, 0.5), (0.5, 0.5, 0.5), (-0.5, 0.5, 0.5)]),
        ((0, 0, -1), [(-0.5, -0.5, -0.5), (-0.5, 0.5, -0.5), (0.5, 0.5, -0.5), (0.5, -0.5, -0.5)]),
    ]
    positions, normals, uvs, triangles = [], [], [], []
    for normal, corners in faces:
        base = len(positions)
        positions.extend(corners)
        normals.extend([normal] * 4)
        uvs.extend([(0, 0), (1, 0), (1, 1), (0, 1)])
        triangles.extend([(base, base + 1, base + 2), (base, base + 2, base + 3)])
    return Mesh(positions, normals, uvs, triangles)


def uv_sphere(longitude=64, latitude=32):
    """Unit UV sphere with poles on +-Y, (latitude-1) rings of longitude+1 vertices.

    Same construction as the reference's tessellated test sphere
    (Tests/Backends/CPU/Embree/CornellWavefrontScene.hpp:110-180): 2*longitude*(latitude-1)
    triangles; sin/cos evaluated in float32 arithmetic on float32 angles.
    """
    stride = longitude + 1
    positions, normals, uvs, triangles = [(0, 1, 0)], [(0, 1, 0)], [(0.5, 0)], []
    pi = F32(math.pi)
    for lat in range(1, latitude):
        v = F32(lat) / F32(latitude)
        theta = F32(pi * v)
        sin_t, cos_t = F32(math.sin(theta)), F32(math.cos(theta))
        for lon in range(longitude + 1):
            u = F32(lon) / F32(longitude)
            phi = F32(F32(F32(2.0) * pi) * u)
            # cos/sin of the float angle leave residues like cos(pi/2) = -4.4e-8 where the
            # exact value is zero; they are snapped to zero so the scalar oracle's exact
            # float-expansion arithmetic does not underflow on them.
            cos_phi, sin_phi = F32(math.cos(phi)), F32(math.sin(phi))
            cos_phi = F32(0.0) if abs(cos_phi) < 1e-6 else cos_phi
            sin_phi = F32(0.0) if abs(sin_phi) < 1e-6 else sin_phi
            x = F32(sin_t * cos_phi)
            z = F32(sin_t * sin_phi)
            positions.append((x, cos_t, z))
            normals.append((x, cos_t, z))
            uvs.append((u, v))
    bottom = len(positions)
    positions.append((0, -1, 0))
    normals.append((0, -1, 0))
    uvs.append((0.5, 1))
    first = 1
    for lon in range(longitude):
        triangles.append((0, first + lon + 1, first + lon))
    for lat in range(1, latitude - 1):
        upper_ring = 1 + (lat - 1) * stride
        lower_ring = upper_ring + stride
        for lon in range(longitude):
            upper, lower = upper_ring + lon, lower_ring + lon
            triangles.append((upper, lower + 1, lower))
            triangles.append((upper, upper + 1, lower + 1))
    last = bottom - stride
    for lon in range(longitude):
        triangles.append((bottom, last + lon, last + lon + 1))
    return Mesh(positions, normals, uvs, triangles)


# ------------------------------------------------------------------------------------------------
# scene assembly
# ------------------------------------------------------------------------------------------------

def lambertian(reflectance):
    return [(abi.CLOSURE_LAMBERTIAN, abi.LOBE_DIFFUSE | abi.LOBE_REFLECTION,
             [F32(v) for v in reflectance], [0.0] * 10)]


def rough_conductor(coefficient, eta, k, alpha_x, alpha_y):
    params = list(eta) + list(k) + [alpha_x, alpha_y]
    return [(abi.CLOSURE_ROUGH_CONDUCTOR, abi.LOBE_GLOSSY | abi.LOBE_REFLECTION,
             [F32(v) for v in coefficient], [F32(v) for v in params])]


def rough_dielectric(coefficient, exterior_eta, interior_eta, alpha_x, alpha_y):
    params = [exterior_eta, interior_eta, alpha_x, alpha_y] + [0.0] * 6
    return [(abi.CLOSURE_ROUGH_DIELECTRIC,
             abi.LOBE_GLOSSY | abi.LOBE_REFLECTION | abi.LOBE_TRANSMISSION,
             [F32(v) for v in coefficient], [F32(v) for v in params])]


def rough_diffuse(reflectance, roughness):
    """Energy-preserving Oren-Nayar reflection (ClosureSet::append_rough_diffuse_reflection)."""
    return [(abi.CLOSURE_ROUGH_DIFFUSE, abi.LOBE_DIFFUSE | abi.LOBE_REFLECTION, [F32(v) for v in reflectance],
             [F32(roughness)] + [0.0] * 9)]


def specular_reflection(reflectance):
    return [(abi.CLOSURE_SPECULAR_REFLECTION, abi.LOBE_SPECULAR | abi.LOBE_REFLECTION,
             [F32(v) for v in reflectance], [0.0] * 10)]


def specular_transmission(transmittance, exterior_eta, interior_eta):
    return [(abi.CLOSURE_SPECULAR_TRANSMISSION, abi.LOBE_SPECULAR | abi.LOBE_TRANSMISSION,
             [F32(v) for v in transmittance], [F32(exterior_eta), F32(interior_eta)] + [0.0] * 8)]


class SceneBuilder:
    """Accumulates meshes, materials and root instances; `desc()` returns a SceneDesc whose
    arrays stay alive as long as the builder does."""

    def __init__(self, wavelength_sample=0.1, environment=(0.0, 0.0, 0.0, 0.0)):
        self.nanometers, self.pdfs = sample_uniform_visible_wavelengths(wavelength_sample)
        self.environment = [F32(v) for v in environment]
        self.meshes, self.materials, self.instances = [], [], []
        self.punctual = []  # abi.PunctualLight records, registry order
        self.probabilities = {}  # material index -> component probabilities (default uniform)

    def add_mesh(self, mesh):
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    def add_material(self, closures, emission=(0.0, 0.0, 0.0, 0.0), frame_mode=0, probabilities=None):
        """closures: up to 8 (kind, lobes, weight[4], parameters[10]) records; probabilities: their
        component probabilities (SceneClosureMixture), uniform when not given."""
        self.materials.append((closures, [F32(v) for v in emission], frame_mode))
        if probabilities is not None:
            self.probabilities[len(self.materials) - 1] = [F32(v) for v in probabilities]
        return len(self.materials) - 1

    def add_point_light(self, position, intensity, error=(0.0, 0.0, 0.0)):
        return self._punctual(abi.PUNCTUAL_POINT, position, error, (0.0, 0.0, 0.0), 0.0, 0.0, intensity)

    def add_directional_light(self, propagation_direction, irradiance):
        return self._punctual(abi.PUNCTUAL_DIRECTIONAL, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), propagation_direction, 0.0,
                              0.0, irradiance)

    def add_spot_light(self, position, emission_direction, inner_half_angle, outer_half_angle, intensity,
                       error=(0.0, 0.0, 0.0)):
        return self._punctual(abi.PUNCTUAL_SPOT, position, error, emission_direction, inner_half_angle,
                              outer_half_angle, intensity)

    def _punctual(self, kind, position, error, direction, inner, outer, spectrum):
        light = abi.PunctualLight()
        light.kind = kind
        for a in range(3):
            light.position[a], light.position_error[a] = F32(position[a]), F32(error[a])
            light.direction[a] = F32(direction[a])
        light.inner_half_angle, light.outer_half_angle = F32(inner), F32(outer)
        for lane in range(4):
            light.spectrum[lane] = F32(spectrum[lane])
        self.punctual.append(light)
        return len(self.punctual) - 1

    def add_instance(self, mesh_index, material_index, object_to_world=None, mask=0xFFFFFFFF):
        matrix = identity() if object_to_world is None else np.asarray(object_to_world, F32)
        self.instances.append((mesh_index, material_index, matrix, mask))
        return len(self.instances) - 1

    @property
    def triangle_count(self):
        return sum(len(m.triangles) for m in self.meshes)

    def desc(self):
        geometries = (abi.Geometry * len(self.meshes))()
        positions, normals, uvs, triangles = [], [], [], []
        vertex_offset = triangle_offset = 0
        for index, mesh in enumerate(self.meshes):
            g = geometries[index]
            g.geometry_id = 100 + index
            g.vertex_offset, g.vertex_count = vertex_offset, len(mesh.positions)
            g.triangle_offset, g.triangle_count = triangle_offset, len(mesh.triangles)
            if isinstance(mesh, Sphere):
                g.kind, g.radius = abi.GEOMETRY_SPHERE, float(mesh.radius)
            positions.append(mesh.positions)
            normals.append(mesh.normals)
            uvs.append(mesh.uvs)
            triangles.append(mesh.triangles)
            vertex_offset += len(mesh.positions)
            triangle_offset += len(mesh.triangles)
        self._positions = np.ascontiguousarray(np.concatenate(positions), F32)
        self._normals = np.ascontiguousarray(np.concatenate(normals), F32)
        self._uvs = np.ascontiguousarray(np.concatenate(uvs), F32)
        self._triangles = np.ascontiguousarray(np.concatenate(triangles), np.uint32)

        closure_records = []
        materials = (abi.Material * len(self.materials))()
        for index, (closures, emission, frame_mode) in enumerate(self.materials):
            m = materials[index]
            m.material_id = 200 + index
            m.closure_offset, m.closure_count = len(closure_records), len(closures)
            m.frame_mode = frame_mode
            m.tangent_rotation_radians = 0.0
            for c in range(len(closures)):
                m.component_probabilities[c] = self.probabilities.get(index, [1.0 / len(closures)] * len(closures))[c]
            for lane in range(4):
                m.emitted_radiance[lane] = emission[lane]
            closure_records.extend(closures)
        closures = (abi.Closure * max(1, len(closure_records)))()
        for index, (kind, lobes, weight, params) in enumerate(closure_records):
            closures[index].kind, closures[index].lobes = kind, lobes
            for lane in range(4):
                closures[index].weight[lane] = weight[lane]
            for p in range(10):
                closures[index].parameters[p] = params[p]

        instances = (abi.Instance * len(self.instances))()
        for index, (mesh_index, material_index, matrix, mask) in enumerate(self.instances):
            inst = instances[index]
            inst.instance_id = 300 + index
            inst.object_id = 400 + index
            inst.geometry_index, inst.material_index = mesh_index, material_index
            inst.visibility_mask = mask
            inverse = affine_inverse(matrix)
            for e in range(16):
                inst.object_to_world[e] = matrix.flat[e]
                inst.world_to_object[e] = inverse.flat[e]

        desc = abi.SceneDesc()
        desc.struct_size = C.sizeof(abi.SceneDesc)
        desc.geometry_count = len(self.meshes)
        desc.vertex_count = len(self._positions)
        desc.triangle_count = len(self._triangles)
        desc.material_count = len(self.materials)
        desc.closure_count = len(closure_records)
        desc.instance_count = len(self.instances)
        desc.geometries = geometries
        desc.positions = self._positions.ctypes.data_as(C.POINTER(abi.f32))
        desc.normals = self._normals.ctypes.data_as(C.POINTER(abi.f32))
        desc.texture_coordinates = self._uvs.ctypes.data_as(C.POINTER(abi.f32))
        desc.triangles = self._triangles.ctypes.data_as(C.POINTER(abi.u32))
        desc.materials = materials
        desc.closures = closures
        desc.instances = instances
        for lane in range(4):
            desc.wavelength_nanometers[lane] = self.nanometers[lane]
            desc.wavelength_pdf[lane] = self.pdfs[lane]
            desc.environment_radiance[lane] = self.environment[lane]
        punctual = (abi.PunctualLight * max(1, len(self.punctual)))(*self.punctual)
        desc.punctual_light_count = len(self.punctual)
        desc.punctual_lights = punctual
        self._keep = (geometries, materials, closures, instances, punctual)
        return desc


RED_WALL = [(360, 0.05), (560, 0.06), (600, 0.35), (640, 0.60), (830, 0.62)]
GREEN_WALL = [(360, 0.08), (470, 0.15), (530, 0.55), (580, 0.45), (640, 0.10), (830, 0.08)]
# Gold-like relative IOR (eta, k) tables; resolved at the packet lanes.
GOLD_ETA = [(360, 1.5), (450, 1.3), (500, 0.9), (550, 0.40), (600, 0.25), (700, 0.16),
            (830, 0.19)]
GOLD_K = [(360, 1.9), (450, 1.85), (500, 1.85), (550, 2.3), (600, 2.9), (700, 3.9), (830, 5.3)]


def cornell_box(builder, with_spheres, analytic_spheres=False):
    """Walls, emitter and cuboids of the Cornell workloads; spheres when `with_spheres`: 64 x 32
    UV-sphere meshes, or analytic spheres (centre and radius in world space, identity instance
    transforms, as renderer::Sphere takes them) when `analytic_spheres`."""
    nm = builder.nanometers
    white = builder.add_material(lambertian([0.73] * 4))
    red = builder.add_material(lambertian(tabulated_spectrum(RED_WALL, nm)))
    green = builder.add_material(lambertian(tabulated_spectrum(GREEN_WALL, nm)))
    light = builder.add_material(lambertian([0.0] * 4), emission=(17.0, 17.0, 17.0, 17.0))

    floor = builder.add_mesh(quad([(-1, -1, 0), (-1, -1, 2), (1, -1, 2), (1, -1, 0)], (0, 1, 0)))
    ceiling = builder.add_mesh(quad([(-1, 1, 0), (1, 1, 0), (1, 1, 2), (-1, 1, 2)], (0, -1, 0)))
    back = builder.add_mesh(quad([(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)], (0, 0, 1)))
    left = builder.add_mesh(quad([(-1, -1, 0), (-1, 1, 0), (-1, 1, 2), (-1, -1, 2)], (1, 0, 0)))
    right = builder.add_mesh(quad([(1, -1, 0), (1, -1, 2), (1, 1, 2), (1, 1, 0)], (-1, 0, 0)))
    emitter = builder.add_mesh(quad([(-0.125, 0.985, 0.875), (0.125, 0.985, 0.875),
                                     (0.125, 0.985, 1.125), (-0.125, 0.985, 1.125)],
                                    (0, -1, 0)))
    box = builder.add_mesh(unit_box())

    builder.add_instance(floor, white)
    builder.add_instance(ceiling, white)
    builder.add_instance(back, white)
    builder.add_instance(left, red)
    builder.add_instance(right, green)
    builder.add_instance(emitter, light)
    builder.add_instance(box, white, rotation_y_scale_translate(18.0, (0.6, 1.2, 0.6),
                                                               (-0.35, -0.4, 0.65)))
    builder.add_instance(box, white, rotation_y_scale_translate(-15.0, (0.6, 0.6, 0.6),
                                                               (0.4, -0.7, 1.25)))
    if with_spheres:
        conductor = builder.add_material(rough_conductor(
            [1.0] * 4, tabulated_spectrum(GOLD_ETA, nm), tabulated_spectrum(GOLD_K, nm), 0.2, 0.2))
        dielectric = builder.add_material(rough_dielectric([1.0] * 4, 1.0, 1.5, 0.05, 0.05))
        if analytic_spheres:
            builder.add_instance(builder.add_mesh(Sphere((0.4, -0.15, 1.25), 0.25)), conductor)
            builder.add_instance(builder.add_mesh(Sphere((-0.3, -0.75, 1.55), 0.25)), dielectric)
            return builder
        sphere = builder.add_mesh(uv_sphere())
        builder.add_instance(sphere, conductor, uniform_scale_translate(0.25, (0.4, -0.15, 1.25)))
        builder.add_instance(sphere, dielectric,
                             uniform_scale_translate(0.25, (-0.3, -0.75, 1.55)))
    return builder


def cornell_layered(builder):
    """The Cornell box with every closure kind, closure mixtures and punctual lights: an
    energy-preserving Oren-Nayar back wall, a layered floor (Lambert under a GGX conductor coat,
    component probabilities 0.6 / 0.4), a mirror cuboid, a glass cuboid (specular reflection and
    transmission, 0.1 / 0.9, coincident delta atoms never merge here since their directions
    differ), a rough-diffuse plus conductor sphere, the ceiling emitter, a point light, a spot light
    and a directional light entering through the open front."""
    nm = builder.nanometers
    white = builder.add_material(lambertian([0.73] * 4))
    back_eon = builder.add_material(rough_diffuse([0.7, 0.72, 0.75, 0.73], 0.6))
    red = builder.add_material(lambertian(tabulated_spectrum(RED_WALL, nm)))
    green = builder.add_material(lambertian(tabulated_spectrum(GREEN_WALL, nm)))
    light = builder.add_material(lambertian([0.0] * 4), emission=(17.0, 17.0, 17.0, 17.0))
    gold_eta, gold_k = tabulated_spectrum(GOLD_ETA, nm), tabulated_spectrum(GOLD_K, nm)
    layered = builder.add_material(lambertian([0.5, 0.45, 0.4, 0.42]) +
                                   rough_conductor([0.6] * 4, gold_eta, gold_k, 0.3, 0.15), probabilities=[0.6, 0.4])
    mirror = builder.add_material(specular_reflection([0.9, 0.92, 0.95, 0.9]))
    glass = builder.add_material(specular_reflection([0.08] * 4) + specular_transmission([0.92] * 4, 1.0, 1.5),
                                 probabilities=[0.1, 0.9])
    rough_metal = builder.add_material(rough_diffuse([0.3, 0.5, 0.4, 0.35], 1.0) +
                                       rough_conductor([0.5] * 4, gold_eta, gold_k, 0.2, 0.2))

    floor = builder.add_mesh(quad([(-1, -1, 0), (-1, -1, 2), (1, -1, 2), (1, -1, 0)], (0, 1, 0)))
    ceiling = builder.add_mesh(quad([(-1, 1, 0), (1, 1, 0), (1, 1, 2), (-1, 1, 2)], (0, -1, 0)))
    back = builder.add_mesh(quad([(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)], (0, 0, 1)))
    left = builder.add_mesh(quad([(-1, -1, 0), (-1, 1, 0), (-1, 1, 2), (-1, -1, 2)], (1, 0, 0)))
    right = builder.add_mesh(quad([(1, -1, 0), (1, -1, 2), (1, 1, 2), (1, 1, 0)], (-1, 0, 0)))
    emitter = builder.add_mesh(quad([(-0.125, 0.985, 0.875), (0.125, 0.985, 0.875),
                                     (0.125, 0.985, 1.125), (-0.125, 0.985, 1.125)],
                                    (0, -1, 0)))
    box = builder.add_mesh(unit_box())
    builder.add_instance(floor, layered)
    builder.add_instance(ceiling, white)
    builder.add_instance(back, back_eon)
    builder.add_instance(left, red)
    builder.add_instance(right, green)
    builder.add_instance(emitter, light)
    builder.add_instance(box, mirror, rotation_y_scale_translate(18.0, (0.6, 1.2, 0.6), (-0.35, -0.4, 0.65)))
    builder.add_instance(box, glass, rotation_y_scale_translate(-15.0, (0.6, 0.6, 0.6), (0.4, -0.7, 1.25)))
    sphere = builder.add_mesh(uv_sphere())
    builder.add_instance(sphere, rough_metal, uniform_scale_translate(0.25, (0.45, 0.1, 0.7)))
    builder.add_point_light((-0.5, 0.7, 1.4), (0.8, 0.7, 0.6, 0.5), error=(1e-6, 1e-6, 1e-6))
    builder.add_spot_light((0.6, 0.8, 1.8), (-0.37139067, -0.74278134, -0.55708601), 0.3, 0.6,
                           (2.0, 2.2, 2.4, 2.6))
    builder.add_directional_light((0.0, -0.6, -0.8), (0.4, 0.35, 0.3, 0.25))
    return builder


CAMERA_ORIGIN = (0.0, 0.0, 4.0)
CAMERA_TARGET = (0.0, -0.05, 0.92)
CAMERA_VFOV = 0.70
PATH_TIME = 0.5


def camera_frame_inputs(origin=CAMERA_ORIGIN, target=CAMERA_TARGET):
    """Camera frame seed looking from `origin` at `target` (default: the Cornell workloads):
    normal = -forward, tangent seed +X (the construction of
    Tests/Backends/CPU/Embree/CornellWavefrontScene.hpp:380-395)."""
    origin = np.array(origin, F32)
    target = np.array(target, F32)
    seed = (target - origin).astype(F32)
    length = np.sqrt(F32(F32(F32(seed[0] * seed[0]) + F32(seed[1] * seed[1])) +
                         F32(seed[2] * seed[2])))
    forward = (seed / length).astype(F32)
    normal = (-forward).astype(F32)
    return origin, normal, np.array([1.0, 0.0, 0.0], F32)


# ------------------------------------------------------------------------------------------------
# BVH-stress scene: seeded displaced icospheres, instanced with random affine transforms
# ------------------------------------------------------------------------------------------------

def icosphere(subdivisions):
    """Unit icosphere: the icosahedron with every triangle split in four `subdivisions` times,
    new vertices projected to the sphere (20 * 4^s triangles, 10 * 4^s + 2 vertices); float64."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
                  (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
                  (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
                  (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], np.int64)
    for _ in range(subdivisions):
        n = len(f)
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        unique, inverse = np.unique(np.sort(edges, axis=1), axis=0, return_inverse=True)
        mid = v[unique[:, 0]] + v[unique[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        index = len(v) + inverse.reshape(-1)
        v = np.concatenate([v, mid])
        a, b, c = index[:n], index[n:2 * n], index[2 * n:]
        f = np.concatenate([np.stack([f[:, 0], a, c], 1), np.stack([a, f[:, 1], b], 1),
                            np.stack([c, b, f[:, 2]], 1), np.stack([a, b, c], 1)])
    return v, f


def displaced_icosphere(subdivisions, amplitude, seed):
    """Icosphere with every vertex moved along its normal by amplitude * U[-1, 1] (seeded).

    At subdivision 7 the edges are about 0.01 long, so a 0.05 displacement makes neighbouring
    faces point in very different directions, and averaged vertex normals would leave the
    geometric-normal hemisphere of some faces, which the surface reconstruction rejects
    (no substitution). Faces are therefore flat-shaded: every triangle gets its own three
    vertices (the displaced positions, so the surface stays watertight) carrying its face normal.
    """
    v, f = icosphere(subdivisions)
    rng = np.random.default_rng(seed)
    v = v * (1.0 + amplitude * rng.uniform(-1.0, 1.0, len(v)))[:, None]
    v32 = v.astype(F32)
    corners = v32[f].reshape(-1, 3)
    p = v32[f].astype(np.float64)
    face_n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    face_n /= np.linalg.norm(face_n, axis=1, keepdims=True)
    normals = np.repeat(face_n, 3, axis=0).astype(F32)
    triangles = np.arange(3 * len(f), dtype=np.uint32).reshape(-1, 3)
    return Mesh(corners, normals, np.zeros((len(corners), 2), F32), triangles)


def grid_quad(center, size, divisions, y, normal_down=True):
    """Square of divisions x divisions cells (2 triangles each) in the plane y, facing -y."""
    xs = np.linspace(center[0] - size / 2, center[0] + size / 2, divisions + 1)
    zs = np.linspace(center[1] - size / 2, center[1] + size / 2, divisions + 1)
    gx, gz = np.meshgrid(xs, zs, indexing="ij")
    positions = np.stack([gx.ravel(), np.full(gx.size, y), gz.ravel()], 1)
    idx = np.arange((divisions + 1) ** 2).reshape(divisions + 1, divisions + 1)
    a, b = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel()
    c, d = idx[1:, 1:].ravel(), idx[:-1, 1:].ravel()
    if normal_down:  # counter-clockwise seen from below
        tris = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    else:
        tris = np.concatenate([np.stack([a, c, b], 1), np.stack([a, d, c], 1)])
    normal = (0.0, -1.0, 0.0) if normal_down else (0.0, 1.0, 0.0)
    return Mesh(positions.astype(F32), np.tile(np.array(normal, F32), (len(positions), 1)),
                np.zeros((len(positions), 2), F32), tris.astype(np.uint32))


def random_rotation(rng):
    """Uniform random rotation matrix (normalised Gaussian quaternion)."""
    q = rng.normal(size=4)
    w, x, y, z = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def bvh_stress(builder, subdivisions=7, instances=40, light_divisions=32):
    """The BVH-stress scene: 3 displaced icospheres (amplitude 0.05, seed k) instanced
    `instances` times with uniform rotation, scale U[0.5, 1.5] and translation U[-10, 10]^3
    (seed 1234); materials 50 % Lambert (albedo U[0.2, 0.8] per lane), 30 % anisotropic GGX
    conductor (alpha_x, alpha_y U[0.05, 0.6]), 20 % GGX dielectric (eta 1.5); a ground quad; one
    emissive 2 * light_divisions^2-triangle grid above; the environment is set by the builder."""
    nm = builder.nanometers
    meshes = [builder.add_mesh(displaced_icosphere(subdivisions, 0.05, k)) for k in range(3)]
    rng = np.random.default_rng(1234)
    gold_eta, gold_k = tabulated_spectrum(GOLD_ETA, nm), tabulated_spectrum(GOLD_K, nm)
    for i in range(instances):
        kind = rng.uniform()
        if kind < 0.5:
            material = builder.add_material(lambertian(rng.uniform(0.2, 0.8, 4)))
        elif kind < 0.8:
            ax, ay = rng.uniform(0.05, 0.6, 2)
            material = builder.add_material(rough_conductor([1.0] * 4, gold_eta, gold_k, ax, ay))
        else:
            material = builder.add_material(rough_dielectric([1.0] * 4, 1.0, 1.5, 0.1, 0.1))
        m = identity()
        m[:3, :3] = (random_rotation(rng) * rng.uniform(0.5, 1.5)).astype(F32)
        m[:3, 3] = rng.uniform(-10.0, 10.0, 3).astype(F32)
        builder.add_instance(meshes[i % 3], material, m)
    ground = builder.add_mesh(quad([(-40, -12, -40), (-40, -12, 40), (40, -12, 40), (40, -12, -40)], (0, 1, 0)))
    builder.add_instance(ground, builder.add_material(lambertian([0.5] * 4)))
    light = builder.add_mesh(grid_quad((0.0, 0.0), 16.0, light_divisions, 14.0))
    builder.add_instance(light, builder.add_material(lambertian([0.0] * 4), emission=(10.0, 10.0, 10.0, 10.0)))
    return builder


# ------------------------------------------------------------------------------------------------
# Batch of uneven scenes: seeded Cornell shells holding displaced icospheres
# ------------------------------------------------------------------------------------------------

def batch_job(seed):
    """One job of the 64-scene batch (seed s = 0..63): film side log-uniform in [64, 512],
    unique triangle count log-uniform in [1k, 200k] reached with displaced icospheres (the largest
    subdivision with 20 * 4^s below the target, as many as round to it) inside the Cornell walls
    and light,
    spp log-uniform in [8, 128], depth uniform in {4..16}, materials drawn like the BVH-stress
    scene's. Returns (builder, options, (width, height, spp))."""
    rng = np.random.default_rng(10_000 + seed)
    side = int(round(math.exp(rng.uniform(math.log(64), math.log(512)))))
    target = math.exp(rng.uniform(math.log(1_000), math.log(200_000)))
    spp = int(round(math.exp(rng.uniform(math.log(8), math.log(128)))))
    depth = int(rng.integers(4, 17))
    builder = SceneBuilder()
    nm = builder.nanometers
    white = builder.add_material(lambertian([0.73] * 4))
    red = builder.add_material(lambertian(tabulated_spectrum(RED_WALL, nm)))
    green = builder.add_material(lambertian(tabulated_spectrum(GREEN_WALL, nm)))
    light = builder.add_material(lambertian([0.0] * 4), emission=(17.0, 17.0, 17.0, 17.0))
    walls = [
        (quad([(-1, -1, 0), (-1, -1, 2), (1, -1, 2), (1, -1, 0)], (0, 1, 0)), white),
        (quad([(-1, 1, 0), (1, 1, 0), (1, 1, 2), (-1, 1, 2)], (0, -1, 0)), white),
        (quad([(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)], (0, 0, 1)), white),
        (quad([(-1, -1, 0), (-1, 1, 0), (-1, 1, 2), (-1, -1, 2)], (1, 0, 0)), red),
        (quad([(1, -1, 0), (1, -1, 2), (1, 1, 2), (1, 1, 0)], (-1, 0, 0)), green),
        (quad([(-0.125, 0.985, 0.875), (0.125, 0.985, 0.875), (0.125, 0.985, 1.125), (-0.125, 0.985, 1.125)],
              (0, -1, 0)), light),
    ]
    for mesh, material in walls:
        builder.add_instance(builder.add_mesh(mesh), material)
    subdivision = max(1, int(math.floor(math.log(target / 20.0, 4))))
    copies = max(1, int(round(target / (20 * 4 ** subdivision))))
    gold_eta, gold_k = tabulated_spectrum(GOLD_ETA, nm), tabulated_spectrum(GOLD_K, nm)
    for c in range(copies):
        kind = rng.uniform()
        if kind < 0.5:
            material = builder.add_material(lambertian(rng.uniform(0.2, 0.8, 4)))
        elif kind < 0.8:
            ax, ay = rng.uniform(0.05, 0.6, 2)
            material = builder.add_material(rough_conductor([1.0] * 4, gold_eta, gold_k, ax, ay))
        else:
            material = builder.add_material(rough_dielectric([1.0] * 4, 1.0, 1.5, 0.1, 0.1))
        radius = 0.25 if copies == 1 else 0.2
        centre = (rng.uniform(-0.6, 0.6), rng.uniform(-0.7, 0.3), rng.uniform(0.5, 1.6))
        sphere = builder.add_mesh(displaced_icosphere(subdivision, 0.05, 100 * seed + c))
        builder.add_instance(sphere, material, uniform_scale_translate(radius, centre))
    options = abi.default_options(mis="power", max_depth=depth)
    return builder, options, (side, side, spp)


# ------------------------------------------------------------------------------------------------
# Adjoint workload: the Cornell box and spheres with a displaced icosphere in place of the cuboids;
# Lambert albedos from an 8-coefficient spectral basis
# ------------------------------------------------------------------------------------------------

SPECTRAL_KNOTS = [360.0 + k * 470.0 / 7.0 for k in range(8)]
ADJOINT_WHITE, ADJOINT_RED, ADJOINT_GREEN, ADJOINT_LIGHT, ADJOINT_CONDUCTOR, ADJOINT_DIELECTRIC, ADJOINT_ICOSPHERE = \
    range(7)
ADJOINT_ALBEDO_MATERIALS = (ADJOINT_WHITE, ADJOINT_RED, ADJOINT_GREEN, ADJOINT_ICOSPHERE)
ADJOINT_LIGHT_RADIANCE = 17.0


def spectral_basis(nanometers):
    """B[k, lane]: 8 piecewise-linear tent functions over 360-830 nm with knots every 470/7 nm (a
    partition of unity), evaluated at the packet's wavelengths."""
    step = 470.0 / 7.0
    basis = np.zeros((8, len(nanometers)))
    for lane, nm in enumerate(nanometers):
        for k, knot in enumerate(SPECTRAL_KNOTS):
            basis[k, lane] = max(0.0, 1.0 - abs(float(nm) - knot) / step)
    return basis


def adjoint_parameters():
    """Base parameters of the adjoint workload: albedo coefficients (white, red, green, icosphere
    x 8 knots), the GGX alpha of the conductor and of the dielectric, the light's radiance scale."""
    albedo = np.array([[0.73] * 8, tabulated_spectrum(RED_WALL, SPECTRAL_KNOTS),
                       tabulated_spectrum(GREEN_WALL, SPECTRAL_KNOTS), [0.5] * 8], np.float64)
    return {"albedo": albedo, "alpha": np.array([0.2, 0.05]), "light_scale": 1.0}


def perturbed_parameters(params, seed=7, sigma=0.1):
    """params + N(0, sigma) (seeded), kept in the valid range (albedo in [0.02, 0.98], alpha in
    [0.01, 1], scale > 0.1): the parameters of the target image."""
    rng = np.random.default_rng(seed)
    return {"albedo": np.clip(params["albedo"] + rng.normal(0.0, sigma, params["albedo"].shape), 0.02, 0.98),
            "alpha": np.clip(params["alpha"] + rng.normal(0.0, sigma, 2), 0.01, 1.0),
            "light_scale": max(0.1, params["light_scale"] + rng.normal(0.0, sigma))}


def cornell_shell(builder, white, red, green, light):
    """The five walls and the emitter quad of the Cornell workloads (6 meshes, then 6 instances)."""
    meshes = [quad([(-1, -1, 0), (-1, -1, 2), (1, -1, 2), (1, -1, 0)], (0, 1, 0)),
              quad([(-1, 1, 0), (1, 1, 0), (1, 1, 2), (-1, 1, 2)], (0, -1, 0)),
              quad([(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)], (0, 0, 1)),
              quad([(-1, -1, 0), (-1, 1, 0), (-1, 1, 2), (-1, -1, 2)], (1, 0, 0)),
              quad([(1, -1, 0), (1, -1, 2), (1, 1, 2), (1, 1, 0)], (-1, 0, 0)),
              quad([(-0.125, 0.985, 0.875), (0.125, 0.985, 0.875), (0.125, 0.985, 1.125),
                    (-0.125, 0.985, 1.125)], (0, -1, 0))]
    index = [builder.add_mesh(m) for m in meshes]
    for mesh, material in zip(index, (white, white, white, red, green, light)):
        builder.add_instance(mesh, material)


def adjoint_icosphere(builder, params, subdivisions=6):
    """The adjoint workload's scene at `params` (see adjoint_parameters). The icosphere is
    subdivision 6 (81,920 triangles), displaced by 0.05 * U[-1, 1] (seed 0), radius 0.35. Materials
    are in ADJOINT_* order."""
    nm = builder.nanometers
    lanes = params["albedo"] @ spectral_basis(nm)
    white = builder.add_material(lambertian(lanes[0]))
    red = builder.add_material(lambertian(lanes[1]))
    green = builder.add_material(lambertian(lanes[2]))
    light = builder.add_material(lambertian([0.0] * 4),
                                 emission=(ADJOINT_LIGHT_RADIANCE * params["light_scale"],) * 4)
    conductor = builder.add_material(rough_conductor(
        [1.0] * 4, tabulated_spectrum(GOLD_ETA, nm), tabulated_spectrum(GOLD_K, nm), params["alpha"][0],
        params["alpha"][0]))
    dielectric = builder.add_material(rough_dielectric([1.0] * 4, 1.0, 1.5, params["alpha"][1], params["alpha"][1]))
    ico = builder.add_material(lambertian(lanes[3]))
    cornell_shell(builder, white, red, green, light)
    sphere = builder.add_mesh(uv_sphere())
    builder.add_instance(sphere, conductor, uniform_scale_translate(0.25, (0.4, -0.15, 1.25)))
    builder.add_instance(sphere, dielectric, uniform_scale_translate(0.25, (-0.3, -0.75, 1.55)))
    blob = builder.add_mesh(displaced_icosphere(subdivisions, 0.05, 0))
    builder.add_instance(blob, ico, uniform_scale_translate(0.35, (-0.35, -0.6, 0.75)))
    return builder


def basis_gradients(material_gradients, nanometers):
    """dLoss/d(albedo coefficient k) of each albedo material from the per-lane closure-weight
    gradients (records of 8 doubles: weight lanes 0..3 first): sum over lanes of dLoss/dw_l B_k(l)."""
    basis = spectral_basis(nanometers)
    g = np.asarray(material_gradients, np.float64)
    return np.stack([basis @ g[m, :4] for m in ADJOINT_ALBEDO_MATERIALS])


BVH_STRESS_CAMERA = ((0.0, 2.0, 24.0), (0.0, -3.0, 0.0))  # origin, target
BVH_STRESS_VFOV = 0.9

WORKLOADS = {
    # name: (width, height, spp, max_depth, mis, scene)
    "cornell_plain_64": (64, 64, 16, 8, "balance", "cornell"),
    "cornell_spheres_256": (256, 256, 256, 16, "power", "cornell_spheres"),
    "bvh_stress_1080p": (1920, 1080, 64, 16, "power", "bvh_stress"),
    "adjoint_icosphere_256": (256, 256, 64, 8, "power", "adjoint_icosphere"),
    "cornell_analytic_256": (256, 256, 256, 16, "power", "cornell_analytic"),
    "cornell_layered_256": (256, 256, 64, 16, "power", "cornell_layered"),
}


def build_workload(name):
    width, height, spp, depth, mis, scene = WORKLOADS[name]
    if scene == "bvh_stress":
        builder = bvh_stress(SceneBuilder(environment=(0.5, 0.5, 0.5, 0.5)))
    elif scene == "adjoint_icosphere":
        # Russian roulette off: with fixed samples the weight and emission gradients are then the
        # exact derivatives of the rendered loss
        builder = adjoint_icosphere(SceneBuilder(), adjoint_parameters())
        return builder, abi.default_options(mis=mis, max_depth=depth, roulette=False), (width, height, spp)
    elif scene == "cornell_layered":
        builder = cornell_layered(SceneBuilder())
    else:
        builder = cornell_box(SceneBuilder(), with_spheres=scene in ("cornell_spheres", "cornell_analytic"),
                              analytic_spheres=scene == "cornell_analytic")
    options = abi.default_options(mis=mis, max_depth=depth)
    return builder, options, (width, height, spp)


def workload_camera(name):
    """(origin, normal, tangent seed, vertical fov) of a workload's camera."""
    if WORKLOADS[name][5] == "bvh_stress":
        return (*camera_frame_inputs(*BVH_STRESS_CAMERA), BVH_STRESS_VFOV)
    return (*camera_frame_inputs(), CAMERA_VFOV)
