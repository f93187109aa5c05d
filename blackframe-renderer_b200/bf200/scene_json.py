"""The native scene JSON codec (bf200_scene_json_*): engine::deserialize_scene_description_json and
serialize_scene_description_json (SceneDescriptionJson.hpp) behind this library's C ABI, and the
commit of a document's active selection into a render.

    from bf200 import runtime, scene_json
    with scene_json.SceneJson(text) as doc, runtime.Context(0) as ctx:
        frame = doc.frame()                       # abi.SceneJsonFrame
        scene = ctx.create_scene(None, desc=frame.scene)
        sums, counts, report = ctx.render_film(scene, frame.camera, sensor, frame.options,
                                               frame.samples_per_pixel, seed=frame.seed,
                                               precision=frame.precision)

Failures raise SceneJsonError with the reference's status code (`code`, core::StatusCode
numbering) and message.
"""
import ctypes as C

from . import abi, runtime

DEFAULT_LIMITS = dict(maximum_encoded_bytes=64 << 20, maximum_total_values=64_000_000,
                      maximum_total_string_bytes=16 << 20, maximum_mesh_vertices=4_000_000,
                      maximum_mesh_triangles=4_000_000, maximum_image_scalar_values=16_000_000,
                      maximum_decoded_bytes=512 << 20, maximum_nesting_depth=64,
                      maximum_records_per_registry=1_000_000)


class SceneJsonError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{abi.SCENE_JSON_CODES.get(code, code)}: {message}")
        self.code = code
        self.message = message


def limits(**overrides):
    """abi.SceneJsonLimits: the reference's defaults with `overrides`."""
    values = dict(DEFAULT_LIMITS, **overrides)
    return abi.SceneJsonLimits(**values)


def _lib():
    lib = runtime.library()
    if not getattr(lib, "_scene_json_bound", False):
        vp = C.c_void_p
        lib.bf200_scene_json_parse.argtypes = [C.c_char_p, C.c_uint64, C.POINTER(abi.SceneJsonLimits), C.POINTER(vp),
                                               C.c_char_p, C.c_uint64]
        lib.bf200_scene_json_parse.restype = C.c_uint32
        lib.bf200_scene_json_destroy.argtypes = [vp]
        lib.bf200_scene_json_destroy.restype = None
        lib.bf200_scene_json_write.argtypes = [vp, C.POINTER(abi.SceneJsonLimits), C.c_char_p, C.c_uint64,
                                               C.POINTER(C.c_uint64), C.c_char_p, C.c_uint64]
        lib.bf200_scene_json_write.restype = C.c_uint32
        lib.bf200_scene_json_frame.argtypes = [vp, C.POINTER(abi.SceneJsonFrame), C.c_char_p, C.c_uint64]
        lib.bf200_scene_json_frame.restype = C.c_uint32
        lib._scene_json_bound = True
    return lib


def _bytes(text):
    return text.encode() if isinstance(text, str) else bytes(text)


def parse_status(text, limits=None):
    """(code, message) of bf200_scene_json_parse without keeping the document."""
    try:
        SceneJson(text, limits).close()
    except SceneJsonError as e:
        return e.code, e.message
    return 0, ""


class SceneJson:
    """One parsed and validated document (bf200_scene_json)."""

    def __init__(self, text, limits=None):
        data = _bytes(text)
        handle = C.c_void_p()
        message = C.create_string_buffer(1024)
        code = _lib().bf200_scene_json_parse(data, len(data), C.byref(limits) if limits is not None else None,
                                             C.byref(handle), message, len(message))
        if code != 0:
            raise SceneJsonError(code, message.value.decode(errors="replace"))
        self.handle = handle

    def canonical(self, limits=None):
        """The canonical encoding (bytes) of the document."""
        lib = _lib()
        size = C.c_uint64()
        message = C.create_string_buffer(1024)
        lim = C.byref(limits) if limits is not None else None
        code = lib.bf200_scene_json_write(self.handle, lim, None, 0, C.byref(size), message, len(message))
        if code != 0:
            raise SceneJsonError(code, message.value.decode(errors="replace"))
        out = C.create_string_buffer(max(1, size.value))
        code = lib.bf200_scene_json_write(self.handle, lim, out, size.value, C.byref(size), message, len(message))
        if code != 0:
            raise SceneJsonError(code, message.value.decode(errors="replace"))
        return out.raw[:size.value]

    def frame(self):
        """abi.SceneJsonFrame of the active selection; its scene arrays live as long as this document."""
        out = abi.SceneJsonFrame()
        message = C.create_string_buffer(1024)
        code = _lib().bf200_scene_json_frame(self.handle, C.byref(out), message, len(message))
        if code != 0:
            raise SceneJsonError(code, message.value.decode(errors="replace"))
        out._owner = self
        return out

    def close(self):
        if getattr(self, "handle", None):
            _lib().bf200_scene_json_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
