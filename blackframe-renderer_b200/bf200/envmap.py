"""The environment-map light through the C ABI (bf200_environment_map_*): EnvironmentMapLightT<float>
of EnvironmentLights.hpp -- create, sample_li, pdf_li, le and power -- with the batch queries run on
the context's device. Arrays in and out are numpy; statuses are bf200_environment_status codes."""
import ctypes as C

import numpy as np

from . import runtime

STATUS_OK, INVALID_SAMPLE, INVALID_DIRECTION, ESCAPED, UNSTABLE, NOT_REPRESENTABLE = range(6)

SAMPLE_DTYPE = np.dtype([("direction", "<f4", 3), ("radiance", "<f4", 4), ("pdf", "<f4"), ("status", "<u4"),
                         ("valid", "<u4")])


class EnvironmentMapDesc(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("reserved", C.c_uint32), ("texels", C.c_void_p), ("nanometers", C.c_float * 4),
                ("environment_to_world", C.c_float * 4)]


_DECLARED = False


def _lib():
    global _DECLARED
    lib = runtime.library()
    if not _DECLARED:
        vp, u64 = C.c_void_p, C.c_uint64
        lib.bf200_environment_map_create.argtypes = [vp, C.POINTER(EnvironmentMapDesc), C.POINTER(vp)]
        lib.bf200_environment_map_destroy.argtypes = [vp]
        lib.bf200_environment_map_sample.argtypes = [vp, vp, vp, vp, u64, vp]
        lib.bf200_environment_map_pdf.argtypes = [vp, vp, vp, vp, u64, vp, vp]
        lib.bf200_environment_map_le.argtypes = [vp, vp, vp, vp, u64, vp, vp]
        lib.bf200_environment_map_power.argtypes = [vp, vp, vp, vp, vp, vp]
        for name in ("create", "destroy", "sample", "pdf", "le", "power"):
            getattr(lib, "bf200_environment_map_" + name).restype = C.c_uint32
        _DECLARED = True
    return lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class EnvironmentMap:
    """texels: float32 [height, width, 4] (row 0 at local +Y, column 0 at the +X seam, longitude
    toward +Z); nanometers: the packet the map is bound to; quaternion: x, y, z, w."""

    def __init__(self, ctx, texels, nanometers, quaternion=(0.0, 0.0, 0.0, 1.0)):
        self.ctx = ctx
        self.texels = np.ascontiguousarray(texels, np.float32)
        height, width, lanes = self.texels.shape
        assert lanes == 4
        self.nanometers = np.ascontiguousarray(nanometers, np.float32).reshape(4)
        desc = EnvironmentMapDesc(C.sizeof(EnvironmentMapDesc), width, height, 0, _ptr(self.texels),
                                  (C.c_float * 4)(*self.nanometers), (C.c_float * 4)(*[float(q) for q in quaternion]))
        handle = C.c_void_p()
        ctx._check(_lib().bf200_environment_map_create(ctx.handle, C.byref(desc), C.byref(handle)),
                   "environment_map_create")
        self.handle = handle

    def sample(self, canonical):
        u = np.ascontiguousarray(canonical, np.float32).reshape(-1, 2)
        out = np.zeros(len(u), SAMPLE_DTYPE)
        self.ctx._check(_lib().bf200_environment_map_sample(self.ctx.handle, self.handle, _ptr(self.nanometers),
                                                            _ptr(u), len(u), _ptr(out)), "environment_map_sample")
        return out

    def pdf(self, directions):
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        pdf, status = np.zeros(len(d), np.float32), np.zeros(len(d), np.uint32)
        self.ctx._check(_lib().bf200_environment_map_pdf(self.ctx.handle, self.handle, _ptr(self.nanometers), _ptr(d),
                                                         len(d), _ptr(pdf), _ptr(status)), "environment_map_pdf")
        return pdf, status

    def le(self, directions):
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        radiance, status = np.zeros((len(d), 4), np.float32), np.zeros(len(d), np.uint32)
        self.ctx._check(_lib().bf200_environment_map_le(self.ctx.handle, self.handle, _ptr(self.nanometers), _ptr(d),
                                                        len(d), _ptr(radiance), _ptr(status)), "environment_map_le")
        return radiance, status

    def power(self, lo, hi):
        lo = np.ascontiguousarray(lo, np.float32).reshape(3)
        hi = np.ascontiguousarray(hi, np.float32).reshape(3)
        out = np.zeros(4, np.float32)
        self.ctx._check(_lib().bf200_environment_map_power(self.ctx.handle, self.handle, _ptr(self.nanometers),
                                                           _ptr(lo), _ptr(hi), _ptr(out)), "environment_map_power")
        return out

    def close(self):
        if self.handle:
            _lib().bf200_environment_map_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
