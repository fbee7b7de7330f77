"""ctypes driver for oracle/lib/librumi_oracle.so, the CPU restatement of the rendering
path (oracle/rumi_oracle.c).  Test infrastructure: the checker, never the product."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "lib", "librumi_oracle.so")
FP = C.POINTER(C.c_float)
_lib = None


def lib():
    global _lib
    if _lib is None:
        # (re)built when missing or older than oracle/rumi_oracle.c
        import importlib.util
        spec = importlib.util.spec_from_file_location("build_oracle", os.path.join(ROOT, "oracle", "build_oracle.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
        L = C.CDLL(LIB_PATH)
        L.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_trace.argtypes = [C.c_void_p, C.c_int64, FP, C.c_int, FP, C.POINTER(C.c_int32)]
        L.orc_render_pt.restype = C.c_longlong
        L.orc_render_pt.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, FP]
        L.orc_texture_pattern.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, FP, FP]
        L.orc_render_whitted.restype = C.c_longlong
        L.orc_render_whitted.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, FP]
        L.orc_material_sample.argtypes = [C.c_void_p, FP, FP, FP, FP]
        L.orc_material_fr.argtypes = [C.c_void_p, FP, FP, FP, C.c_int, C.c_float, C.c_float, C.c_float, FP, FP]
        L.orc_fresnel.restype = C.c_float
        L.orc_fresnel.argtypes = [FP, FP, C.c_float, C.c_float]
        L.orc_distance_sample.argtypes = [FP, FP, C.c_float, C.c_float, C.c_float, FP]
        L.orc_phase_sample.argtypes = [FP, C.c_float, C.c_float, C.c_float, FP]
        L.orc_material_sample_n.argtypes = [C.c_void_p, FP, FP, C.c_int64, FP, FP]
        L.orc_phase_sample_n.argtypes = [FP, C.c_float, C.c_int64, FP, FP]
        L.orc_distance_sample_n.argtypes = [FP, FP, C.c_float, C.c_int64, FP, FP]
        L.orc_hg_eval.restype = C.c_float
        L.orc_hg_eval.argtypes = [C.c_float, C.c_float]
        L.orc_camera_ray.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                     C.c_float, FP]
        L.orc_pixel_sample.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_uint64, FP]
        L.orc_perm.restype = C.c_int
        L.orc_perm.argtypes = [C.c_int, C.c_int, C.c_uint32]
        _lib = L
    return _lib


def f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


def P(a):
    return a.ctypes.data_as(FP) if a is not None else None


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return [o[i] for i in range(4)]


def material_struct(m):
    """orc_material (same layout as rumi_material) for a scene.Material."""
    import rumi_b200._capi as capi
    s = capi.rumi_material()
    s.type = m.type
    s.kd, s.ks, s.exponent = m.kd, m.ks, m.exponent
    s.rgb = capi.f3(*m.rgb)
    s.eta_in, s.eta_out = m.eta_in, m.eta_out
    s.rgb2 = capi.f3(*m.rgb2)
    s.density = m.density
    return s


class OracleScene:
    """A flattened scene description shared with the C-ABI layout."""

    def __init__(self, scene):
        from rumi_b200 import build_desc
        self.flat = scene.flatten()
        self.desc, self._keep = build_desc(self.flat)
        self.width, self.height = self.flat.image.width, self.flat.image.height

    def trace(self, rays8: np.ndarray, anyhit=False):
        r = f32(rays8).reshape(-1, 8)
        n = r.shape[0]
        t = np.zeros(n, np.float32)
        p = np.zeros(n, np.int32)
        lib().orc_trace(C.byref(self.desc), n, P(r), 1 if anyhit else 0, P(t), p.ctypes.data_as(C.POINTER(C.c_int32)))
        return t, p

    def render_pt(self, max_depth, spp, seed, row0=0, row1=None):
        film = np.zeros((self.height, self.width, 3), np.float32)
        nan = lib().orc_render_pt(C.byref(self.desc), max_depth, spp, seed, row0,
                                  self.height if row1 is None else row1, P(film))
        return film, int(nan)

    def texture_pattern(self, prim, pts):
        prim = np.ascontiguousarray(prim, np.int32)
        p = f32(np.asarray(pts).reshape(-1, 3))
        out = np.zeros_like(p)
        lib().orc_texture_pattern(C.byref(self.desc), p.shape[0], prim.ctypes.data, P(p), P(out))
        return out

    def render_whitted(self, max_depth, spp, seed, row0=0, row1=None):
        """RayTracer(scene, max_depth) frame: film (H, W, 3) B,G,R sums and NaN count."""
        film = np.zeros((self.height, self.width, 3), np.float32)
        nan = lib().orc_render_whitted(C.byref(self.desc), max_depth, spp, seed, row0,
                                       self.height if row1 is None else row1, P(film))
        return film, int(nan)

    def camera_ray(self, w, h, sx, sy, lu1=0.0, lu2=0.0):
        out = np.zeros(6, np.float32)
        lib().orc_camera_ray(C.byref(self.desc.camera), self.width, self.height, w, h, sx, sy, lu1, lu2, P(out))
        return out
