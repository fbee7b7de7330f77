"""ctypes declarations of include/rumi_b200.h and the loader of lib/librumi_b200.so.

The library is the only implementation: there is no CPU fallback, and loading fails
loudly when the CUDA build is missing."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RUMI_B200_LIB") or os.path.join(os.path.dirname(HERE), "lib", "librumi_b200.so")

f3 = C.c_float * 3
f16 = C.c_float * 16


class rumi_material(C.Structure):
    _fields_ = [("type", C.c_int32), ("kd", C.c_float), ("ks", C.c_float), ("exponent", C.c_float),
                ("rgb", f3), ("eta_in", C.c_float), ("eta_out", C.c_float), ("rgb2", f3), ("density", C.c_float)]


class rumi_light(C.Structure):
    _fields_ = [("type", C.c_int32), ("shape_type", C.c_int32), ("shape_index", C.c_int32),
                ("position", f3), ("direction", f3), ("cone_deg", C.c_float), ("intensity", f3)]


class rumi_volume(C.Structure):
    _fields_ = [("present", C.c_int32), ("pmin", f3), ("pmax", f3), ("sigma_s", f3), ("sigma_a", f3),
                ("g", C.c_float)]


class rumi_camera(C.Structure):
    _fields_ = [("position", f3), ("basis", f16), ("y_ratio", C.c_float), ("fov_deg", C.c_float),
                ("focal_distance", C.c_float), ("lens_radius", C.c_float)]


FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int32)


class rumi_texture(C.Structure):
    _fields_ = [("type", C.c_int32), ("repeat_u", C.c_float), ("repeat_v", C.c_float), ("color1", f3),
                ("color2", f3), ("gamma", C.c_float), ("img_width", C.c_int32), ("img_height", C.c_int32),
                ("bytes_per_pixel", C.c_int32), ("pixels", C.c_void_p)]


class rumi_scene_desc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32),
                ("n_triangles", C.c_int32), ("tri_vertices", FP), ("tri_normals", FP), ("tri_material", IP),
                ("tri_albedo", FP),
                ("n_rects", C.c_int32), ("rects", FP), ("rect_material", IP),
                ("n_spheres", C.c_int32), ("spheres", FP), ("sphere_material", IP),
                ("n_materials", C.c_int32), ("materials", C.POINTER(rumi_material)),
                ("n_lights", C.c_int32), ("lights", C.POINTER(rumi_light)),
                ("volume", rumi_volume), ("camera", rumi_camera),
                ("n_textures", C.c_int32), ("textures", C.POINTER(rumi_texture)), ("tri_texture", IP),
                ("rect_texture", IP), ("sphere_texture", IP), ("sphere_frame", FP)]


class rumi_render_params(C.Structure):
    _fields_ = [("integrator", C.c_int32), ("max_depth", C.c_int32), ("n_light", C.c_int32), ("n_eye", C.c_int32),
                ("spp", C.c_int32), ("seed", C.c_uint64), ("wave_paths", C.c_int32), ("flags", C.c_int32),
                ("stream", C.c_void_p), ("trace_mode", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("refill_min", C.c_int32), ("stack_depth", C.c_int32)]


class rumi_render_stats(C.Structure):
    _fields_ = [("paths", C.c_int64), ("nan_samples", C.c_int64), ("extend_launches", C.c_int64),
                ("extend_ms", C.c_double), ("shade_launches", C.c_int64), ("shade_ms", C.c_double),
                ("shadow_launches", C.c_int64), ("shadow_ms", C.c_double), ("total_ms", C.c_double),
                ("rays_extend", C.c_int64), ("rays_shadow", C.c_int64), ("extend_node_fetches", C.c_int64),
                ("extend_prim_tests", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class rumi_batch_params(C.Structure):
    _fields_ = [("max_depth", C.c_int32), ("spp", C.POINTER(C.c_int32)), ("seeds", C.POINTER(C.c_uint64)),
                ("wave_paths", C.c_int32), ("flags", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("stream", C.c_void_p)]


BATCH_GRAPH = 4


class rumi_bvh_info(C.Structure):
    _fields_ = [("large_levels", C.c_int32), ("small_tasks", C.c_int32), ("n_nodes", C.c_int32),
                ("build_ms", C.c_double)]


# every symbol include/rumi_b200.h and include/rumi_b200_test.h declare
EXPORTS = ["rumi_scene_create", "rumi_scene_destroy", "rumi_scene_bvh_info", "rumi_render", "rumi_render_noalloc",
           "rumi_trace_rays", "rumi_batch_create", "rumi_batch_destroy", "rumi_batch_film_floats",
           "rumi_render_batch", "rumi_forward", "rumi_backward", "rumi_scene_set_albedo", "rumi_scene_set_volume",
           "rumi_film_tonemap", "rumi_film_fireflies",
           "rumi_last_error_string", "rumi_version",
           "rumi_test_philox", "rumi_test_material_sample", "rumi_test_material_fr", "rumi_test_distance_sample",
           "rumi_test_phase_sample", "rumi_test_camera_rays", "rumi_test_pixel_samples",
           "rumi_test_read_bandwidth", "rumi_test_texture_pattern", "rumi_test_trace_scheme"]

_lib = None


def load(path: str = LIB_PATH):
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run `python rumi-renderer_b200/build.py`")
    L = C.CDLL(path)
    L.rumi_scene_create.restype = C.c_int
    L.rumi_scene_create.argtypes = [C.POINTER(rumi_scene_desc), C.POINTER(C.c_void_p)]
    L.rumi_scene_destroy.restype = C.c_int
    L.rumi_scene_destroy.argtypes = [C.c_void_p]
    L.rumi_scene_bvh_info.restype = C.c_int
    L.rumi_scene_bvh_info.argtypes = [C.c_void_p, C.POINTER(rumi_bvh_info)]
    L.rumi_render.restype = C.c_int
    L.rumi_render.argtypes = [C.c_void_p, C.POINTER(rumi_render_params), C.c_void_p, C.c_int32,
                              C.POINTER(rumi_render_stats)]
    L.rumi_render_noalloc.restype = C.c_int
    L.rumi_render_noalloc.argtypes = [C.c_void_p, C.POINTER(rumi_render_params), C.c_void_p,
                                      C.POINTER(rumi_render_stats)]
    L.rumi_trace_rays.restype = C.c_int
    L.rumi_trace_rays.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                  C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_void_p]
    L.rumi_batch_create.restype = C.c_int
    L.rumi_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]
    L.rumi_batch_destroy.restype = C.c_int
    L.rumi_batch_destroy.argtypes = [C.c_void_p]
    L.rumi_batch_film_floats.restype = C.c_int64
    L.rumi_batch_film_floats.argtypes = [C.c_void_p]
    L.rumi_render_batch.restype = C.c_int
    L.rumi_render_batch.argtypes = [C.c_void_p, C.POINTER(rumi_batch_params), C.c_void_p, C.c_int32,
                                    C.POINTER(rumi_render_stats)]
    L.rumi_forward.restype = C.c_int
    L.rumi_forward.argtypes = [C.c_void_p, C.POINTER(rumi_render_params), C.c_void_p, C.c_int32,
                               C.POINTER(rumi_render_stats)]
    L.rumi_backward.restype = C.c_int
    L.rumi_backward.argtypes = [C.c_void_p, C.POINTER(rumi_render_params), C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_int32, C.POINTER(rumi_render_stats)]
    L.rumi_scene_set_albedo.restype = C.c_int
    L.rumi_scene_set_albedo.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    L.rumi_scene_set_volume.restype = C.c_int
    L.rumi_scene_set_volume.argtypes = [C.c_void_p, C.POINTER(rumi_volume)]
    vp = C.c_void_p
    L.rumi_test_philox.argtypes = [C.c_int64, vp, vp, vp]
    L.rumi_test_material_sample.argtypes = [C.POINTER(rumi_material), C.c_int64, vp, vp, vp, vp]
    L.rumi_test_material_fr.argtypes = [C.POINTER(rumi_material), C.c_int64, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.rumi_test_distance_sample.argtypes = [vp, vp, C.c_int64, vp, vp, vp, vp]
    L.rumi_test_phase_sample.argtypes = [C.c_int64, vp, C.c_float, vp, vp]
    L.rumi_test_camera_rays.argtypes = [C.POINTER(rumi_camera), C.c_int32, C.c_int32, C.c_int64, vp, vp, vp, vp]
    L.rumi_test_pixel_samples.argtypes = [C.c_int64, vp, C.c_int32, vp, C.c_uint64, vp]
    L.rumi_film_tonemap.restype = C.c_int
    L.rumi_film_tonemap.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_int32, vp, C.c_int32, vp]
    L.rumi_film_fireflies.restype = C.c_int
    L.rumi_film_fireflies.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int32, vp]
    L.rumi_test_read_bandwidth.restype = C.c_int
    L.rumi_test_read_bandwidth.argtypes = [vp, C.c_int64, C.c_int32, vp, C.POINTER(C.c_double)]
    L.rumi_test_texture_pattern.argtypes = [vp, C.c_int64, vp, vp, vp]
    L.rumi_test_trace_scheme.argtypes = [vp, C.c_int64, vp, C.c_int32, C.c_int32, vp, vp]
    L.rumi_last_error_string.restype = C.c_char_p
    L.rumi_version.restype = C.c_char_p
    _lib = L
    return L


class RumiError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = load().rumi_last_error_string().decode(errors="replace")
        super().__init__(f"{where} failed with status {status}: {msg}")
        self.status = status


def check(status: int, where: str):
    if status != 0:
        raise RumiError(status, where)
