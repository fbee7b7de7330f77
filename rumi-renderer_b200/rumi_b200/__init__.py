"""B200 rendering path for Rumi-Renderer scenes.

``GpuScene(scene)`` uploads a ``scene.Scene`` (the reference-shaped scene API) through
``rumi_scene_create`` and renders it with ``rumi_render``; ``trace`` queries the BVH
like the reference's ``BVHAccel::Travel``.  Everything runs in lib/librumi_b200.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .scene import (Scene, FlatScene, PathTracer, BidirectionalPathTracer, RayTracer, PATH_TRACER, BDPT, RAY_TRACER,
                    LIGHT_AREA, LIGHT_SPOT, LIGHT_IBL, TEX_CHECKER, TEX_IMAGE)

__all__ = ["GpuScene", "render", "Scene"]


def _fp(a):
    return a.ctypes.data_as(_capi.FP) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(_capi.IP) if a is not None else None


def build_desc(fs: FlatScene):
    """rumi_scene_desc for a flattened scene; returns (desc, keep-alive list)."""
    keep = []

    def arr(a, dt):
        if a is None:
            return None
        b = np.ascontiguousarray(a, dtype=dt)
        keep.append(b)
        return b

    d = _capi.rumi_scene_desc()
    d.width, d.height = fs.image.width, fs.image.height
    tv = arr(fs.tri_vertices.reshape(-1, 9), np.float32)
    tn = arr(fs.tri_normals.reshape(-1, 9), np.float32)
    tm = arr(fs.tri_material, np.int32)
    ta = arr(fs.tri_albedo, np.float32)
    d.n_triangles = tv.shape[0]
    d.tri_vertices, d.tri_normals, d.tri_material, d.tri_albedo = _fp(tv), _fp(tn), _ip(tm), _fp(ta)
    r = arr(fs.rects, np.float32)
    rm = arr(fs.rect_material, np.int32)
    d.n_rects, d.rects, d.rect_material = r.shape[0], _fp(r), _ip(rm)
    s = arr(fs.spheres, np.float32)
    sm = arr(fs.sphere_material, np.int32)
    d.n_spheres, d.spheres, d.sphere_material = s.shape[0], _fp(s), _ip(sm)
    mats = (_capi.rumi_material * max(1, len(fs.materials)))()
    for i, m in enumerate(fs.materials):
        mats[i].type = m.type
        mats[i].kd, mats[i].ks, mats[i].exponent = m.kd, m.ks, m.exponent
        mats[i].rgb = _capi.f3(*m.rgb)
        mats[i].eta_in, mats[i].eta_out = m.eta_in, m.eta_out
        mats[i].rgb2 = _capi.f3(*m.rgb2)
        mats[i].density = m.density
    keep.append(mats)
    d.n_materials, d.materials = len(fs.materials), C.cast(mats, C.POINTER(_capi.rumi_material))
    lights = (_capi.rumi_light * max(1, len(fs.lights)))()
    for i, L in enumerate(fs.lights):
        lights[i].type = L["type"]
        if L["type"] in (LIGHT_AREA, LIGHT_IBL):
            lights[i].shape_type, lights[i].shape_index = L["shape_type"], L["shape_index"]
        else:
            lights[i].position = _capi.f3(*L["position"])
            lights[i].direction = _capi.f3(*L["direction"])
            lights[i].cone_deg = L["cone_deg"]
            lights[i].intensity = _capi.f3(*L["intensity"])
    keep.append(lights)
    d.n_lights, d.lights = len(fs.lights), C.cast(lights, C.POINTER(_capi.rumi_light))
    if fs.volume is not None:
        v = fs.volume
        d.volume.present = 1
        d.volume.pmin, d.volume.pmax = _capi.f3(*v.pmin), _capi.f3(*v.pmax)
        d.volume.sigma_s, d.volume.sigma_a = _capi.f3(*v.sigma_s), _capi.f3(*v.sigma_a)
        d.volume.g = v.g
    cam = fs.camera
    d.camera.position = _capi.f3(*cam.position)
    d.camera.basis = _capi.f16(*np.asarray(cam.basis, np.float32).reshape(16))
    d.camera.y_ratio = cam.y_ratio
    d.camera.fov_deg = cam.fov
    d.camera.focal_distance = float(getattr(cam, "focal_distance", 0.0))
    d.camera.lens_radius = float(getattr(cam, "lens_radius", 0.0))
    texs = getattr(fs, "textures", None) or []
    if texs:
        tarr = (_capi.rumi_texture * len(texs))()
        for i, t in enumerate(texs):
            tarr[i].type = t.kind
            if t.kind == TEX_CHECKER:
                tarr[i].repeat_u, tarr[i].repeat_v = t.width, t.height
                tarr[i].color1, tarr[i].color2 = _capi.f3(*t.c1), _capi.f3(*t.c2)
            elif t.kind == TEX_IMAGE:
                tarr[i].gamma = t.gamma
                tarr[i].img_height, tarr[i].img_width, tarr[i].bytes_per_pixel = t.pixels.shape
                tarr[i].pixels = t.pixels.ctypes.data
                keep.append(t.pixels)
            else:
                tarr[i].img_height, tarr[i].img_width = t.data.shape[:2]
                tarr[i].bytes_per_pixel = 12
                tarr[i].pixels = t.data.ctypes.data
                keep.append(t.data)
        keep.append(tarr)
        d.n_textures, d.textures = len(texs), C.cast(tarr, C.POINTER(_capi.rumi_texture))
        tt = arr(fs.tri_texture, np.int32)
        rt = arr(fs.rect_texture, np.int32)
        st_ = arr(fs.sphere_texture, np.int32)
        sf = arr(fs.sphere_frame, np.float32)
        d.tri_texture, d.rect_texture, d.sphere_texture, d.sphere_frame = _ip(tt), _ip(rt), _ip(st_), _fp(sf)
    return d, keep


class GpuScene:
    """A scene resident on the GPU (rumi_scene)."""

    def __init__(self, scene: Scene):
        self.lib = _capi.load()
        self.flat = scene.flatten() if isinstance(scene, Scene) else scene
        self.width, self.height = self.flat.image.width, self.flat.image.height
        desc, keep = build_desc(self.flat)
        h = C.c_void_p()
        _capi.check(self.lib.rumi_scene_create(C.byref(desc), C.byref(h)), "rumi_scene_create")
        self.h = h

    def bvh_info(self) -> dict:
        info = _capi.rumi_bvh_info()
        _capi.check(self.lib.rumi_scene_bvh_info(self.h, C.byref(info)), "rumi_scene_bvh_info")
        return {k: getattr(info, k) for k, _ in info._fields_}

    def render(self, spp: int = None, seed: int = 1, tracer=None, wave_paths: int = 0, timing: bool = False,
               film_device_ptr: int = None, stream: int = None, count_stats: bool = False, trace_mode: int = 0,
               blocks_per_sm: int = 0, refill_min: int = 0, tuning: dict = None, serial: bool = False):
        """Renders one frame.  Returns (film (H, W, 3) B,G,R sums, stats dict); with
        film_device_ptr the film stays on the device and the first value is None.
        serial=True (RUMI_FLAG_SERIAL) runs every launch in order on one stream, so that
        timing=True reports each kernel's time alone on the GPU; the film is the same."""
        tr = tracer or self.flat.tracer
        p = _capi.rumi_render_params()
        if isinstance(tr, BidirectionalPathTracer):
            p.integrator, p.n_light, p.n_eye = BDPT, tr.nL, tr.nE
            p.max_depth = tr.nL + tr.nE
        elif isinstance(tr, RayTracer):
            p.integrator, p.max_depth = RAY_TRACER, tr.max_depth
        else:
            p.integrator, p.max_depth = PATH_TRACER, tr.max_depth
        p.spp = int(spp if spp is not None else self.flat.image.n_samples)
        p.seed = int(seed)
        p.wave_paths = int(wave_paths)
        p.flags = (1 if timing else 0) | (2 if count_stats else 0) | (4 if serial else 0)
        p.stream = stream
        t = dict(tuning or {})
        p.trace_mode = int(t.get("trace_mode", trace_mode))
        p.blocks_per_sm = int(t.get("blocks_per_sm", blocks_per_sm))
        p.refill_min = int(t.get("refill_min", refill_min))
        p.stack_depth = int(t.get("stack_depth", 0))
        if "wave_paths" in t and not wave_paths:
            p.wave_paths = int(t["wave_paths"])
        st = _capi.rumi_render_stats()
        if film_device_ptr is not None:
            _capi.check(self.lib.rumi_render(self.h, C.byref(p), C.c_void_p(film_device_ptr), 1, C.byref(st)),
                        "rumi_render")
            return None, st.as_dict()
        film = np.zeros((self.height, self.width, 3), np.float32)
        _capi.check(self.lib.rumi_render(self.h, C.byref(p), film.ctypes.data_as(C.c_void_p), 0, C.byref(st)),
                    "rumi_render")
        return film, st.as_dict()

    def _pt_params(self, spp, seed, max_depth=None, wave_paths=0, timing=False, stream=None):
        p = _capi.rumi_render_params()
        p.integrator = PATH_TRACER
        p.max_depth = int(max_depth if max_depth is not None else self.flat.tracer.max_depth)
        p.spp = int(spp if spp is not None else self.flat.image.n_samples)
        p.seed = int(seed)
        p.wave_paths = int(wave_paths)
        p.flags = 1 if timing else 0
        p.stream = stream
        return p

    def forward(self, spp: int = None, seed: int = 1, max_depth: int = None, wave_paths: int = 0,
                film_device_ptr: int = None, stream: int = None, timing: bool = False, keep: bool = False):
        """rumi_forward: the path-traced film that backward() differentiates.  keep=True
        (RUMI_FLAG_KEEP_RADIANCE) keeps every path's radiance on the device (16 bytes per
        path) so that the next backward() with the same seed, spp and max_depth skips its
        first pass."""
        p = self._pt_params(spp, seed, max_depth, wave_paths, timing, stream)
        if keep:
            p.flags |= 8
        st = _capi.rumi_render_stats()
        if film_device_ptr is not None:
            _capi.check(self.lib.rumi_forward(self.h, C.byref(p), C.c_void_p(film_device_ptr), 1, C.byref(st)),
                        "rumi_forward")
            return None, st.as_dict()
        film = np.zeros((self.height, self.width, 3), np.float32)
        _capi.check(self.lib.rumi_forward(self.h, C.byref(p), film.ctypes.data_as(C.c_void_p), 0, C.byref(st)),
                    "rumi_forward")
        return film, st.as_dict()

    def backward(self, d_film, spp: int = None, seed: int = 1, max_depth: int = None, albedo: bool = True,
                 volume: bool = True, wave_paths: int = 0, timing: bool = False):
        """rumi_backward with host buffers: d_film (H, W, 3) in the film's B,G,R layout.
        Returns (grad_albedo (n_tris, 3) r,g,b or None, grad_volume (7,) or None, stats)."""
        p = self._pt_params(spp, seed, max_depth, wave_paths, timing)
        df = np.ascontiguousarray(d_film, np.float32)
        assert df.size == self.height * self.width * 3
        ga = np.zeros((self.flat.tri_vertices.shape[0], 3), np.float32) if albedo else None
        gv = np.zeros(7, np.float32) if volume else None
        st = _capi.rumi_render_stats()
        _capi.check(self.lib.rumi_backward(self.h, C.byref(p), df.ctypes.data_as(C.c_void_p),
                                           None if ga is None else ga.ctypes.data_as(C.c_void_p),
                                           None if gv is None else gv.ctypes.data_as(C.c_void_p), 0, C.byref(st)),
                    "rumi_backward")
        return ga, gv, st.as_dict()

    def backward_device(self, d_film_ptr: int, grad_albedo_ptr, grad_volume_ptr, spp: int = None, seed: int = 1,
                        max_depth: int = None, wave_paths: int = 0, stream: int = None, timing: bool = False):
        """rumi_backward with device buffers (pointers as ints; gradient pointers may be None)."""
        p = self._pt_params(spp, seed, max_depth, wave_paths, timing, stream)
        st = _capi.rumi_render_stats()
        _capi.check(self.lib.rumi_backward(self.h, C.byref(p), C.c_void_p(d_film_ptr),
                                           None if grad_albedo_ptr is None else C.c_void_p(grad_albedo_ptr),
                                           None if grad_volume_ptr is None else C.c_void_p(grad_volume_ptr), 1,
                                           C.byref(st)), "rumi_backward")
        return st.as_dict()

    def set_albedo(self, albedo=None, device_ptr: int = None):
        """Replaces the per-triangle albedo ((n_tris, 3) r,g,b host array, or a device pointer)."""
        if device_ptr is not None:
            _capi.check(self.lib.rumi_scene_set_albedo(self.h, C.c_void_p(device_ptr), 1), "rumi_scene_set_albedo")
            return
        a = np.ascontiguousarray(albedo, np.float32)
        assert a.size == self.flat.tri_vertices.shape[0] * 3
        _capi.check(self.lib.rumi_scene_set_albedo(self.h, a.ctypes.data_as(C.c_void_p), 0), "rumi_scene_set_albedo")

    def set_volume(self, sigma_s, sigma_a, g: float, pmin=None, pmax=None):
        """Replaces the medium's coefficients (and optionally its box)."""
        v = _capi.rumi_volume()
        cur = self.flat.volume
        v.present = 1
        v.pmin = _capi.f3(*(pmin if pmin is not None else cur.pmin))
        v.pmax = _capi.f3(*(pmax if pmax is not None else cur.pmax))
        v.sigma_s = _capi.f3(*[float(x) for x in sigma_s])
        v.sigma_a = _capi.f3(*[float(x) for x in sigma_a])
        v.g = float(g)
        _capi.check(self.lib.rumi_scene_set_volume(self.h, C.byref(v)), "rumi_scene_set_volume")

    def trace(self, rays: np.ndarray, anyhit: bool = False, in_object=None):
        """rays (n, 7) o, d, tmax (or (n, 8) in the C-ABI layout).  Returns (t, prim,
        node_visits, prim_tests)."""
        r = np.asarray(rays, np.float32)
        if r.shape[-1] == 7:
            r8 = np.zeros((r.shape[0], 8), np.float32)
            r8[:, 0:3] = r[:, 0:3]
            r8[:, 4:7] = r[:, 3:6]
            r8[:, 7] = r[:, 6]
            if in_object is not None:
                r8[:, 3] = np.asarray(in_object, np.float32)
            r = r8
        r = np.ascontiguousarray(r)
        n = r.shape[0]
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        nv, pt = C.c_int64(), C.c_int64()
        _capi.check(self.lib.rumi_trace_rays(self.h, n, r.ctypes.data_as(C.c_void_p), 1 if anyhit else 0,
                                             t.ctypes.data_as(C.c_void_p), prim.ctypes.data_as(C.c_void_p), 0,
                                             C.byref(nv), C.byref(pt), None), "rumi_trace_rays")
        return t, prim, nv.value, pt.value

    def trace_device(self, n: int, rays_ptr: int, t_ptr: int, prim_ptr: int, anyhit: bool = False, stream=None,
                     count: bool = True):
        """rumi_trace_rays on device buffers; count=False skips the node / primitive
        counters (the plain kernel).  Returns (node_visits, prim_tests) or (None, None)."""
        nv, pt = C.c_int64(), C.c_int64()
        _capi.check(self.lib.rumi_trace_rays(self.h, n, C.c_void_p(rays_ptr), 1 if anyhit else 0, C.c_void_p(t_ptr),
                                             C.c_void_p(prim_ptr), 1, C.byref(nv) if count else None,
                                             C.byref(pt) if count else None, stream), "rumi_trace_rays")
        return (nv.value, pt.value) if count else (None, None)

    def close(self):
        if getattr(self, "h", None):
            self.lib.rumi_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuBatch:
    """Many GpuScenes path traced as one frame from shared ray queues (rumi_batch).  The
    scenes must stay open while the batch lives."""

    def __init__(self, scenes):
        self.lib = _capi.load()
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(self.scenes))(*[g.h.value for g in self.scenes])
        h = C.c_void_p()
        _capi.check(self.lib.rumi_batch_create(arr, len(self.scenes), C.byref(h)), "rumi_batch_create")
        self.h = h
        self.sizes = [(g.height, g.width) for g in self.scenes]
        self.n_floats = int(self.lib.rumi_batch_film_floats(self.h))

    def render(self, spp, seeds, max_depth: int, graph: bool = False, timing: bool = False, wave_paths: int = 0,
               blocks_per_sm: int = 0, films_device_ptr: int = None, stream: int = None):
        """One frame of every scene.  Returns (list of (H, W, 3) films, stats dict); with
        films_device_ptr the concatenated films stay on the device and the list is None."""
        n = len(self.scenes)
        spp_a = (C.c_int32 * n)(*[int(x) for x in (spp if hasattr(spp, "__len__") else [spp] * n)])
        seed_a = (C.c_uint64 * n)(*[int(x) for x in (seeds if hasattr(seeds, "__len__") else [seeds] * n)])
        p = _capi.rumi_batch_params()
        p.max_depth = int(max_depth)
        p.spp = spp_a
        p.seeds = seed_a
        p.wave_paths = int(wave_paths)
        p.flags = (1 if timing else 0) | (_capi.BATCH_GRAPH if graph else 0)
        p.blocks_per_sm = int(blocks_per_sm)
        p.stream = stream
        st = _capi.rumi_render_stats()
        if films_device_ptr is not None:
            _capi.check(self.lib.rumi_render_batch(self.h, C.byref(p), C.c_void_p(films_device_ptr), 1, C.byref(st)),
                        "rumi_render_batch")
            return None, st.as_dict()
        flat = np.zeros(self.n_floats, np.float32)
        _capi.check(self.lib.rumi_render_batch(self.h, C.byref(p), flat.ctypes.data_as(C.c_void_p), 0, C.byref(st)),
                    "rumi_render_batch")
        films, o = [], 0
        for H, W in self.sizes:
            films.append(flat[o:o + H * W * 3].reshape(H, W, 3))
            o += H * W * 3
        return films, st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.rumi_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render(scene: Scene, seed: int = 1, **kw):
    """One-shot: upload, render, release."""
    g = GpuScene(scene)
    try:
        return g.render(seed=seed, **kw)
    finally:
        g.close()
