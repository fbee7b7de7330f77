"""ctypes driver for oracle/_ref/librumi_ref.so: the reference renderer's own classes,
compiled from its sources by oracle/build_ref.py.  Test infrastructure only -- used as
the parity checker and never as the thing measured."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "_ref", "librumi_ref.so")

_lib = None
fp = C.POINTER(C.c_float)
ip = C.POINTER(C.c_int)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `python oracle/build_ref.py`")
        L = C.CDLL(LIB_PATH)
        L.ref_scene_new.restype = C.c_void_p
        L.ref_scene_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float]
        L.ref_add_triangles.argtypes = [C.c_void_p, C.c_int, fp, fp, C.c_int, fp, C.c_int]
        L.ref_add_model.argtypes = [C.c_void_p, C.c_int, fp, fp, C.c_int, fp]
        L.ref_add_rect.argtypes = [C.c_void_p, fp, fp, fp, C.c_int, C.c_int, fp]
        L.ref_add_sphere.argtypes = [C.c_void_p, fp, C.c_float, C.c_int, C.c_int, fp]
        L.ref_add_area_light.argtypes = [C.c_void_p, C.c_int]
        L.ref_set_volume.argtypes = [C.c_void_p, fp, fp, fp, fp]
        L.ref_set_camera.argtypes = [C.c_void_p, fp, fp, C.c_float, C.c_float]
        L.ref_finalize.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_ulonglong]
        L.ref_render_rows.restype = C.c_longlong
        L.ref_render_rows.argtypes = [C.c_void_p, C.c_ulonglong, C.c_int, C.c_int, fp, fp]
        L.ref_sample_count.argtypes = [C.c_void_p]
        L.ref_trace.argtypes = [C.c_void_p, C.c_int, fp, C.c_int, fp, ip, fp]
        L.ref_scene_free.argtypes = [C.c_void_p]
        L.ref_seed.argtypes = [C.c_ulonglong]
        L.ref_inject.argtypes = [fp, C.c_int]
        L.ref_material_sample.argtypes = [C.c_int, fp, fp, fp, fp]
        L.ref_material_fr.argtypes = [C.c_int, fp, fp, fp, fp, C.c_int, C.c_float, C.c_float, C.c_float,
                                      fp, fp, fp]
        L.ref_material_pdfw.restype = C.c_float
        L.ref_material_pdfw.argtypes = [C.c_int, fp, fp, fp, fp, C.c_float]
        L.ref_fresnel.restype = C.c_float
        L.ref_fresnel.argtypes = [fp, fp, C.c_float, C.c_float]
        L.ref_isotropic_sample.argtypes = [fp, fp]
        L.ref_onb.argtypes = [fp, fp]
        L.ref_volume_distance_sampling.argtypes = [fp, fp, C.c_float, fp]
        L.ref_volume_segment.argtypes = [fp, fp, fp, fp, C.c_float, fp]
        L.ref_volume_shadow_tr.argtypes = [fp, fp, fp, fp, fp, fp, C.c_float, fp]
        L.ref_subsurface_distance_sampling.argtypes = [fp, C.c_float, fp]
        L.ref_camera_cast.argtypes = [fp, fp, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_float, C.c_float, fp]
        L.ref_camera_params.argtypes = [C.c_void_p, fp]
        L.ref_camera_cast_dof.argtypes = [fp, fp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int,
                                          C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint, fp]
        L.ref_set_camera_dof.argtypes = [C.c_void_p, C.c_float, C.c_float]
        L.ref_add_texture.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, fp, fp, C.c_char_p,
                                      C.c_float]
        L.ref_set_shape_transform.argtypes = [C.c_void_p, C.c_int, fp]
        L.ref_add_ibl_light.argtypes = [C.c_void_p, C.c_int]
        L.ref_texture_pattern.argtypes = [C.c_void_p, C.c_int, C.c_int, fp, fp]
        L.ref_load_hdr.argtypes = [C.c_char_p, C.c_int, fp, C.POINTER(C.c_int)]
        L.ref_load_bmp.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.POINTER(C.c_uint)]
        _lib = L
    return _lib


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def P(a):
    """float* into a contiguous float32 array (caller keeps the array alive)."""
    return a.ctypes.data_as(fp) if a is not None else None


def morton_order(tris: np.ndarray) -> np.ndarray:
    """Permutation putting triangles in Morton order of their centroids (10 bits/axis)."""
    c = tris.astype(np.float64).mean(1)
    lo, hi = c.min(0), c.max(0)
    q = ((c - lo) / np.maximum(hi - lo, 1e-12) * 1023).astype(np.uint64)

    def spread(x):
        x = (x | (x << np.uint64(16))) & np.uint64(0x030000FF)
        x = (x | (x << np.uint64(8))) & np.uint64(0x0300F00F)
        x = (x | (x << np.uint64(4))) & np.uint64(0x030C30C3)
        x = (x | (x << np.uint64(2))) & np.uint64(0x09249249)
        return x
    code = (spread(q[:, 0]) << np.uint64(2)) | (spread(q[:, 1]) << np.uint64(1)) | spread(q[:, 2])
    return np.argsort(code, kind="stable")


class RefScene:
    """A reference Scene built from a ``rumi_b200.scene.Scene``.

    Triangles of ``Model`` shapes with a per-triangle albedo become standalone Triangle
    shapes (each with its own Matte), since the reference's Model shares one material;
    other Models keep the reference's two-level Model BVH.

    presort_over: meshes with more triangles than this are handed to the reference in
    Morton order.  Only the input order changes -- the reference's object-median build
    produces the same partitions -- but its shell sort then runs on nearly sorted data
    (a 1,048,576-triangle build takes seconds instead of minutes).  ``id_map`` maps the
    reference's primitive numbering back to the canonical ids."""

    def __init__(self, scene, seed: int = 1, integrator=None, presort_over: int = 200000):
        from rumi_b200.scene import (Triangle, Model, Rect, Sphere, AreaLight, PathTracer,
                                     BidirectionalPathTracer, RayTracer, ImageBasedLight, MATTE)
        L = lib()
        self._keep = []
        img = scene.image
        self.width, self.height = img.width, img.height
        self.h = L.ref_scene_new(img.width, img.height, img.n_samples, img.gamma)
        # primitive ids follow the canonical order: triangles, rects, spheres.  The
        # harness numbers shapes in insertion order, so insert in that order.
        order = ([s for s in scene.objects if isinstance(s, (Triangle, Model))] +
                 [s for s in scene.objects if isinstance(s, Rect)] +
                 [s for s in scene.objects if isinstance(s, Sphere)])
        obj_index = {}
        id_map = []
        next_canon = 0
        for s in order:
            mp = f32(s.material.ref_params())
            self._keep.append(mp)
            if not isinstance(s, Model):
                id_map.append(np.array([next_canon]))
                next_canon += 1
            if isinstance(s, Triangle):
                v = f32(s.v.reshape(1, 9))
                n = f32(s.n.reshape(1, 9)) if s.n is not None else None
                self._keep += [v, n]
                obj_index[id(s)] = L.ref_add_triangles(self.h, 1, P(v), P(n), s.material.type, P(mp), 0)
            elif isinstance(s, Model):
                from rumi_b200.scene import _face_normal
                k = s.vertices.shape[0]
                perm = morton_order(s.vertices) if k > presort_over else np.arange(k)
                v = f32(s.vertices[perm].reshape(-1, 9))
                if s.normals is not None:
                    n = f32(s.normals[perm].reshape(-1, 9))
                else:
                    n = f32(np.repeat(_face_normal(s.vertices[perm])[:, None, :], 3, axis=1).reshape(-1, 9))
                self._keep += [v, n]
                id_map.append(next_canon + perm)
                next_canon += k
                if s.albedo is not None:
                    assert s.material.type == MATTE
                    per = np.tile(mp, (k, 1))
                    per[:, 3:6] = s.albedo[perm]
                    per = f32(per)
                    self._keep.append(per)
                    obj_index[id(s)] = L.ref_add_triangles(self.h, k, P(v), P(n), s.material.type, P(per),
                                                           per.shape[1])
                else:
                    obj_index[id(s)] = L.ref_add_model(self.h, k, P(v), P(n), s.material.type, P(mp))
            elif isinstance(s, Rect):
                a, b, c = f32(s.p), f32(s.l), f32(s.w)
                self._keep += [a, b, c]
                obj_index[id(s)] = L.ref_add_rect(self.h, P(a), P(b), P(c), s.n_samples, s.material.type, P(mp))
            elif isinstance(s, Sphere):
                c = f32(s.c)
                self._keep.append(c)
                obj_index[id(s)] = L.ref_add_sphere(self.h, P(c), s.r, s.n_samples, s.material.type, P(mp))
        self.id_map = np.concatenate(id_map).astype(np.int32) if id_map else np.zeros(0, np.int32)
        self.obj_index = obj_index
        self._tmpdir = None
        for s in scene.objects:
            if isinstance(s, Sphere):
                tr = f32(getattr(s, "transform", np.eye(4, dtype=np.float32).reshape(16)))
                self._keep.append(tr)
                L.ref_set_shape_transform(self.h, obj_index[id(s)], P(tr))
            t = getattr(s, "texture", None)
            if t is not None:
                self._add_texture(obj_index[id(s)], t)
        for light in scene.lights:
            if isinstance(light, ImageBasedLight):
                L.ref_add_ibl_light(self.h, obj_index[id(light.sphere)])
                continue
            if not isinstance(light, AreaLight):
                raise NotImplementedError("the reference has area and image-based lights only")
            L.ref_add_area_light(self.h, obj_index[id(light.shape)])
        if scene.volume is not None:
            v = scene.volume
            if v.g != 0.0:
                raise NotImplementedError("the reference's medium is isotropic (g = 0)")
            arrs = [f32(v.pmin), f32(v.pmax), f32(v.sigma_s), f32(v.sigma_a)]
            self._keep += arrs
            L.ref_set_volume(self.h, *[P(a) for a in arrs])
        cam = scene.camera
        pos, basis = f32(cam.position), f32(cam.basis)
        self._keep += [pos, basis]
        L.ref_set_camera(self.h, P(pos), P(basis), cam.y_ratio, cam.fov)
        if getattr(cam, "focal_distance", 0.0) > 0.0:
            L.ref_set_camera_dof(self.h, cam.focal_distance, cam.lens_radius)
        tr = integrator or scene.tracer
        if isinstance(tr, PathTracer):
            L.ref_finalize(self.h, 0, tr.max_depth, 0, seed)
        elif isinstance(tr, BidirectionalPathTracer):
            L.ref_finalize(self.h, 1, tr.nL, tr.nE, seed)
        elif isinstance(tr, RayTracer):
            L.ref_finalize(self.h, 2, tr.max_depth, 0, seed)
        else:
            L.ref_finalize(self.h, 0, 1, 0, seed)

    def _add_texture(self, obj, t):
        """Shape::AddingTexture through the harness; image textures without a file are
        written to a BMP first (the reference reads textures from files only)."""
        import tempfile
        from rumi_b200.scene import TEX_CHECKER, TEX_IMAGE
        from rumi_b200.film import save_bmp
        L = lib()
        if t.kind == TEX_CHECKER:
            c1, c2 = f32(t.c1), f32(t.c2)
            self._keep += [c1, c2]
            L.ref_add_texture(self.h, obj, 0, t.width, t.height, P(c1), P(c2), None, 1.0)
            return
        path = getattr(t, "path", None)
        if path is None:
            if t.kind != TEX_IMAGE:
                raise ValueError("an HDR texture for the reference needs its file (HDRTexture.from_hdr)")
            if self._tmpdir is None:
                self._tmpdir = tempfile.TemporaryDirectory()
            path = os.path.join(self._tmpdir.name, "tex%d.bmp" % obj)
            save_bmp(path, t.pixels)
        L.ref_add_texture(self.h, obj, 1 if t.kind == TEX_IMAGE else 2, 0.0, 0.0, None, None, path.encode(),
                          float(getattr(t, "gamma", 1.0)))

    def texture_pattern(self, shape, pts):
        """Texture::Pattern(shape, p) of the reference at points (n, 3) -> (n, 3) r, g, b."""
        p = f32(np.asarray(pts).reshape(-1, 3))
        out = np.zeros_like(p)
        lib().ref_texture_pattern(self.h, self.obj_index[id(shape)], p.shape[0], P(p), P(out))
        return out

    def render_rows(self, seed: int, row0: int, row1: int):
        """Film pixel sums (H, W, 3) in B,G,R order for rows [row0, row1), the light
        buffer, and the NaN sample count."""
        L = lib()
        film = np.zeros((self.height, self.width, 3), np.float32)
        light = np.zeros((self.height, self.width, 3), np.float32)
        nans = L.ref_render_rows(self.h, seed, row0, row1, P(film), P(light))
        return film, light, int(nans)

    def render(self, seed: int):
        film, light, nans = self.render_rows(seed, 0, self.height)
        return film + light, nans

    @property
    def spp(self) -> int:
        return lib().ref_sample_count(self.h)

    def trace(self, rays: np.ndarray, anyhit: bool = False, want_normals: bool = False):
        """rays (n, 7): o, d, tmax.  Returns t (0 = miss), id (-1 = miss; any-hit: 0/1) and
        optionally the shading normal."""
        L = lib()
        r = f32(rays).reshape(-1, 7)
        n = r.shape[0]
        t = np.zeros(n, np.float32)
        ids = np.zeros(n, np.int32)
        nn = np.zeros((n, 3), np.float32) if want_normals else None
        L.ref_trace(self.h, n, P(r), 1 if anyhit else 0, P(t), ids.ctypes.data_as(ip), P(nn))
        if not anyhit:
            ids = np.where(ids >= 0, self.id_map[np.maximum(ids, 0)], ids).astype(np.int32)
        return (t, ids, nn) if want_normals else (t, ids)

    def close(self):
        if self.h:
            lib().ref_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_obj(path: str, m16=None, cap: int = 1 << 20):
    """The reference's Model(path, transform): (vertices (F,3,3), normals (F,3,3))."""
    L = lib()
    L.ref_load_obj.restype = C.c_int
    L.ref_load_obj.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    v = np.zeros((cap, 9), np.float32)
    n = np.zeros((cap, 9), np.float32)
    m = None if m16 is None else f32(np.asarray(m16, np.float32).reshape(16))
    k = L.ref_load_obj(path.encode(), None if m is None else m.ctypes.data_as(C.c_void_p), cap,
                       v.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p))
    return v[:k].reshape(-1, 3, 3), n[:k].reshape(-1, 3, 3)


def inject(u: np.ndarray):
    """Make the reference's rand() return exactly the uniforms u (each m * 2^-24)."""
    u = f32(u)
    lib().ref_inject(P(u), u.shape[0])
    return u
