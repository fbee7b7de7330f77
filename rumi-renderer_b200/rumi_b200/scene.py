"""Scene description mirroring Rumi-Renderer's host-side classes.

A host program written against the reference builds a scene with ``Rect``, ``Sphere``,
``Triangle``/``Model`` shapes, ``AddingMaterial(Matte(...))``, ``AreaLight``,
``HomogeneousVolume``, ``Pinhole``, ``Film`` and an integrator
(``src/Scene/scene.cpp:135-204``).  The same names and argument meanings are kept here;
``Scene.flatten()`` turns the object graph into the plain arrays that the C-ABI
``rumi_scene_create`` copies to the GPU (``include/rumi_b200.h``).

Colours are given as (red, green, blue) like the reference's ``Color(r, g, b)``
constructor; film buffers come back in the reference's B,G,R storage order
(``src/Kernel/color.h:7-9``, ``src/Camera/film.cpp:83-97``).

Primitive ids (returned by ray queries) follow one canonical order: all triangles
(in insertion order, meshes expanded), then rects, then spheres.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

# material kinds (rumi_material.type)
MATTE, GLOSSY, SPECULAR, EMISSIVE, DIELECTRIC, SUBSURFACE = range(6)
# shape kinds (rumi_light.shape_type)
SHAPE_TRIANGLE, SHAPE_RECT, SHAPE_SPHERE = range(3)
# light kinds
LIGHT_AREA, LIGHT_SPOT = range(2)
# integrators
PATH_TRACER, BDPT, RAY_TRACER = range(3)
# light kinds (continued) and texture kinds
LIGHT_IBL = 2
TEX_CHECKER, TEX_IMAGE, TEX_HDR = range(3)


def _v3(x) -> np.ndarray:
    a = np.asarray(x, dtype=np.float32).reshape(3)
    return a


@dataclass
class Material:
    """Flat material record; see the subclasses for the reference constructors."""
    type: int
    kd: float = 0.0
    ks: float = 0.0
    exponent: float = 0.0
    rgb: Sequence[float] = (0.0, 0.0, 0.0)
    eta_in: float = 1.0
    eta_out: float = 1.0
    rgb2: Sequence[float] = (0.0, 0.0, 0.0)
    density: float = 1.0

    def ref_params(self) -> np.ndarray:
        """Parameter vector of oracle/ref_harness.cpp make_material (test side)."""
        p = np.zeros(10, np.float32)
        if self.type == MATTE or self.type == SPECULAR or self.type == EMISSIVE:
            p[0] = self.kd
        elif self.type == GLOSSY:
            p[0], p[1], p[2] = self.kd, self.ks, self.exponent
        else:  # DIELECTRIC, SUBSURFACE
            p[0], p[1] = self.eta_in, self.eta_out
        p[3:6] = self.rgb
        p[6:9] = self.rgb2
        p[9] = self.density
        return p


def Matte(kd: float, rgb) -> Material:
    """``Matte(kd, rgb)``: Lambertian, f = kd * rgb / pi (src/Material/matte.cpp:27-31)."""
    return Material(MATTE, kd=kd, rgb=tuple(rgb))


def Glossy(kd: float, ks: float, e: float, rgb) -> Material:
    """``Glossy(kd, ks, e, rgb)``: Lambertian + Phong lobe picked with kd/(kd+ks)
    (src/Material/glossy.cpp:19-25)."""
    return Material(GLOSSY, kd=kd, ks=ks, exponent=e, rgb=tuple(rgb))


def Specular(kr: float, rgb) -> Material:
    """``Specular(kr, rgb)``: perfect mirror (src/Material/specular.cpp:18-23)."""
    return Material(SPECULAR, kd=kr, rgb=tuple(rgb))


def Emissive(ls: float, rgb) -> Material:
    """``Emissive(ls, rgb)``: Le = ls * rgb, front side only (src/Material/emissive.cpp:17-48)."""
    return Material(EMISSIVE, kd=ls, rgb=tuple(rgb))


def Dielectric(eta_in: float, eta_out: float, absorption) -> Material:
    """``Dielectric(eta_in, eta_out, absorption)``: Fresnel-weighted reflect/refract with
    Beer-Lambert absorption inside (src/Material/dielectric.cpp:18-98)."""
    return Material(DIELECTRIC, eta_in=eta_in, eta_out=eta_out, rgb=tuple(absorption))


def Subsurface(eta_in: float, eta_out: float, sigma_s, sigma_a, density: float = 1.0) -> Material:
    """``Subsurface(eta_in, eta_out, sigma_s, sigma_a, density)``: dielectric boundary with a
    random walk inside (src/Material/subsurface.cpp:21-40)."""
    return Material(SUBSURFACE, eta_in=eta_in, eta_out=eta_out, rgb=tuple(sigma_s), rgb2=tuple(sigma_a),
                    density=density)


class Texture:
    """Base of the reference's textures (src/Texture/texture.h): Pattern(shape, p) =
    Pixel(shape.TextureMapping(p))."""
    kind: int


@dataclass
class Checker(Texture):
    """``Checker(width, height, c1, c2)``: c2 where floor(u*width) and floor(v*height) have
    the same parity, else c1 (src/Texture/checker.cpp:17-32)."""
    width: float
    height: float
    c1: Sequence[float]
    c2: Sequence[float]
    kind: int = TEX_CHECKER


class ImageTexture(Texture):
    """``ImageTexture(bmp_file, gamma)`` (src/Texture/imagetexture.cpp:18-61).  ``pixels``:
    uint8 (height, width, bytes_per_pixel) in the order LoadBmp returns them -- rows as
    stored in the file (bottom row first), B,G,R[,A]."""
    kind = TEX_IMAGE

    def __init__(self, pixels, gamma: float = 1.0):
        self.pixels = np.ascontiguousarray(pixels, dtype=np.uint8)
        if self.pixels.ndim != 3 or self.pixels.shape[2] not in (3, 4):
            raise ValueError("image texture pixels must be (height, width, 3 or 4) bytes")
        self.gamma = float(gamma)

    path: Optional[str] = None

    @classmethod
    def from_bmp(cls, path: str, gamma: float = 1.0) -> "ImageTexture":
        from .textures import load_bmp
        t = cls(load_bmp(path), gamma)
        t.path = path
        return t


class HDRTexture(Texture):
    """``HDRTexture(hdr_file)`` (src/Texture/hdrtexture.cpp:22-59).  ``data``: float32
    (height, width, 3) as LoadHDR returns it -- first scanline first, R,G,B."""
    kind = TEX_HDR

    def __init__(self, data):
        self.data = np.ascontiguousarray(data, dtype=np.float32)
        if self.data.ndim != 3 or self.data.shape[2] != 3:
            raise ValueError("HDR texture data must be (height, width, 3) floats")

    path: Optional[str] = None

    @classmethod
    def from_hdr(cls, path: str) -> "HDRTexture":
        from .textures import load_hdr
        t = cls(load_hdr(path))
        t.path = path
        return t


class Shape:
    material: Optional[Material] = None
    texture: Optional[Texture] = None

    def AddingMaterial(self, material: Material) -> bool:
        self.material = material
        return True

    def AddingTexture(self, texture: Texture) -> bool:
        """``Shape::AddingTexture`` (src/Shape/shape.cpp:71-84)."""
        self.texture = texture
        return True


class Triangle(Shape):
    """``Triangle(v0, v1, v2)`` + ``Normal(n0, n1, n2)`` (src/Shape/triangle.cpp:25-39)."""

    def __init__(self, v0, v1, v2):
        self.v = np.stack([_v3(v0), _v3(v1), _v3(v2)])
        self.n = None

    def Normal(self, n0, n1, n2):
        self.n = np.stack([_v3(n0), _v3(n1), _v3(n2)])


class Model(Shape):
    """A triangle mesh with one material (src/Shape/model.cpp:35-74).  ``vertices`` is
    (n, 3, 3) float32; ``normals`` (n, 3, 3) or None for face normals; ``albedo`` (n, 3)
    optionally overrides a Matte material's colour per triangle."""

    def __init__(self, vertices, normals=None, albedo=None):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3, 3)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3, 3)
        self.albedo = None if albedo is None else np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)

    @classmethod
    def from_obj(cls, path: str, transform=None, albedo=None) -> "Model":
        """``Model(file, transform)``: an OBJ file read by the reference's rules
        (rumi_b200.obj); transform is a row-major 4x4 (16 floats), None = identity."""
        from .obj import load_obj
        v, n = load_obj(path, transform)
        return cls(v, normals=n, albedo=albedo)


class Rect(Shape):
    """``Rect(p, l, w[, n_samples])``: parallelogram p + a*l + b*w, normal
    Normalize(Cross(l, w)) (src/Shape/rect.cpp:12-38)."""

    def __init__(self, p, l, w, n_samples: int = 0):
        self.p, self.l, self.w = _v3(p), _v3(l), _v3(w)
        self.n_samples = int(n_samples)


class Sphere(Shape):
    """``Sphere(c, r[, n_samples])`` (src/Shape/sphere.cpp:18-38).  ``transform``: the public
    ``Shape::_transform`` (row-major 4x4), whose upper 3x3 rows orient the sphere's texture."""

    def __init__(self, c, r: float, n_samples: int = 0, transform=None):
        self.c = _v3(c)
        self.r = float(r)
        self.n_samples = int(n_samples)
        self.transform = np.eye(4, dtype=np.float32).reshape(16) if transform is None else \
            np.asarray(transform, np.float32).reshape(16)


@dataclass
class AreaLight:
    """``AreaLight(shape, material)`` over an emissive Rect or Sphere (src/Light/arealight.cpp)."""
    shape: Shape


@dataclass
class ImageBasedLight:
    """``ImageBasedLight(sphere, material, texture)`` (src/Light/imagebasedlight.cpp): the
    emissive, textured sphere around the scene as a light, sampled by cosine-weighted
    directions about the shading normal; radiance = the sphere's texture where the
    direction leaves it."""
    sphere: Shape


@dataclass
class SpotLight:
    """Point emitter with a cone (not in the reference; the volumetric-caustic workload
    needs it): intensity I within ``cone_deg`` half-angle of ``direction``."""
    position: Sequence[float]
    direction: Sequence[float]
    cone_deg: float
    intensity: Sequence[float]


@dataclass
class HomogeneousVolume:
    """``HomogeneousVolume(BBox(pmin, pmax), sigma_s, sigma_a)`` (src/Volume/homogeneousvolume.cpp:24-44);
    ``g`` is the Henyey-Greenstein asymmetry (0 = the reference's isotropic phase)."""
    pmin: Sequence[float]
    pmax: Sequence[float]
    sigma_s: Sequence[float]
    sigma_a: Sequence[float]
    g: float = 0.0


def identity16() -> np.ndarray:
    return np.eye(4, dtype=np.float32).reshape(16)


def RotationX(rad: float) -> np.ndarray:
    c, s = math.cos(rad), math.sin(rad)
    return np.array([1, 0, 0, 0, 0, c, -s, 0, 0, s, c, 0, 0, 0, 0, 1], np.float32)


def RotationY(rad: float) -> np.ndarray:
    c, s = math.cos(rad), math.sin(rad)
    return np.array([c, 0, s, 0, 0, 1, 0, 0, -s, 0, c, 0, 0, 0, 0, 1], np.float32)


def RotationZ(rad: float) -> np.ndarray:
    c, s = math.cos(rad), math.sin(rad)
    return np.array([c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1], np.float32)


def matmul16(a, b) -> np.ndarray:
    return (np.asarray(a, np.float32).reshape(4, 4) @ np.asarray(b, np.float32).reshape(4, 4)).reshape(16)


@dataclass
class Pinhole:
    """``Pinhole(position, basis_transform, y_ratio)``; the reference fixes fov at 20
    degrees (src/Camera/pinhole.cpp:36) -- ``fov`` sets the same public member.
    ``focal_distance`` / ``lens_radius``: ``Pinhole::DepthOfField`` (thin lens when the
    focal distance is > 0)."""
    position: Sequence[float]
    basis: np.ndarray = field(default_factory=identity16)
    y_ratio: float = 1.0
    fov: float = 20.0
    focal_distance: float = 0.0
    lens_radius: float = 0.0


@dataclass
class Film:
    """``Film(width, height, bpp, n_samples, gamma)``: float sum-of-samples buffer
    (src/Camera/film.cpp:28-50).  The reference draws ``floor(sqrt(n))**2`` samples per
    pixel; ``samples_per_pixel`` reports that count."""
    width: int
    height: int
    n_samples: int
    gamma: float = 2.2

    @property
    def samples_per_pixel(self) -> int:
        d = int(math.isqrt(max(self.n_samples, 1)))
        return d * d


@dataclass
class PathTracer:
    """``PathTracer(scene, max_depth)`` (src/Integrator/pathtracer.cpp:27-44)."""
    max_depth: int


@dataclass
class BidirectionalPathTracer:
    """``BidirectionalPathTracer(scene, nL, nE)`` (src/Integrator/bidirectionalpathtracer.cpp:43-96)."""
    nL: int
    nE: int


@dataclass
class RayTracer:
    """``RayTracer(scene, max_depth)`` (src/Integrator/raytracer.cpp:30-86): the Whitted
    integrator -- mirror and glass chains up to trace depth ``max_depth``, direct lighting
    at the first other surface."""
    max_depth: int


class Scene:
    """Container with the reference's public members: objects, lights, volume, camera,
    image and tracer (src/Scene/scene.h:18-38)."""

    def __init__(self):
        self.objects: List[Shape] = []
        self.lights: list = []
        self.volume: Optional[HomogeneousVolume] = None
        self.camera: Optional[Pinhole] = None
        self.image: Optional[Film] = None
        self.tracer = None

    def add(self, shape: Shape, material: Optional[Material] = None) -> Shape:
        if material is not None:
            shape.AddingMaterial(material)
        if shape.material is None:
            raise ValueError("shape has no material")
        self.objects.append(shape)
        return shape

    # ------------------------------------------------------------------ flattening
    def flatten(self) -> "FlatScene":
        mats: List[Material] = []
        mat_index = {}

        def mid(m: Material) -> int:
            key = id(m)
            if key not in mat_index:
                mat_index[key] = len(mats)
                mats.append(m)
            return mat_index[key]

        texs: List[Texture] = []
        tex_index = {}

        def tid(t: Optional[Texture]) -> int:
            if t is None:
                return -1
            if id(t) not in tex_index:
                tex_index[id(t)] = len(texs)
                texs.append(t)
            return tex_index[id(t)]

        tri_t, rect_t, sphere_t, sphere_f = [], [], [], []
        tri_v, tri_n, tri_m, tri_alb = [], [], [], []
        has_alb = False
        rects, rect_m, spheres, sphere_m = [], [], [], []
        rect_samples, sphere_samples = [], []
        shape_loc = {}
        n_tri = 0
        for s in self.objects:
            if isinstance(s, Triangle):
                tri_v.append(s.v[None])
                n = s.n if s.n is not None else np.repeat(_face_normal(s.v[None]), 3, axis=0)[None]
                tri_n.append(np.asarray(n, np.float32).reshape(1, 3, 3))
                tri_m.append(np.full(1, mid(s.material), np.int32))
                tri_alb.append(np.asarray(s.material.rgb, np.float32).reshape(1, 3))
                tri_t.append(np.full(1, tid(s.texture), np.int32))
                shape_loc[id(s)] = (SHAPE_TRIANGLE, n_tri)
                n_tri += 1
            elif isinstance(s, Model):
                k = s.vertices.shape[0]
                tri_v.append(s.vertices)
                if s.normals is not None:
                    tri_n.append(s.normals)
                else:
                    tri_n.append(np.repeat(_face_normal(s.vertices)[:, None, :], 3, axis=1))
                tri_m.append(np.full(k, mid(s.material), np.int32))
                if s.albedo is not None:
                    has_alb = True
                    tri_alb.append(s.albedo)
                else:
                    tri_alb.append(np.tile(np.asarray(s.material.rgb, np.float32), (k, 1)))
                tri_t.append(np.full(k, tid(s.texture), np.int32))
                shape_loc[id(s)] = (SHAPE_TRIANGLE, n_tri)
                n_tri += k
            elif isinstance(s, Rect):
                shape_loc[id(s)] = (SHAPE_RECT, len(rects))
                rects.append(np.concatenate([s.p, s.l, s.w]))
                rect_m.append(mid(s.material))
                rect_samples.append(s.n_samples)
                rect_t.append(tid(s.texture))
            elif isinstance(s, Sphere):
                shape_loc[id(s)] = (SHAPE_SPHERE, len(spheres))
                spheres.append(np.array([*s.c, s.r], np.float32))
                sphere_m.append(mid(s.material))
                sphere_samples.append(s.n_samples)
                sphere_t.append(tid(s.texture))
                tr = np.asarray(getattr(s, "transform", np.eye(4, dtype=np.float32).reshape(16)), np.float32)
                sphere_f.append(tr.reshape(4, 4)[:3, :3].reshape(9))
            else:
                raise TypeError(type(s))
        lights = []
        for L in self.lights:
            if isinstance(L, AreaLight):
                st, si = shape_loc[id(L.shape)]
                lights.append(dict(type=LIGHT_AREA, shape_type=st, shape_index=si))
            elif isinstance(L, ImageBasedLight):
                st, si = shape_loc[id(L.sphere)]
                if st != SHAPE_SPHERE:
                    raise TypeError("an image-based light needs a Sphere")
                lights.append(dict(type=LIGHT_IBL, shape_type=st, shape_index=si))
            elif isinstance(L, SpotLight):
                lights.append(dict(type=LIGHT_SPOT, position=L.position, direction=L.direction,
                                   cone_deg=L.cone_deg, intensity=L.intensity))
            else:
                raise TypeError(type(L))
        fs = FlatScene()
        fs.tri_vertices = np.concatenate(tri_v).astype(np.float32) if tri_v else np.zeros((0, 3, 3), np.float32)
        fs.tri_normals = np.concatenate(tri_n).astype(np.float32) if tri_n else np.zeros((0, 3, 3), np.float32)
        fs.tri_material = np.concatenate(tri_m).astype(np.int32) if tri_m else np.zeros(0, np.int32)
        fs.tri_albedo = np.concatenate(tri_alb).astype(np.float32) if (tri_alb and has_alb) else None
        fs.rects = np.asarray(rects, np.float32).reshape(-1, 9)
        fs.rect_material = np.asarray(rect_m, np.int32)
        fs.rect_samples = np.asarray(rect_samples, np.int32)
        fs.spheres = np.asarray(spheres, np.float32).reshape(-1, 4)
        fs.sphere_material = np.asarray(sphere_m, np.int32)
        fs.sphere_samples = np.asarray(sphere_samples, np.int32)
        fs.materials = mats
        fs.lights = lights
        fs.textures = texs
        if texs:
            fs.tri_texture = np.concatenate(tri_t).astype(np.int32) if tri_t else np.zeros(0, np.int32)
            fs.rect_texture = np.asarray(rect_t, np.int32)
            fs.sphere_texture = np.asarray(sphere_t, np.int32)
            fs.sphere_frame = np.asarray(sphere_f, np.float32).reshape(-1, 9)
        else:
            fs.tri_texture = fs.rect_texture = fs.sphere_texture = fs.sphere_frame = None
        fs.volume = self.volume
        fs.camera = self.camera
        fs.image = self.image
        fs.tracer = self.tracer
        fs.source = self
        return fs


def _face_normal(v: np.ndarray) -> np.ndarray:
    """Normalize(Cross(v1 - v0, v2 - v0)) per triangle, in float32 like the reference."""
    v = np.asarray(v, np.float32)
    e1 = v[:, 1] - v[:, 0]
    e2 = v[:, 2] - v[:, 0]
    c = np.cross(e1, e2).astype(np.float32)
    inv = (np.float32(1.0) / np.sqrt((c * c).sum(axis=1, dtype=np.float32))).astype(np.float32)
    return (c * inv[:, None]).astype(np.float32)


class FlatScene:
    """Plain arrays handed to ``rumi_scene_create``."""
    tri_vertices: np.ndarray
    tri_normals: np.ndarray
    tri_material: np.ndarray
    tri_albedo: Optional[np.ndarray]
    rects: np.ndarray
    rect_material: np.ndarray
    rect_samples: np.ndarray
    spheres: np.ndarray
    sphere_material: np.ndarray
    sphere_samples: np.ndarray
    materials: List[Material]
    lights: list
    textures: list = []
    tri_texture: Optional[np.ndarray] = None
    rect_texture: Optional[np.ndarray] = None
    sphere_texture: Optional[np.ndarray] = None
    sphere_frame: Optional[np.ndarray] = None
    volume: Optional[HomogeneousVolume]
    camera: Optional[Pinhole]
    image: Optional[Film]

    @property
    def n_prims(self) -> int:
        return self.tri_vertices.shape[0] + self.rects.shape[0] + self.spheres.shape[0]
