"""Seeded synthetic workloads (the reference ships no benchmark scenes).

Every builder returns a ``scene.Scene`` assembled with the reference-shaped API, so the
same object graph drives the GPU path and the reference oracle.

Geometry generation uses float32 numpy arithmetic restricted to + - * / sqrt and integer
hashing, all correctly rounded in IEEE-754, so a mesh is bit-identical on every x86-64
host (no libm transcendental functions are involved).
"""
from __future__ import annotations

import math

import numpy as np

from .scene import (Scene, Rect, Sphere, Model, Matte, Specular, Emissive, Dielectric, Glossy, Subsurface, AreaLight,
                    SpotLight, HomogeneousVolume, Pinhole, Film, PathTracer, BidirectionalPathTracer,
                    RayTracer, identity16)

F32 = np.float32

# Cornell-box palette of the plain path-tracer workload.
RED = (0.63, 0.065, 0.05)
GREEN = (0.14, 0.45, 0.09)
WHITE = (0.73, 0.73, 0.73)
LIGHT_RADIANCE = (17.0, 12.0, 4.0)


def cornell_walls() -> list:
    """Five walls of [0,1]^3 (front z=0 open) as 10 triangles with face normals.
    Returns a list of (vertices (2,3,3), albedo)."""
    P = np.array
    quads = [
        (P([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]], F32), WHITE),  # floor y=0
        (P([[0, 1, 0], [0, 1, 1], [1, 1, 1], [1, 1, 0]], F32), WHITE),  # ceiling y=1
        (P([[0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], F32), WHITE),  # back z=1
        (P([[0, 0, 0], [0, 0, 1], [0, 1, 1], [0, 1, 0]], F32), RED),    # left x=0
        (P([[1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], F32), GREEN),  # right x=1
    ]
    out = []
    for q, alb in quads:
        tris = np.stack([np.stack([q[0], q[1], q[2]]), np.stack([q[0], q[2], q[3]])]).astype(F32)
        out.append((tris, alb))
    return out


def add_cornell_box(sc: Scene, light_samples: int = 256) -> Rect:
    for tris, alb in cornell_walls():
        sc.add(Model(tris), Matte(1.0, alb))
    light = Rect((0.375, 0.999, 0.375), (0.25, 0.0, 0.0), (0.0, 0.0, 0.25), light_samples)
    sc.add(light, Emissive(1.0, LIGHT_RADIANCE))
    sc.lights.append(AreaLight(light))
    return light


def cornell_camera() -> Pinhole:
    return Pinhole((0.5, 0.5, -1.4), identity16(), 1.0, fov=40.0)


def whitted(sc: Scene, max_depth: int = 10) -> Scene:
    """The scene rendered by ``RayTracer(scene, max_depth)`` (the reference's scene presets
    construct it with depth 10)."""
    sc.tracer = RayTracer(max_depth)
    return sc


def cornell_dof_pt(width: int = 256, height: int = 256, spp: int = 16, max_depth: int = 8,
                   focal_distance: float = 2.0, lens_radius: float = 0.08) -> Scene:
    """``cornell_pt`` seen through a thin lens (``Pinhole::DepthOfField``): in focus at the
    white sphere's depth (z = 0.6), the back wall and the mirror sphere blurred."""
    sc = cornell_pt(width, height, spp, max_depth)
    sc.camera.focal_distance = focal_distance
    sc.camera.lens_radius = lens_radius
    return sc


def cornell_pt(width: int = 256, height: int = 256, spp: int = 16, max_depth: int = 8) -> Scene:
    """Plain path tracer, Cornell box: 10 wall triangles, 0.25 x 0.25 quad light at y=0.999
    with radiance (17,12,4), a white Lambertian sphere r=0.15 at (0.3,0.15,0.6), a mirror
    sphere r=0.1 at (0.7,0.1,0.4), pinhole at (0.5,0.5,-1.4) with 40 degree fov."""
    sc = Scene()
    add_cornell_box(sc)
    sc.add(Sphere((0.3, 0.15, 0.6), 0.15), Matte(1.0, WHITE))
    sc.add(Sphere((0.7, 0.1, 0.4), 0.1), Specular(1.0, (0.9, 0.9, 0.9)))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def absorbing_glass_cornell(width: int = 32, height: int = 32, spp: int = 16, max_depth: int = 10) -> Scene:
    """The Cornell box holding a coloured glass sphere (Dielectric(1.5, 1.0, rgb): Beer-Lambert
    absorption exp(-rgb * length) on every segment travelled inside it,
    src/Material/material.cpp:18-26) and the mirror sphere, path traced."""
    sc = Scene()
    add_cornell_box(sc)
    sc.add(Sphere((0.35, 0.2, 0.55), 0.2), Dielectric(1.5, 1.0, (0.5, 1.5, 4.0)))
    sc.add(Sphere((0.72, 0.12, 0.35), 0.12), Specular(1.0, (0.9, 0.9, 0.9)))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def with_medium(sc: Scene, sigma_s=(0.3, 0.3, 0.3), sigma_a=(0.05, 0.05, 0.05), g: float = 0.0) -> Scene:
    """The scene with a homogeneous medium filling the unit box (the Cornell interior)."""
    sc.volume = HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), tuple(sigma_s), tuple(sigma_a), float(g))
    return sc


def with_bdpt(sc: Scene, nL: int = 4, nE: int = 5) -> Scene:
    """The scene rendered by ``BidirectionalPathTracer(scene, nL, nE)``."""
    sc.tracer = BidirectionalPathTracer(nL, nE)
    return sc


def cornell_sphere_light_pt(width: int = 32, height: int = 32, spp: int = 16, max_depth: int = 8) -> Scene:
    """The Cornell walls lit by a spherical emitter instead of the quad: an Emissive sphere
    of radius 0.06 under the ceiling with a 4096-point sample set and an AreaLight over it
    (the arrangement the reference's "RGB Sphere" preset keeps as its alternative light,
    Sphere(c, r, 4096) + Emissive; its points come from Sphere::ShapeSampling,
    src/Shape/sphere.cpp:152-170), a white Lambertian sphere and a glossy sphere."""
    sc = Scene()
    for tris, alb in cornell_walls():
        sc.add(Model(tris), Matte(1.0, alb))
    light = Sphere((0.5, 0.86, 0.5), 0.06, 4096)
    sc.add(light, Emissive(1.0, (60.0, 48.0, 30.0)))
    sc.lights.append(AreaLight(light))
    sc.add(Sphere((0.3, 0.15, 0.6), 0.15), Matte(1.0, WHITE))
    sc.add(Sphere((0.72, 0.12, 0.38), 0.12), Glossy(0.6, 0.4, 25.0, (0.8, 0.75, 0.7)))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def cornell_two_lights_pt(width: int = 32, height: int = 32, spp: int = 16, max_depth: int = 8) -> Scene:
    """The Cornell box with two area lights of different size and colour under the ceiling:
    next-event estimation picks one of them uniformly per sample (Scene::
    LightsUniformSampling, src/Scene/scene.cpp:91-97, pdf = (1/n) / area)."""
    sc = Scene()
    for tris, alb in cornell_walls():
        sc.add(Model(tris), Matte(1.0, alb))
    a = Rect((0.15, 0.999, 0.55), (0.2, 0.0, 0.0), (0.0, 0.0, 0.3), 256)
    b = Rect((0.7, 0.999, 0.2), (0.12, 0.0, 0.0), (0.0, 0.0, 0.12), 64)
    sc.add(a, Emissive(1.0, (14.0, 10.0, 6.0)))
    sc.add(b, Emissive(1.0, (6.0, 12.0, 24.0)))
    sc.lights += [AreaLight(a), AreaLight(b)]
    sc.add(Sphere((0.3, 0.15, 0.6), 0.15), Matte(1.0, WHITE))
    sc.add(Sphere((0.7, 0.1, 0.4), 0.1), Specular(1.0, (0.9, 0.9, 0.9)))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


# ----------------------------------------------------------------------------- meshes
def _hash3(ix, iy, iz, seed):
    """32-bit integer hash of lattice coordinates -> float32 in [-1, 1)."""
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343)) ^ (iy.astype(np.uint32) * np.uint32(0xD8163841)) \
        ^ (iz.astype(np.uint32) * np.uint32(0xCB1AB31F)) ^ np.uint32(seed * 0x9E3779B9 & 0xFFFFFFFF)
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x7FEB352D)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x846CA68B)
    h ^= h >> np.uint32(16)
    return (h >> np.uint32(8)).astype(F32) * F32(2.0 / 16777216.0) - F32(1.0)


def _value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise with smoothstep weights; p (n,3) float32."""
    fl = np.floor(p).astype(F32)
    f = (p - fl).astype(F32)
    w = (f * f * (F32(3.0) - F32(2.0) * f)).astype(F32)
    i = fl.astype(np.int64) + 4096  # keep lattice coordinates positive before hashing
    acc = np.zeros(p.shape[0], F32)
    for dz in (0, 1):
        wz = w[:, 2] if dz else (F32(1.0) - w[:, 2])
        for dy in (0, 1):
            wy = w[:, 1] if dy else (F32(1.0) - w[:, 1])
            for dx in (0, 1):
                wx = w[:, 0] if dx else (F32(1.0) - w[:, 0])
                v = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                acc = (acc + ((wx * wy).astype(F32) * wz).astype(F32) * v).astype(F32)
    return acc


def fbm(p: np.ndarray, seed: int, octaves: int = 6) -> np.ndarray:
    """Fractal sum of value noise, lacunarity 2, gain 0.5, normalised to about [-1, 1]."""
    total = np.zeros(p.shape[0], F32)
    amp = F32(0.5)
    norm = F32(0.0)
    q = p.astype(F32)
    for o in range(octaves):
        total = (total + amp * _value_noise(q, seed + 101 * o)).astype(F32)
        norm = F32(norm + amp)
        amp = F32(amp * F32(0.5))
        q = (q * F32(2.0)).astype(F32)
    return (total / norm).astype(F32)


def subdivided_tetrahedron(levels: int):
    """Regular tetrahedron subdivided ``levels`` times (4 * 4**levels faces), vertices
    projected to the unit sphere.  Returns (vertices (V,3) float32, faces (F,3) int64)."""
    s = F32(1.0) / np.sqrt(F32(3.0))
    verts = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], F32) * s
    faces = np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]], np.int64)
    for _ in range(levels):
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = (verts[uniq[:, 0]] + verts[uniq[:, 1]]).astype(F32)
        nrm = np.sqrt((mid * mid).sum(axis=1, dtype=F32)).astype(F32)
        mid = (mid / nrm[:, None]).astype(F32)
        base = verts.shape[0]
        verts = np.concatenate([verts, mid]).astype(F32)
        nf = faces.shape[0]
        m01 = base + inv[0:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:3 * nf]
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.concatenate([
            np.stack([a, m01, m20], 1), np.stack([m01, b, m12], 1),
            np.stack([m20, m12, c], 1), np.stack([m01, m12, m20], 1)])
    return verts, faces


def displaced_sphere(levels: int, center, radius: float, amplitude: float, seed: int, freq: float = 4.0):
    """Seeded displaced sphere: subdivided tetrahedron, each vertex moved along its
    direction by ``amplitude * fbm(freq * dir)`` (6 octaves).  Returns (F,3,3) float32."""
    verts, faces = subdivided_tetrahedron(levels)
    disp = fbm((verts * F32(freq)).astype(F32), seed)
    r = (F32(radius) + F32(amplitude) * disp).astype(F32)
    pos = (verts * r[:, None] + np.asarray(center, F32)[None, :]).astype(F32)
    return np.ascontiguousarray(pos[faces], dtype=F32)


def random_albedo(n: int, seed: int, lo: float = 0.2, hi: float = 0.8) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return (F32(lo) + rng.random((n, 3), dtype=F32) * F32(hi - lo)).astype(F32)


def mesh_checksum(tris: np.ndarray) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(tris, np.float32).tobytes()).hexdigest()[:16]


def bvh_bound_pt(width: int = 1024, height: int = 1024, spp: int = 64, max_depth: int = 10,
                 levels: int = 9, seed: int = 7) -> Scene:
    """BVH-bound path tracing: the Cornell box (walls + light) holding a displaced sphere of
    4 * 4**levels triangles (levels=9: 1,048,576) centred at (0.5,0.35,0.5), radius 0.25,
    displaced by 0.05 * fBm, with uniform random per-triangle albedo in [0.2,0.8]^3."""
    sc = Scene()
    add_cornell_box(sc)
    tris = displaced_sphere(levels, (0.5, 0.35, 0.5), 0.25, 0.05, seed)
    alb = random_albedo(tris.shape[0], seed + 1)
    sc.add(Model(tris, albedo=alb), Matte(1.0, WHITE))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def volumetric_caustic(width: int = 512, height: int = 512, spp: int = 32, nL: int = 6, nE: int = 7,
                       parity: bool = False) -> Scene:
    """BDPT with MIS, volumetric caustic: a glass sphere (IOR 1.5, r=0.3) at (0.5, 0.35, 0.5)
    inside the Cornell box filled with a homogeneous medium (sigma_a=0.05, sigma_s=0.4,
    RGB-uniform).  Workload: Henyey-Greenstein g=0.7, 30 degree spot light of intensity 50
    at (0.5, 0.98, 0.5) pointing down.  ``parity``: the reference-expressible variant -- the
    reference's isotropic phase (g=0) and a small area light under the ceiling in place of
    the spot (the reference's "Volumetric Caustics" preset uses the same arrangement).
    Max path length nL + nE - 1."""
    sc = Scene()
    for tris, alb in cornell_walls():
        sc.add(Model(tris), Matte(1.0, alb))
    sc.add(Sphere((0.5, 0.35, 0.5), 0.3), Dielectric(1.5, 1.0, (0.0, 0.0, 0.0)))
    if parity:
        light = Rect((0.45, 0.98, 0.45), (0.1, 0.0, 0.0), (0.0, 0.0, 0.1), 64)
        sc.add(light, Emissive(1.0, (120.0, 120.0, 120.0)))
        sc.lights.append(AreaLight(light))
        g = 0.0
    else:
        sc.lights.append(SpotLight((0.5, 0.98, 0.5), (0.0, -1.0, 0.0), 30.0, (50.0, 50.0, 50.0)))
        g = 0.7
    sc.volume = HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.4, 0.4, 0.4), (0.05, 0.05, 0.05), g)
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = BidirectionalPathTracer(nL, nE)
    return sc


def cornell_bdpt(width: int = 32, height: int = 32, spp: int = 16, nL: int = 4, nE: int = 5) -> Scene:
    """The plain path-tracer Cornell scene rendered by BDPT (parity scene without a medium)."""
    sc = cornell_pt(width, height, spp, 8)
    sc.tracer = BidirectionalPathTracer(nL, nE)
    return sc


def subsurface_cornell(width: int = 32, height: int = 32, spp: int = 16, max_depth: int = 12) -> Scene:
    """The Cornell box with a subsurface-scattering sphere (Subsurface(1.3, 1.0, sigma_s,
    sigma_a)) and a glossy sphere, path traced (reference semantics of
    src/Material/subsurface.cpp and src/Material/glossy.cpp)."""
    sc = Scene()
    add_cornell_box(sc)
    sc.add(Sphere((0.35, 0.2, 0.55), 0.2), Subsurface(1.3, 1.0, (6.0, 4.0, 2.0), (0.3, 0.6, 1.2), 1.0))
    sc.add(Sphere((0.72, 0.15, 0.35), 0.15), Glossy(0.5, 0.5, 30.0, (0.8, 0.7, 0.6)))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def heightfield(n_target: int, seed: int, lo=(0.1, 0.1), hi=(0.9, 0.9), base: float = 0.12, amp: float = 0.12):
    """Seeded fBm terrain over [lo, hi] in x/z: an nx-by-nx grid split into 2 nx^2
    triangles, nx = max(2, round(sqrt(n_target / 2))).  Returns (F,3,3) float32."""
    nx = max(2, int(round(math.sqrt(n_target / 2.0))))
    g = np.arange(nx + 1, dtype=F32) / F32(nx)
    x = (F32(lo[0]) + g * F32(hi[0] - lo[0])).astype(F32)
    z = (F32(lo[1]) + g * F32(hi[1] - lo[1])).astype(F32)
    X, Z = np.meshgrid(x, z, indexing="ij")
    p = np.stack([X, np.zeros_like(X), Z], -1).reshape(-1, 3).astype(F32)
    y = (F32(base) + F32(amp) * fbm((p * F32(4.0)).astype(F32), seed)).astype(F32)
    p[:, 1] = y
    P = p.reshape(nx + 1, nx + 1, 3)
    a, b, c, d = P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]
    t0 = np.stack([a, c, b], -2).reshape(-1, 3, 3)
    t1 = np.stack([a, d, c], -2).reshape(-1, 3, 3)
    return np.ascontiguousarray(np.concatenate([t0, t1]), dtype=F32)


BATCH_RESOLUTIONS = (64, 128, 256, 512)
BATCH_SPP = (4, 16, 64)


def batch_scene(i: int, max_depth: int = 8, res: int = None, spp: int = None, n_tris: int = None) -> Scene:
    """Scene i of the batched workload: the Cornell box holding a seeded fBm terrain whose
    triangle count is drawn log-uniform in [1k, 200k] (rounded to the terrain grid), with
    per-triangle albedo, and a sphere; the terrain is Lambertian and the sphere glass, or
    the other way round, by the seed.  Resolution from {64,128,256,512}^2, spp from
    {4,16,64}, path depth 8.  res / spp / n_tris override the draws."""
    rng = np.random.Generator(np.random.PCG64(1000 + i))
    u_tris, u_res, u_spp, u_mat, u_pos = rng.random(5)
    if n_tris is None:
        n_tris = int(round(math.exp(math.log(1000.0) + u_tris * (math.log(200000.0) - math.log(1000.0)))))
    if res is None:
        res = BATCH_RESOLUTIONS[min(3, int(u_res * 4))]
    if spp is None:
        spp = BATCH_SPP[min(2, int(u_spp * 3))]
    sc = Scene()
    add_cornell_box(sc)
    tris = heightfield(n_tris, 50 + i)
    glass_terrain = u_mat < 0.5
    if glass_terrain:
        sc.add(Model(tris), Dielectric(1.5, 1.00029, (0.0, 0.0, 0.0)))
        sc.add(Sphere((0.3 + 0.4 * float(u_pos), 0.55, 0.5), 0.12), Matte(1.0, WHITE))
    else:
        sc.add(Model(tris, albedo=random_albedo(tris.shape[0], 70 + i)), Matte(1.0, WHITE))
        sc.add(Sphere((0.3 + 0.4 * float(u_pos), 0.55, 0.5), 0.12), Dielectric(1.5, 1.00029, (0.0, 0.0, 0.0)))
    sc.camera = cornell_camera()
    sc.image = Film(res, res, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


# Inverse-rendering workload: hidden parameters of the target image.
INVERSE_TARGET_MEDIUM = dict(sigma_s=(0.45, 0.35, 0.25), sigma_a=(0.04, 0.06, 0.09), g=0.35)
INVERSE_START_MEDIUM = dict(sigma_s=(0.3, 0.3, 0.3), sigma_a=(0.05, 0.05, 0.05), g=0.1)


def inverse_rendering(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8, levels: int = 7,
                      albedo=None, medium: dict = None, albedo_seed: int = 23) -> Scene:
    """Differentiable inverse rendering: the Cornell box holding a seeded displaced sphere of
    4 * 4**levels triangles (levels=7: 65,536) with per-triangle RGB albedo, the whole box
    filled with a homogeneous medium (sigma_s, sigma_a RGB, Henyey-Greenstein g).
    albedo: (n_mesh, 3) or None for the hidden target albedo (uniform in [0.2, 0.8]^3,
    seeded by albedo_seed); medium: dict(sigma_s, sigma_a, g), default the hidden target."""
    sc = Scene()
    add_cornell_box(sc)
    tris = displaced_sphere(levels, (0.5, 0.35, 0.5), 0.25, 0.05, 11)
    if albedo is None:
        albedo = random_albedo(tris.shape[0], albedo_seed)
    sc.add(Model(tris, albedo=np.asarray(albedo, np.float32)), Matte(1.0, WHITE))
    m = medium or INVERSE_TARGET_MEDIUM
    sc.volume = HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), tuple(m["sigma_s"]), tuple(m["sigma_a"]),
                                  float(m["g"]))
    sc.camera = cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc
