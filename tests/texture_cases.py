"""Seeded texture images and textured scenes shared by the texture tests and the fixture
generator (tests/golden/make_golden.py): the same files come out on every machine, so the
reference's frames in tests/golden/ match the scenes the tests rebuild."""
from __future__ import annotations

import os

import numpy as np

from rumi_b200 import scenes
from rumi_b200.scene import (Scene, Rect, Sphere, Matte, Specular, Emissive, Checker, ImageTexture, HDRTexture,
                             ImageBasedLight, Film, PathTracer, Pinhole, RotationY, RotationX, matmul16, identity16)
from rumi_b200.textures import rgbe_from_float, save_hdr
from rumi_b200.film import save_bmp


def image_pixels(width: int = 20, height: int = 12, bpp: int = 3, seed: int = 5) -> np.ndarray:
    """Blocky seeded colours, (height, width, bpp) uint8 in LoadBmp order."""
    rng = np.random.default_rng(seed)
    blocks = rng.integers(0, 256, size=(height // 2 + 1, width // 4 + 1, bpp), dtype=np.uint8)
    img = np.repeat(np.repeat(blocks, 2, axis=0), 4, axis=1)[:height, :width]
    return np.ascontiguousarray(img)


def write_image(path: str, **kw) -> str:
    save_bmp(path, image_pixels(**kw))
    return path


def sky_rgbe(width: int = 64, height: int = 32, seed: int = 9) -> np.ndarray:
    """A latitude-longitude sky: blue-to-white gradient, a warm horizon band and a small
    bright sun, with seeded noise; (height, width, 4) RGBE bytes."""
    rng = np.random.default_rng(seed)
    y = (np.arange(height) + 0.5)[:, None] / height
    x = (np.arange(width) + 0.5)[None, :] / width
    rgb = np.zeros((height, width, 3))
    rgb[..., 0] = 0.3 + 0.7 * y
    rgb[..., 1] = 0.45 + 0.5 * y
    rgb[..., 2] = 0.9 + 0.1 * y
    band = np.exp(-((y - 0.55) / 0.06) ** 2)
    rgb += band[..., None] * np.array([0.8, 0.5, 0.2])
    sun = np.exp(-(((x - 0.3) / 0.03) ** 2 + ((y - 0.25) / 0.05) ** 2))
    rgb += sun[..., None] * np.array([40.0, 36.0, 30.0])
    rgb *= 1.0 + 0.05 * rng.standard_normal((height, width, 1))
    return rgbe_from_float(np.maximum(rgb, 0.0))


def write_sky(path: str, **kw) -> str:
    save_hdr(path, sky_rgbe(**kw))
    return path


def textured_cornell(width: int, height: int, spp: int, max_depth: int, image_path: str) -> Scene:
    """Cornell box with a checker-textured floor rect (Checker(8, 8)), a white Matte sphere
    with an image texture (rotated by its transform) and the mirror sphere."""
    sc = Scene()
    scenes.add_cornell_box(sc)
    floor = Rect((0.05, 0.002, 0.05), (0.0, 0.0, 0.9), (0.9, 0.0, 0.0))
    sc.add(floor, Matte(1.0, (1.0, 1.0, 1.0)))
    floor.AddingTexture(Checker(8.0, 8.0, (0.9, 0.85, 0.8), (0.15, 0.2, 0.55)))
    ball = Sphere((0.3, 0.17, 0.6), 0.15, transform=matmul16(RotationY(0.7), RotationX(-0.4)))
    sc.add(ball, Matte(1.0, (1.0, 1.0, 1.0)))
    ball.AddingTexture(ImageTexture.from_bmp(image_path, 1.0))
    sc.add(Sphere((0.7, 0.1, 0.4), 0.1), Specular(1.0, (0.9, 0.9, 0.9)))
    sc.camera = scenes.cornell_camera()
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def textured_bdpt(width: int, height: int, spp: int, image_path: str) -> Scene:
    """textured_cornell under BidirectionalPathTracer(4, 5)."""
    from rumi_b200.scene import BidirectionalPathTracer
    sc = textured_cornell(width, height, spp, 8, image_path)
    sc.tracer = BidirectionalPathTracer(4, 5)
    return sc


def ibl_scene(width: int, height: int, spp: int, max_depth: int, hdr_path: str) -> Scene:
    """An emissive sphere of radius 15 carrying the sky (HDRTexture, turned by RotationY(-PI)
    like the reference's image-based-lighting preset) as the only light, a Matte ball, a
    mirror ball and a Matte floor."""
    sc = Scene()
    env = Sphere((0.5, 0.5, 0.5), 15.0, transform=RotationY(-np.pi))
    sc.add(env, Emissive(1.0, (1.0, 1.0, 1.0)))
    env.AddingTexture(HDRTexture.from_hdr(hdr_path))
    sc.lights.append(ImageBasedLight(env))
    sc.add(Rect((-1.5, 0.0, -1.0), (0.0, 0.0, 3.0), (3.5, 0.0, 0.0)), Matte(0.8, (0.8, 0.8, 0.8)))
    sc.add(Sphere((0.35, 0.25, 0.6), 0.25), Matte(1.0, (0.9, 0.6, 0.4)))
    sc.add(Sphere((0.8, 0.15, 0.35), 0.15), Specular(1.0, (0.95, 0.95, 0.95)))
    sc.camera = Pinhole((0.5, 0.45, -1.4), identity16(), 1.0, fov=40.0)
    sc.image = Film(width, height, spp)
    sc.tracer = PathTracer(max_depth)
    return sc


def case_files(directory: str):
    """(image BMP path, sky HDR path) written into `directory`."""
    return (write_image(os.path.join(directory, "ball.bmp")), write_sky(os.path.join(directory, "sky.hdr")))
