"""Textures and image-based lights: the file loaders against the reference's LoadHDR /
LoadBmp, Texture::Pattern of the oracle and the GPU against the reference's own, and
frames of textured and image-lit scenes against the reference's PathTracer and RayTracer
frames (tests/golden/image_{tex,ibl}_{pt,whitted}32.npz, made by make_golden.py textures
from the seeded files of texture_cases.py)."""
import ctypes as C
import os

import numpy as np
import pytest

import oraclelib as O
import refimpl
import texture_cases as TC
from rumi_b200 import scenes, textures as T
from rumi_b200.scene import RayTracer, Sphere, Rect, BidirectionalPathTracer

from test_oracle_golden import frames_vs_reference


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("tex")
    return TC.case_files(str(d))


def _cases(img, hdr):
    return [("image_tex_pt32.npz", TC.textured_cornell(32, 32, 16, 8, img)),
            ("image_tex_whitted32.npz", scenes.whitted(TC.textured_cornell(32, 32, 16, 8, img))),
            ("image_ibl_pt32.npz", TC.ibl_scene(32, 32, 16, 8, hdr)),
            ("image_ibl_whitted32.npz", scenes.whitted(TC.ibl_scene(32, 32, 16, 8, hdr)))]


def _ref_hdr(path, cap=1 << 20):
    buf = np.zeros(cap, np.float32)
    wh = (C.c_int * 2)()
    n = refimpl.lib().ref_load_hdr(path.encode(), cap, refimpl.P(buf), wh)
    return buf[:3 * n].reshape(wh[1], wh[0], 3)


def _ref_bmp(path, cap=1 << 20):
    buf = np.zeros(cap, np.uint8)
    whb = (C.c_uint * 3)()
    n = refimpl.lib().ref_load_bmp(path.encode(), cap, buf.ctypes.data, whb)
    return buf[:n].reshape(whb[1], whb[0], whb[2])


@pytest.mark.parametrize("width,height,comment,extra", [(64, 32, b"# sky", b""),
                                                        (40, 9, b"#c1\n#c2", b"EXPOSURE=1.0\nGAMMA=2.2\n"),
                                                        (8, 3, b"#", b"PRIMARIES=0 0 0 0 0 0 0 0\n")])
def test_hdr_loader_matches_reference(tmp_path, width, height, comment, extra):
    """load_hdr = LoadHDR (hdr.cpp:4-107) bit for bit: header lines, run-length scanlines."""
    rgbe = TC.sky_rgbe(width, height, seed=width)
    rgbe[0, : width // 2] = rgbe[0, 0]  # a long run
    rgbe[1, ::3, 3] = 0                  # e = 0 -> black
    p = str(tmp_path / "a.hdr")
    T.save_hdr(p, rgbe, comment=comment, extra=extra)
    ours = T.load_hdr(p)
    assert ours.shape == (height, width, 3)
    np.testing.assert_array_equal(ours, _ref_hdr(p))
    e = rgbe[..., 3].astype(np.int64)
    exp = np.where(e[..., None] > 0, rgbe[..., :3] * np.ldexp(1.0, e - 136)[..., None], 0.0)
    np.testing.assert_array_equal(ours, exp.astype(np.float32))


def test_hdr_loader_rejects_what_the_reference_cannot_read(tmp_path):
    """Widths whose low byte is >= 128 fail the reference's signed-char width check, and
    flat (old-style) scanlines are not decoded: ValueError, where the reference prints an
    error and leaves its buffer unwritten."""
    p = str(tmp_path / "w200.hdr")
    T.save_hdr(p, TC.sky_rgbe(200, 2))
    with pytest.raises(ValueError):
        T.load_hdr(p)
    flat = b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 1 +X 8\n" + bytes([10, 20, 30, 130]) * 8
    with pytest.raises(ValueError):
        T.load_hdr_bytes(flat)
    with pytest.raises(ValueError):
        T.load_hdr_bytes(b"#?RGBE\n")


@pytest.mark.parametrize("width,height,bpp", [(20, 12, 3), (7, 5, 3), (8, 6, 4), (1, 3, 3)])
def test_bmp_loader_matches_reference(tmp_path, width, height, bpp):
    """load_bmp = LoadBmp (bmp.cpp:3-57): rows in file order, width % 4 bytes skipped."""
    p = str(tmp_path / "a.bmp")
    TC.write_image(p, width=width, height=height, bpp=bpp, seed=width * 7 + bpp)
    ours = T.load_bmp(p)
    np.testing.assert_array_equal(ours, _ref_bmp(p))
    np.testing.assert_array_equal(ours, TC.image_pixels(width, height, bpp, seed=width * 7 + bpp))


def _surface_points(sc, flat, n=3000, seed=1):
    """Points on every textured rect / sphere of sc with their canonical primitive ids."""
    rng = np.random.default_rng(seed)
    nt, nr = flat.tri_vertices.shape[0], flat.rects.shape[0]
    rects = [o for o in sc.objects if isinstance(o, Rect)]
    spheres = [o for o in sc.objects if isinstance(o, Sphere)]
    out = []
    for s in sc.objects:
        if getattr(s, "texture", None) is None:
            continue
        if isinstance(s, Sphere):
            d = rng.normal(size=(n, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            pts = (s.c + s.r * d).astype(np.float32)
            pid = nt + nr + spheres.index(s)
        else:
            a = rng.random((n, 2)).astype(np.float32)
            pts = (s.p + a[:, :1] * s.l + a[:, 1:] * s.w).astype(np.float32)
            pid = nt + rects.index(s)
        out.append((s, pts, np.full(n, pid, np.int32)))
    return out


def test_oracle_texture_pattern_matches_reference(files):
    """Checker, ImageTexture and HDRTexture through Rect / Sphere::TextureMapping (a rotated
    sphere frame included): the oracle's Texture::Pattern equals the reference's bit for bit."""
    img, hdr = files
    for sc in (TC.textured_cornell(8, 8, 1, 2, img), TC.ibl_scene(8, 8, 1, 2, hdr)):
        rs = refimpl.RefScene(sc, seed=1)
        os_ = O.OracleScene(sc)
        for s, pts, pid in _surface_points(sc, os_.flat):
            np.testing.assert_array_equal(os_.texture_pattern(pid, pts), rs.texture_pattern(s, pts))
        rs.close()


@pytest.mark.parametrize("k", range(4))
def test_oracle_textured_frames_match_reference_3sigma(golden, files, k):
    name, sc = _cases(*files)[k]
    os_ = O.OracleScene(sc)
    frames = []
    for s in range(24):
        if isinstance(sc.tracer, RayTracer):
            film, nan = os_.render_whitted(sc.tracer.max_depth, 16, seed=2000 + s)
        else:
            film, nan = os_.render_pt(sc.tracer.max_depth, 16, seed=2000 + s)
        assert nan == 0
        frames.append(film / 16.0)
    frames_vs_reference(frames, golden(name))


# ------------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_gpu_texture_pattern_matches_reference(files):
    """The device's Texture::Pattern against the reference's: the same texel on all but a
    handful of points (device acosf / atan2f / sinf may differ from the host's in the last
    bit, which moves a point across a texel edge only at the edge)."""
    import rumi_b200
    img, hdr = files
    for sc in (TC.textured_cornell(8, 8, 1, 2, img), TC.ibl_scene(8, 8, 1, 2, hdr)):
        rs = refimpl.RefScene(sc, seed=1)
        gs = rumi_b200.GpuScene(sc)
        for s, pts, pid in _surface_points(sc, gs.flat):
            out = np.zeros_like(pts)
            assert gs.lib.rumi_test_texture_pattern(gs.h, len(pid), pid.ctypes.data, pts.ctypes.data,
                                                    out.ctypes.data) == 0
            ref = rs.texture_pattern(s, pts)
            same = np.all(np.abs(out - ref) <= 1e-6 * np.maximum(1.0, np.abs(ref)), axis=1)
            assert same.mean() >= 0.995, (type(s.texture).__name__, same.mean())
        gs.close()
        rs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(4))
def test_gpu_textured_frames_match_reference_3sigma(golden, files, k):
    from test_gpu_parity import gpu_frames
    name, sc = _cases(*files)[k]
    frames_vs_reference(gpu_frames(sc, 32, 16000 + 100 * k), golden(name))


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(4))
def test_gpu_textured_frame_matches_oracle_per_pixel(files, k):
    """Same Philox streams: per-pixel agreement on paths of two vertices (the image-based
    light's sampled direction goes through device sinf / cosf / acosf, so a light sample
    may land on a neighbouring texel: a few pixels may differ)."""
    import rumi_b200
    name, sc = _cases(*files)[k]
    sc.tracer = RayTracer(1) if isinstance(sc.tracer, RayTracer) else scenes.PathTracer(2)
    gs = rumi_b200.GpuScene(sc)
    film, st = gs.render(spp=4, seed=41)
    gs.close()
    os_ = O.OracleScene(sc)
    if isinstance(sc.tracer, RayTracer):
        ofilm, onan = os_.render_whitted(1, 4, 41)
    else:
        ofilm, onan = os_.render_pt(2, 4, 41)
    assert st["nan_samples"] == onan == 0
    rel = np.abs(film - ofilm) / np.maximum(np.abs(ofilm), 1e-3)
    assert np.mean(rel.max(2) > 1e-3) <= 0.02, float(np.mean(rel.max(2) > 1e-3))
    assert abs(film.sum() / ofilm.sum() - 1.0) < 5e-3


@pytest.mark.gpu
def test_gpu_textured_bdpt_matches_reference_3sigma(golden, files):
    """BDPT with textures: subpath throughputs take each surface vertex's pattern and a
    connection both connecting vertices' (bidirectionalpathtracer.cpp:350-364, 660-661,
    971-972), against the reference's BidirectionalPathTracer frames."""
    from test_gpu_parity import gpu_frames
    frames_vs_reference(gpu_frames(TC.textured_bdpt(32, 32, 16, files[0]), 32, 17000),
                        golden("image_tex_bdpt32.npz"))


@pytest.mark.gpu
def test_gpu_bdpt_rejects_image_based_lights(files):
    import rumi_b200
    from rumi_b200 import _capi
    sc = TC.ibl_scene(8, 8, 1, 2, files[1])
    gs = rumi_b200.GpuScene(sc)
    with pytest.raises(_capi.RumiError):
        gs.render(spp=1, tracer=BidirectionalPathTracer(3, 3))
    gs.close()


def test_oracle_textured_scene_in_a_medium_matches_reference_3sigma(golden, files):
    """The textured Cornell scene inside a homogeneous medium, path traced: a medium vertex
    takes no texture, a surface vertex its own."""
    sc = scenes.with_medium(TC.textured_cornell(32, 32, 16, 8, files[0]))
    os_ = O.OracleScene(sc)
    frames = []
    for s in range(24):
        film, nan = os_.render_pt(sc.tracer.max_depth, 16, seed=2100 + s)
        assert nan == 0
        frames.append(film / 16.0)
    frames_vs_reference(frames, golden("image_tex_medium_pt32.npz"))


@pytest.mark.gpu
@pytest.mark.parametrize("fixture,bdpt", [("image_tex_medium_pt32.npz", False), ("image_tex_medium_bdpt32.npz", True)])
def test_gpu_textured_scene_in_a_medium_matches_reference_3sigma(golden, files, fixture, bdpt):
    """The textured Cornell scene inside a medium, path traced and under BDPT (where a medium
    connection vertex takes the texture of the surface its segment was headed for)."""
    from test_gpu_parity import gpu_frames
    sc = TC.textured_bdpt(32, 32, 16, files[0]) if bdpt else TC.textured_cornell(32, 32, 16, 8, files[0])
    frames_vs_reference(gpu_frames(scenes.with_medium(sc), 32, 18000), golden(fixture))


def test_oracle_image_based_light_around_a_medium_matches_reference_3sigma(golden, files):
    """An image-based light (an emissive textured sphere around the scene) lighting the
    Cornell scene through a medium, path traced."""
    sc = scenes.with_medium(TC.ibl_scene(32, 32, 16, 8, files[1]))
    os_ = O.OracleScene(sc)
    frames = []
    for s in range(24):
        film, nan = os_.render_pt(sc.tracer.max_depth, 16, seed=2200 + s)
        assert nan == 0
        frames.append(film / 16.0)
    frames_vs_reference(frames, golden("image_ibl_medium_pt32.npz"))


@pytest.mark.gpu
def test_gpu_image_based_light_around_a_medium_matches_reference_3sigma(golden, files):
    from test_gpu_parity import gpu_frames
    frames_vs_reference(gpu_frames(scenes.with_medium(TC.ibl_scene(32, 32, 16, 8, files[1])), 32, 19000),
                        golden("image_ibl_medium_pt32.npz"))
