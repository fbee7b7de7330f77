"""The reference-side adapter (rumi-renderer_b200/adapter/rumi_gpu_integrators.cpp):
GpuPathTracer / GpuBDPT installed as Scene::_tracer_ptr of a Scene built through the
reference's own classes, rendered by the reference's own Scene::Rendering loop
(src/Scene/scene.cpp:206-258).

CPU: the adapter compiles against the reference's headers, and its walk over the
reference's Scene (RumiFlattenScene) yields the same geometry, per-primitive materials,
lights, medium and camera as the Python host mirror's Scene.flatten() of the same scene.
GPU: frames rendered through Scene::Rendering with the GPU integrators installed match the
reference's CPU integrators' frames (golden fixtures) within 3 sigma."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import refimpl
from rumi_b200 import _capi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "oracle", "_ref", "librumi_ref_gpuhost.so")
ADAPTER = os.path.join(ROOT, "rumi-renderer_b200", "adapter")

need_host = pytest.mark.skipif(not (refimpl.available() and os.path.exists(HOST)),
                               reason="reference build with the adapter host (python oracle/build_ref.py) missing")

_host = None


def host():
    global _host
    if _host is None:
        refimpl.lib()  # the reference build first: the host library links the same copy
        L = C.CDLL(HOST)
        fp, ip, vp = C.POINTER(C.c_float), C.POINTER(C.c_int), C.c_void_p
        L.ref_gpu_rendering.restype = C.c_int
        L.ref_gpu_rendering.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_int, fp, C.c_char_p,
                                        C.c_int]
        L.ref_gpu_flatten.restype = C.c_int
        L.ref_gpu_flatten.argtypes = [vp, ip, fp, fp, fp, ip, fp, ip, fp, ip, vp, vp, vp, vp, C.c_char_p, C.c_int]
        refimpl.lib().ref_scene_ptr.restype = C.c_void_p
        refimpl.lib().ref_scene_ptr.argtypes = [C.c_void_p]
        _host = L
    return _host


def scene_ptr(rs):
    return refimpl.lib().ref_scene_ptr(rs.h)


def adapter_flatten(rs):
    L = host()
    counts = (C.c_int * 5)()
    err = C.create_string_buffer(256)
    nul = [None] * 8
    assert L.ref_gpu_flatten(scene_ptr(rs), counts, *nul, None, None, None, None, err, 256) == 0, err.value
    nT, nR, nS, nM, nL = list(counts)
    out = dict(tri_v=np.zeros((nT, 3, 3), np.float32), tri_n=np.zeros((nT, 3, 3), np.float32),
               tri_alb=np.zeros((nT, 3), np.float32), tri_mat=np.zeros(nT, np.int32),
               rects=np.zeros((nR, 9), np.float32), rect_mat=np.zeros(nR, np.int32),
               spheres=np.zeros((nS, 4), np.float32), sphere_mat=np.zeros(nS, np.int32))
    mats = (_capi.rumi_material * max(nM, 1))()
    lights = (_capi.rumi_light * max(nL, 1))()
    cam, vol = _capi.rumi_camera(), _capi.rumi_volume()

    def P(a, t=C.c_float):
        return a.ctypes.data_as(C.POINTER(t))
    assert L.ref_gpu_flatten(scene_ptr(rs), counts, P(out["tri_v"]), P(out["tri_n"]), P(out["tri_alb"]),
                             P(out["tri_mat"], C.c_int), P(out["rects"]), P(out["rect_mat"], C.c_int),
                             P(out["spheres"]), P(out["sphere_mat"], C.c_int), C.cast(mats, C.c_void_p),
                             C.cast(lights, C.c_void_p), C.byref(cam), C.byref(vol), err, 256) == 0, err.value
    out["mats"] = [mats[i] for i in range(nM)]
    out["lights"] = [lights[i] for i in range(nL)]
    out["camera"], out["volume"] = cam, vol
    return out


def _effective(mat_type, kd, ks, e, rgb, eta_in, eta_out, rgb2, density):
    f = lambda x: float(np.float32(x))  # noqa: E731
    return (int(mat_type), f(kd), f(ks), f(e), tuple(np.float32(rgb).tolist()), f(eta_in), f(eta_out),
            tuple(np.float32(rgb2).tolist()), round(f(density), 5))


def _py_mat(m, rgb=None):
    return _effective(m.type, m.kd, m.ks, m.exponent, m.rgb if rgb is None else rgb, m.eta_in, m.eta_out, m.rgb2,
                      m.density)


def _c_mat(m, rgb=None):
    return _effective(m.type, m.kd, m.ks, m.exponent, list(m.rgb) if rgb is None else rgb, m.eta_in, m.eta_out,
                      list(m.rgb2), m.density)


CASES = {
    "cornell_pt": lambda: scenes.cornell_pt(16, 16, 4, 8),
    "caustic_parity": lambda: scenes.volumetric_caustic(16, 16, 4, 4, 5, parity=True),
    "subsurface": lambda: scenes.subsurface_cornell(16, 16, 4, 12),
    "per_triangle_albedo": lambda: scenes.bvh_bound_pt(16, 16, 4, 10, levels=3, seed=7),
}


def test_adapter_compiles_against_the_reference_headers():
    """rumi_gpu_integrators.cpp with the reference's own headers (the portability-patched
    copy oracle/build_ref.py writes): its Trace overrides the reference's
    Integrator::Trace(w, h, camera, film) (src/Integrator/integrator.h:15-28) and both
    classes can be constructed with the CPU integrators' signatures."""
    ref_src = os.path.join(ROOT, "oracle", "_ref", "src")
    if not os.path.isdir(ref_src) or not shutil.which("g++"):
        pytest.skip("reference headers (python oracle/build_ref.py) or g++ not present")
    probe = ('#include "rumi_gpu_integrators.h"\n'
             'Integrator *make_pt(Scene *s) { return new GpuPathTracer(s, 15); }\n'
             'Integrator *make_bdpt(Scene *s) { return new GpuBDPT(s, 6, 7); }\n'
             'Integrator *make_rt(Scene *s) { return new GpuRayTracer(s, 10); }\n'
             'static_assert(sizeof(GpuPathTracer) > sizeof(Integrator), "derived");\n')
    for src in (os.path.join(ADAPTER, "rumi_gpu_integrators.cpp"), "-"):
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable", "-include",
                            os.path.join(ROOT, "oracle", "ref_shim.h"), "-I", ref_src, "-I", ADAPTER, "-I",
                            os.path.join(ROOT, "include"), "-x", "c++", src],
                           input=probe if src == "-" else None, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]


@need_host
@pytest.mark.parametrize("case", sorted(CASES))
def test_adapter_flatten_matches_the_host_mirror(case):
    sc = CASES[case]()
    fs = sc.flatten()
    rs = refimpl.RefScene(sc, seed=1)
    a = adapter_flatten(rs)
    # a Model keeps its triangles in the order its own BVH build left them
    # (src/Acceleration/bvh.cpp:72-103 sorts the array in place), so triangles compare as
    # sets: vertices, normals and the material the GPU shades each with (colour from
    # tri_albedo)
    alb = fs.tri_albedo

    def tri_rows(v, n, mat_of):
        return sorted((tuple(v[i].reshape(-1).tolist()), tuple(n[i].reshape(-1).tolist()), mat_of(i))
                      for i in range(v.shape[0]))
    want = tri_rows(fs.tri_vertices, fs.tri_normals,
                    lambda i: _py_mat(fs.materials[fs.tri_material[i]], alb[i] if alb is not None else None))
    got = tri_rows(a["tri_v"], a["tri_n"], lambda i: _c_mat(a["mats"][a["tri_mat"][i]], list(a["tri_alb"][i])))
    assert len(got) == len(want)
    for g_, w_ in zip(got, want):
        assert g_ == w_, (g_, w_)
    np.testing.assert_array_equal(a["rects"], fs.rects)
    np.testing.assert_array_equal(a["spheres"], fs.spheres)
    for i in range(fs.rects.shape[0]):
        assert _c_mat(a["mats"][a["rect_mat"][i]]) == _py_mat(fs.materials[fs.rect_material[i]])
    for i in range(fs.spheres.shape[0]):
        assert _c_mat(a["mats"][a["sphere_mat"][i]]) == _py_mat(fs.materials[fs.sphere_material[i]])
    assert [(l.type, l.shape_type, l.shape_index) for l in a["lights"]] == \
        [(l["type"], l["shape_type"], l["shape_index"]) for l in fs.lights]
    cam = a["camera"]
    np.testing.assert_array_equal(np.array(cam.position, np.float32), np.float32(fs.camera.position))
    np.testing.assert_array_equal(np.array(cam.basis, np.float32), np.float32(fs.camera.basis).reshape(16))
    assert np.float32(cam.fov_deg) == np.float32(fs.camera.fov)
    assert np.float32(cam.y_ratio) == np.float32(fs.camera.y_ratio)
    vol = a["volume"]
    assert bool(vol.present) == (fs.volume is not None)
    if fs.volume is not None:
        np.testing.assert_array_equal(np.array(vol.sigma_s, np.float32), np.float32(fs.volume.sigma_s))
        np.testing.assert_array_equal(np.array(vol.sigma_a, np.float32), np.float32(fs.volume.sigma_a))
        np.testing.assert_array_equal(np.array(vol.pmin, np.float32), np.float32(fs.volume.pmin))
        np.testing.assert_array_equal(np.array(vol.pmax, np.float32), np.float32(fs.volume.pmax))
    rs.close()


def _render_through_reference_loop(sc, integrator, a, b, frames, seed, tmp_path):
    """Frames of Scene::Rendering with GpuPathTracer (integrator 0), GpuBDPT (1) or
    GpuRayTracer (2)."""
    import torch
    torch.cuda.set_device(0)
    rs = refimpl.RefScene(sc, seed=1)
    n = rs.width * rs.height * 3
    out = np.zeros((frames, rs.height, rs.width, 3), np.float32)
    err = C.create_string_buffer(512)
    cwd = os.getcwd()
    os.chdir(tmp_path)  # Film::Save writes "<seconds>s.bmp" into the working directory
    try:
        rc = host().ref_gpu_rendering(scene_ptr(rs), integrator, a, b, seed, frames,
                                      out.ctypes.data_as(C.POINTER(C.c_float)), err, 512)
    finally:
        os.chdir(cwd)
    spp = rs.spp
    rs.close()
    assert rc == 0, err.value
    assert out.size == frames * n
    return [f / spp for f in out]


@pytest.mark.gpu
@need_host
def test_gpu_pathtracer_adapter_in_the_reference_rendering_loop(golden, tmp_path):
    from test_oracle_golden import frames_vs_reference
    g = golden("image_cornell32.npz")
    frames = _render_through_reference_loop(scenes.cornell_pt(32, 32, 16, 8), 0, 8, 0, 32, 41000, tmp_path)
    assert all(np.isfinite(f).all() for f in frames)
    frames_vs_reference(frames, g)
    # each Rendering call rendered a new frame (the seed advances)
    assert not np.array_equal(frames[0], frames[1])


@pytest.mark.gpu
@need_host
def test_gpu_bdpt_adapter_in_the_reference_rendering_loop(golden, tmp_path):
    from test_oracle_golden import frames_vs_reference
    g = golden("image_cornell_bdpt32.npz")
    frames = _render_through_reference_loop(scenes.cornell_bdpt(32, 32, 16, 4, 5), 1, 4, 5, 32, 42000, tmp_path)
    frames_vs_reference(frames, g)


@pytest.mark.gpu
@need_host
def test_gpu_raytracer_adapter_in_the_reference_rendering_loop(golden, tmp_path):
    """GpuRayTracer (the Whitted integrator) installed in place of RayTracer(scene, 10)."""
    from test_oracle_golden import frames_vs_reference
    g = golden("image_whitted_cornell32.npz")
    sc = scenes.whitted(scenes.cornell_pt(32, 32, 16, 8))
    frames = _render_through_reference_loop(sc, 2, sc.tracer.max_depth, 0, 32, 43000, tmp_path)
    frames_vs_reference(frames, g)
