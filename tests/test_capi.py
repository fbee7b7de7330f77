"""Host-side checks that need no GPU: the C-ABI library loads and exports every symbol
its headers declare, argument validation returns status codes, scene flattening and
the synthetic workloads are deterministic."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import rumi_b200
from rumi_b200 import _capi, scenes
from rumi_b200.scene import Scene, Rect, Sphere, Model, Matte, Emissive, AreaLight, Pinhole, Film, PathTracer

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("rumi_b200.h", "rumi_b200_test.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^\s*(?:rumi_status|const char \*|int64_t)\s*(rumi_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _capi.load()
    decl = declared_symbols()
    assert decl == set(_capi.EXPORTS)
    for name in decl:
        assert getattr(L, name) is not None
    assert L.rumi_version().decode().startswith("rumi_b200")


def _prototypes():
    """{name: number of parameters} of every function declared in the two headers."""
    out = {}
    for h in ("rumi_b200.h", "rumi_b200_test.h"):
        text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", h)).read(), flags=re.S)
        for name, args in re.findall(r"\b(rumi_\w+)\s*\(([^;{]*?)\)\s*;", text, re.S):
            args = args.strip()
            out[name] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_ctypes_bindings_take_the_declared_parameters():
    """Every entry point the ctypes layer binds has as many argtypes as the header's
    prototype has parameters (a missing or extra argument would shift every later one)."""
    L = _capi.load()
    protos = _prototypes()
    assert "rumi_render" in protos and "rumi_trace_rays" in protos
    bound = 0
    for name, n in protos.items():
        fn = getattr(L, name)
        if fn.argtypes is None:
            continue
        bound += 1
        assert len(fn.argtypes) == n, (name, len(fn.argtypes), n)
    assert bound >= 15


def test_invalid_arguments_return_status_without_touching_the_gpu():
    L = _capi.load()
    h = C.c_void_p()
    assert L.rumi_scene_create(None, C.byref(h)) == 1  # RUMI_ERR_INVALID_ARG
    assert h.value is None
    assert b"NULL" in L.rumi_last_error_string()
    d = _capi.rumi_scene_desc()
    d.width, d.height = 0, 10
    assert L.rumi_scene_create(C.byref(d), C.byref(h)) == 1
    # material index out of range
    sc = scenes.cornell_pt(8, 8, 1, 2)
    desc, keep = rumi_b200.build_desc(sc.flatten())
    bad = np.full(desc.n_triangles, 99, np.int32)
    desc.tri_material = bad.ctypes.data_as(_capi.IP)
    assert L.rumi_scene_create(C.byref(desc), C.byref(h)) == 1
    assert b"material index" in L.rumi_last_error_string()
    # light referring to a missing rect
    desc, keep = rumi_b200.build_desc(sc.flatten())
    lights = (_capi.rumi_light * 1)()
    lights[0].type, lights[0].shape_type, lights[0].shape_index = 0, 1, 7
    desc.lights = C.cast(lights, C.POINTER(_capi.rumi_light))
    assert L.rumi_scene_create(C.byref(desc), C.byref(h)) == 1
    assert L.rumi_render(None, None, None, 0, None) == 1
    assert L.rumi_trace_rays(None, 1, None, 0, None, None, 0, None, None, None) == 1


def _tex_table(*types, pixels=None, bpp=3):
    t = (_capi.rumi_texture * len(types))()
    for i, ty in enumerate(types):
        t[i].type = ty
        t[i].repeat_u = t[i].repeat_v = 4.0
        t[i].img_width = t[i].img_height = 2
        t[i].bytes_per_pixel = bpp
        t[i].pixels = pixels
    return t


def _set_volume(d, sigma_s=(0.4, 0.4, 0.4), sigma_a=(0.05, 0.05, 0.05), g=0.0):
    d.volume.present = 1
    d.volume.pmin = _capi.f3(0, 0, 0)
    d.volume.pmax = _capi.f3(1, 1, 1)
    d.volume.sigma_s = _capi.f3(*sigma_s)
    d.volume.sigma_a = _capi.f3(*sigma_a)
    d.volume.g = g


def _ibl(d, keep, with_texture=True):
    d.lights[0].type, d.lights[0].shape_type, d.lights[0].shape_index = 2, 2, 0
    if with_texture:
        keep.append(_tex_table(0))
        d.n_textures, d.textures = 1, C.cast(keep[-1], C.POINTER(_capi.rumi_texture))
        keep.append(np.array([0, -1], np.int32))
        d.sphere_texture = keep[-1].ctypes.data_as(_capi.IP)


# (what is wrong, how to make it, text of the error): every rejection of rumi_scene_create's
# descriptor check, reached before any device call
DESC_FAULTS = [
    ("negative count", lambda d, k: setattr(d, "n_lights", -1), "negative count"),
    ("too many primitives", lambda d, k: setattr(d, "n_triangles", 0x3FFFFFFF), "too many primitives"),
    ("no triangle vertices", lambda d, k: setattr(d, "tri_vertices", None), "triangle arrays missing"),
    ("no rect materials", lambda d, k: setattr(d, "rect_material", None), "rect arrays missing"),
    ("no sphere array", lambda d, k: setattr(d, "spheres", None), "sphere arrays missing"),
    ("no materials", lambda d, k: setattr(d, "materials", None), "materials missing"),
    ("no lights", lambda d, k: setattr(d, "lights", None), "lights missing"),
    ("unknown material", lambda d, k: setattr(d.materials[0], "type", 9), "unknown material type"),
    ("light on a missing rect", lambda d, k: setattr(d.lights[0], "shape_index", 7), "light rect index"),
    ("light on a missing sphere", lambda d, k: (setattr(d.lights[0], "shape_type", 2),
                                                setattr(d.lights[0], "shape_index", 5)), "light sphere index"),
    ("triangle area light", lambda d, k: setattr(d.lights[0], "shape_type", 0), "rects or spheres"),
    ("image light on a rect", lambda d, k: (_ibl(d, k), setattr(d.lights[0], "shape_type", 1)), "sphere index"),
    ("image light without texture", lambda d, k: _ibl(d, k, with_texture=False), "has no texture"),
    ("unknown light", lambda d, k: setattr(d.lights[0], "type", 7), "unknown light type"),
    ("no texture table", lambda d, k: setattr(d, "n_textures", 1), "textures missing"),
    ("unknown texture", lambda d, k: (k.append(_tex_table(5)), setattr(d, "n_textures", 1),
                                      setattr(d, "textures", C.cast(k[-1], C.POINTER(_capi.rumi_texture)))),
     "unknown texture type"),
    ("image texture without pixels", lambda d, k: (k.append(_tex_table(1)), setattr(d, "n_textures", 1),
                                                   setattr(d, "textures", C.cast(k[-1], C.POINTER(_capi.rumi_texture)))),
     "texture image missing"),
    ("two bytes per pixel", lambda d, k: (k.append(np.zeros(16, np.uint8)),
                                          k.append(_tex_table(1, pixels=k[-1].ctypes.data, bpp=2)),
                                          setattr(d, "n_textures", 1),
                                          setattr(d, "textures", C.cast(k[-1], C.POINTER(_capi.rumi_texture)))),
     "3 or 4 bytes per pixel"),
    ("texture index past the table", lambda d, k: (k.append(_tex_table(0)), setattr(d, "n_textures", 1),
                                                   setattr(d, "textures", C.cast(k[-1], C.POINTER(_capi.rumi_texture))),
                                                   k.append(np.full(d.n_triangles, 1, np.int32)),
                                                   setattr(d, "tri_texture", k[-1].ctypes.data_as(_capi.IP))),
     "texture index out of range"),
    ("negative scattering", lambda d, k: _set_volume(d, sigma_s=(-0.1, 0.4, 0.4)), "positive extinction"),
    ("a clear channel", lambda d, k: _set_volume(d, sigma_s=(0.4, 0.0, 0.4), sigma_a=(0.05, 0.0, 0.05)),
     "positive extinction"),
    ("NaN absorption", lambda d, k: _set_volume(d, sigma_a=(float("nan"), 0.05, 0.05)), "positive extinction"),
    ("g of one", lambda d, k: _set_volume(d, g=1.0), "medium g"),
]


@pytest.mark.parametrize("what,fault,message", DESC_FAULTS, ids=[f[0] for f in DESC_FAULTS])
def test_scene_descriptor_faults_are_rejected_before_the_device(what, fault, message):
    """Host-side fault injection: a descriptor broken in one way returns
    RUMI_ERR_INVALID_ARG with its reason and no scene, without a GPU."""
    L = _capi.load()
    desc, keep = rumi_b200.build_desc(scenes.cornell_pt(8, 8, 1, 2).flatten())
    fault(desc, keep)
    h = C.c_void_p()
    assert L.rumi_scene_create(C.byref(desc), C.byref(h)) == 1
    assert h.value is None
    assert message.encode() in L.rumi_last_error_string(), L.rumi_last_error_string()


def test_every_entry_point_rejects_null_handles_without_a_gpu():
    """NULL scenes, batches, parameter blocks and buffers: RUMI_ERR_INVALID_ARG from every
    entry point that takes them, a no-op from the destroy calls (as free(NULL))."""
    L = _capi.load()
    p = _capi.rumi_render_params()
    p.integrator, p.max_depth, p.spp = 0, 2, 1
    buf = np.zeros(16, np.float32)
    ptr = buf.ctypes.data_as(C.c_void_p)
    out = C.c_void_p()
    assert L.rumi_scene_destroy(None) == 0
    assert L.rumi_batch_destroy(None) == 0
    assert L.rumi_batch_film_floats(None) == 0
    assert L.rumi_scene_bvh_info(None, None) == 1
    assert L.rumi_render_noalloc(None, C.byref(p), ptr, None) == 1
    assert L.rumi_forward(None, C.byref(p), ptr, 0, None) == 1
    assert L.rumi_forward(None, None, ptr, 0, None) == 1
    assert L.rumi_backward(None, C.byref(p), ptr, ptr, ptr, 0, None) == 1
    assert L.rumi_scene_set_albedo(None, ptr, 0) == 1
    assert L.rumi_scene_set_volume(None, None) == 1
    assert L.rumi_batch_create(None, 0, C.byref(out)) == 1 and out.value is None
    arr = (C.c_void_p * 2)(None, None)
    assert L.rumi_batch_create(arr, 0, C.byref(out)) == 1
    assert b"empty batch" in L.rumi_last_error_string()
    bp = _capi.rumi_batch_params()
    assert L.rumi_render_batch(None, C.byref(bp), ptr, 0, None) == 1


def test_flatten_canonical_order_and_lights():
    sc = Scene()
    r = sc.add(Rect((0, 1, 0), (1, 0, 0), (0, 0, 1)), Emissive(2.0, (1, 1, 1)))
    sc.add(Sphere((0, 0, 0), 0.5), Matte(1, (0.5, 0.5, 0.5)))
    tris = np.random.default_rng(0).uniform(size=(3, 3, 3)).astype(np.float32)
    sc.add(Model(tris), Matte(1, (0.2, 0.3, 0.4)))
    sc.lights.append(AreaLight(r))
    sc.camera, sc.image, sc.tracer = Pinhole((0, 0, -2)), Film(4, 4, 1), PathTracer(3)
    fs = sc.flatten()
    assert fs.n_prims == 5
    assert fs.tri_vertices.shape == (3, 3, 3) and fs.rects.shape == (1, 9) and fs.spheres.shape == (1, 4)
    assert fs.lights == [dict(type=0, shape_type=1, shape_index=0)]
    # face normals exactly as Normalize(Cross(v1 - v0, v2 - v0)) in float32
    e1, e2 = tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0]
    c = np.cross(e1, e2).astype(np.float32)
    n = c * (np.float32(1) / np.sqrt((c * c).sum(1, dtype=np.float32)))[:, None]
    np.testing.assert_array_equal(fs.tri_normals[:, 0], n.astype(np.float32))


def test_synthetic_meshes_are_deterministic():
    t5 = scenes.displaced_sphere(5, (0.5, 0.35, 0.5), 0.25, 0.05, 7)
    assert t5.shape == (4 * 4 ** 5, 3, 3)
    assert scenes.mesh_checksum(t5) == scenes.mesh_checksum(scenes.displaced_sphere(5, (0.5, 0.35, 0.5), 0.25, 0.05, 7))
    assert scenes.mesh_checksum(t5) != scenes.mesh_checksum(scenes.displaced_sphere(5, (0.5, 0.35, 0.5), 0.25, 0.05, 8))
    # the 1,048,576-triangle workload mesh: count is 4 * 4^9
    assert 4 * 4 ** 9 == 1048576
    r = np.linalg.norm(t5.reshape(-1, 3) - np.array([0.5, 0.35, 0.5], np.float32), axis=1)
    assert r.min() > 0.19 and r.max() < 0.31
    alb = scenes.random_albedo(1000, 8)
    assert alb.min() >= 0.2 and alb.max() <= 0.8


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++11")])
def test_headers_compile_for_plain_c_and_cxx_hosts(tmp_path, compiler, std):
    """The boundary headers are what a reference-side host includes: they must compile as
    plain C99 (cgo / FFI generators) and as C++ without anything from the library's own
    build (no CUDA headers), with every struct field the ctypes mirror declares."""
    import shutil
    import subprocess
    if shutil.which(compiler) is None:
        pytest.skip(compiler + " not installed")
    inc = os.path.join(ROOT, "include")
    src = tmp_path / ("h.c" if compiler == "gcc" else "h.cpp")
    src.write_text('#include "rumi_b200.h"\n#include "rumi_b200_test.h"\n'
                   "int main(void) {\n"
                   "    rumi_scene_desc d; rumi_render_params p; rumi_texture t;\n"
                   "    (void)d; (void)p; (void)t;\n"
                   "    return (int)sizeof(rumi_scene_desc) + RUMI_FLAG_KEEP_RADIANCE + RUMI_LIGHT_IBL + RUMI_TEX_HDR;\n"
                   "}\n")
    r = subprocess.run([compiler, std, "-Wall", "-Werror", "-fsyntax-only", "-I", inc, str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """sizeof and field offsets of the C structs equal those of the ctypes mirror in
    rumi_b200/_capi.py (a mismatch would hand the library misread scene descriptions)."""
    import ctypes as C
    import shutil
    import subprocess
    from rumi_b200 import _capi
    if shutil.which("gcc") is None:
        pytest.skip("gcc not installed")
    structs = ["rumi_material", "rumi_light", "rumi_volume", "rumi_camera", "rumi_texture", "rumi_scene_desc",
               "rumi_render_params", "rumi_render_stats"]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rumi_b200.h"', "int main(void) {"]
    for sname in structs:
        cls = getattr(_capi, sname)
        lines.append('    printf("%s %%zu\\n", sizeof(%s));' % (sname, sname))
        for fname, _ in cls._fields_:
            lines.append('    printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (sname, fname, sname, fname))
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for sname in structs:
        cls = getattr(_capi, sname)
        assert int(got[sname]) == C.sizeof(cls), sname
        for fname, _ in cls._fields_:
            assert int(got[f"{sname}.{fname}"]) == getattr(cls, fname).offset, (sname, fname)
