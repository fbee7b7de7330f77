"""Runs a host build of the renderer's kernels (bdpt_host.cpp or pt_host.cpp, built with
address and undefined-behaviour checks) over the parity scenes and prints one JSON object:
per case its status, a hash of every value the kernels produced, the image mean and (BDPT)
the kernel's index-check record or (path tracer) the hash of the other shading
instantiation.  Run as a separate process with the sanitizer runtime preloaded (the Python
interpreter itself is not built with it):

    LD_PRELOAD=$(g++ -print-file-name=libasan.so) python tests/host_build/run_cases.py bdpt|pt LIB [CASE ...]
    LD_PRELOAD=... python tests/host_build/run_cases.py films LIB OUTDIR   (frames for the oracle)
"""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "rumi-renderer_b200"))
sys.path.insert(0, os.path.join(HERE, ".."))

from rumi_b200 import scenes, build_desc  # noqa: E402
from rumi_b200.scene import PathTracer, RayTracer  # noqa: E402


def _bdpt45(sc):
    sc.tracer = scenes.BidirectionalPathTracer(4, 5)
    return sc


def _pt(sc, depth):
    sc.tracer = PathTracer(depth)
    return sc


_FILES = []


def _tex_files():
    """(image BMP path, sky HDR path) of the textured cases, written once per process into a
    temporary folder that is removed when the process exits."""
    if not _FILES:
        import atexit
        import tempfile
        import texture_cases as TC
        folder = tempfile.TemporaryDirectory(prefix="rumi_tex_")
        atexit.register(folder.cleanup)
        _FILES.extend(TC.case_files(folder.name))
    return _FILES


def _textured(kind, medium=False):
    import texture_cases as TC
    img, hdr = _tex_files()
    if kind == "tex":
        sc = TC.textured_cornell(32, 32, 16, 8, img)
    elif kind == "tex_bdpt":
        sc = TC.textured_bdpt(32, 32, 16, img)
    else:
        sc = TC.ibl_scene(32, 32, 16, 8, hdr)
    return scenes.with_medium(sc) if medium else sc


def bdpt_cases():
    from test_oracle_golden import lights_in_medium, sss_in_medium
    S = scenes
    return {
        # (scene builder, samples per pixel, golden fixture of the reference's frames or None)
        "cornell": (lambda: S.cornell_bdpt(32, 32, 16, 4, 5), 16, "image_cornell_bdpt32.npz"),
        "caustic45": (lambda: S.volumetric_caustic(32, 32, 16, 4, 5, parity=True), 16, "image_caustic_bdpt32.npz"),
        "caustic67": (lambda: S.volumetric_caustic(32, 32, 16, 6, 7, parity=True), 16,
                      "image_caustic_bdpt67_32.npz"),
        "sss": (lambda: _bdpt45(S.subsurface_cornell(32, 32, 16, 12)), 16, "image_sss_bdpt32.npz"),
        "dof": (lambda: _bdpt45(S.cornell_dof_pt(32, 32, 16, 8)), 16, "image_dof_bdpt32.npz"),
        "mesh": (lambda: _bdpt45(S.bvh_bound_pt(32, 32, 16, 10, levels=3, seed=7)), 4, "image_mesh_bdpt32.npz"),
        "glass": (lambda: S.with_bdpt(S.absorbing_glass_cornell()), 16, "image_glass_bdpt32.npz"),
        "sphere_light": (lambda: _bdpt45(S.cornell_sphere_light_pt(32, 32, 16, 8)), 16,
                         "image_sphere_light_bdpt32.npz"),
        "two_lights": (lambda: _bdpt45(S.cornell_two_lights_pt(32, 32, 16, 8)), 16, "image_two_lights_bdpt32.npz"),
        "sphere_light_medium": (lambda: S.with_bdpt(S.with_medium(S.cornell_sphere_light_pt(32, 32, 16, 8))), 16,
                                "image_sphere_light_medium_bdpt32.npz"),
        "cornell_medium": (lambda: S.with_medium(S.cornell_bdpt(32, 32, 16, 4, 5)), 16,
                           "image_cornell_medium_bdpt32.npz"),
        "two_lights_medium": (lambda: lights_in_medium("two_bdpt"), 16, "image_two_lights_medium_bdpt32.npz"),
        "sss_medium": (lambda: sss_in_medium(True), 16, "image_sss_medium_bdpt32.npz"),
        # the volumetric-caustic workload itself (spot light, Henyey-Greenstein g = 0.7,
        # subpaths of 6 and 7 vertices) and the 16-vertex kernel instantiation
        "workload": (lambda: S.volumetric_caustic(32, 32, 8, 6, 7), 8, None),
        "long": (lambda: S.cornell_bdpt(16, 16, 4, 12, 16), 4, None),
        # textures (an image texture and checkers)
        "textured": (lambda: _textured("tex_bdpt"), 16, "image_tex_bdpt32.npz"),
        "textured_medium": (lambda: _textured("tex_bdpt", medium=True), 16, "image_tex_medium_bdpt32.npz"),
    }


def pt_cases():
    from test_oracle_golden import lights_in_medium, sss_in_medium
    S = scenes
    return {
        "cornell": (lambda: S.cornell_pt(32, 32, 16, 8), 16, "image_cornell32.npz"),
        "caustic": (lambda: _pt(S.volumetric_caustic(32, 32, 16, 4, 5, parity=True), 8), 16,
                    "image_caustic_pt32.npz"),
        "sss": (lambda: S.subsurface_cornell(32, 32, 16, 12), 16, "image_sss_pt32.npz"),
        "glass": (lambda: S.absorbing_glass_cornell(), 16, "image_glass_pt32.npz"),
        "sphere_light": (lambda: S.cornell_sphere_light_pt(32, 32, 16, 8), 16, "image_sphere_light_pt32.npz"),
        "two_lights": (lambda: S.cornell_two_lights_pt(32, 32, 16, 8), 16, "image_two_lights_pt32.npz"),
        "sphere_light_medium": (lambda: lights_in_medium("sphere"), 16, "image_sphere_light_medium_pt32.npz"),
        "two_lights_medium": (lambda: S.with_medium(S.cornell_two_lights_pt(32, 32, 16, 8)), 16,
                              "image_two_lights_medium_pt32.npz"),
        "sss_medium": (lambda: sss_in_medium(False), 16, "image_sss_medium_pt32.npz"),
        # the BVH-bound workload's scene kind (displaced-sphere mesh, per-triangle albedo)
        "mesh": (lambda: S.bvh_bound_pt(32, 32, 4, 10, levels=3, seed=7), 4, None),
        # the Whitted ray tracer
        "whitted_cornell": (lambda: S.whitted(S.cornell_pt(32, 32, 16, 8)), 16, "image_whitted_cornell32.npz"),
        "whitted_caustic": (lambda: S.whitted(S.volumetric_caustic(32, 32, 16, 4, 5, parity=True)), 16,
                            "image_whitted_caustic32.npz"),
        "whitted_glass": (lambda: S.whitted(S.absorbing_glass_cornell()), 16, "image_glass_whitted32.npz"),
        "whitted_dof": (lambda: S.whitted(S.cornell_dof_pt(32, 32, 16, 8)), 16, "image_dof_whitted32.npz"),
        # textures and an image-based light, alone and around a medium
        "textured": (lambda: _textured("tex"), 16, "image_tex_pt32.npz"),
        "textured_medium": (lambda: _textured("tex", medium=True), 16, "image_tex_medium_pt32.npz"),
        "ibl": (lambda: _textured("ibl"), 16, "image_ibl_pt32.npz"),
        "ibl_medium": (lambda: _textured("ibl", medium=True), 16, "image_ibl_medium_pt32.npz"),
        "whitted_textured": (lambda: S.whitted(_textured("tex")), 16, "image_tex_whitted32.npz"),
        "whitted_ibl": (lambda: S.whitted(_textured("ibl")), 16, "image_ibl_whitted32.npz"),
    }


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def run_bdpt(lib, names):
    fn = lib.rumi_host_bdpt
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                   C.c_void_p]
    cases = bdpt_cases()
    out = {}
    for name in names:
        build, spp, fixture = cases[name]
        sc = build()
        fs = sc.flatten()
        desc, keep = build_desc(fs)
        W, H = fs.image.width, fs.image.height
        L = np.zeros((W * H * spp, 4), np.float32)
        light = np.zeros((H, W, 3), np.float32)
        chk = np.zeros(4, np.int32)
        rc = fn(C.addressof(desc), sc.tracer.nL, sc.tracer.nE, spp, 20000, 0, W * H, L.ctypes.data,
                light.ctypes.data, chk.ctypes.data)
        # the kernel's per-sample values are R, G, B; the film and the light splats B, G, R
        film = L[:, :3].reshape(H, W, spp, 3).sum(2)[..., ::-1] + light
        finite = bool(np.isfinite(L).all() and np.isfinite(light).all())
        out[name] = {"rc": rc, "chk": chk.tolist(), "finite": finite, "hash": _digest(L, light),
                     "mean": float(film.mean() / spp) if finite else None, "fixture": fixture}
    return out


def run_pt(lib, names):
    fn = lib.rumi_host_pt
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
    cases = pt_cases()
    out = {}
    for name in names:
        build, spp, fixture = cases[name]
        sc = build()
        fs = sc.flatten()
        desc, keep = build_desc(fs)
        W, H = fs.image.width, fs.image.height
        whitted = isinstance(sc.tracer, RayTracer)
        integrator = 2 if whitted else 0
        res = {}
        for lean in (-1, 0, 1):
            film = np.zeros((H, W, 3), np.float32)
            stats = np.zeros(16, np.uint64)
            rc = fn(C.addressof(desc), integrator, sc.tracer.max_depth, spp, 30000, lean, film.ctypes.data,
                    stats.ctypes.data)
            res[lean] = (rc, film, stats)
        rc, film, stats = res[-1]
        finite = bool(np.isfinite(film).all())
        out[name] = {"rc": rc, "finite": finite, "hash": _digest(film, stats),
                     "general_hash": _digest(res[0][1], res[0][2]) if res[0][0] == 0 else None,
                     "lean_hash": _digest(res[1][1], res[1][2]) if res[1][0] == 0 else None,
                     "mean": float(film.mean() / spp) if finite else None, "fixture": fixture,
                     "rays": int(stats[0])}
    return out


def film_cases():
    """Frames compared with the oracle pixel by pixel: (scene builder, integrator, depth,
    samples per pixel, seed), the settings of the GPU's per-pixel tests."""
    from test_oracle_golden import WHITTED_CASES
    S = scenes
    out = {"pt_cornell_d2": (lambda: S.cornell_pt(32, 32, 4, 2), 0, 2, 4, 21),
           "pt_dof_d2": (lambda: S.cornell_dof_pt(32, 32, 4, 2), 0, 2, 4, 21),
           # full depth: paths part ways on some pixels once a float difference moves a
           # scattering decision, without bias
           "deep_cornell8": (lambda: S.cornell_pt(32, 32, 4, 8), 0, 8, 4, 21),
           "deep_mesh10": (lambda: S.bvh_bound_pt(32, 32, 4, 10, levels=3, seed=7), 0, 10, 4, 21),
           "deep_caustic8": (lambda: S.volumetric_caustic(32, 32, 4, 4, 5, parity=True), 0, 8, 4, 21),
           "deep_sss12": (lambda: S.subsurface_cornell(32, 32, 4, 12), 0, 12, 4, 21)}
    for fixture, builder in WHITTED_CASES:
        out["whitted_" + fixture[len("image_"):-len(".npz")]] = (builder, 2, None, 4, 31)
    return out


def run_films(lib, outdir):
    fn = lib.rumi_host_pt
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
    out = {}
    for name, (build, integrator, depth, spp, seed) in sorted(film_cases().items()):
        sc = build()
        fs = sc.flatten()
        desc, keep = build_desc(fs)
        film = np.zeros((fs.image.height, fs.image.width, 3), np.float32)
        stats = np.zeros(16, np.uint64)
        d = depth if depth is not None else sc.tracer.max_depth
        rc = fn(C.addressof(desc), integrator, d, spp, seed, -1, film.ctypes.data, stats.ctypes.data)
        np.save(os.path.join(outdir, name + ".npy"), film)
        out[name] = {"rc": rc, "nan": int(stats[2])}
    return out


if __name__ == "__main__":
    kind, lib_path, rest = sys.argv[1], sys.argv[2], sys.argv[3:]
    lib = C.CDLL(lib_path)
    if kind == "bdpt":
        print(json.dumps(run_bdpt(lib, rest or sorted(bdpt_cases()))))
    elif kind == "films":
        print(json.dumps(run_films(lib, rest[0])))
    else:
        print(json.dumps(run_pt(lib, rest or sorted(pt_cases()))))
