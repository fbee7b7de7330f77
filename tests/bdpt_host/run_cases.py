"""Runs the host build of the BDPT kernel (bdpt_host.cpp, built with address and
undefined-behaviour checks) over the BDPT scenes of the parity tests and prints one JSON
object: per case its status, the kernel's index-check record, a hash of every sample value
and the frame's image mean.  Run as a separate process with the sanitizer runtime
preloaded (the Python interpreter itself is not built with it):

    LD_PRELOAD=$(g++ -print-file-name=libasan.so) python tests/bdpt_host/run_cases.py LIB [CASE ...]
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


def _bdpt45(sc):
    sc.tracer = scenes.BidirectionalPathTracer(4, 5)
    return sc


def _cases():
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
    }


def run(lib_path, names):
    lib = C.CDLL(lib_path)
    fn = lib.rumi_host_bdpt
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                   C.c_void_p]
    cases = _cases()
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
        out[name] = {
            "rc": rc, "chk": chk.tolist(), "finite": finite,
            "hash": hashlib.sha256(L.tobytes() + light.tobytes()).hexdigest(),
            "mean": float(film.mean() / spp) if finite else None, "fixture": fixture, "spp": spp,
            "pixels": W * H,
        }
    return out


if __name__ == "__main__":
    lib_path, names = sys.argv[1], sys.argv[2:]
    print(json.dumps(run(lib_path, names or sorted(_cases().keys()))))
