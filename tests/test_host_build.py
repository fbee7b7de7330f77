"""The renderer's kernels built by g++ for the host and run over the parity scenes
(tests/host_build): the BDPT kernel (rumi-renderer_b200/csrc/bdpt.cu) one camera sample after
another, and the path tracer's kernels (rumi-renderer_b200/csrc/pt.cu: generation,
closest-hit and any-hit traversal, shading, Whitted shading) in the launch order of the
library's serial schedule, over every BDPT / path-traced / Whitted parity scene without
textures, the volumetric-caustic BDPT workload (spot light, HG g = 0.7, subpaths of 6 and 7
vertices), the 16-vertex BDPT instantiation and the BVH-bound workload's mesh kind:

* under AddressSanitizer and UndefinedBehaviorSanitizer: every access stays inside its
  object and no arithmetic is undefined;
* with every automatic variable initialised to a pattern, and again to zero: the two builds
  produce the same values bit for bit, so no result depends on a variable read before it is
  written;
* with the BDPT kernel's own index checks (bd_index) silent;
* with the path tracer's two shading instantiations (general and lean) bit-identical on the
  scenes the lean one applies to: on the host nothing contracts multiply-adds, so this shows
  the lean instantiation only leaves out branches such scenes never take;
* with image means near the reference's frames (within 10%, or 4 sigma of the reference's
  frame-to-frame spread where that is larger; the host's libm is not the device's, so the
  values are not the GPU's bit for bit).

This checks the kernels' logic on the CPU, where a fault cannot reach a GPU."""
import json
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HOST_DIR = os.path.join(HERE, "host_build")
sys.path.insert(0, HOST_DIR)

import run_cases  # noqa: E402

BDPT_CASES = sorted(run_cases.bdpt_cases())
PT_CASES = sorted(run_cases.pt_cases())


def _cuda_include():
    for root in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if root and os.path.isfile(os.path.join(root, "include", "cuda_runtime.h")):
            return os.path.join(root, "include")
    nvcc = shutil.which("nvcc")
    if nvcc:
        inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
        if os.path.isfile(os.path.join(inc, "cuda_runtime.h")):
            return inc
    return None


@pytest.fixture(scope="module")
def host_runs(tmp_path_factory):
    gxx = shutil.which("g++")
    inc = _cuda_include()
    if not gxx or not inc:
        pytest.skip("g++ or the CUDA headers are missing")
    asan = subprocess.run([gxx, "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    if not os.path.isabs(asan) or not os.path.exists(asan):
        pytest.skip("no AddressSanitizer runtime for g++")
    out = tmp_path_factory.mktemp("host_build")
    flags = ["-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
             "-fno-sanitize-recover=undefined", "-ffp-contract=off", "-fPIC", "-shared", "-I" + inc]
    libs, procs = {}, []
    for kind in ("bdpt", "pt"):
        for init in ("pattern", "zero"):
            lib = str(out / ("lib%s_host_%s.so" % (kind, init)))
            libs[(kind, init)] = lib
            src = os.path.join(HOST_DIR, "%s_host.cpp" % kind)
            procs.append(subprocess.Popen([gxx, *flags, "-ftrivial-auto-var-init=" + init, src, "-o", lib],
                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    for p in procs:
        _, se = p.communicate(timeout=900)
        assert p.returncode == 0, se[-4000:]
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0", UBSAN_OPTIONS="print_stacktrace=1")
    runs = {}
    for (kind, init), lib in libs.items():
        r = subprocess.run([sys.executable, os.path.join(HOST_DIR, "run_cases.py"), kind, lib], capture_output=True,
                           text=True, env=env, timeout=1800)
        assert r.returncode == 0, r.stderr[-6000:]
        assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-6000:]
        runs[(kind, init)] = json.loads(r.stdout.strip().splitlines()[-1])
    films = out / "films"
    films.mkdir()
    r = subprocess.run([sys.executable, os.path.join(HOST_DIR, "run_cases.py"), "films", libs[("pt", "pattern")],
                        str(films)], capture_output=True, text=True, env=env, timeout=1800)
    assert r.returncode == 0, r.stderr[-6000:]
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-6000:]
    runs["films"] = (str(films), json.loads(r.stdout.strip().splitlines()[-1]))
    return runs


def _mean_close(golden, res):
    if not res["fixture"]:
        return
    g = golden(res["fixture"])
    ref = float(g["mean"].mean())
    tol = 0.10
    if "frame_means" in g.files:
        fm = g["frame_means"]
        tol = max(tol, 4.0 * float(fm.std(ddof=1) / fm.mean()))
    assert abs(res["mean"] / ref - 1.0) < tol, (res["mean"], ref, tol)


@pytest.mark.parametrize("case", BDPT_CASES)
def test_bdpt_kernel_body_stays_in_range_and_reads_nothing_uninitialised(host_runs, golden, case):
    pat, zero = host_runs[("bdpt", "pattern")][case], host_runs[("bdpt", "zero")][case]
    assert pat["rc"] == 0, pat
    assert pat["chk"] == [0, 0, 0, 0], pat          # bd_index: no index left its range
    assert pat["finite"], pat
    assert pat["hash"] == zero["hash"], case        # nothing read before it is written
    _mean_close(golden, pat)


@pytest.mark.parametrize("case", PT_CASES)
def test_path_tracer_kernels_stay_in_range_and_lean_shading_equals_general(host_runs, golden, case):
    pat, zero = host_runs[("pt", "pattern")][case], host_runs[("pt", "zero")][case]
    assert pat["rc"] == 0, pat
    assert pat["finite"], pat
    assert pat["rays"] > 0, pat
    assert pat["hash"] == zero["hash"], case        # nothing read before it is written
    assert pat["general_hash"] == pat["hash"] or pat["lean_hash"] == pat["hash"], pat
    if pat["lean_hash"] is not None:                # the lean instantiation applies
        assert pat["lean_hash"] == pat["general_hash"], case
    _mean_close(golden, pat)


@pytest.mark.parametrize("case", sorted(run_cases.film_cases()))
def test_path_tracer_kernels_match_the_oracle_per_pixel(host_runs, case):
    """The kernels' source on the CPU against the oracle with the same Philox streams, with
    the GPU per-pixel tests' settings: paths of two vertices, and the Whitted ray tracer (no
    hemisphere sampling).  Both use the host's libm, so pixels agree to a few ulps (3.7e-5
    relative at most here, most of them exactly); two pixels may differ more, for a lobe or
    shadow decision that lands within an ulp of its threshold under another libm."""
    import oraclelib as O
    build, integrator, depth, spp, seed = run_cases.film_cases()[case]
    folder, meta = host_runs["films"]
    assert meta[case]["rc"] == 0, meta[case]
    film = np.load(os.path.join(folder, case + ".npy"))
    sc = build()
    if integrator == 0:
        ofilm, onan = O.OracleScene(sc).render_pt(depth, spp, seed)
    else:
        ofilm, onan = O.OracleScene(sc).render_whitted(sc.tracer.max_depth, spp, seed)
    assert meta[case]["nan"] == onan == 0
    rel = np.abs(film - ofilm) / np.maximum(np.abs(ofilm), 1e-3)
    if case.startswith("deep_"):
        # full-depth paths: 6-10% of the pixels part ways here, the film sums agree to 0.15%
        assert np.mean(rel.max(2) > 1e-3) <= 0.15, float(np.mean(rel.max(2) > 1e-3))
        assert abs(film.sum() / ofilm.sum() - 1.0) < 5e-3
        return
    assert np.sum(rel.max(2) > 1e-4) <= 2, float(rel.max())
    assert abs(film.sum() / ofilm.sum() - 1.0) < 1e-4
