"""The BDPT kernel's body (rumi-renderer_b200/csrc/bdpt.cu) built by g++ for the host and
run over every BDPT parity scene, the volumetric-caustic workload (spot light, HG g = 0.7,
subpaths of 6 and 7 vertices) and the 16-vertex instantiation, one camera sample after
another (tests/bdpt_host):

* under AddressSanitizer and UndefinedBehaviorSanitizer: every access to a subpath array,
  a stack or a scene array stays inside its object, and no arithmetic is undefined;
* with every automatic variable set to a non-zero pattern, and again to zero: the two
  builds produce the same sample values bit for bit, so no result depends on a variable
  read before it is written;
* with the kernel's own index checks (bd_index) silent;
* with image means within 10% of the reference's frames at 16 spp (the host's libm differs
  from the device's, so the values are not the GPU's bit for bit; the mean shows the host
  build computes the same estimator).

This checks the kernel's logic on the CPU, where a fault cannot reach a GPU."""
import json
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HOST_DIR = os.path.join(HERE, "bdpt_host")
sys.path.insert(0, HOST_DIR)

import run_cases  # noqa: E402

CASES = sorted(run_cases._cases())


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
    out = tmp_path_factory.mktemp("bdpt_host")
    flags = ["-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
             "-fno-sanitize-recover=undefined", "-ffp-contract=off", "-fPIC", "-shared", "-I" + inc]
    builds = {}
    procs = []
    for init in ("pattern", "zero"):
        lib = str(out / ("libbdpt_host_%s.so" % init))
        builds[init] = lib
        procs.append(subprocess.Popen([gxx, *flags, "-ftrivial-auto-var-init=" + init, os.path.join(HOST_DIR, "bdpt_host.cpp"),
                                       "-o", lib], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    for p in procs:
        so, se = p.communicate(timeout=900)
        assert p.returncode == 0, se[-4000:]
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0", UBSAN_OPTIONS="print_stacktrace=1")
    runs = {}
    for init, lib in builds.items():
        r = subprocess.run([sys.executable, os.path.join(HOST_DIR, "run_cases.py"), lib], capture_output=True, text=True,
                           env=env, timeout=1800)
        assert r.returncode == 0, r.stderr[-6000:]
        assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-6000:]
        runs[init] = json.loads(r.stdout.strip().splitlines()[-1])
    return runs


@pytest.mark.parametrize("case", CASES)
def test_bdpt_kernel_body_stays_in_range_and_reads_nothing_uninitialised(host_runs, golden, case):
    pat, zero = host_runs["pattern"][case], host_runs["zero"][case]
    assert pat["rc"] == 0, pat
    assert pat["chk"] == [0, 0, 0, 0], pat          # bd_index: no index left its range
    assert pat["finite"], pat
    assert pat["hash"] == zero["hash"], case        # nothing read before it is written
    if pat["fixture"]:
        ref = float(golden(pat["fixture"])["mean"].mean())
        assert abs(pat["mean"] / ref - 1.0) < 0.10, (pat["mean"], ref)
