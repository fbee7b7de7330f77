#!/usr/bin/env python3
"""Build recipe for ``oracle/_ref/librumi_ref.so`` -- the reference renderer itself,
compiled from its own sources, used ONLY as the parity checker and as the timed CPU
baseline.  Test infrastructure: nothing in the product links or loads it.

What this script does (and nothing more):

1. copies ``src/**/*.{cpp,h}`` of the reference checkout (``--ref``, else the
   ``RUMI_REFERENCE`` environment variable, else ``DEFAULT_REF``) into
   ``oracle/_ref/src`` (git-ignored, never committed);
2. applies portability-only patches so that the MSVC-dialect sources build with g++ on
   LP64 Linux.  None of them changes rendering logic; each is listed in ``PATCHES``;
3. compiles every reference ``.cpp`` except ``main.cpp`` together with
   ``oracle/ref_harness.cpp`` (our own driver code) into one shared library, with
   ``oracle/ref_shim.h`` force-included into every translation unit.

The shim routes the reference's ``rand()``/``srand()`` to a seedable generator owned by
the harness (so CPU renders are reproducible and unit checks can inject uniforms) and
opens ``private``/``protected`` members so the harness can read them (``Scene::_objects``,
``Pinhole::_fov`` ...).  Run: ``python oracle/build_ref.py [--ref /path/to/reference]``.
"""
import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC_OUT = os.path.join(OUT, "src")
OBJ_OUT = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "librumi_ref.so")
# Where the read-only reference checkout is mounted in the container that builds the
# checker; machines without it use the prebuilt oracle/_ref.
DEFAULT_REF = "/root/reference"


def reference_dir():
    """The reference checkout to build from: $RUMI_REFERENCE, else DEFAULT_REF."""
    return os.environ.get("RUMI_REFERENCE") or DEFAULT_REF

# (file, old text, new text, reason) -- applied after CRLF -> LF normalisation.
PATCHES = [
    ("Kernel/intersection.h",
     "\t// Volume factor\n\tstruct\n\t{\n\t\tfloat _volumetric_s;\n\t\tfloat _volumetric_smax;\n"
     "\t\tColor _volumetric_tau;\n\t\tColor _volumetric_pdf;\n\t};\n",
     "\t// Volume factor\n\tfloat _volumetric_s;\n\tfloat _volumetric_smax;\n"
     "\tColor _volumetric_tau;\n\tColor _volumetric_pdf;\n",
     "anonymous struct with non-trivial members is MSVC-only; same members, same order"),
    ("Acceleration/bvh.cpp",
     "\t: _bound()\n\t, _offset_idx(0)\n\t, _contain_n(0)\n\t, _left(0x00)\n\t, _right(0x00)\n",
     "\t: _bound()\n\t, _left(0x00)\n\t, _right(0x00)\n",
     "g++ rejects initialising two members of one union; the pointer pair covers all bytes"),
    ("Kernel/matrix.h",
     "};\n\n#endif",
     "};\n\nMat4x4 Inverse(const Mat4x4 &matrix);\nMat4x4 Transpose(const Mat4x4 &matrix);\n"
     "Mat4x4 Translation(float x, float y, float z);\nMat4x4 Scaling(float x, float y, float z);\n"
     "Mat4x4 RotationX(float radian);\nMat4x4 RotationY(float radian);\nMat4x4 RotationZ(float radian);\n\n#endif",
     "friend-only declarations are not visible to callers under ISO C++"),
    ("Shape/model.cpp", "\t\t\tuv = 0.0f;\n", "\t\t\tuv = Point2();\n",
     "Point2 has no float constructor; Point2() is the zero point"),
    ("Shape/model.cpp", "if (n0 == Vector3())",
     "if (n0._x == 0.0f && n0._y == 0.0f && n0._z == 0.0f)", "Vector3 has no operator=="),
    ("Shape/model.cpp", "if (n1 == Vector3())",
     "if (n1._x == 0.0f && n1._y == 0.0f && n1._z == 0.0f)", "Vector3 has no operator=="),
    ("Shape/model.cpp", "if (n2 == Vector3())",
     "if (n2._x == 0.0f && n2._y == 0.0f && n2._z == 0.0f)", "Vector3 has no operator=="),
    ("Scene/scene.cpp", "\t_image->OutputBuffer();\n", "",
     "Film::OutputBuffer is declared nowhere and defined nowhere"),
    ("Kernel/bmp.h", "\tunsigned long file_size;", "\tuint32_t file_size;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long bitmap_data_offset;", "\tuint32_t bitmap_data_offset;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  bitmap_header_size;", "\tuint32_t  bitmap_header_size;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  width;", "\tuint32_t  width;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  height;", "\tuint32_t  height;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  compression;", "\tuint32_t  compression;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  bitmap_data_size;", "\tuint32_t  bitmap_data_size;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  H_resolution;", "\tuint32_t  H_resolution;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  V_resolution;", "\tuint32_t  V_resolution;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  used_colors;", "\tuint32_t  used_colors;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
    ("Kernel/bmp.h", "\tunsigned long  important_color;", "\tuint32_t  important_color;",
     "BMP header fields are 32-bit; unsigned long is 64-bit on LP64 and breaks the header"),
]

INCLUDE_RE = re.compile(r'^(\s*#\s*include\s*")([^"]+)(")', re.M)


def _resolve_include(cur_dir, path, all_files_lower):
    """Rewrite a backslash / wrong-case include path to the real relative path."""
    p = path.replace("\\\\", "/").replace("\\", "/")
    target = os.path.normpath(os.path.join(cur_dir, p))
    real = all_files_lower.get(target.lower())
    if real is None:
        raise RuntimeError(f"cannot resolve include {path!r} from {cur_dir}")
    return os.path.relpath(real, cur_dir).replace(os.sep, "/")


def copy_and_patch(ref_root):
    src = os.path.join(ref_root, "src")
    if not os.path.isdir(src):
        raise SystemExit(f"reference sources not found under {src}")
    if os.path.isdir(SRC_OUT):
        shutil.rmtree(SRC_OUT)
    files = []
    for dp, _, fns in os.walk(src):
        for fn in fns:
            if fn.endswith((".cpp", ".h")):
                rel = os.path.relpath(os.path.join(dp, fn), src)
                files.append(rel)
    all_lower = {os.path.normpath(os.path.join(SRC_OUT, f)).lower(): os.path.normpath(os.path.join(SRC_OUT, f))
                 for f in files}
    for rel in files:
        with open(os.path.join(src, rel), "r", encoding="latin-1") as fh:
            text = fh.read().replace("\r\n", "\n").replace("\r", "\n")
        dst = os.path.join(SRC_OUT, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        cur_dir = os.path.dirname(dst)
        text = INCLUDE_RE.sub(lambda m: m.group(1) + _resolve_include(cur_dir, m.group(2), all_lower) + m.group(3),
                              text)
        with open(dst, "w", encoding="latin-1") as fh:
            fh.write(text)
    for rel, old, new, why in PATCHES:
        dst = os.path.join(SRC_OUT, rel)
        with open(dst, "r", encoding="latin-1") as fh:
            text = fh.read()
        if old not in text:
            raise RuntimeError(f"patch site not found in {rel}: {why}")
        text = text.replace(old, new, 1)
        with open(dst, "w", encoding="latin-1") as fh:
            fh.write(text)
    return [f for f in files if f.endswith(".cpp") and f != "main.cpp"]


def compile_all(cpp_files, jobs):
    os.makedirs(OBJ_OUT, exist_ok=True)
    flags = ["g++", "-O2", "-fPIC", "-std=c++17", "-w", "-fno-strict-aliasing",
             "-include", os.path.join(HERE, "ref_shim.h"), "-I", SRC_OUT]
    jobs_list = []
    for rel in cpp_files:
        obj = os.path.join(OBJ_OUT, rel.replace("/", "_").replace(".cpp", ".o"))
        jobs_list.append(flags + ["-c", os.path.join(SRC_OUT, rel), "-o", obj])
    harness_obj = os.path.join(OBJ_OUT, "ref_harness.o")
    jobs_list.append(flags + ["-c", os.path.join(HERE, "ref_harness.cpp"), "-o", harness_obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: " + " ".join(cmd) + "\n" + r.stderr[-4000:])
        return cmd[-1]

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(run, jobs_list))
    cmd = ["g++", "-shared", "-Wl,-soname,librumi_ref.so", "-o", LIB] + objs + ["-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    return LIB


REPO = os.path.dirname(HERE)
ADAPTER = os.path.join(REPO, "rumi-renderer_b200", "adapter")
PRODUCT_LIB_DIR = os.path.join(REPO, "rumi-renderer_b200", "lib")
GPU_HOST_LIB = os.path.join(OUT, "librumi_ref_gpuhost.so")


def build_gpu_host():
    """oracle/_ref/librumi_ref_gpuhost.so: the reference-side adapter
    (rumi-renderer_b200/adapter/rumi_gpu_integrators.cpp, compiled against the reference's
    headers like any reference source) plus the test host oracle/ref_gpu_host.cpp, linked
    with the reference build and librumi_b200.so.  Skipped while librumi_b200.so is not
    built."""
    if not os.path.exists(os.path.join(PRODUCT_LIB_DIR, "librumi_b200.so")):
        return None
    flags = ["g++", "-O2", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-variable", "-fno-strict-aliasing",
             "-include", os.path.join(HERE, "ref_shim.h"), "-I", SRC_OUT, "-I", ADAPTER,
             "-I", os.path.join(REPO, "include")]
    objs = []
    for src in (os.path.join(ADAPTER, "rumi_gpu_integrators.cpp"), os.path.join(HERE, "ref_gpu_host.cpp")):
        obj = os.path.join(OBJ_OUT, "gpuhost_" + os.path.basename(src).replace(".cpp", ".o"))
        r = subprocess.run(flags + ["-c", src, "-o", obj], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: " + src + "\n" + r.stderr[-4000:])
        objs.append(obj)
    tmp = GPU_HOST_LIB + ".tmp"
    rel_lib = os.path.relpath(PRODUCT_LIB_DIR, OUT)
    cmd = ["g++", "-shared", "-o", tmp] + objs + [
        "-L", OUT, "-lrumi_ref", "-L", PRODUCT_LIB_DIR, "-lrumi_b200",
        "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,$ORIGIN/" + rel_lib]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    os.replace(tmp, GPU_HOST_LIB)
    return GPU_HOST_LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=reference_dir())
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args(argv)
    cpp = copy_and_patch(a.ref)
    lib = compile_all(cpp, a.j)
    print(lib)
    host = build_gpu_host()
    if host:
        print(host)
    return 0


if __name__ == "__main__":
    sys.exit(main())
