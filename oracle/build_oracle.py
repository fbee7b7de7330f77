#!/usr/bin/env python3
"""Builds oracle/lib/librumi_oracle.so from oracle/rumi_oracle.c (the CPU restatement
used as the checker by tests/).  -ffp-contract=off keeps every float operation rounded
separately, as in the reference's x86 build."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "rumi_oracle.c")
LIB = os.path.join(HERE, "lib", "librumi_oracle.so")


def build(force=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    # built under a private name and renamed into place, so a process loading the library
    # while another rebuilds it never sees a partly written file
    tmp = f"{LIB}.{os.getpid()}.tmp"
    cmd = ["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-Wall",
           "-Wno-unused-function", "-o", tmp, SRC, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
