"""Build libfoggy_b200.so in-tree with nvcc for sm_100a.

    python -m itofoggysim_b200.build          # or: python itofoggysim_b200/build.py

The shared library lands next to this file (itofoggysim_b200/libfoggy_b200.so) so that it
travels with the source tree; nothing is installed elsewhere.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfoggy_b200.so")
SOURCES = ["foggy_api.cu", "k_direct.cu", "k_pair_tables.cu", "k_translation.cu", "k_scene.cu", "k_gmres.cu", "k_tree.cu", "gaunt.cpp", "fmm_tree.cpp", "server.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(HERE, "..", "include", "foggy_gpu.h")
    return os.path.getmtime(hdr) > t


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-ccbin", "/usr/bin/g++", "-I" + CSRC, "-I" + os.path.join(HERE, "..", "include"),
           "-o", OUT + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
