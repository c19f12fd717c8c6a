"""The C-ABI library: builds, loads, exports every declared symbol, host-side pieces (CPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "foggy_gpu.h")) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(foggy_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_exports_every_symbol(native):
    from itofoggysim_b200 import _native
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(native, n), n
    assert sorted(_native.EXPORTS) == names


def test_nm_exports_match_header(native):
    import subprocess
    from itofoggysim_b200 import _native
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    syms = set(l.split()[-1] for l in out.splitlines() if l.strip())
    for n in declared_functions():
        assert n in syms, n


def test_default_params_are_reference_defaults(native):
    from itofoggysim_b200 import _native
    p = _native.FoggyParams()
    native.foggy_default_params(C.byref(p))
    # lib_solver_GMRES.f90:93-106 and lib_mie_multi_sphere.f90:145 (tolerance 1e-6)
    assert p.gmres_restart == 10 and p.gmres_max_iterations == 1000
    assert p.gmres_tolerance == 1e-6 and p.z_coupling == 1 and p.tree_s_opt == 10


@pytest.mark.parametrize("j1,j2,m", [(3, 5, 0), (10, 7, 3), (16, 20, -15), (30, 30, 30), (30, 29, 0),
                                     (45, 44, 12), (5, 5, 5)])
def test_wigner_3j_recurrence_matches_wigxjpf(native, oracle, j1, j2, m):
    # the product's own 3j (used for the axial tables) against the reference's wigxjpf
    worst = 0.0
    for j3 in range(abs(j1 - j2), j1 + j2 + 1):
        for mm in (m, 0):
            v = native.foggy_wigner_3j(j1, j2, j3, -mm, mm, 0)
            r = oracle.wigner_3j(j1, j2, j3, -mm, mm, 0)
            worst = max(worst, abs(v - r) / max(abs(r), 1e-300) if abs(r) > 1e-14 else abs(v - r))
    assert worst < 1e-12, worst


def test_wigner_3j_general_golden(native, golden):
    g = golden["wigner_3j"]
    for j3, ref in zip(g["j3"], g["values"]):
        v = native.foggy_wigner_3j(g["j1"], g["j2"], j3, g["m1"], g["m2"], g["m3"])
        assert abs(v - ref) <= 1e-13, (j3, v, ref)


def test_wigner_3j_exhaustive_small(native, oracle):
    worst = 0.0
    for j1 in range(0, 9):
        for j2 in range(0, 9):
            for m1 in range(-j1, j1 + 1):
                for m2 in range(-j2, j2 + 1):
                    for j3 in range(abs(j1 - j2), j1 + j2 + 1):
                        if abs(m1 + m2) > j3:
                            continue
                        v = native.foggy_wigner_3j(j1, j2, j3, m1, m2, -m1 - m2)
                        r = oracle.wigner_3j(j1, j2, j3, m1, m2, -m1 - m2)
                        worst = max(worst, abs(v - r))
    assert worst < 1e-14, worst


def test_no_cpu_fallback_without_gpu(native):
    """Without a CUDA device the product refuses to run instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from itofoggysim_b200 import _native, scene, solver
    sc = scene.random_cluster(3, seed=1, p=3)
    with pytest.raises(_native.FoggyError) as e:
        solver.MultiSphereSolver(sc)
    assert e.value.code == _native.FOGGY_ERR_CUDA


def test_argument_errors_are_reported(native):
    from itofoggysim_b200 import _native
    p = _native.FoggyParams()
    native.foggy_default_params(C.byref(p))
    p.n_range[1] = 99
    h = C.c_void_p()
    rc = native.foggy_create(C.byref(p), 0, C.byref(h))
    assert rc == _native.FOGGY_ERR_ARGUMENT
    assert b"n_range" in native.foggy_last_error(None)
    p.n_range[1] = 5
    p.gmres_restart = 500
    assert native.foggy_create(C.byref(p), 0, C.byref(h)) == _native.FOGGY_ERR_ARGUMENT


C_PROGRAM = r"""
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "foggy_gpu.h"

int main(void) {
    foggy_params p;
    foggy_handle h = NULL;
    int64_t parent = -1, kids[8];
    double c[3];
    foggy_default_params(&p);
    if (p.gmres_restart != 10 || p.gmres_max_iterations != 1000) return 1;
    if (fabs(foggy_wigner_3j(2, 2, 2, 0, 0, 0) + sqrt(2.0 / 35.0)) > 1e-15) return 2;
    if (foggy_tree_parent(6, 1, 1, &parent) != FOGGY_OK || parent != 0) return 3;
    if (foggy_tree_children(1, 1, kids) != FOGGY_OK || kids[0] != 8 || kids[7] != 15) return 4;
    if (foggy_tree_centre_of_box(1, 1, c) != FOGGY_OK || c[0] != 0.25 || c[2] != 0.75) return 5;
    p.n_range[1] = 99;
    if (foggy_create(&p, 0, &h) != FOGGY_ERR_ARGUMENT || h != NULL) return 6;
    if (strstr(foggy_last_error(NULL), "n_range") == NULL) return 7;
    puts("ok");
    return 0;
}
"""


def test_c_program_links_and_runs(native, tmp_path):
    """The header is plain C (C99, pedantic) and a C program linked against the library calls it."""
    import subprocess
    from itofoggysim_b200 import _native
    src = tmp_path / "use_abi.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "use_abi"
    libdir = os.path.dirname(_native.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                        "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L" + libdir, "-l:" + os.path.basename(_native.LIB_PATH), "-Wl,-rpath," + libdir, "-lm"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)


def test_handle_less_errors_are_per_thread(native):
    """Threads whose foggy_create calls fail side by side each read their own message."""
    import threading
    from itofoggysim_b200 import _native

    def bad_params(kind):
        p = _native.FoggyParams()
        native.foggy_default_params(C.byref(p))
        if kind == 0:
            p.n_range[1] = 99
        else:
            p.lambda_0 = -1.0
        return p

    expect = [b"n_range", b"lambda_0"]
    wrong = []

    def run(kind):
        p = bad_params(kind)
        h = C.c_void_p()
        for _ in range(2000):
            native.foggy_create(C.byref(p), 0, C.byref(h))
            if expect[kind] not in native.foggy_last_error(None):
                wrong.append(kind)

    ts = [threading.Thread(target=run, args=(k % 2,)) for k in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert wrong == []


def test_fortran_module_binds_every_header_symbol():
    """The iso_c_binding module declares a bind(c) interface for every entry point of the header."""
    with open(os.path.join(ROOT, "itofoggysim_b200", "fortran", "foggy_gpu_f.f90")) as f:
        bound = set(re.findall(r'name="(foggy_[a-z0-9_]+)"', f.read()))
    assert set(declared_functions()) - bound == set()
