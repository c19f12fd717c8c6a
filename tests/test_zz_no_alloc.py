"""foggy_matvec_static: the operator for callers that may not allocate device memory.

Some callers can't call cudaMalloc after their set-up: a host code whose memory pool owns the
rest of the GPU, or an outer loop checked to allocate nothing after warm-up.  This entry point
works in a fixed array of device memory inside the library instead.  It must give the same
y = A x as foggy_matvec (the path checked against the oracle), within the tolerance of the
operator parity tests (1e-12, max error over max entry, in the scaled basis x / g_nm), call
after call: the array keeps the previous call's contents, which must not leak into the next.

This file is collected last so that it runs both alone and after every other test.
"""
import ctypes as C
import dataclasses
import math

import numpy as np
import pytest

from itofoggysim_b200 import _native, scene as S, solver

pytestmark = pytest.mark.gpu

TOL = 1e-12
STATIC_BYTES = 32 << 20


def _g(sc):
    g = [math.sqrt(math.factorial(n + m) / math.factorial(n - m))
         for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)]
    g = np.array(g)
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def _err(y, ref, g):
    a, r = y / g, ref / g
    return np.max(np.abs(a - r)) / max(np.max(np.abs(r)), 1e-300)


def _vector(sc, seed):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(sc.vector_length()) + 1j * rng.standard_normal(sc.vector_length())) * _g(sc)
    return x


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def _static(s, torch, x):
    xd = _dev(torch, x)
    yd = torch.full_like(xd, complex(float("nan"), float("nan")))
    _native.check(s.L.foggy_matvec_static(s.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr())), s.h)
    return yd.cpu().numpy()


def _plain(s, torch, x):
    xd = _dev(torch, x)
    yd = torch.zeros_like(xd)
    s.matvec_device(xd.data_ptr(), yd.data_ptr())
    return yd.cpu().numpy()


@pytest.mark.parametrize("case", ["mixed_orders", "small_cluster"])
def test_static_matches_matvec_twice(native, case):
    torch = pytest.importorskip("torch")
    if case == "mixed_orders":
        sc = S.random_cluster(12, seed=21, p=None, z_coupling=1, reference_row_rule=False)
    else:
        sc = S.small_cluster()
    g = _g(sc)
    x1, x2 = _vector(sc, 1), _vector(sc, 2)
    with solver.MultiSphereSolver(sc) as s:
        # first on a fresh handle (no pair tables built yet), two calls in a row
        ys1 = _static(s, torch, x1)
        ys2 = _static(s, torch, x2)
        yp1 = _plain(s, torch, x1)
        yp2 = _plain(s, torch, x2)
        assert _err(ys1, yp1, g) < TOL
        assert _err(ys2, yp2, g) < TOL
        # again now that foggy_matvec has built the pair tables, with the inputs swapped so the
        # array holds the other vector's partial sums from the call before
        ys3 = _static(s, torch, x2)
        ys4 = _static(s, torch, x1)
        assert _err(ys3, yp2, g) < TOL
        assert _err(ys4, yp1, g) < TOL


def test_static_after_radial_function_change(native):
    """The static entry reads pair tables it does not build: after foggy_matvec built them for
    z = j_n, a switch to z = h_n through foggy_set_params must not let it read the old ones."""
    torch = pytest.importorskip("torch")
    sc = S.random_cluster(10, seed=23, p=None, z_coupling=1, reference_row_rule=False)
    g = _g(sc)
    x1, x2 = _vector(sc, 3), _vector(sc, 4)
    with solver.MultiSphereSolver(sc) as s:
        y1 = _plain(s, torch, x1)             # builds the z = 1 tables
        assert _err(_static(s, torch, x1), y1, g) < TOL
        s.params.z_coupling = 3
        s._set()
        ys = _static(s, torch, x2)            # before any z = 3 tables exist
        yp = _plain(s, torch, x2)             # rebuilds the tables for z = 3
        assert _err(ys, yp, g) < TOL
        assert _err(_static(s, torch, x2), yp, g) < TOL   # now with the z = 3 tables
        assert _err(yp, _plain_fresh(sc, torch, x2, 3), g) < TOL


def _plain_fresh(sc, torch, x, z):
    sc2 = dataclasses.replace(sc, z_coupling=z)
    with solver.MultiSphereSolver(sc2) as s:
        return _plain(s, torch, x)


def test_static_on_mixed_precision_handle(native):
    """A mixed-precision solve builds the single-precision tables (and the double ones when both
    fit); the static entry is FP64 and must match foggy_matvec on that handle, also after a
    precision switch and a radial-function change in between."""
    torch = pytest.importorskip("torch")
    sc = S.random_cluster(10, seed=24, p=None, z_coupling=3, reference_row_rule=False)
    g = _g(sc)
    x = _vector(sc, 5)
    with solver.MultiSphereSolver(sc, precision=1) as s:
        _, st = s.solve()
        assert st["status"] == 0
        yp = _plain(s, torch, x)
        assert _err(_static(s, torch, x), yp, g) < TOL
        # FP64 at z = 1, then mixed again at z = 1: the FP32 tables of z = 3 must be rebuilt
        s.params.precision = 0
        s.params.z_coupling = 1
        s._set()
        y1 = _plain(s, torch, x)
        s.params.precision = 1
        s._set()
        _, st1 = s.solve()
        assert st1["status"] == 0
        assert _err(_static(s, torch, x), y1, g) < TOL
    # the mixed solve at z = 1 on that handle takes the same Arnoldi steps as on a fresh handle
    sc1 = dataclasses.replace(sc, z_coupling=1)
    with solver.MultiSphereSolver(sc1, precision=1) as s:
        _, st_fresh = s.solve()
    assert st1["iterations"] == st_fresh["iterations"]


def test_static_rejects_scene_above_limit(native):
    torch = pytest.importorskip("torch")
    # 400 spheres of degree 30: 16 * 400 * 2 * 30 * 32 * (2 + 1) bytes of working memory > 32 MiB
    sc = S.random_cluster(400, seed=3, p=30, radii=np.full(400, 0.3))
    with solver.MultiSphereSolver(sc) as s:
        xd = torch.zeros(s.n, dtype=torch.complex128, device="cuda:0")
        yd = torch.zeros_like(xd)
        rc = s.L.foggy_matvec_static(s.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()))
        assert rc == _native.FOGGY_ERR_ARGUMENT
        msg = s.L.foggy_last_error(s.h).decode()
        assert "32" in msg or str(STATIC_BYTES) in msg
        assert "foggy_matvec" in msg
