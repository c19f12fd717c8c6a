"""Scattered field of a solved cluster at observation points: foggy_get_field against the oracle
(lib_mie_ms_get_field, FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:379-434, summing
lib_mie_ss_get_field, lib_mie_single_sphere.f90:1397-1582, over the spheres).  Points are random
in and around the cluster, on the z axis of a sphere (the poles of its frame, where the
reference switches to its tabulated pi_nm, tau_nm) and inside a sphere (field zero).
Tolerance: 1e-12 of the largest field component."""
import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu


def _points(sc, rng, n):
    c = sc.centres
    lo, hi = c.min(axis=0) - 1.0, c.max(axis=0) + 1.0
    pts = lo + (hi - lo) * rng.random((n, 3))
    c0 = c[0]
    r0 = float(sc.radius[sc.param_index[0]])
    extra = np.array([c0 + np.array([0.0, 0.0, 2.5 * r0]),     # theta = 0 in sphere 0's frame
                      c0 - np.array([0.0, 0.0, 3.0 * r0]),     # theta = pi
                      c0 + np.array([0.1 * r0, 0.0, 0.0])])    # inside sphere 0
    return np.vstack([pts, extra])


@pytest.mark.parametrize("p,z", [(4, 3), (None, 3), (6, 1)])
def test_field_matches_oracle(native, oracle, p, z):
    sc = S.random_cluster(8, seed=4, p=p, z_coupling=z)
    rng = np.random.default_rng(17)
    pts = _points(sc, rng, 60)
    P = oracle.Problem(sc)
    with solver.MultiSphereSolver(sc) as s:
        x, st = s.solve()
        E, H = s.get_field(x, pts, e_field_0=1.3)
    Eo, Ho = P.field(x, pts, 1.3)
    assert np.max(np.abs(Eo[:-1])) > 0
    assert np.max(np.abs(E - Eo)) <= 1e-12 * np.max(np.abs(Eo))
    assert np.max(np.abs(H - Ho)) <= 1e-12 * np.max(np.abs(Ho))
    assert np.all(E[-1] == 0) and np.all(H[-1] == 0)


def test_field_device_pointers(native, oracle):
    torch = pytest.importorskip("torch")
    import ctypes as C
    from itofoggysim_b200 import _native
    sc = S.small_cluster()
    rng = np.random.default_rng(3)
    pts = _points(sc, rng, 20)
    x = rng.standard_normal(sc.vector_length()) + 1j * rng.standard_normal(sc.vector_length())
    with solver.MultiSphereSolver(sc) as s:
        xd = torch.from_numpy(x).to("cuda:0")
        pd = torch.from_numpy(np.ascontiguousarray(pts)).to("cuda:0")
        Ed = torch.zeros((len(pts), 3), dtype=torch.complex128, device="cuda:0")
        Hd = torch.zeros_like(Ed)
        _native.check(s.L.foggy_get_field(s.h, C.c_void_p(xd.data_ptr()), _native.FOGGY_MEM_DEVICE, len(pts),
                                          C.c_void_p(pd.data_ptr()), 1.0, C.c_void_p(Ed.data_ptr()),
                                          C.c_void_p(Hd.data_ptr())), s.h)
        Eh, Hh = s.get_field(x, pts)
    assert np.max(np.abs(Ed.cpu().numpy() - Eh)) <= 1e-14 * np.max(np.abs(Eh))
    assert np.max(np.abs(Hd.cpu().numpy() - Hh)) <= 1e-14 * np.max(np.abs(Hh))
