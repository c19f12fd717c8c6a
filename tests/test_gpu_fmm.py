"""ML-FMM path on the GPU against the oracle's restatement of the reference's ML-FMM.

Tree lists (E1, E2, I4 of lib_tree_get_domain_*) must be identical; the operator must match the
oracle FMM within 1e-12 (max error over max entry, scaled basis x_nm / g_nm, as for the direct
operator), in both conventions: 0 = the reference's passes as written, 1 = the consistent
expansion.  The consistent FMM must also stay close to the direct operator on a scene whose
boxes are small against the wavelength (the expansion order is the global order, as in the
reference), and a GMRES solve through it must reach its tolerance.
"""
import math

import numpy as np
import pytest

from itofoggysim_b200 import scene as S, solver

pytestmark = pytest.mark.gpu


def _g(sc):
    g = [math.sqrt(math.factorial(n + m) / math.factorial(n - m))
         for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)]
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def _err(y, ref, g):
    return np.max(np.abs((y - ref) / g)) / max(np.max(np.abs(ref / g)), 1e-300)


def _x(sc, seed):
    rng = np.random.default_rng(seed)
    n = sc.vector_length()
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * _g(sc)


def long_wave_scene(p, z=3, n=20):
    rng = np.random.default_rng(7)
    radii = rng.uniform(0.1, 0.3, n)
    return S.make_scene(radii, 8.0, 5, lambda_0=6.0, n_max=p, z_coupling=z, reference_row_rule=False,
                        tree_l_max=3)


def test_tree_lists_match_oracle(native, oracle):
    sc = S.random_cluster(40, seed=11, p=3)
    sc.tree_l_max = 3
    with solver.MultiSphereSolver(sc, use_ml_fmm=True) as s:
        u, order, lmin, lmax = s.build_tree()
        assert (lmin, lmax) == (2, 3)
        for l in (2, 3):
            for n in sorted(set((uu >> (3 * (lmax - l))) for uu in u))[:12]:
                for kind in (1, 2, 4):
                    got = s.tree_domain(l, n, kind)
                    ref = oracle.tree_domain(sc.centres, 3, l, n, kind)
                    assert np.array_equal(got, ref), (l, n, kind)


CASES = [
    # n, p, z, convention, row rule, l_max
    (16, 3, 1, 0, True, 2),
    (24, 4, 3, 0, True, 3),
    (24, 4, 1, 1, False, 3),
    (30, 5, 3, 1, False, 3),
    (20, None, 3, 0, True, 3),    # polydisperse orders: the row rule drops the lower-order spheres
    (20, None, 1, 1, False, 3),
]


@pytest.mark.parametrize("n,p,z,conv,rule,lmax", CASES)
def test_fmm_matvec_matches_oracle(native, oracle, n, p, z, conv, rule, lmax):
    sc = S.random_cluster(n, seed=n + (p or 0), p=p, z_coupling=z, reference_row_rule=rule)
    sc.tree_l_max = lmax
    P = oracle.Problem(sc)
    x = _x(sc, 3)
    ref = P.fmm_matvec(x, l_max=lmax, convention=conv, z_gt_r=3)
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=conv, z_translation_gt_r=3) as s:
        y = s.calculate_vector_b(x)
        y2 = s.calculate_vector_b(x)
    assert _err(y, ref, _g(sc)) < 1e-12
    assert np.array_equal(y, y2), "FMM operator is not bit-reproducible"


def test_consistent_fmm_close_to_direct(native, oracle):
    sc = long_wave_scene(8)
    x = _x(sc, 5)
    with solver.MultiSphereSolver(sc) as d:
        yd = d.calculate_vector_b(x)
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=1) as f:
        yf = f.calculate_vector_b(x)
    P = oracle.Problem(sc)
    assert _err(yf, P.fmm_matvec(x, l_max=3, convention=1), _g(sc)) < 1e-12
    assert _err(yf, yd, _g(sc)) < 2e-3   # expansion truncation at order 8


def test_fmm_solve(native):
    sc = long_wave_scene(8)
    sc.gmres_restart = 20
    sc.gmres_tolerance = 1e-8
    with solver.MultiSphereSolver(sc, use_ml_fmm=True, fmm_convention=1) as f:
        xf, st = f.solve()
        b = f.get_vector_b()
        r = f.calculate_vector_b(xf) - b
    assert st["status"] == 0 and st["backward_error"] <= 1e-8
    g = _g(sc)
    assert np.max(np.abs(r / g)) / np.max(np.abs(b / g)) < 1e-7
    with solver.MultiSphereSolver(sc) as d:
        xd, _ = d.solve()
    assert _err(xf, xd, g) < 5e-3
